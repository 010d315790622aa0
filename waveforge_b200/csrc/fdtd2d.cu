// fdtd2d.cu -- plain (one solve per launch sequence) 2D TM Yee kernel and
// the wf_fdtd2d_run C entry point.
//
// A run is a sequence of passes; each pass is ONE launch of k2d_pass that
// advances every tile of the grid by k steps (temporal block depth k), reading
// the pass-input buffers and writing the pass-output buffers (ping-pong
// between the caller's state and scratch).  The pass plan makes the last pass
// land in the caller's state buffers.
#include <algorithm>

#include "tile2d.cuh"

namespace wf {

template <bool MAT>
__global__ void __launch_bounds__(512, 1) k2d_pass(Tile2D P, int ti, int tj, int tiles_j,
                                                 int step0, int k) {
  extern __shared__ float sm[];
  __shared__ Lists2D L;
  const int bi = blockIdx.x / tiles_j, bj = blockIdx.x - bi * tiles_j;
  const int ci0 = bi * ti, cj0 = bj * tj;
  const int ci1 = min(ci0 + ti, P.nx), cj1 = min(cj0 + tj, P.ny);
  tile2d<MAT>(P, ci0, ci1, cj0, cj1, step0, k, sm, L);
}

__global__ void k_copy3(const float* __restrict__ a, const float* __restrict__ b,
                        const float* __restrict__ c, float* __restrict__ x,
                        float* __restrict__ y, float* __restrict__ z, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    x[i] = a[i];
    y[i] = b[i];
    z[i] = c[i];
  }
}

wf_tune default_tune2d(int nx, int ny) {
  wf_tune t{};
  if ((long long)nx * ny >= 1024LL * 1024) {
    t.steps_per_pass = 4;
    t.tile_i = 24;
    t.tile_j = 120;
    t.threads = 512;
  } else {
    t.steps_per_pass = 4;
    t.tile_i = 24;
    t.tile_j = 56;
    t.threads = 256;
  }
  t.tile_k = 1;
  return t;
}

int validate_tune2d(const wf_tune& t) {
  if (t.steps_per_pass < 1 || t.steps_per_pass > 64 || t.tile_i < 2 || t.tile_j < 2 ||
      t.threads < 32 || t.threads > 512 || (t.threads & 31))
    return set_error(WF_E_ARG, "bad 2D tune: k=%d tile=%dx%d threads=%d", t.steps_per_pass,
                     t.tile_i, t.tile_j, t.threads);
  return WF_OK;
}

template <bool MAT>
static int launch_pass(const Tile2D& P, const wf_tune& t, int step0, int k, cudaStream_t st) {
  const int tiles_i = (P.nx + t.tile_i - 1) / t.tile_i;
  const int tiles_j = (P.ny + t.tile_j - 1) / t.tile_j;
  const int rh = std::min(t.tile_i + 2 * k, P.nx), rw = std::min(t.tile_j + 2 * k, P.ny);
  const size_t smem = tile2d_smem(rh, rw, MAT);
  cudaError_t e = cudaFuncSetAttribute(k2d_pass<MAT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(k2d_pass)");
  k2d_pass<MAT><<<tiles_i * tiles_j, t.threads, smem, st>>>(P, t.tile_i, t.tile_j, tiles_j, step0, k);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "launch k2d_pass");
  return WF_OK;
}

}  // namespace wf

using namespace wf;

extern "C" int32_t wf_fdtd2d_run(const wf_grid2d* g, float* ex, float* ey, float* hz, float* sx,
                                 float* sy, float* sz, const float* ca, const float* cb,
                                 const wf_source* src, int32_t nsrc, const wf_probe* probes,
                                 int32_t nprobe, float* traces, int64_t trace_ld,
                                 int32_t trace_step0, int32_t step0, int32_t nsteps,
                                 int32_t n_check, uint32_t* check_max, const wf_tune* tune,
                                 void* stream) {
  if (g == nullptr || ex == nullptr || ey == nullptr || hz == nullptr || sx == nullptr ||
      sy == nullptr || sz == nullptr)
    return set_error(WF_E_ARG, "wf_fdtd2d_run: null grid/state/scratch pointer");
  if (g->nx < 4 || g->ny < 4)
    return set_error(WF_E_ARG, "wf_fdtd2d_run: grid %dx%d below the 4x4 stencil minimum", g->nx,
                     g->ny);
  if ((ca == nullptr) != (cb == nullptr))
    return set_error(WF_E_ARG, "wf_fdtd2d_run: Ca and Cb must be given together");
  if (nsteps < 0 || step0 < 0 || nsrc < 0 || nprobe < 0 || (nsrc > 0 && src == nullptr) ||
      (nprobe > 0 && (probes == nullptr || traces == nullptr)))
    return set_error(WF_E_ARG, "wf_fdtd2d_run: bad counts or null descriptor arrays");
  if (nsrc > 32767 || nprobe > 32767)
    return set_error(WF_E_LIMIT, "wf_fdtd2d_run: at most 32767 sources and probes");
  if (nsteps == 0) return WF_OK;
  const wf_tune t = tune ? *tune : default_tune2d(g->nx, g->ny);
  if (int rc = validate_tune2d(t)) return rc;
  cudaStream_t st = (cudaStream_t)stream;

  Tile2D P{};
  P.nx = g->nx;
  P.ny = g->ny;
  P.dh = g->dh;
  P.de = g->de;
  P.dx = g->dx;
  P.dy = g->dy;
  P.mx = g->mur_x;
  P.my = g->mur_y;
  P.ca = ca;
  P.cb = cb;
  P.src = src;
  P.nsrc = nsrc;
  P.prb = probes;
  P.nprb = nprobe;
  P.traces = traces;
  P.trace_ld = trace_ld;
  P.trace_step0 = trace_step0;
  P.n_check = n_check;
  P.check_max = check_max;
  P.check_base = n_check > 0 ? step0 / n_check : 0;
  P.status = nullptr;

  float* A[3] = {ex, ey, hz};
  float* B[3] = {sx, sy, sz};
  const PassPlan plan(nsteps, t.steps_per_pass);
  for (int p = 0; p < plan.passes(); ++p) {
    float** in = (p & 1) ? B : A;
    float** out = (p & 1) ? A : B;
    P.ex_in = in[0];
    P.ey_in = in[1];
    P.hz_in = in[2];
    P.ex_out = out[0];
    P.ey_out = out[1];
    P.hz_out = out[2];
    const int s0 = step0 + plan.offset(p), k = plan.len(p);
    const int rc = ca ? launch_pass<true>(P, t, s0, k, st) : launch_pass<false>(P, t, s0, k, st);
    if (rc) return rc;
  }
  if (plan.needs_copy()) {
    const long long n = (long long)g->nx * g->ny;
    k_copy3<<<592, 256, 0, st>>>(sx, sy, sz, ex, ey, hz, n);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "launch k_copy3");
  }
  return WF_OK;
}
