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
#include "tile2d_cfg.cuh"

namespace wf {

template <class C, bool MAT, bool FDIV>
__global__ void __launch_bounds__(C::THREADS, 1) k2d_pass(Tile2D P, int ci, int cj, int tiles_j,
                                                          int step0, int k) {
  extern __shared__ __align__(16) unsigned char smraw[];
  TileSmem<C>& S = *reinterpret_cast<TileSmem<C>*>(smraw);
  const int bi = blockIdx.x / tiles_j, bj = blockIdx.x - bi * tiles_j;
  const int ci0 = bi * ci, cj0 = bj * cj;
  tile2d<C, MAT, FDIV>(P, ci0, min(ci0 + ci, P.nx), cj0, min(cj0 + cj, P.ny), step0, k, S);
}

// One single-step pass for each of gridDim.y transmitter runs that share the
// grid and coefficients: run t reads slot P.*_in + t*tx_stride, writes the
// matching output slot, and uses sources [t*src_per_tx, (t+1)*src_per_tx).
template <class C, bool MAT, bool FDIV>
__global__ void __launch_bounds__(C::THREADS, 1) k2d_states_tx(Tile2D P, int ci, int cj,
                                                               int tiles_j, int step0,
                                                               long long tx_stride,
                                                               int src_per_tx) {
  extern __shared__ __align__(16) unsigned char smraw[];
  TileSmem<C>& S = *reinterpret_cast<TileSmem<C>*>(smraw);
  const long long o = blockIdx.y * tx_stride;
  P.ex_in += o;
  P.ey_in += o;
  P.hz_in += o;
  P.ex_out += o;
  P.ey_out += o;
  P.hz_out += o;
  P.src += blockIdx.y * src_per_tx;
  const int bi = blockIdx.x / tiles_j, bj = blockIdx.x - bi * tiles_j;
  const int ci0 = bi * ci, cj0 = bj * cj;
  tile2d<C, MAT, FDIV>(P, ci0, min(ci0 + ci, P.nx), cj0, min(cj0 + cj, P.ny), step0, 1, S);
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
    // 64 x 128 regions on 512 threads of 4 x 4 cells: the fastest compiled
    // layout on large grids (2048^2, depth 6: 177.8 Gcell-upd/s against
    // 170.8 for 48 x 128 on 512 threads and 163.1 for 64 x 128 on 1024)
    t.steps_per_pass = 6;
    t.tile_i = 64;
    t.tile_j = 128;
    t.threads = 512;
  } else {
    t.steps_per_pass = 4;
    t.tile_i = 32;
    t.tile_j = 64;
  }
  t.tile_k = 1;
  return t;
}

template <class C, bool MAT, bool FDIV>
static int launch_pass_cfg(const Tile2D& P, int k, int step0, cudaStream_t st) {
  const int ci = C::RH - 2 * k, cj = C::RW - 2 * k;
  const int tiles_i = (P.nx + ci - 1) / ci, tiles_j = (P.ny + cj - 1) / cj;
  const size_t smem = sizeof(TileSmem<C>);
  static bool attr_done = false;
  if (!attr_done) {
    cudaError_t e = cudaFuncSetAttribute(k2d_pass<C, MAT, FDIV>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(k2d_pass)");
    attr_done = true;
  }
  const long long nblk = (long long)tiles_i * tiles_j;
  if (nblk > 0x7fffffffLL) return set_error(WF_E_LIMIT, "wf_fdtd2d_run: too many tiles");
  k2d_pass<C, MAT, FDIV><<<(unsigned)nblk, C::THREADS, smem, st>>>(P, ci, cj, tiles_j, step0, k);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "launch k2d_pass");
  return WF_OK;
}

struct LaunchPass {
  const Tile2D& P;
  int k, step0;
  cudaStream_t st;
  bool mat, fdiv;
  template <class C>
  int operator()() const {
    if (mat) return fdiv ? launch_pass_cfg<C, true, true>(P, k, step0, st)
                         : launch_pass_cfg<C, true, false>(P, k, step0, st);
    return fdiv ? launch_pass_cfg<C, false, true>(P, k, step0, st)
                : launch_pass_cfg<C, false, false>(P, k, step0, st);
  }
};

template <class C, bool MAT, bool FDIV>
static int launch_states_cfg(const Tile2D& P, int step0, int ntx, long long tx_stride,
                             int src_per_tx, cudaStream_t st) {
  const int ci = C::RH - 2, cj = C::RW - 2;
  const int tiles_i = (P.nx + ci - 1) / ci, tiles_j = (P.ny + cj - 1) / cj;
  const size_t smem = sizeof(TileSmem<C>);
  static bool attr_done = false;
  if (!attr_done) {
    cudaError_t e = cudaFuncSetAttribute(k2d_states_tx<C, MAT, FDIV>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(k2d_states_tx)");
    attr_done = true;
  }
  const long long nblk = (long long)tiles_i * tiles_j;
  if (nblk > 0x7fffffffLL || ntx > 65535) return set_error(WF_E_LIMIT, "wf_fdtd2d_states: grid too large");
  dim3 grid((unsigned)nblk, (unsigned)ntx);
  k2d_states_tx<C, MAT, FDIV><<<grid, C::THREADS, smem, st>>>(P, ci, cj, tiles_j, step0, tx_stride,
                                                              src_per_tx);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "launch k2d_states_tx");
  return WF_OK;
}

struct LaunchStates {
  const Tile2D& P;
  int step0, ntx;
  long long tx_stride;
  int src_per_tx;
  cudaStream_t st;
  bool mat, fdiv;
  template <class C>
  int operator()() const {
    if (mat) return fdiv ? launch_states_cfg<C, true, true>(P, step0, ntx, tx_stride, src_per_tx, st)
                         : launch_states_cfg<C, true, false>(P, step0, ntx, tx_stride, src_per_tx, st);
    return fdiv ? launch_states_cfg<C, false, true>(P, step0, ntx, tx_stride, src_per_tx, st)
                : launch_states_cfg<C, false, false>(P, step0, ntx, tx_stride, src_per_tx, st);
  }
};

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
  if (int rc = check_tune2d(t)) return rc;
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
  P.fastdiv = g->flags;
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
  const bool fdiv = (g->flags & (WF_FASTDIV_X | WF_FASTDIV_Y)) == (WF_FASTDIV_X | WF_FASTDIV_Y);

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
    const int rc = dispatch_cfg2d(t, LaunchPass{P, k, s0, st, ca != nullptr, fdiv});
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

extern "C" int32_t wf_fdtd2d_states(const wf_grid2d* g, float* states, int64_t tx_stride,
                                    int32_t ntx, int32_t nsteps, const float* ca, const float* cb,
                                    const wf_source* src, int32_t src_per_tx, int32_t step0,
                                    void* stream) {
  if (g == nullptr || states == nullptr)
    return set_error(WF_E_ARG, "wf_fdtd2d_states: null grid/states pointer");
  if (g->nx < 4 || g->ny < 4)
    return set_error(WF_E_ARG, "wf_fdtd2d_states: grid %dx%d below the 4x4 stencil minimum",
                     g->nx, g->ny);
  if ((ca == nullptr) != (cb == nullptr))
    return set_error(WF_E_ARG, "wf_fdtd2d_states: Ca and Cb must be given together");
  const long long cells = (long long)g->nx * g->ny;
  if (nsteps < 0 || step0 < 0 || src_per_tx < 0 || ntx < 1 ||
      (src_per_tx > 0 && src == nullptr) ||
      (ntx > 1 && tx_stride < (long long)(nsteps + 1) * 3 * cells))
    return set_error(WF_E_ARG, "wf_fdtd2d_states: bad counts, stride or null source array");
  if (src_per_tx > 32767) return set_error(WF_E_LIMIT, "wf_fdtd2d_states: at most 32767 sources");
  if (nsteps == 0) return WF_OK;
  wf_tune t = default_tune2d(g->nx, g->ny);
  t.steps_per_pass = 1;
  if (int rc = check_tune2d(t)) return rc;
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
  P.fastdiv = g->flags;
  P.ca = ca;
  P.cb = cb;
  P.src = src;
  P.nsrc = src_per_tx;
  const bool fdiv = (g->flags & (WF_FASTDIV_X | WF_FASTDIV_Y)) == (WF_FASTDIV_X | WF_FASTDIV_Y);
  for (int s = 0; s < nsteps; ++s) {
    float* in = states + (long long)s * 3 * cells;
    float* out = in + 3 * cells;
    P.ex_in = in;
    P.ey_in = in + cells;
    P.hz_in = in + 2 * cells;
    P.ex_out = out;
    P.ey_out = out + cells;
    P.hz_out = out + 2 * cells;
    const int rc = dispatch_cfg2d(t, LaunchStates{P, step0 + s, ntx, tx_stride, src_per_tx, st,
                                                  ca != nullptr, fdiv});
    if (rc) return rc;
  }
  return WF_OK;
}
