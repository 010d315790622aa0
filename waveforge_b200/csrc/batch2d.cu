// batch2d.cu -- persistent batched kernel for many independent, uneven 2D
// TM solves (e.g. every transmitter of every phantom of a MIMO study).
//
// Resident CTAs pull solve indices from a device work queue (an atomic
// counter over a largest-first order, i.e. LPT list scheduling) and run each
// solve through ALL of its passes with the same tile routine as the plain
// kernel: for every pass the CTA sweeps the solve's tiles, then a CTA barrier
// orders the pass before the next one.  No inter-CTA synchronisation exists,
// so there is no spin-wait anywhere, and each solve's arithmetic is exactly
// what wf_fdtd2d_run performs for it alone.
#include <algorithm>

#include "tile2d.cuh"

namespace wf {

template <bool MAT>
__device__ void run_solve(const wf_solve2d& S, int K, int ti, int tj, float* sm, Lists2D& L,
                          int* status) {
  Tile2D P{};
  P.nx = S.g.nx;
  P.ny = S.g.ny;
  P.dh = S.g.dh;
  P.de = S.g.de;
  P.dx = S.g.dx;
  P.dy = S.g.dy;
  P.mx = S.g.mur_x;
  P.my = S.g.mur_y;
  P.ca = S.ca;
  P.cb = S.cb;
  P.src = S.src;
  P.nsrc = S.nsrc;
  P.prb = S.probes;
  P.nprb = S.nprobe;
  P.traces = S.traces;
  P.trace_ld = S.trace_ld;
  P.trace_step0 = S.trace_step0;
  P.n_check = S.n_check;
  P.check_max = S.check_max;
  P.check_base = S.n_check > 0 ? S.step0 / S.n_check : 0;
  P.status = status;
  float* A[3] = {S.ex, S.ey, S.hz};
  float* B[3] = {S.sx, S.sy, S.sz};
  const int tiles_i = (P.nx + ti - 1) / ti, tiles_j = (P.ny + tj - 1) / tj;
  const PassPlan plan(S.nsteps, K);
  for (int p = 0; p < plan.passes(); ++p) {
    float** in = (p & 1) ? B : A;
    float** out = (p & 1) ? A : B;
    P.ex_in = in[0];
    P.ey_in = in[1];
    P.hz_in = in[2];
    P.ex_out = out[0];
    P.ey_out = out[1];
    P.hz_out = out[2];
    const int s0 = S.step0 + plan.offset(p), k = plan.len(p);
    for (int bi = 0; bi < tiles_i; ++bi)
      for (int bj = 0; bj < tiles_j; ++bj) {
        const int ci0 = bi * ti, cj0 = bj * tj;
        tile2d<MAT>(P, ci0, min(ci0 + ti, P.nx), cj0, min(cj0 + tj, P.ny), s0, k, sm, L);
      }
    // tile2d ends with a CTA barrier; global writes of this pass are visible
    // to every thread of the CTA before the next pass reads them.
    __threadfence_block();
  }
  if (plan.needs_copy()) {
    const long long n = (long long)P.nx * P.ny;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) {
      S.ex[i] = S.sx[i];
      S.ey[i] = S.sy[i];
      S.hz[i] = S.sz[i];
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(512, 1) k_batch2d(const wf_solve2d* __restrict__ solves,
                                                  const int* __restrict__ order, int nsolve,
                                                  int* queue, int K, int ti, int tj) {
  extern __shared__ float sm[];
  __shared__ Lists2D L;
  __shared__ int s_item;
  __shared__ int s_status;
  for (;;) {
    if (threadIdx.x == 0) {
      s_item = atomicAdd(queue, 1);
      s_status = 0;
    }
    __syncthreads();
    const int it = s_item;
    if (it >= nsolve) return;
    const int si = order[it];
    const wf_solve2d& S = solves[si];
    if (S.nsteps > 0) {
      if (S.ca != nullptr) run_solve<true>(S, K, ti, tj, sm, L, &s_status);
      else run_solve<false>(S, K, ti, tj, sm, L, &s_status);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      // Overwrite the solve's status word (it is only written by its owner).
      const_cast<wf_solve2d&>(S).status = s_status;
    }
    __syncthreads();
  }
}

}  // namespace wf

using namespace wf;

extern "C" int32_t wf_batch2d_run(const wf_solve2d* solves, int32_t nsolve, const int32_t* order,
                                  int32_t* queue, const wf_tune* tune, int32_t ctas_per_sm,
                                  void* stream) {
  if (nsolve < 0 || (nsolve > 0 && (solves == nullptr || order == nullptr || queue == nullptr)))
    return set_error(WF_E_ARG, "wf_batch2d_run: null descriptor/order/queue pointer");
  if (nsolve == 0) return WF_OK;
  wf_tune t{};
  if (tune) {
    t = *tune;
  } else {
    t.steps_per_pass = 4;
    t.tile_i = 24;
    t.tile_j = 56;
    t.threads = 256;
    t.tile_k = 1;
  }
  if (t.steps_per_pass < 1 || t.steps_per_pass > 64 || t.tile_i < 2 || t.tile_j < 2 ||
      t.threads < 32 || t.threads > 512 || (t.threads & 31))
    return set_error(WF_E_ARG, "wf_batch2d_run: bad tune k=%d tile=%dx%d threads=%d",
                     t.steps_per_pass, t.tile_i, t.tile_j, t.threads);
  int dev = 0, nsm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute(SM count)");
  // The region of any tile is at most (tile + 2k) per side; always size for
  // the material path so one launch serves every solve.
  const size_t smem =
      tile2d_smem(t.tile_i + 2 * t.steps_per_pass, t.tile_j + 2 * t.steps_per_pass, true);
  e = cudaFuncSetAttribute(k_batch2d, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(k_batch2d)");
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch2d, t.threads, smem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
  if (per_sm < 1)
    return set_error(WF_E_LIMIT, "wf_batch2d_run: tune does not fit on an SM (smem %zu B)", smem);
  if (ctas_per_sm > 0) per_sm = std::min(per_sm, (int)ctas_per_sm);
  const int grid = std::min(nsm * per_sm, (int)nsolve);
  k_batch2d<<<grid, t.threads, smem, (cudaStream_t)stream>>>(solves, order, nsolve, queue,
                                                              t.steps_per_pass, t.tile_i, t.tile_j);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "launch k_batch2d");
  return WF_OK;
}
