// batch2d.cu -- batched kernels for many independent, uneven 2D TM solves
// (e.g. every transmitter of every phantom of a MIMO study): a persistent
// solve queue (k_batch2d), one launch per temporal pass over every solve's
// tiles (k_batch_pass), and a persistent tile queue over all passes
// (k_batch_queue).
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
#include "tile2d_cfg.cuh"

namespace wf {

template <class C, bool MAT, bool FDIV>
__device__ void run_solve(const wf_solve2d& S, int K, TileSmem<C>& sm, int* status) {
  Tile2D P{};
  P.nx = S.g.nx;
  P.ny = S.g.ny;
  P.dh = S.g.dh;
  P.de = S.g.de;
  P.dx = S.g.dx;
  P.dy = S.g.dy;
  P.mx = S.g.mur_x;
  P.my = S.g.mur_y;
  P.fastdiv = S.g.flags;
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
    const int ci = C::RH - 2 * k, cj = C::RW - 2 * k;
    for (int ci0 = 0; ci0 < P.nx; ci0 += ci)
      for (int cj0 = 0; cj0 < P.ny; cj0 += cj)
        tile2d<C, MAT, FDIV>(P, ci0, min(ci0 + ci, P.nx), cj0, min(cj0 + cj, P.ny), s0, k, sm);
    // tile2d ends with a CTA barrier, so this pass's global writes are
    // visible to every thread of the CTA before the next pass reads them.
  }
  if (plan.needs_copy()) {
    const long long n = (long long)P.nx * P.ny;
    for (long long i = threadIdx.x; i < n; i += C::THREADS) {
      S.ex[i] = S.sx[i];
      S.ey[i] = S.sy[i];
      S.hz[i] = S.sz[i];
    }
    __syncthreads();
  }
}

template <class C, bool FDIV>
__global__ void __launch_bounds__(C::THREADS, 1) k_batch2d(const wf_solve2d* __restrict__ solves,
                                                           const int* __restrict__ order,
                                                           int nsolve, int* queue, int K) {
  extern __shared__ __align__(16) unsigned char smraw[];
  TileSmem<C>& sm = *reinterpret_cast<TileSmem<C>*>(smraw);
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
    const wf_solve2d& S = solves[order[it]];
    const bool flagged = (S.g.flags & (WF_FASTDIV_X | WF_FASTDIV_Y)) == (WF_FASTDIV_X | WF_FASTDIV_Y);
    if (FDIV && !flagged) {
      // a launch in fast-division mode only runs solves whose spacings passed
      // wf_check_fastdiv; anything else is reported, not computed
      if (threadIdx.x == 0) s_status = WF_E_ARG;
    } else if (S.nsteps > 0) {
      if (S.ca != nullptr) run_solve<C, true, FDIV>(S, K, sm, &s_status);
      else run_solve<C, false, FDIV>(S, K, sm, &s_status);
    }
    __syncthreads();
    if (threadIdx.x == 0) const_cast<wf_solve2d&>(S).status = s_status;
    __syncthreads();
  }
}

struct LaunchBatch {
  const wf_solve2d* solves;
  const int* order;
  int nsolve;
  int* queue;
  int K, ctas_per_sm, nsm;
  bool fdiv;
  cudaStream_t st;
  template <class C>
  int operator()() const {
    return fdiv ? go<C, true>() : go<C, false>();
  }
  template <class C, bool FDIV>
  int go() const {
    const size_t smem = sizeof(TileSmem<C>);
    cudaError_t e = cudaFuncSetAttribute(k_batch2d<C, FDIV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(k_batch2d)");
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch2d<C, FDIV>, C::THREADS, smem);
    if (e != cudaSuccess) return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    if (per_sm < 1) return set_error(WF_E_LIMIT, "wf_batch2d_run: layout does not fit on an SM");
    if (ctas_per_sm > 0) per_sm = std::min(per_sm, ctas_per_sm);
    const int grid = std::min(nsm * per_sm, nsolve);
    k_batch2d<C, FDIV><<<grid, C::THREADS, smem, st>>>(solves, order, nsolve, queue, K);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "launch k_batch2d");
    return WF_OK;
  }
};

// ---------------------------------------------------------------------------
// Tile-queue form: one launch = one temporal pass of every listed solve.
// Work items are (solve, tile origin) triplets; each CTA takes one item and
// runs the same tile routine as the plain kernel on it, so every solve's
// result is bit-identical to its plain run, while a large grid's tiles spread
// over all SMs instead of one.  All solves of one pass sequence advance the
// same number of steps from their own step0; pass p reads the state buffers
// when `parity` is 0 and the scratch buffers when it is 1, and writes the other.
// ---------------------------------------------------------------------------
template <class C, bool FDIV>
__global__ void __launch_bounds__(C::THREADS, 1) k_batch_pass(const wf_solve2d* __restrict__ solves,
                                                              const int* __restrict__ items,
                                                              int parity, int s_off, int k) {
  extern __shared__ __align__(16) unsigned char smraw[];
  TileSmem<C>& sm = *reinterpret_cast<TileSmem<C>*>(smraw);
  const int* it = items + 3 * (long long)blockIdx.x;
  const wf_solve2d& S = solves[it[0]];
  const int ci0 = it[1], cj0 = it[2];
  Tile2D P{};
  P.nx = S.g.nx;
  P.ny = S.g.ny;
  P.dh = S.g.dh;
  P.de = S.g.de;
  P.dx = S.g.dx;
  P.dy = S.g.dy;
  P.mx = S.g.mur_x;
  P.my = S.g.mur_y;
  P.fastdiv = S.g.flags;
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
  P.status = nullptr;
  const float* A[3] = {S.ex, S.ey, S.hz};
  const float* B[3] = {S.sx, S.sy, S.sz};
  P.ex_in = parity ? B[0] : A[0];
  P.ey_in = parity ? B[1] : A[1];
  P.hz_in = parity ? B[2] : A[2];
  P.ex_out = const_cast<float*>(parity ? A[0] : B[0]);
  P.ey_out = const_cast<float*>(parity ? A[1] : B[1]);
  P.hz_out = const_cast<float*>(parity ? A[2] : B[2]);
  const int ci = C::RH - 2 * k, cj = C::RW - 2 * k;
  const int ci1 = min(ci0 + ci, P.nx), cj1 = min(cj0 + cj, P.ny);
  const int s0 = S.step0 + s_off;
  if (S.ca != nullptr) tile2d<C, true, FDIV>(P, ci0, ci1, cj0, cj1, s0, k, sm);
  else tile2d<C, false, FDIV>(P, ci0, ci1, cj0, cj1, s0, k, sm);
}

struct LaunchPassBatch {
  const wf_solve2d* solves;
  const int* items;
  int nitems, parity, s_off, k;
  bool fdiv;
  cudaStream_t st;
  template <class C>
  int operator()() const {
    return fdiv ? go<C, true>() : go<C, false>();
  }
  template <class C, bool FDIV>
  int go() const {
    const size_t smem = sizeof(TileSmem<C>);
    static bool attr_done = false;
    if (!attr_done) {
      cudaError_t e = cudaFuncSetAttribute(k_batch_pass<C, FDIV>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(k_batch_pass)");
      attr_done = true;
    }
    k_batch_pass<C, FDIV><<<nitems, C::THREADS, smem, st>>>(solves, items, parity, s_off, k);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "launch k_batch_pass");
    return WF_OK;
  }
};

// ---------------------------------------------------------------------------
// Persistent tile queue: ONE launch for all temporal passes of many solves.
// Resident CTAs (one per SM) pull items from a device work queue; item i is
// pass i / ntiles of tile i % ntiles (pass-major order, tiles largest solve
// first).  Before it runs, an item waits until its own tile and the (up to 8)
// neighbouring tiles of its solve have finished the previous pass: their
// cores cover this tile's region (core + k-cell halo, k <= core side), so
// the wait covers both the data this pass reads and the buffer it overwrites
// (the previous pass's input, still read by a neighbour until it finishes).
// Every item an item waits for sits earlier in the queue and was therefore
// taken by a CTA that is already running, so the waits always end; they are
// bounded all the same (wait_limit polls, then WF_E_TIMEOUT in the solve's
// status, the tile is skipped and still marked done so nothing waits on it).
// Region loads go through L2 (ld.global.cg): this SM may hold lines of the
// same buffer from an earlier pass in its L1.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release_gpu(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

template <class C, bool FDIV>
__global__ void __launch_bounds__(C::THREADS, 1) k_batch_queue(
    wf_solve2d* __restrict__ solves, const int* __restrict__ tiles, int ntiles,
    const int* __restrict__ nbr, int* done, int* queue, int nsteps, int K,
    unsigned wait_limit) {
  extern __shared__ __align__(16) unsigned char smraw[];
  TileSmem<C>& sm = *reinterpret_cast<TileSmem<C>*>(smraw);
  __shared__ int s_item, s_ok;
  const PassPlan plan(nsteps, K);
  const long long nitems = (long long)ntiles * plan.passes();
  const int ci = C::RH - 2 * K, cj = C::RW - 2 * K;  // core of every pass
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(queue, 1);
    __syncthreads();
    const long long it = s_item;
    if (it >= nitems || it < 0) return;
    const int pass = (int)(it / ntiles), tile = (int)(it - (long long)pass * ntiles);
    const int* T = tiles + 3 * (long long)tile;
    wf_solve2d& S = solves[T[0]];
    // lanes 0..8 of warp 0 wait for the tile itself and its neighbours
    if (threadIdx.x < 32) {
      bool ok = true;
      if (threadIdx.x < 9) {
        const int nb = nbr[9 * (long long)tile + threadIdx.x];
        if (nb >= 0) {
          unsigned spin = 0;
          while (ld_acquire_gpu(done + nb) < pass) {
            if (spin++ >= wait_limit) {
              ok = false;
              break;
            }
            __nanosleep(128);
          }
        }
      }
      ok = __all_sync(0xffffffffu, ok);
      if (threadIdx.x == 0) {
        s_ok = ok ? 1 : 0;
        if (!ok) atomicExch(&S.status, WF_E_TIMEOUT);
      }
    }
    __syncthreads();
    const bool flagged = (S.g.flags & (WF_FASTDIV_X | WF_FASTDIV_Y)) == (WF_FASTDIV_X | WF_FASTDIV_Y);
    if (FDIV && !flagged) {
      if (threadIdx.x == 0) atomicExch(&S.status, WF_E_ARG);
    } else if (s_ok) {
      Tile2D P{};
      P.nx = S.g.nx;
      P.ny = S.g.ny;
      P.dh = S.g.dh;
      P.de = S.g.de;
      P.dx = S.g.dx;
      P.dy = S.g.dy;
      P.mx = S.g.mur_x;
      P.my = S.g.mur_y;
      P.fastdiv = S.g.flags;
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
      P.status = nullptr;
      const bool par = pass & 1;
      P.ex_in = par ? S.sx : S.ex;
      P.ey_in = par ? S.sy : S.ey;
      P.hz_in = par ? S.sz : S.hz;
      P.ex_out = par ? S.ex : S.sx;
      P.ey_out = par ? S.ey : S.sy;
      P.hz_out = par ? S.hz : S.sz;
      const int ci0 = T[1], cj0 = T[2];
      const int ci1 = min(ci0 + ci, P.nx), cj1 = min(cj0 + cj, P.ny);
      const int s0 = S.step0 + plan.offset(pass), k = plan.len(pass);
      if (S.ca != nullptr) tile2d<C, true, FDIV>(P, ci0, ci1, cj0, cj1, s0, k, sm);
      else tile2d<C, false, FDIV>(P, ci0, ci1, cj0, cj1, s0, k, sm);
    }
    // tile2d ends with a CTA barrier after its stores: publish the pass
    if (threadIdx.x == 0) {
      __threadfence();
      st_release_gpu(done + tile, pass + 1);
    }
    __syncthreads();
  }
}

struct LaunchQueueBatch {
  wf_solve2d* solves;
  const int* tiles;
  int ntiles;
  const int* nbr;
  int* done;
  int* queue;
  int nsteps, K;
  unsigned wait_limit;
  bool fdiv;
  cudaStream_t st;
  template <class C>
  int operator()() const {
    return fdiv ? go<C, true>() : go<C, false>();
  }
  template <class C, bool FDIV>
  int go() const {
    const size_t smem = sizeof(TileSmem<C>);
    cudaError_t e = cudaFuncSetAttribute(k_batch_queue<C, FDIV>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(k_batch_queue)");
    int dev = 0, nsm = 0, per_sm = 0;
    e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute(SM count)");
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_queue<C, FDIV>, C::THREADS,
                                                      smem);
    if (e != cudaSuccess) return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    if (per_sm < 1) return set_error(WF_E_LIMIT, "wf_batch2d_queue: layout does not fit on an SM");
    const long long nitems = (long long)ntiles * PassPlan(nsteps, K).passes();
    const int grid = (int)std::min<long long>((long long)nsm * per_sm, nitems);
    k_batch_queue<C, FDIV><<<grid, C::THREADS, smem, st>>>(solves, tiles, ntiles, nbr, done,
                                                           queue, nsteps, K, wait_limit);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "launch k_batch_queue");
    return WF_OK;
  }
};

}  // namespace wf

using namespace wf;

extern "C" int32_t wf_batch2d_queue(wf_solve2d* solves, const int32_t* tiles, int32_t ntiles,
                                    const int32_t* nbr, int32_t* done, int32_t* queue,
                                    int32_t nsteps, const wf_tune* tune, int32_t fastdiv,
                                    int64_t wait_limit, void* stream) {
  if (ntiles < 0 || nsteps < 0 ||
      (ntiles > 0 && (solves == nullptr || tiles == nullptr || nbr == nullptr ||
                      done == nullptr || queue == nullptr)))
    return set_error(WF_E_ARG, "wf_batch2d_queue: null pointer or negative count");
  if (ntiles == 0 || nsteps == 0) return WF_OK;
  wf_tune t{};
  if (tune) {
    t = *tune;
  } else {
    t.steps_per_pass = 6;
    t.tile_i = 48;
    t.tile_j = 128;
  }
  if (int rc = check_tune2d(t)) return rc;
  const int K = t.steps_per_pass;
  if (3 * K > t.tile_i || 3 * K > t.tile_j)
    return set_error(WF_E_ARG,
                     "wf_batch2d_queue: depth %d needs a core of at least %d cells per side "
                     "(region %dx%d)", K, K, t.tile_i, t.tile_j);
  if ((long long)ntiles * PassPlan(nsteps, K).passes() > 0x7fffffffLL)
    return set_error(WF_E_LIMIT, "wf_batch2d_queue: more than 2^31-1 items");
  const unsigned lim = wait_limit < 0 ? (1u << 24) : (unsigned)std::min<long long>(wait_limit, 0xffffffffLL);
  return dispatch_cfg2d(t, LaunchQueueBatch{solves, tiles, ntiles, nbr, done, queue, nsteps, K,
                                            lim, fastdiv != 0, (cudaStream_t)stream});
}

extern "C" int32_t wf_batch2d_run(const wf_solve2d* solves, int32_t nsolve, const int32_t* order,
                                  int32_t* queue, const wf_tune* tune, int32_t ctas_per_sm,
                                  int32_t fastdiv, void* stream) {
  if (nsolve < 0 || (nsolve > 0 && (solves == nullptr || order == nullptr || queue == nullptr)))
    return set_error(WF_E_ARG, "wf_batch2d_run: null descriptor/order/queue pointer");
  if (nsolve == 0) return WF_OK;
  wf_tune t{};
  if (tune) {
    t = *tune;
  } else {
    t.steps_per_pass = 6;
    t.tile_i = 48;
    t.tile_j = 128;
  }
  if (int rc = check_tune2d(t)) return rc;
  int dev = 0, nsm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute(SM count)");
  return dispatch_cfg2d(t, LaunchBatch{solves, order, nsolve, queue, t.steps_per_pass,
                                       ctas_per_sm, nsm, fastdiv != 0, (cudaStream_t)stream});
}

extern "C" int32_t wf_batch2d_pass(const wf_solve2d* solves, const int32_t* items,
                                   int32_t nitems, int32_t parity, int32_t step_offset,
                                   int32_t k, const wf_tune* tune, int32_t fastdiv,
                                   void* stream) {
  if (nitems < 0 || (nitems > 0 && (solves == nullptr || items == nullptr)))
    return set_error(WF_E_ARG, "wf_batch2d_pass: null descriptor/item pointer");
  if (nitems == 0) return WF_OK;
  if (parity != 0 && parity != 1) return set_error(WF_E_ARG, "wf_batch2d_pass: parity is 0 or 1");
  if (step_offset < 0) return set_error(WF_E_ARG, "wf_batch2d_pass: negative step offset");
  wf_tune t{};
  if (tune) {
    t = *tune;
  } else {
    t.tile_i = 48;
    t.tile_j = 128;
  }
  t.steps_per_pass = k;
  if (int rc = check_tune2d(t)) return rc;
  return dispatch_cfg2d(t, LaunchPassBatch{solves, items, nitems, parity, step_offset, k,
                                           fastdiv != 0, (cudaStream_t)stream});
}
