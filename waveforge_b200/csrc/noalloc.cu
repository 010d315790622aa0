// noalloc.cu -- wf_fdtd2d_run_noalloc: the 2D run for callers that cannot
// allocate device memory.
//
// wf_fdtd2d_run needs a caller-owned scratch copy of the three fields (the
// ping-pong partner of its temporally blocked passes).  Some callers cannot
// provide one: applications that hand all GPU memory to their own pool
// allocator (a cudaMalloc from a library would fail or fragment that pool),
// and latency-critical loops that must not call cudaMalloc/cudaFree because
// those can synchronise the whole device.  For them this entry point keeps
// the scratch in a file-scope device array that is part of the library
// image, sized for grids of up to WF_NOALLOC_MAX_CELLS cells, and allocates
// nothing: no cudaMalloc, no cudaFree, no allocating library call.
//
// The array is reserved on every GPU that loads this library's device code,
// and stays until the process exits.  All calls on a device share it, and it
// keeps whatever the previous call left there; that is harmless because every
// pass writes every scratch cell before it is read, so nothing has to start at
// zero.  Calls that can overlap on the GPU (e.g. on two streams) race on the
// array and must be serialised by the caller.
#include <mutex>

#include "wf_common.cuh"

namespace {

constexpr long long kMaxCells = WF_NOALLOC_MAX_CELLS;

// Ex, Ey, Hz scratch planes, kMaxCells floats each.
static __device__ __align__(256) float g_scratch[3 * kMaxCells];

// Device address of g_scratch per device (looked up once per device).  It is
// the address in the device's current CUDA context: after cudaDeviceReset
// the cached value is stale, so a process that resets a device must reload
// this library before calling it again.
constexpr int kMaxDevices = 64;
std::mutex g_mu;
float* g_addr[kMaxDevices] = {};

}  // namespace

extern "C" int32_t wf_fdtd2d_run_noalloc(const wf_grid2d* g, float* ex, float* ey, float* hz,
                                         const float* ca, const float* cb, const wf_source* src,
                                         int32_t nsrc, const wf_probe* probes, int32_t nprobe,
                                         float* traces, int64_t trace_ld, int32_t trace_step0,
                                         int32_t step0, int32_t nsteps, int32_t n_check,
                                         uint32_t* check_max, const wf_tune* tune, void* stream) {
  if (g == nullptr) return wf::set_error(WF_E_ARG, "wf_fdtd2d_run_noalloc: null grid");
  if (g->nx < 0 || g->ny < 0)
    return wf::set_error(WF_E_ARG, "wf_fdtd2d_run_noalloc: negative grid size %dx%d", g->nx,
                         g->ny);
  const long long cells = (long long)g->nx * g->ny;
  if (cells > kMaxCells)
    return wf::set_error(WF_E_LIMIT,
                         "wf_fdtd2d_run_noalloc: grid %dx%d has %lld cells, above the %lld-cell "
                         "limit of the built-in scratch (use wf_fdtd2d_run with your own scratch)",
                         g->nx, g->ny, cells, kMaxCells);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return wf::cuda_fail(e, "wf_fdtd2d_run_noalloc: cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices)
    return wf::set_error(WF_E_LIMIT, "wf_fdtd2d_run_noalloc: device %d out of range", dev);
  float* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (g_addr[dev] == nullptr) {
      // One-time set-up on this device (the current one): the host-side name
      // g_scratch is only a stand-in, the kernels need its device address.
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_scratch);
      if (e != cudaSuccess)
        return wf::cuda_fail(e, "wf_fdtd2d_run_noalloc: cudaGetSymbolAddress(scratch)");
      g_addr[dev] = static_cast<float*>(p);
    }
    base = g_addr[dev];
  }
  return wf_fdtd2d_run(g, ex, ey, hz, base, base + kMaxCells, base + 2 * kMaxCells, ca, cb, src,
                       nsrc, probes, nprobe, traces, trace_ld, trace_step0, step0, nsteps, n_check,
                       check_max, tune, stream);
}
