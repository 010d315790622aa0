// fdtd2d_f64.cu -- the 2D TM leapfrog in float64, for grids whose FieldSet is
// float64 (the reference's YeeGrid / FieldSet accept dtype=torch.float64,
// src/core/grid.py:226-239, src/core/fields.py:124-130).
//
// One step is the reference's sequence of whole-grid operations
// (src/core/fdtd2d.py:219-257), one launch each, every operation a separately
// rounded IEEE float64 op in the reference's order:
//   snapshot Hz (boundaries.py:237) -> soft sources in collection order
//   (sources.py:863-887, 1060-1071) -> Faraday on i<Nx-1, j<Ny-1 -> Mur x
//   edges, then y edges (boundaries.py:259-274) -> dHz/dy, dHz/dx of the final
//   Hz and the Ampere updates of Ex (j>=1) and Ey (i>=1) -> detector samples.
// This path exists for float64 verification runs, not for speed: the float32
// engine is the temporally blocked one.
#include <algorithm>

#include "wf_common.cuh"

namespace wf {

__global__ void k64_copy(const double* __restrict__ a, double* __restrict__ b, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    b[i] = a[i];
}

// Every source in array order, one CTA: a barrier separates the sources so
// overlapping boxes accumulate in collection order.  wave / amp point at
// float64 tables in this path.
__global__ void k64_inject(const wf_source* __restrict__ src, int nsrc, double* ex, double* ey,
                           double* hz, int ny, int n) {
  for (int s = 0; s < nsrc; ++s) {
    const wf_source Q = src[s];
    double* f = Q.comp == WF_EX ? ex : (Q.comp == WF_EY ? ey : hz);
    const double* wave = reinterpret_cast<const double*>(Q.wave);
    const double* amp = reinterpret_cast<const double*>(Q.amp);
    const double w = wave[n];
    const int bw = Q.j1 - Q.j0, cells = (Q.i1 - Q.i0) * bw;
    for (int c = threadIdx.x; c < cells; c += blockDim.x) {
      const long long g = (long long)(Q.i0 + c / bw) * ny + (Q.j0 + c % bw);
      const double v = amp == nullptr ? w : __dmul_rn(w, amp[c]);
      f[g] = __dadd_rn(f[g], v);
    }
    __syncthreads();
  }
}

__global__ void k64_faraday(const double* __restrict__ ex, const double* __restrict__ ey,
                            double* __restrict__ hz, int nx, int ny, double dh, double dx,
                            double dy) {
  const long long n = (long long)(nx - 1) * (ny - 1);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / (ny - 1)), j = (int)(t % (ny - 1));
    const long long g = (long long)i * ny + j;
    const double a = __ddiv_rn(__dsub_rn(ex[g + 1], ex[g]), dy);
    const double b = __ddiv_rn(__dsub_rn(ey[g + ny], ey[g]), dx);
    hz[g] = __dadd_rn(hz[g], __dmul_rn(dh, __dsub_rn(a, b)));
  }
}

// x edges (rows 0 and Nx-1) from the snapshot and the curl-updated row next
// to them.
__global__ void k64_mur_x(double* hz, const double* __restrict__ hp, int nx, int ny, double cx) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < ny; j += gridDim.x * blockDim.x) {
    const long long r1 = ny, rl = (long long)(nx - 1) * ny, rl1 = (long long)(nx - 2) * ny;
    hz[j] = __dadd_rn(hp[r1 + j], __dmul_rn(cx, __dsub_rn(hz[r1 + j], hp[j])));
    hz[rl + j] = __dadd_rn(hp[rl1 + j], __dmul_rn(cx, __dsub_rn(hz[rl1 + j], hp[rl + j])));
  }
}

// y edges (columns 0 and Ny-1), after the x edges.
__global__ void k64_mur_y(double* hz, const double* __restrict__ hp, int nx, int ny, double cy) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nx; i += gridDim.x * blockDim.x) {
    const long long r = (long long)i * ny;
    hz[r] = __dadd_rn(hp[r + 1], __dmul_rn(cy, __dsub_rn(hz[r + 1], hp[r])));
    hz[r + ny - 1] = __dadd_rn(hp[r + ny - 2], __dmul_rn(cy, __dsub_rn(hz[r + ny - 2], hp[r + ny - 1])));
  }
}

template <bool MAT>
__global__ void k64_ampere(double* ex, double* ey, const double* __restrict__ hz,
                           const double* __restrict__ ca, const double* __restrict__ cb, int nx,
                           int ny, double de, double dx, double dy) {
  const long long n = (long long)nx * ny;
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < n;
       g += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(g / ny), j = (int)(g % ny);
    if (j >= 1) {
      const double d = __ddiv_rn(__dsub_rn(hz[g], hz[g - 1]), dy);
      ex[g] = MAT ? __dadd_rn(__dmul_rn(ca[g], ex[g]), __dmul_rn(cb[g], d))
                  : __dadd_rn(ex[g], __dmul_rn(de, d));
    }
    if (i >= 1) {
      const double d = __ddiv_rn(__dsub_rn(hz[g], hz[g - ny]), dx);
      ey[g] = MAT ? __dsub_rn(__dmul_rn(ca[g], ey[g]), __dmul_rn(cb[g], d))
                  : __dsub_rn(ey[g], __dmul_rn(de, d));
    }
  }
}

__global__ void k64_probe(const wf_probe* __restrict__ prb, int nprb, const double* ex,
                          const double* ey, const double* hz, int ny, double* traces,
                          long long ld, int col) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nprb; q += gridDim.x * blockDim.x) {
    const wf_probe p = prb[q];
    const double* f = p.comp == WF_EX ? ex : (p.comp == WF_EY ? ey : hz);
    traces[q * ld + col] = f[(long long)p.i * ny + p.j];
  }
}

// |field| maxima of the three components as ordered float64 bits.
__global__ void k64_max(const double* ex, const double* ey, const double* hz, long long n,
                        unsigned long long* out) {
  unsigned long long m[3] = {0ull, 0ull, 0ull};
  const double* f[3] = {ex, ey, hz};
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < n;
       g += (long long)gridDim.x * blockDim.x)
    for (int c = 0; c < 3; ++c)
      m[c] = max(m[c], (unsigned long long)__double_as_longlong(f[c][g]) & 0x7fffffffffffffffull);
  for (int c = 0; c < 3; ++c) {
    for (int sh = 16; sh > 0; sh >>= 1) m[c] = max(m[c], __shfl_xor_sync(0xffffffffu, m[c], sh));
    if ((threadIdx.x & 31) == 0) atomicMax(&out[c], m[c]);
  }
}

static int launched(const char* what) {
  cudaError_t e = cudaGetLastError();
  return e != cudaSuccess ? cuda_fail(e, what) : WF_OK;
}

}  // namespace wf

using namespace wf;

extern "C" int32_t wf_fdtd2d_run_f64(const wf_grid2d_f64* g, double* ex, double* ey, double* hz,
                                     double* hz_prev, const double* ca, const double* cb,
                                     const wf_source* src, int32_t nsrc, const wf_probe* probes,
                                     int32_t nprobe, double* traces, int64_t trace_ld,
                                     int32_t trace_step0, int32_t step0, int32_t nsteps,
                                     int32_t n_check, uint64_t* check_max, void* stream) {
  if (g == nullptr || ex == nullptr || ey == nullptr || hz == nullptr || hz_prev == nullptr)
    return set_error(WF_E_ARG, "wf_fdtd2d_run_f64: null grid/state/snapshot pointer");
  if (g->nx < 4 || g->ny < 4)
    return set_error(WF_E_ARG, "wf_fdtd2d_run_f64: grid %dx%d below the 4x4 stencil minimum",
                     g->nx, g->ny);
  if ((ca == nullptr) != (cb == nullptr))
    return set_error(WF_E_ARG, "wf_fdtd2d_run_f64: Ca and Cb must be given together");
  if (nsteps < 0 || step0 < 0 || nsrc < 0 || nprobe < 0 || (nsrc > 0 && src == nullptr) ||
      (nprobe > 0 && (probes == nullptr || traces == nullptr)) || trace_ld < 0 ||
      (nprobe > 0 && (trace_step0 > step0 || step0 + nsteps - trace_step0 > trace_ld)))
    return set_error(WF_E_ARG, "wf_fdtd2d_run_f64: bad counts, trace window or null arrays");
  if (nsteps == 0) return WF_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const int nx = g->nx, ny = g->ny;
  const long long cells = (long long)nx * ny;
  const int T = 256;
  const unsigned gc = (unsigned)std::min<long long>((cells + T - 1) / T, 148LL * 8);
  const unsigned gf = (unsigned)std::min<long long>(((long long)(nx - 1) * (ny - 1) + T - 1) / T,
                                                    148LL * 8);
  const long long cbase = n_check > 0 ? step0 / n_check : 0;
  for (int s = 0; s < nsteps; ++s) {
    const int n = step0 + s;
    k64_copy<<<gc, T, 0, st>>>(hz, hz_prev, cells);
    if (nsrc > 0) k64_inject<<<1, 512, 0, st>>>(src, nsrc, ex, ey, hz, ny, n);
    k64_faraday<<<gf, T, 0, st>>>(ex, ey, hz, nx, ny, g->dh, g->dx, g->dy);
    k64_mur_x<<<(ny + T - 1) / T, T, 0, st>>>(hz, hz_prev, nx, ny, g->mur_x);
    k64_mur_y<<<(nx + T - 1) / T, T, 0, st>>>(hz, hz_prev, nx, ny, g->mur_y);
    if (ca != nullptr)
      k64_ampere<true><<<gc, T, 0, st>>>(ex, ey, hz, ca, cb, nx, ny, g->de, g->dx, g->dy);
    else
      k64_ampere<false><<<gc, T, 0, st>>>(ex, ey, hz, ca, cb, nx, ny, g->de, g->dx, g->dy);
    if (nprobe > 0)
      k64_probe<<<(nprobe + 127) / 128, 128, 0, st>>>(probes, nprobe, ex, ey, hz, ny, traces,
                                                      trace_ld, n - trace_step0);
    if (check_max != nullptr && n_check > 0 && (n + 1) % n_check == 0) {
      unsigned long long* out =
          reinterpret_cast<unsigned long long*>(check_max) + 3 * ((n + 1) / n_check - cbase - 1);
      k64_max<<<gc, T, 0, st>>>(ex, ey, hz, cells, out);
    }
    if (int rc = launched("launch float64 step")) return rc;
  }
  return WF_OK;
}
