// paint2d.cu -- per-cell Ca/Cb of a region-painted 2D material map, on the device.
//
// MaterialMap.build (src/core/materials.py:200-252) evaluates each region's
// mask on float32 index grids I, J in painter's order (later regions win)
// and stores the float32-rounded Material.ca/cb (:61-82) of the winning
// material.  The masks are float32 PyTorch expressions with Python-float
// parameters, which PyTorch rounds to float32 before each op:
//   circle   (I - ci)**2 + (J - cj)**2 <= r*r            (materials.py:143-163)
//   rectangle I >= i0 & I <= i1 & J >= j0 & J <= j1        (:165-185)
//   ellipse  ((I - ci)/a)**2 + ((J - cj)/b)**2 <= 1.0     (axis-aligned; the
//            benchmark phantoms paint it through add_custom)
//   shell    ellipse(outer) & ~ellipse(inner)
// Here every parameter arrives float32-rounded by the host and each op is a
// separately rounded _rn intrinsic in the same order (x**2 is x*x), so the
// label of every cell, and therefore Ca/Cb, is bit-identical to the host
// painter.  The material table (ca, cb per material, index 0 = default) is
// computed by the host exactly as Material.ca/cb do.
#include "wf_common.cuh"

namespace wf {

constexpr int kMaxRegions = 1024;

__device__ __forceinline__ bool in_ellipse(float fi, float fj, float ci, float cj, float a,
                                           float b) {
  const float u = fdiv(fsub(fi, ci), a);
  const float v = fdiv(fsub(fj, cj), b);
  return fadd(fmul(u, u), fmul(v, v)) <= 1.0f;
}

__device__ __forceinline__ bool in_region(const wf_region2d& r, float fi, float fj) {
  const float* p = r.p;
  switch (r.kind) {
    case WF_REGION_CIRCLE: {
      const float u = fsub(fi, p[0]), v = fsub(fj, p[1]);
      return fadd(fmul(u, u), fmul(v, v)) <= p[2];
    }
    case WF_REGION_RECT:
      return fi >= p[0] && fi <= p[1] && fj >= p[2] && fj <= p[3];
    case WF_REGION_ELLIPSE:
      return in_ellipse(fi, fj, p[0], p[1], p[2], p[3]);
    case WF_REGION_SHELL:
      return in_ellipse(fi, fj, p[0], p[1], p[2], p[3]) &&
             !in_ellipse(fi, fj, p[4], p[5], p[6], p[7]);
    default:
      return false;
  }
}

__global__ void k_paint2d(int nx, int ny, const wf_region2d* __restrict__ regions, int nreg,
                          const float* __restrict__ tca, const float* __restrict__ tcb,
                          const double* __restrict__ teps, const double* __restrict__ tsig,
                          int nmat, float* __restrict__ ca, float* __restrict__ cb,
                          double* __restrict__ eps, double* __restrict__ sig, int* status) {
  __shared__ wf_region2d R[128];
  const long long n = (long long)nx * ny;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long first = blockIdx.x * (long long)blockDim.x;
  for (long long base = first; base < n; base += stride) {
    const long long q = base + threadIdx.x;
    const int i = q < n ? (int)(q / ny) : 0;
    const int j = q < n ? (int)(q - (long long)i * ny) : 0;
    const float fi = (float)i, fj = (float)j;
    int label = 0;
    for (int r0 = 0; r0 < nreg; r0 += 128) {
      const int m = min(128, nreg - r0);
      __syncthreads();
      for (int t = threadIdx.x; t < m; t += blockDim.x) R[t] = regions[r0 + t];
      __syncthreads();
      for (int t = 0; t < m; ++t)
        if (in_region(R[t], fi, fj)) label = R[t].material;
    }
    if (label < 0 || label >= nmat) {
      // a material index outside the table: report it, paint the default
      if (status != nullptr) atomicExch(status, WF_E_ARG);
      label = 0;
    }
    if (q < n) {
      ca[q] = tca[label];
      cb[q] = tcb[label];
      if (eps != nullptr) {
        eps[q] = teps[label];
        sig[q] = tsig[label];
      }
    }
  }
}

}  // namespace wf

using namespace wf;

extern "C" int32_t wf_paint2d(int32_t nx, int32_t ny, const wf_region2d* regions, int32_t nreg,
                              const float* table_ca, const float* table_cb,
                              const double* table_eps, const double* table_sigma, int32_t nmat,
                              float* ca, float* cb, double* eps_r, double* sigma,
                              int32_t* status, void* stream) {
  if (nx < 1 || ny < 1 || nreg < 0 || nmat < 1 || table_ca == nullptr || table_cb == nullptr ||
      ca == nullptr || cb == nullptr || (nreg > 0 && regions == nullptr))
    return set_error(WF_E_ARG, "wf_paint2d: bad sizes or null pointers");
  if ((eps_r == nullptr) != (sigma == nullptr) ||
      (eps_r != nullptr && (table_eps == nullptr || table_sigma == nullptr)))
    return set_error(WF_E_ARG, "wf_paint2d: eps_r/sigma outputs need both tables and both planes");
  if (nreg > kMaxRegions)
    return set_error(WF_E_LIMIT, "wf_paint2d: at most %d regions", kMaxRegions);
  int dev = 0, nsm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
  const long long n = (long long)nx * ny;
  const long long want = (n + 255) / 256;
  const int blocks = (int)(want < 8LL * nsm ? want : 8LL * nsm);
  k_paint2d<<<blocks, 256, 0, (cudaStream_t)stream>>>(nx, ny, regions, nreg, table_ca, table_cb,
                                                       table_eps, table_sigma, nmat, ca, cb, eps_r,
                                                       sigma, status);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "launch k_paint2d");
  return WF_OK;
}
