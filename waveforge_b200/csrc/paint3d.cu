// paint3d.cu -- per-cell Ca/Cb of a region-painted 3D material map, on the device.
//
// MaterialMap3D.build3d (src/core/materials.py:425-478) evaluates each
// region's mask on float32 index grids I, J, K in painter's order (later
// regions win) and stores the float32 Material.ca/cb of the winning
// material.  The masks are float32 PyTorch expressions whose Python-float
// parameters are rounded to float32 before each op (materials.py:297-423):
//   sphere     (I-ci)**2 + (J-cj)**2 + (K-ck)**2 <= r*r
//   box        I >= i0 & I <= i1 & J >= j0 & J <= j1 & K >= k0 & K <= k1
//   ellipsoid  (I-ci)**2 / a**2 + (J-cj)**2 / b**2 + (K-ck)**2 / c**2 <= 1
//   cylinder   along x: (J-cj)**2 + (K-ck)**2 <= r*r & |I-ci| <= h/2
//              (y, z alike with the roles of the axes exchanged)
// The host passes every parameter float32-rounded; each op here is one
// separately rounded _rn intrinsic in the same order (x**2 is x*x), so the
// label of every cell, and Ca/Cb, are bit-identical to the host painter.
#include "wf_common.cuh"

namespace wf {

constexpr int kMaxRegions3 = 1024;
constexpr int kStage3 = 128;  // regions staged in shared memory per pass

__device__ __forceinline__ float sq(float x) { return fmul(x, x); }

__device__ __forceinline__ bool in_region3(const wf_region3d& r, float fi, float fj, float fk) {
  const float* p = r.p;
  switch (r.kind) {
    case WF_REGION3_SPHERE:
      return fadd(fadd(sq(fsub(fi, p[0])), sq(fsub(fj, p[1]))), sq(fsub(fk, p[2]))) <= p[3];
    case WF_REGION3_BOX:
      return fi >= p[0] && fi <= p[1] && fj >= p[2] && fj <= p[3] && fk >= p[4] && fk <= p[5];
    case WF_REGION3_ELLIPSOID:
      return fadd(fadd(fdiv(sq(fsub(fi, p[0])), p[3]), fdiv(sq(fsub(fj, p[1])), p[4])),
                  fdiv(sq(fsub(fk, p[2])), p[5])) <= 1.0f;
    case WF_REGION3_CYL_X:
      return fadd(sq(fsub(fj, p[1])), sq(fsub(fk, p[2]))) <= p[3] &&
             fabsf(fsub(fi, p[0])) <= p[4];
    case WF_REGION3_CYL_Y:
      return fadd(sq(fsub(fi, p[0])), sq(fsub(fk, p[2]))) <= p[3] &&
             fabsf(fsub(fj, p[1])) <= p[4];
    case WF_REGION3_CYL_Z:
      return fadd(sq(fsub(fi, p[0])), sq(fsub(fj, p[1]))) <= p[3] &&
             fabsf(fsub(fk, p[2])) <= p[4];
    default:
      return false;
  }
}

// One thread per cell (grid-stride); the region list passes through shared
// memory kStage3 regions at a time, so every block reads it once per pass.
__global__ void k_paint3d(int nx, int ny, int nz, const wf_region3d* __restrict__ regions,
                          int nreg, const float* __restrict__ tca, const float* __restrict__ tcb,
                          int nmat, float* __restrict__ ca, float* __restrict__ cb, int* status) {
  __shared__ wf_region3d R[kStage3];
  const long long plane = (long long)ny * nz, n = (long long)nx * plane;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long base = blockIdx.x * (long long)blockDim.x; base < n; base += stride) {
    const long long q = base + threadIdx.x;
    const long long qq = q < n ? q : 0;
    const int i = (int)(qq / plane);
    const long long rem = qq - (long long)i * plane;
    const int j = (int)(rem / nz), k = (int)(rem - (long long)j * nz);
    const float fi = (float)i, fj = (float)j, fk = (float)k;
    int label = 0;
    for (int r0 = 0; r0 < nreg; r0 += kStage3) {
      const int m = min(kStage3, nreg - r0);
      __syncthreads();
      for (int t = threadIdx.x; t < m; t += blockDim.x) R[t] = regions[r0 + t];
      __syncthreads();
      for (int t = 0; t < m; ++t)
        if (in_region3(R[t], fi, fj, fk)) label = R[t].material;
    }
    if (label < 0 || label >= nmat) {
      // a material index outside the table: report it, paint the default
      if (status != nullptr) atomicExch(status, WF_E_ARG);
      label = 0;
    }
    if (q < n) {
      ca[q] = tca[label];
      cb[q] = tcb[label];
    }
  }
}

}  // namespace wf

using namespace wf;

extern "C" int32_t wf_paint3d(int32_t nx, int32_t ny, int32_t nz, const wf_region3d* regions,
                              int32_t nreg, const float* table_ca, const float* table_cb,
                              int32_t nmat, float* ca, float* cb, int32_t* status, void* stream) {
  if (nx < 1 || ny < 1 || nz < 1 || nreg < 0 || nmat < 1 || table_ca == nullptr ||
      table_cb == nullptr || ca == nullptr || cb == nullptr || (nreg > 0 && regions == nullptr))
    return set_error(WF_E_ARG, "wf_paint3d: bad sizes or null pointers");
  if (nreg > kMaxRegions3)
    return set_error(WF_E_LIMIT, "wf_paint3d: at most %d regions", kMaxRegions3);
  int dev = 0, nsm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
  const long long n = (long long)nx * ny * nz;
  const long long want = (n + 255) / 256;
  const int blocks = (int)(want < 8LL * nsm ? want : 8LL * nsm);
  k_paint3d<<<blocks, 256, 0, (cudaStream_t)stream>>>(nx, ny, nz, regions, nreg, table_ca,
                                                       table_cb, nmat, ca, cb, status);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "launch k_paint3d");
  return WF_OK;
}
