// fastdiv.cu -- exhaustive check that div_fast(x, RN64(1/d)) equals the IEEE
// quotient __fdiv_rn(x, d) for every float32 bit pattern x (NaN inputs only
// need to give NaN).  The engines use the fast division for a spacing d only
// after this check reported zero mismatches for that d.
#include "wf_common.cuh"

namespace wf {

__global__ void k_check_fastdiv(float d, unsigned* mismatches) {
  const double r = __drcp_rn((double)d);
  unsigned bad = 0;
  const unsigned long long total = 1ULL << 32;
  for (unsigned long long u = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; u < total;
       u += (unsigned long long)gridDim.x * blockDim.x) {
    const float x = __uint_as_float((unsigned)u);
    const float a = __fdiv_rn(x, d);
    const float b = div_fast(x, r);
    const bool both_nan = (a != a) && (b != b);
    bad += (!both_nan && __float_as_uint(a) != __float_as_uint(b)) ? 1u : 0u;
  }
  for (int s = 16; s > 0; s >>= 1) bad += __shfl_xor_sync(0xffffffffu, bad, s);
  if ((threadIdx.x & 31) == 0 && bad) atomicAdd(mismatches, bad);
}

}  // namespace wf

using namespace wf;

extern "C" int32_t wf_check_fastdiv(float d, uint32_t* mismatches, void* stream) {
  if (mismatches == nullptr) return set_error(WF_E_ARG, "wf_check_fastdiv: null counter");
  if (!(d > 0.f) || d != d || __builtin_isinf(d))
    return set_error(WF_E_ARG, "wf_check_fastdiv: divisor must be positive and finite");
  int dev = 0, nsm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
  k_check_fastdiv<<<nsm * 8, 256, 0, (cudaStream_t)stream>>>(d, mismatches);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "launch k_check_fastdiv");
  return WF_OK;
}
