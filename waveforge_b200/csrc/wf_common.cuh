// wf_common.cuh -- shared helpers of the waveforge_b200 CUDA library (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "waveforge_b200.h"

namespace wf {

// ---------------------------------------------------------------------------
// Exactly rounded single-precision operations.  The reference evaluates every
// update as a sequence of separately rounded float32 PyTorch ops (a sub, a
// true division by the Python-float spacing, a multiply by the Python-float
// coefficient, an add).  Using the _rn intrinsics forbids FMA contraction and
// approximate division, so the device reproduces that sequence bit for bit.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }

// Division of a float32 x by a float32 spacing d through float64:
// q = RN32( RN64( (double)x * rd ) ) with rd = RN64(1/d).  The exact
// quotient x/d of two 24-bit-significand numbers lies either exactly on, or
// at least ~2^-48 (relative) away from, every float32 rounding midpoint (the
// numerator of the difference is a non-zero integer multiple of the midpoint
// spacing over d); for d not a power of two it is never exactly on one.  The
// float64 product is within ~2^-52 of x/d, so its rounding to float32 equals
// the correctly rounded IEEE quotient for every x, including subnormals,
// zeros of either sign, infinities and NaN (the argument behind "innocuous"
// double rounding, S. A. Figueroa 1995; J.-M. Muller et al., "Handbook of
// Floating-Point Arithmetic", ch. on double rounding).  Because the engines'
// bit-exactness rests on it, wf_check_fastdiv still compares it with
// __fdiv_rn on all 2^32 inputs for each spacing before it is enabled.
__device__ __forceinline__ float div_fast(float x, double rd) {
  return __double2float_rn(__dmul_rn((double)x, rd));
}

// |x| as ordered bits: for non-negative floats the unsigned bit pattern is
// monotone in the value, and NaN (0x7fc00000..) sorts above +inf, so a NaN
// field shows up as "above any threshold" in the stability check.
__device__ __forceinline__ unsigned abs_bits(float x) {
  return __float_as_uint(x) & 0x7fffffffu;
}

// Pass schedule of a temporally blocked run: nsteps split into passes of at
// most K steps.  When the plain count is odd the first pass is split in two so
// the ping-pong ends in the caller's state buffers (no copy-back); only a run
// made of single-step passes of odd length needs a final copy.
struct PassPlan {
  int nsteps, K, P0, split, a;
  __host__ __device__ PassPlan(int nsteps_, int K_) : nsteps(nsteps_), K(K_) {
    P0 = (nsteps + K - 1) / K;
    const int L0 = nsteps < K ? nsteps : K;
    split = ((P0 & 1) && L0 >= 2) ? 1 : 0;
    a = L0 / 2;
  }
  __host__ __device__ int passes() const { return P0 + split; }
  __host__ __device__ int unsplit_len(int q) const {
    return q < P0 - 1 ? K : nsteps - K * (P0 - 1);
  }
  __host__ __device__ int len(int p) const {
    if (!split) return unsplit_len(p);
    if (p == 0) return a;
    if (p == 1) return unsplit_len(0) - a;
    return unsplit_len(p - 1);
  }
  __host__ __device__ int offset(int p) const {
    if (!split) return p * K;
    if (p == 0) return 0;
    if (p == 1) return a;
    return (p - 1) * K;
  }
  __host__ __device__ bool needs_copy() const { return (passes() & 1) != 0; }
};

// Host-side error plumbing (thread-local message, see capi.cu).
int set_error(int code, const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what);

}  // namespace wf
