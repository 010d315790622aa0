// das.cu -- delay-and-sum backprojection, bit-identical to the reference's
// NumPy float64 loop (examples/brain_mimo_imaging.py:211-266).
//
// One thread owns one pixel.  The per-antenna distances are evaluated once
// per pixel (the reference recomputes them per pair, with identical float64
// results), then the pair loop accumulates in the reference's tx-major,
// rx-minor order so the float64 sum rounds identically.  All float64 ops are
// the correctly rounded _rn intrinsics: no FMA contraction, IEEE sqrt/div,
// rint() is round-half-to-even like np.round.
#include "wf_common.cuh"

namespace wf {

constexpr int kDasThreads = 128;
constexpr int kDasMaxAnt = 64;

__global__ void __launch_bounds__(kDasThreads) k_das2d(
    const float* __restrict__ tr, const float* __restrict__ tr_ref, int nant, int n_steps, const double* __restrict__ ax,
    const double* __restrict__ ay, const double* __restrict__ px, int nxi,
    const double* __restrict__ py, int nyi, double v, double dt, int gate, int skip_self,
    double* __restrict__ img) {
  extern __shared__ double d[];  // [nant][kDasThreads]
  const long long p = blockIdx.x * (long long)kDasThreads + threadIdx.x;
  const bool live = p < (long long)nxi * nyi;
  const int ix = live ? (int)(p / nyi) : 0, iy = live ? (int)(p - (long long)ix * nyi) : 0;
  const double x = px[ix], y = py[iy];
  for (int a = 0; a < nant; ++a) {
    const double u = __dsub_rn(x, ax[a]), w = __dsub_rn(y, ay[a]);
    d[a * kDasThreads + threadIdx.x] = __dsqrt_rn(__dadd_rn(__dmul_rn(u, u), __dmul_rn(w, w)));
  }
  if (!live) return;
  double acc = 0.0;
  const double hi = (double)(n_steps - 1);
  for (int t = 0; t < nant; ++t) {
    const double dt_t = d[t * kDasThreads + threadIdx.x];
    const float* row = tr + (long long)t * nant * n_steps;
    const float* rrow = tr_ref ? tr_ref + (long long)t * nant * n_steps : nullptr;
    for (int r = 0; r < nant; ++r) {
      if (skip_self && r == t) continue;
      const double tau = __ddiv_rn(__dadd_rn(dt_t, d[r * kDasThreads + threadIdx.x]), v);
      double q = rint(__ddiv_rn(tau, dt));
      q = q < 0.0 ? 0.0 : (q > hi ? hi : q);
      const int n = (int)q;
      if (n < gate) continue;  // gated samples are exact zeros
      const long long o = (long long)r * n_steps + n;
      // delta_S = S - S_ref is a float32 subtraction in the reference
      const float sample = rrow ? __fsub_rn(row[o], rrow[o]) : row[o];
      acc = __dadd_rn(acc, (double)sample);
    }
  }
  img[p] = __dmul_rn(acc, acc);
}

}  // namespace wf

using namespace wf;

extern "C" int32_t wf_das2d(const float* traces, const float* traces_ref, int32_t nant, int32_t n_steps,
                            const double* ant_x, const double* ant_y, const double* px,
                            int32_t nxi, const double* py, int32_t nyi, double v_medium,
                            double dt, int32_t gate_start, int32_t skip_self, double* image,
                            void* stream) {
  if (traces == nullptr || ant_x == nullptr || ant_y == nullptr || px == nullptr ||
      py == nullptr || image == nullptr)
    return set_error(WF_E_ARG, "wf_das2d: null pointer");
  if (nant < 1 || n_steps < 1 || nxi < 1 || nyi < 1)
    return set_error(WF_E_ARG, "wf_das2d: bad sizes nant=%d n_steps=%d image=%dx%d", nant,
                     n_steps, nxi, nyi);
  if (nant > kDasMaxAnt)
    return set_error(WF_E_LIMIT, "wf_das2d: at most %d antennas (got %d)", kDasMaxAnt, nant);
  if (!(v_medium > 0.0) || !(dt > 0.0))
    return set_error(WF_E_ARG, "wf_das2d: v_medium and dt must be > 0");
  const long long npx = (long long)nxi * nyi;
  const unsigned blocks = (unsigned)((npx + kDasThreads - 1) / kDasThreads);
  const size_t smem = (size_t)nant * kDasThreads * sizeof(double);
  cudaError_t e = cudaFuncSetAttribute(k_das2d, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(k_das2d)");
  k_das2d<<<blocks, kDasThreads, smem, (cudaStream_t)stream>>>(traces, traces_ref, nant, n_steps, ant_x, ant_y,
                                                            px, nxi, py, nyi, v_medium, dt,
                                                            gate_start, skip_self, image);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "launch k_das2d");
  return WF_OK;
}
