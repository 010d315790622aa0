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


// ---------------------------------------------------------------------------
// AntennaRing.compute_das_image (src/datasets/brain/antenna.py:216-341).
// Travel times: one thread per (antenna, pixel row, pixel column), float64 ops
// in the reference's order (x**2 is x*x; Python max(0.0, v) keeps v only when
// v > 0.0, min(L, v) keeps v only when v < L), stored as float32 like the
// reference's float32 table.  Image: one thread per pixel, tx-major/rx-minor
// float64 accumulation of envelope samples at rint(tt[tx] + tt[rx]) (float32
// add, half-to-even), then the float64 square rounded to float32.
// ---------------------------------------------------------------------------
constexpr int kMaxLayers = 16;

struct Layers {
  int n;
  double r[kMaxLayers], eps[kMaxLayers];
};

__device__ __forceinline__ double pymax0(double v) { return v > 0.0 ? v : 0.0; }
__device__ __forceinline__ double pymin(double a, double v) { return v < a ? v : a; }

__device__ double ray_chord(double ax, double ay, double bx, double by, double cx, double cy,
                            double r) {
  const double dx_ = __dsub_rn(bx, ax), dy_ = __dsub_rn(by, ay);
  const double seg = __dadd_rn(__dsqrt_rn(__dadd_rn(__dmul_rn(dx_, dx_), __dmul_rn(dy_, dy_))), 1e-30);
  const double ux = __ddiv_rn(dx_, seg), uy = __ddiv_rn(dy_, seg);
  const double ox = __dsub_rn(ax, cx), oy = __dsub_rn(ay, cy);
  const double b = __dadd_rn(__dmul_rn(ox, ux), __dmul_rn(oy, uy));
  const double c = __dsub_rn(__dadd_rn(__dmul_rn(ox, ox), __dmul_rn(oy, oy)), __dmul_rn(r, r));
  const double disc = __dsub_rn(__dmul_rn(b, b), c);
  if (disc <= 0.0) return 0.0;
  const double sq = __dsqrt_rn(disc);
  const double t0 = pymax0(pymin(seg, __dsub_rn(-b, sq)));
  const double t1 = pymax0(pymin(seg, __dadd_rn(-b, sq)));
  return pymax0(__dsub_rn(t1, t0));
}

__global__ void k_das_tt(int nant, const double* __restrict__ ax, const double* __restrict__ ay,
                         const double* __restrict__ px, int nxi, const double* __restrict__ py,
                         int nyi, double cx, double cy, Layers L, double dt,
                         float* __restrict__ tt) {
  const long long total = (long long)nant * nyi * nxi;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const int a = (int)(q / ((long long)nyi * nxi));
    const int rem = (int)(q - (long long)a * nyi * nxi);
    const int iy = rem / nxi, ix = rem - iy * nxi;
    const double x0 = ax[a], y0 = ay[a], bx = px[ix], by = py[iy];
    const double C0 = 3e8;
    double t;
    if (L.n == 0) {
      const double u = __dsub_rn(bx, x0), v = __dsub_rn(by, y0);
      const double d = __dsqrt_rn(__dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v)));
      t = __ddiv_rn(__ddiv_rn(__dmul_rn(d, 1e-3), C0), dt);
    } else {
      const double u = __dsub_rn(bx, x0), v = __dsub_rn(by, y0);
      const double total_d = __dadd_rn(__dsqrt_rn(__dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v))), 1e-30);
      double prev = 0.0, acc = 0.0;
      for (int l = 0; l < L.n; ++l) {
        const double co = ray_chord(x0, y0, bx, by, cx, cy, L.r[l]);
        const double ci = l + 1 < L.n ? ray_chord(x0, y0, bx, by, cx, cy, L.r[l + 1]) : 0.0;
        const double sc = pymax0(__dsub_rn(co, ci));
        acc = __dadd_rn(acc, __ddiv_rn(__dmul_rn(sc, 1e-3), __ddiv_rn(C0, __dsqrt_rn(L.eps[l]))));
        prev = __dadd_rn(prev, sc);
      }
      acc = __dadd_rn(acc, __ddiv_rn(__dmul_rn(pymax0(__dsub_rn(total_d, prev)), 1e-3), C0));
      t = __ddiv_rn(acc, dt);
    }
    tt[q] = __double2float_rn(t);
  }
}

__global__ void k_das_env_image(const float* __restrict__ env, int nant, int n_steps,
                                const float* __restrict__ tt, int npix,
                                float* __restrict__ image) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int tx = 0; tx < nant; ++tx) {
      const float ttx = tt[(long long)tx * npix + p];
      for (int rx = 0; rx < nant; ++rx) {
        const float s = rintf(__fadd_rn(ttx, tt[(long long)rx * npix + p]));
        if (s >= 0.f && s < (float)n_steps)
          acc = __dadd_rn(acc, (double)env[((long long)tx * nant + rx) * n_steps + (int)s]);
      }
    }
    image[p] = __double2float_rn(__dmul_rn(acc, acc));
  }
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

extern "C" int32_t wf_das_travel_times(int32_t nant, const double* ant_x_mm, const double* ant_y_mm,
                                       const double* px_mm, int32_t nxi, const double* py_mm,
                                       int32_t nyi, double cx_mm, double cy_mm,
                                       const double* layer_r_mm, const double* layer_eps,
                                       int32_t nlayer, double dt, float* tt, void* stream) {
  if (nant < 1 || nxi < 1 || nyi < 1 || ant_x_mm == nullptr || ant_y_mm == nullptr ||
      px_mm == nullptr || py_mm == nullptr || tt == nullptr || !(dt > 0.0))
    return set_error(WF_E_ARG, "wf_das_travel_times: bad sizes, null pointers or dt <= 0");
  if (nlayer < 0 || nlayer > kMaxLayers || (nlayer > 0 && (layer_r_mm == nullptr || layer_eps == nullptr)))
    return set_error(WF_E_LIMIT, "wf_das_travel_times: 0..%d layers (host arrays)", kMaxLayers);
  Layers L{};
  L.n = nlayer;
  for (int l = 0; l < nlayer; ++l) {
    L.r[l] = layer_r_mm[l];
    L.eps[l] = layer_eps[l];
  }
  const long long total = (long long)nant * nyi * nxi;
  const int blocks = (int)((total + 255) / 256 < 4096 ? (total + 255) / 256 : 4096);
  k_das_tt<<<blocks, 256, 0, (cudaStream_t)stream>>>(nant, ant_x_mm, ant_y_mm, px_mm, nxi, py_mm,
                                                     nyi, cx_mm, cy_mm, L, dt, tt);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "launch k_das_tt");
  return WF_OK;
}

extern "C" int32_t wf_das_envelope_image(const float* env, int32_t nant, int32_t n_steps,
                                         const float* tt, int32_t npix, float* image,
                                         void* stream) {
  if (nant < 1 || n_steps < 1 || npix < 1 || env == nullptr || tt == nullptr || image == nullptr)
    return set_error(WF_E_ARG, "wf_das_envelope_image: bad sizes or null pointers");
  const int blocks = (npix + 127) / 128;
  k_das_env_image<<<blocks, 128, 0, (cudaStream_t)stream>>>(env, nant, n_steps, tt, npix, image);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "launch k_das_env_image");
  return WF_OK;
}
