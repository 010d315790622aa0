// adjoint2d.cu -- reverse-mode (adjoint, time-reversed Yee) step of the 2D TM
// update, and the material-coefficient kernels of the differentiable misfit.
//
// The reference has no adjoint (its design exists only as a document,
// docs/architecture/DIFFERENTIABLE_PHYSICS.md); the forward it differentiates
// is the step of src/core/fdtd2d.py:187-266 with the Mur edges of
// src/core/boundaries.py:237-274 and the lossy coefficients of
// src/core/materials.py:61-82.  One forward step n maps x_n = (Ex, Ey, Hz) to
// x_{n+1}:
//   hp = Hz;  Hz += s_n (soft source)
//   Hc = Hz + Dh*((Ex[i,j+1]-Ex[i,j])/dy - (Ey[i+1,j]-Ey[i,j])/dx)   (i<Nx-1, j<Ny-1)
//   Hx = Mur-x(Hc, hp)      rows 0 and Nx-1 replaced
//   H' = Mur-y(Hx, hp)      columns 0 and Ny-1 replaced (corners see Hx)
//   Ex'[i,j] = Ca Ex + Cb (H'[i,j]-H'[i,j-1])/dy   (j>=1)
//   Ey'[i,j] = Ca Ey - Cb (H'[i,j]-H'[i-1,j])/dx   (i>=1)
// Traces record x_{n+1} at the probes.  With L = 1/2 sum (trace - target)^2
// and lambda_{n+1} = dL/dx_{n+1} (residual r_n already added at the probes),
// one reverse step is the transpose of that linear map, taken in reverse
// order (Ampere^T, Mur-y^T, Mur-x^T, Faraday^T, snapshot^T), plus the
// parameter terms
//   dL/dCa[i,j] += aEx'[i,j] Ex^n[i,j] (j>=1) + aEy'[i,j] Ey^n[i,j] (i>=1)
//   dL/dCb[i,j] += aEx'[i,j] dyH'[i,j] (j>=1) - aEy'[i,j] dxH'[i,j] (i>=1)
// which need E^n and H^{n+1} of the forward run (recomputed per checkpoint
// segment by wf_fdtd2d_states).
//
// k_adj2d_step: one CTA produces a TI x TJ tile of lambda_n from a region of
// lambda_{n+1} with a 3-cell halo staged in shared memory; the chain
// aHy -> aHx -> aHc needs radius 3.  blockIdx.y selects one of several
// transmitter runs that share the grid and coefficients, so one launch per
// reverse step covers all of them.  Gradient accumulators are float64, one
// plane pair per run (one read-modify-write per cell and step by its owning
// thread); wf_material_grad sums them in run order, so the result does not
// depend on how runs are grouped into launches.
#include "wf_common.cuh"

namespace wf {

constexpr int kAdjHalo = 3;
constexpr int kAdjTI = 26, kAdjTJ = 58;
constexpr int kAdjRI = kAdjTI + 2 * kAdjHalo, kAdjRJ = kAdjTJ + 2 * kAdjHalo;  // 32 x 64
constexpr int kAdjThreads = 256;

struct Adj2D {
  int nx, ny;
  float dh, de, rdx, rdy, mx, my;
  const float *ex_n, *ey_n, *hz_n1;  // forward E^n and H^{n+1}
  const float *ca, *cb;              // NULL = vacuum (scalar De) path
  const float *lin[3];               // lambda_{n+1}: aEx, aEy, aHz
  float* lout[3];                    // lambda_n
  const wf_probe* prb;
  int nprb;
  const float* resid;                // resid[p * resid_ld + col], col = step n
  long long resid_ld;
  int col;
  double *gca, *gcb;                 // accumulated dL/dCa, dL/dCb (MAT only)
  // per-run strides (blockIdx.y = run): states, adjoint planes, residual rows,
  // accumulator planes
  long long st_stride, lam_stride, resid_stride, g_stride;
};

template <bool MAT>
__global__ void __launch_bounds__(kAdjThreads) k_adj2d_step(Adj2D A, int tiles_j) {
  __shared__ float sEx[kAdjRI][kAdjRJ];  // aEx' (+ residual)
  __shared__ float sEy[kAdjRI][kAdjRJ];  // aEy' (+ residual)
  __shared__ float sH[kAdjRI][kAdjRJ];   // aH' (+ residual), later aHx
  __shared__ float sB[kAdjRI][kAdjRJ];   // Cb (or De), later aHc
  __shared__ float sY[kAdjRI][kAdjRJ];   // aHy
  const int nx = A.nx, ny = A.ny;
  {
    // this CTA's transmitter run
    const long long r = blockIdx.y;
    A.ex_n += r * A.st_stride;
    A.ey_n += r * A.st_stride;
    A.hz_n1 += r * A.st_stride;
    for (int c = 0; c < 3; ++c) {
      A.lin[c] += r * A.lam_stride;
      A.lout[c] += r * A.lam_stride;
    }
    A.resid += r * A.resid_stride;
    if (MAT) {
      A.gca += r * A.g_stride;
      A.gcb += r * A.g_stride;
    }
  }
  const int bi = blockIdx.x / tiles_j, bj = blockIdx.x - bi * tiles_j;
  const int i0 = bi * kAdjTI - kAdjHalo, j0 = bj * kAdjTJ - kAdjHalo;  // region origin
  const int tid = threadIdx.x;
  constexpr int RN = kAdjRI * kAdjRJ;
  auto inside = [&](int i, int j) { return i >= 0 && i < nx && j >= 0 && j < ny; };

  // ---- phase 0: stage lambda_{n+1} and Cb over the region ------------------
  for (int q = tid; q < RN; q += kAdjThreads) {
    const int r = q / kAdjRJ, c = q - r * kAdjRJ;
    const int i = i0 + r, j = j0 + c;
    float ax = 0.f, ay = 0.f, ah = 0.f, b = 0.f;
    if (inside(i, j)) {
      // read-only for the whole launch: non-coherent loads the compiler may
      // issue together
      const long long g = (long long)i * ny + j;
      ax = __ldg(&A.lin[0][g]);
      ay = __ldg(&A.lin[1][g]);
      ah = __ldg(&A.lin[2][g]);
      b = MAT ? __ldg(&A.cb[g]) : A.de;
    }
    sEx[r][c] = ax;
    sEy[r][c] = ay;
    sH[r][c] = ah;
    sB[r][c] = b;
  }
  __syncthreads();
  // residual r_n of the traces recorded after this step, at the probes
  for (int p = tid; p < A.nprb; p += kAdjThreads) {
    const wf_probe pr = A.prb[p];
    const int r = pr.i - i0, c = pr.j - j0;
    if (r >= 0 && r < kAdjRI && c >= 0 && c < kAdjRJ) {
      const float v = A.resid[(long long)p * A.resid_ld + A.col];
      if (pr.comp == WF_EX) atomicAdd(&sEx[r][c], v);
      else if (pr.comp == WF_EY) atomicAdd(&sEy[r][c], v);
      else if (pr.comp == WF_HZ) atomicAdd(&sH[r][c], v);
    }
  }
  __syncthreads();

  // ---- phase 1: adjoint of H' through the Ampere update ----------------------
  // qx = Cb aEx' on columns 1..Ny-1, qy = Cb aEy' on rows 1..Nx-1
  auto qx = [&](int r, int c) -> float {
    const int i = i0 + r, j = j0 + c;
    return (i >= 0 && i < nx && j >= 1 && j < ny) ? sB[r][c] * sEx[r][c] : 0.f;
  };
  auto qy = [&](int r, int c) -> float {
    const int i = i0 + r, j = j0 + c;
    return (i >= 1 && i < nx && j >= 0 && j < ny) ? sB[r][c] * sEy[r][c] : 0.f;
  };
  for (int q = tid; q < RN; q += kAdjThreads) {
    const int r = q / kAdjRJ, c = q - r * kAdjRJ;
    float y = 0.f;
    if (r + 1 < kAdjRI && c + 1 < kAdjRJ && inside(i0 + r, j0 + c))
      y = sH[r][c] + (qx(r, c) - qx(r, c + 1)) * A.rdy + (qy(r + 1, c) - qy(r, c)) * A.rdx;
    sY[r][c] = y;
  }
  __syncthreads();

  // ---- phase 2: Mur-y transpose -> adjoint of Hx (into sH) -------------------
  for (int q = tid; q < RN; q += kAdjThreads) {
    const int r = q / kAdjRJ, c = q - r * kAdjRJ;
    const int i = i0 + r, j = j0 + c;
    float x = 0.f;
    if (c >= 1 && c + 1 < kAdjRJ && inside(i, j) && j != 0 && j != ny - 1) {
      x = sY[r][c];
      if (j == 1) x += A.my * sY[r][c - 1];
      if (j == ny - 2) x += A.my * sY[r][c + 1];
    }
    sH[r][c] = x;
  }
  __syncthreads();

  // ---- phase 3: Mur-x transpose -> adjoint of Hc (into sB) -------------------
  for (int q = tid; q < RN; q += kAdjThreads) {
    const int r = q / kAdjRJ, c = q - r * kAdjRJ;
    const int i = i0 + r, j = j0 + c;
    float h = 0.f;
    if (r >= 1 && r + 1 < kAdjRI && inside(i, j) && i != 0 && i != nx - 1) {
      h = sH[r][c];
      if (i == 1) h += A.mx * sH[r - 1][c];
      if (i == nx - 2) h += A.mx * sH[r + 1][c];
    }
    sB[r][c] = h;
  }
  __syncthreads();

  // ---- phase 4: Faraday transpose, snapshot transpose, outputs --------------
  // p = Dh * aHc on the curl-updated cells (i<Nx-1, j<Ny-1)
  auto pf = [&](int r, int c) -> float {
    const int i = i0 + r, j = j0 + c;
    return (i >= 0 && i < nx - 1 && j >= 0 && j < ny - 1) ? A.dh * sB[r][c] : 0.f;
  };
#pragma unroll 2
  for (int q = tid; q < kAdjTI * kAdjTJ; q += kAdjThreads) {
    const int rr = q / kAdjTJ, cc = q - rr * kAdjTJ;
    const int r = rr + kAdjHalo, c = cc + kAdjHalo;
    const int i = i0 + r, j = j0 + c;
    if (!inside(i, j)) continue;
    const long long g = (long long)i * ny + j;
    // every global input of the cell first (the stores below could alias
    // plain loads issued after them); the accumulators belong to this cell only
    const float ca = MAT ? __ldg(&A.ca[g]) : 1.f;
    float h = 0.f, hjm = 0.f, him = 0.f, exn = 0.f, eyn = 0.f;
    double gca0 = 0.0, gcb0 = 0.0;
    if (MAT) {
      h = __ldg(&A.hz_n1[g]);
      if (j >= 1) {
        hjm = __ldg(&A.hz_n1[g - 1]);
        exn = __ldg(&A.ex_n[g]);
      }
      if (i >= 1) {
        him = __ldg(&A.hz_n1[g - ny]);
        eyn = __ldg(&A.ey_n[g]);
      }
      gca0 = A.gca[g];
      gcb0 = A.gcb[g];
    }
    // adjoint of the Mur snapshot hp (pre-injection Hz)
    float ahp = 0.f;
    if (j == 1) ahp += sY[r][c - 1];
    if (j == 0) ahp -= A.my * sY[r][c];
    if (j == ny - 2) ahp += sY[r][c + 1];
    if (j == ny - 1) ahp -= A.my * sY[r][c];
    if (i == 1) ahp += sH[r - 1][c];
    if (i == 0) ahp -= A.mx * sH[r][c];
    if (i == nx - 2) ahp += sH[r + 1][c];
    if (i == nx - 1) ahp -= A.mx * sH[r][c];
    const float aex1 = sEx[r][c], aey1 = sEy[r][c];
    const float aex = (j >= 1 ? ca * aex1 : aex1) + (pf(r, c - 1) - pf(r, c)) * A.rdy;
    const float aey = (i >= 1 ? ca * aey1 : aey1) + (pf(r, c) - pf(r - 1, c)) * A.rdx;
    A.lout[0][g] = aex;
    A.lout[1][g] = aey;
    A.lout[2][g] = sB[r][c] + ahp;
    if (MAT) {
      double gca = 0.0, gcb = 0.0;
      if (j >= 1) {
        gca += (double)aex1 * (double)exn;
        gcb += (double)aex1 * ((double)(h - hjm) * (double)A.rdy);
      }
      if (i >= 1) {
        gca += (double)aey1 * (double)eyn;
        gcb -= (double)aey1 * ((double)(h - him) * (double)A.rdx);
      }
      A.gca[g] = gca0 + gca;
      A.gcb[g] = gcb0 + gcb;
    }
  }
}

__global__ void k_copy3f(const float* __restrict__ s, float* __restrict__ d, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    d[i] = s[i];
}

// Ca/Cb from per-cell eps_r, sigma exactly as src/core/materials.py:61-82
// evaluates them in Python float64, then rounded to float32 like the
// float32 tensors of MaterialMap.build (:200-252).
constexpr double kEps0 = 8.8541878128e-12;

__global__ void k_material_coeffs(const double* __restrict__ eps, const double* __restrict__ sig,
                                  long long n, double dt, float* __restrict__ ca,
                                  float* __restrict__ cb) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const double e = eps[q], s = sig[q];
    const double alpha = __ddiv_rn(__dmul_rn(s, dt), __dmul_rn(__dmul_rn(2.0, kEps0), e));
    const double opa = __dadd_rn(1.0, alpha);
    ca[q] = __double2float_rn(__ddiv_rn(__dsub_rn(1.0, alpha), opa));
    cb[q] = __double2float_rn(__ddiv_rn(__ddiv_rn(dt, __dmul_rn(kEps0, e)), opa));
  }
}

// Chain rule from dL/dCa, dL/dCb to dL/deps_r, dL/dsigma (float64), scaled.
// With D = eps_r (1 + alpha) = eps_r + sigma dt / (2 eps0):
//   dCa/dalpha = -2 / (1+alpha)^2,  dalpha/deps = -alpha/eps,
//   dalpha/dsigma = dt / (2 eps0 eps),  dCb/deps = -(dt/eps0) / D^2,
//   dCb/dsigma = -(dt/eps0) / D^2 * dt / (2 eps0).
__global__ void k_material_grad(const double* __restrict__ eps, const double* __restrict__ sig,
                                long long n, double dt, const double* __restrict__ gca,
                                const double* __restrict__ gcb, int count, double scale,
                                double* __restrict__ geps, double* __restrict__ gsig) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    // sum of the per-run accumulators, always in run order
    double ga = gca[q], gb = gcb[q];
    for (int c = 1; c < count; ++c) {
      ga += gca[c * n + q];
      gb += gcb[c * n + q];
    }
    const double e = eps[q], s = sig[q];
    const double k = dt / (2.0 * kEps0);
    const double alpha = s * k / e;
    const double opa = 1.0 + alpha;
    const double dca_da = -2.0 / (opa * opa);
    const double D = e + s * k;
    const double dcb_dD = -(dt / kEps0) / (D * D);
    geps[q] = scale * (ga * dca_da * (-alpha / e) + gb * dcb_dD);
    gsig[q] = scale * (ga * dca_da * (k / e) + gb * dcb_dD * k);
  }
}

}  // namespace wf

using namespace wf;

extern "C" int32_t wf_adjoint2d_run(const wf_grid2d* g, const float* states, int64_t states_stride,
                                    int32_t ntx, int32_t nsteps, const float* ca, const float* cb,
                                    const wf_probe* probes, int32_t nprobe, const float* resid,
                                    int64_t resid_ld, int64_t resid_stride, int32_t resid_step0,
                                    int32_t step0, float* lam, float* lam_scratch, double* g_ca,
                                    double* g_cb, void* stream) {
  if (g == nullptr || states == nullptr || lam == nullptr || lam_scratch == nullptr)
    return set_error(WF_E_ARG, "wf_adjoint2d_run: null grid/states/adjoint pointer");
  if (g->nx < 4 || g->ny < 4)
    return set_error(WF_E_ARG, "wf_adjoint2d_run: grid %dx%d below the 4x4 stencil minimum",
                     g->nx, g->ny);
  if ((ca == nullptr) != (cb == nullptr))
    return set_error(WF_E_ARG, "wf_adjoint2d_run: Ca and Cb must be given together");
  if (ca != nullptr && (g_ca == nullptr || g_cb == nullptr))
    return set_error(WF_E_ARG, "wf_adjoint2d_run: gradient accumulators required with Ca/Cb");
  const long long cells = (long long)g->nx * g->ny;
  if (nsteps < 0 || step0 < 0 || nprobe < 0 || ntx < 1 || ntx > 65535 ||
      (nprobe > 0 && (probes == nullptr || resid == nullptr)) ||
      (ntx > 1 && states_stride < (long long)(nsteps + 1) * 3 * cells))
    return set_error(WF_E_ARG, "wf_adjoint2d_run: bad counts, stride or null probe/residual arrays");
  if (nprobe > 0 && step0 < resid_step0)
    return set_error(WF_E_ARG, "wf_adjoint2d_run: step0 %d precedes the residual's first step %d",
                     step0, resid_step0);
  if (nsteps == 0) return WF_OK;
  cudaStream_t st = (cudaStream_t)stream;
  Adj2D A{};
  A.nx = g->nx;
  A.ny = g->ny;
  A.dh = g->dh;
  A.de = g->de;
  A.rdx = 1.0f / g->dx;
  A.rdy = 1.0f / g->dy;
  A.mx = g->mur_x;
  A.my = g->mur_y;
  A.ca = ca;
  A.cb = cb;
  A.prb = probes;
  A.nprb = nprobe;
  A.resid = resid;
  A.resid_ld = resid_ld;
  A.gca = g_ca;
  A.gcb = g_cb;
  A.st_stride = states_stride;
  A.lam_stride = 3 * cells;
  A.resid_stride = resid_stride;
  A.g_stride = cells;
  const int tiles_i = (g->nx + kAdjTI - 1) / kAdjTI, tiles_j = (g->ny + kAdjTJ - 1) / kAdjTJ;
  float* L[2] = {lam, lam_scratch};
  for (int t = nsteps - 1, p = 0; t >= 0; --t, ++p) {
    const float* x_n = states + (long long)t * 3 * cells;
    const float* x_n1 = states + (long long)(t + 1) * 3 * cells;
    A.ex_n = x_n;
    A.ey_n = x_n + cells;
    A.hz_n1 = x_n1 + 2 * cells;
    float* in = L[p & 1];
    float* out = L[(p + 1) & 1];
    for (int c = 0; c < 3; ++c) {
      A.lin[c] = in + c * cells;
      A.lout[c] = out + c * cells;
    }
    A.col = step0 + t - resid_step0;
    dim3 grid(tiles_i * tiles_j, ntx);
    if (ca) k_adj2d_step<true><<<grid, kAdjThreads, 0, st>>>(A, tiles_j);
    else k_adj2d_step<false><<<grid, kAdjThreads, 0, st>>>(A, tiles_j);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "launch k_adj2d_step");
  }
  if (nsteps & 1) {
    k_copy3f<<<296, 256, 0, st>>>(lam_scratch, lam, 3 * cells * ntx);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "launch k_copy3f");
  }
  return WF_OK;
}

extern "C" int32_t wf_material_coeffs(const double* eps_r, const double* sigma, int64_t n,
                                      double dt, float* ca, float* cb, void* stream) {
  if (n < 0 || (n > 0 && (eps_r == nullptr || sigma == nullptr || ca == nullptr || cb == nullptr)))
    return set_error(WF_E_ARG, "wf_material_coeffs: null pointer or negative size");
  if (!(dt > 0.0)) return set_error(WF_E_ARG, "wf_material_coeffs: dt must be positive");
  if (n == 0) return WF_OK;
  k_material_coeffs<<<592, 256, 0, (cudaStream_t)stream>>>(eps_r, sigma, n, dt, ca, cb);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "launch k_material_coeffs");
  return WF_OK;
}

extern "C" int32_t wf_material_grad(const double* eps_r, const double* sigma, int64_t n,
                                    double dt, const double* g_ca, const double* g_cb,
                                    int32_t count, double scale, double* g_eps, double* g_sigma,
                                    void* stream) {
  if (n < 0 || count < 1 || (n > 0 && (eps_r == nullptr || sigma == nullptr || g_ca == nullptr ||
                                       g_cb == nullptr || g_eps == nullptr || g_sigma == nullptr)))
    return set_error(WF_E_ARG, "wf_material_grad: null pointer, negative size or count < 1");
  if (!(dt > 0.0)) return set_error(WF_E_ARG, "wf_material_grad: dt must be positive");
  if (n == 0) return WF_OK;
  k_material_grad<<<592, 256, 0, (cudaStream_t)stream>>>(eps_r, sigma, n, dt, g_ca, g_cb, count,
                                                         scale, g_eps, g_sigma);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "launch k_material_grad");
  return WF_OK;
}
