// fdtd3d.cu -- 3D six-component Yee kernel and the wf_fdtd3d_run entry point.
//
// Same scheme as the 2D tile routine: one CTA advances one (i,j,k) tile by k
// time steps in shared memory from a halo-extended copy, H is double-buffered
// (a = previous step = Mur snapshot, b = new), E is updated in place.  Per
// step, in the reference order (src/core/fdtd3d.py:261-402):
//   E-component soft injection; Faraday updates of Hx (j<Ny-1,k<Nz-1),
//   Hy (i<Nx-1,k<Nz-1), Hz (i<Nx-1,j<Ny-1) with H-component injection folded
//   in; Mur on the tangential H of each face, x faces (Hy,Hz) then y faces
//   (Hx,Hz) then z faces (Hx,Hy, only when Nz>1) (boundaries.py:499-583),
//   evaluated as pure functions of pre-step and curl-updated H; Ampere
//   updates of Ex (j,k>=1), Ey (i,k>=1), Ez (i,j>=1); detectors; maxima.
#include <algorithm>

#include "wf_common.cuh"

namespace wf {

constexpr int kMaxLocalSrc3 = 64;
constexpr int kMaxLocalProbe3 = 256;

struct Tile3D {
  int nx, ny, nz;
  float dh, de, dx, dy, dz, mx, my, mz;
  const float* in[6];
  float* out[6];
  const float *ca, *cb;
  const wf_source* src;
  int nsrc;
  const wf_probe* prb;
  int nprb;
  float* traces;
  long long trace_ld;
  int trace_step0;
  int n_check;
  unsigned* check_max;
  int check_base;
};

struct Lists3D {
  int nh, ne, np;
  short h[kMaxLocalSrc3];
  short e[kMaxLocalSrc3];
  short p[kMaxLocalProbe3];
  unsigned bmax[6];
};

__host__ __device__ inline size_t tile3d_smem(int ri, int rj, int rk, bool mat) {
  return (size_t)ri * rj * rk * (mat ? 11 : 9) * sizeof(float);
}

__device__ __forceinline__ float src3_value(const wf_source& s, int i, int j, int k, int n) {
  const float w = s.wave[n];
  if (s.amp == nullptr) return w;
  const int c = ((i - s.i0) * (s.j1 - s.j0) + (j - s.j0)) * (s.k1 - s.k0) + (k - s.k0);
  return fmul(w, s.amp[c]);
}

template <bool FDIV>
__device__ __forceinline__ float dv(float a, float d, double r) {
  return FDIV ? div_fast(a, r) : fdiv(a, d);
}

template <bool MAT, bool FDIV>
__global__ void __launch_bounds__(512, 1) k3d_pass(Tile3D P, int ti, int tj, int tk, int tiles_j,
                                                int tiles_k, int step0, int kst) {
  extern __shared__ float sm[];
  __shared__ Lists3D L;
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  int b = blockIdx.x;
  const int bk = b % tiles_k;
  b /= tiles_k;
  const int bj = b % tiles_j, bi = b / tiles_j;
  const int ci0 = bi * ti, cj0 = bj * tj, ck0 = bk * tk;
  const int ci1 = min(ci0 + ti, nx), cj1 = min(cj0 + tj, ny), ck1 = min(ck0 + tk, nz);
  const int ri0 = max(ci0 - kst, 0), ri1 = min(ci1 + kst, nx);
  const int rj0 = max(cj0 - kst, 0), rj1 = min(cj1 + kst, ny);
  const int rk0 = max(ck0 - kst, 0), rk1 = min(ck1 + kst, nz);
  const int RI = ri1 - ri0, RJ = rj1 - rj0, RK = rk1 - rk0;
  const int RN = RI * RJ * RK, SJ = RK, SI = RJ * RK;
  float* E[3] = {sm, sm + RN, sm + 2 * RN};
  float* Ha[3] = {sm + 3 * RN, sm + 4 * RN, sm + 5 * RN};
  float* Hb[3] = {sm + 6 * RN, sm + 7 * RN, sm + 8 * RN};
  float* ca = sm + 9 * RN;
  float* cb = sm + 10 * RN;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  const float dh = P.dh, de = P.de, dx = P.dx, dy = P.dy, dz = P.dz;
  const float mx = P.mx, my = P.my, mz = P.mz;
  const double rdx = __drcp_rn((double)dx), rdy = __drcp_rn((double)dy),
               rdz = __drcp_rn((double)dz);

  if (tid == 0) {
    int nh = 0, ne = 0;
    for (int s = 0; s < P.nsrc; ++s) {
      const wf_source& S = P.src[s];
      if (S.i1 <= ri0 || S.i0 >= ri1 || S.j1 <= rj0 || S.j0 >= rj1 || S.k1 <= rk0 || S.k0 >= rk1)
        continue;
      if (S.comp >= WF_HX) {
        if (nh < kMaxLocalSrc3) L.h[nh++] = (short)s;
      } else {
        if (ne < kMaxLocalSrc3) L.e[ne++] = (short)s;
      }
    }
    L.nh = nh;
    L.ne = ne;
    L.np = 0;
    for (int c = 0; c < 6; ++c) L.bmax[c] = 0u;
  }
  __syncthreads();
  for (int q = tid; q < P.nprb; q += blockDim.x) {
    const wf_probe& pr = P.prb[q];
    if (pr.i >= ci0 && pr.i < ci1 && pr.j >= cj0 && pr.j < cj1 && pr.k >= ck0 && pr.k < ck1) {
      const int slot = atomicAdd(&L.np, 1);
      if (slot < kMaxLocalProbe3) L.p[slot] = (short)q;
    }
  }
  // load
  for (int row = warp; row < RI * RJ; row += nw) {
    const int r = row / RJ, s = row - r * RJ;
    const long long g = ((long long)(ri0 + r) * ny + (rj0 + s)) * nz + rk0;
    for (int u = lane; u < RK; u += 32) {
      const int o = row * RK + u;
      E[0][o] = P.in[0][g + u];
      E[1][o] = P.in[1][g + u];
      E[2][o] = P.in[2][g + u];
      Ha[0][o] = P.in[3][g + u];
      Ha[1][o] = P.in[4][g + u];
      Ha[2][o] = P.in[5][g + u];
      if (MAT) {
        ca[o] = P.ca[g + u];
        cb[o] = P.cb[g + u];
      }
    }
  }
  __syncthreads();
  const int np = min(L.np, kMaxLocalProbe3), nh = L.nh, ne = L.ne;
  const bool faces = (ri0 == 0) || (ri1 == nx) || (rj0 == 0) || (rj1 == ny) ||
                     (nz > 1 && ((rk0 == 0) || (rk1 == nz)));

  for (int t = 0; t < kst; ++t) {
    const int n = step0 + t;
    if (ne > 0) {
      if (tid == 0) {
        for (int q = 0; q < ne; ++q) {
          const wf_source& S = P.src[L.e[q]];
          float* f = E[S.comp];
          for (int i = max(S.i0, ri0); i < min(S.i1, ri1); ++i)
            for (int j = max(S.j0, rj0); j < min(S.j1, rj1); ++j)
              for (int k = max(S.k0, rk0); k < min(S.k1, rk1); ++k) {
                const int o = (i - ri0) * SI + (j - rj0) * SJ + (k - rk0);
                f[o] = fadd(f[o], src3_value(S, i, j, k, n));
              }
        }
      }
      __syncthreads();
    }
    // Faraday
    for (int row = warp; row < RI * RJ; row += nw) {
      const int r = row / RJ, s = row - r * RJ;
      const int gi = ri0 + r, gj = rj0 + s;
      for (int u = lane; u < RK; u += 32) {
        const int gk = rk0 + u;
        const int o = row * RK + u;
        float vx = Ha[0][o], vy = Ha[1][o], vz = Ha[2][o];
        if (nh > 0) {
          for (int q = 0; q < nh; ++q) {
            const wf_source& S = P.src[L.h[q]];
            if (gi >= S.i0 && gi < S.i1 && gj >= S.j0 && gj < S.j1 && gk >= S.k0 && gk < S.k1) {
              const float w = src3_value(S, gi, gj, gk, n);
              if (S.comp == WF_HX) vx = fadd(vx, w);
              else if (S.comp == WF_HY) vy = fadd(vy, w);
              else vz = fadd(vz, w);
            }
          }
        }
        if (gj < ny - 1 && gk < nz - 1 && s + 1 < RJ && u + 1 < RK) {
          const float t1 = dv<FDIV>(fsub(E[1][o + 1], E[1][o]), dz, rdz);
          const float t2 = dv<FDIV>(fsub(E[2][o + SJ], E[2][o]), dy, rdy);
          vx = fadd(vx, fmul(dh, fsub(t1, t2)));
        }
        if (gi < nx - 1 && gk < nz - 1 && r + 1 < RI && u + 1 < RK) {
          const float t1 = dv<FDIV>(fsub(E[2][o + SI], E[2][o]), dx, rdx);
          const float t2 = dv<FDIV>(fsub(E[0][o + 1], E[0][o]), dz, rdz);
          vy = fadd(vy, fmul(dh, fsub(t1, t2)));
        }
        if (gi < nx - 1 && gj < ny - 1 && r + 1 < RI && s + 1 < RJ) {
          const float t1 = dv<FDIV>(fsub(E[0][o + SJ], E[0][o]), dy, rdy);
          const float t2 = dv<FDIV>(fsub(E[1][o + SI], E[1][o]), dx, rdx);
          vz = fadd(vz, fmul(dh, fsub(t1, t2)));
        }
        Hb[0][o] = vx;
        Hb[1][o] = vy;
        Hb[2][o] = vz;
      }
    }
    __syncthreads();
    // Mur faces. Reads touch only non-face H cells of the written component.
    if (faces) {
      auto xface = [&](int c, int r, int s, int u) -> float {  // after x faces
        const int gi = ri0 + r, o = s * SJ + u;
        if (gi == 0) return fadd(Ha[c][SI + o], fmul(mx, fsub(Hb[c][SI + o], Ha[c][o])));
        if (gi == nx - 1)
          return fadd(Ha[c][(RI - 2) * SI + o],
                      fmul(mx, fsub(Hb[c][(RI - 2) * SI + o], Ha[c][(RI - 1) * SI + o])));
        return Hb[c][r * SI + o];
      };
      auto yface_hx = [&](int r, int s, int u) -> float {  // Hx after y faces
        const int gj = rj0 + s, b0 = r * SI + u;
        if (gj == 0) return fadd(Ha[0][b0 + SJ], fmul(my, fsub(Hb[0][b0 + SJ], Ha[0][b0])));
        if (gj == ny - 1)
          return fadd(Ha[0][b0 + (RJ - 2) * SJ],
                      fmul(my, fsub(Hb[0][b0 + (RJ - 2) * SJ], Ha[0][b0 + (RJ - 1) * SJ])));
        return Hb[0][b0 + s * SJ];
      };
      for (int row = warp; row < RI * RJ; row += nw) {
        const int r = row / RJ, s = row - r * RJ;
        const int gi = ri0 + r, gj = rj0 + s;
        const bool xf = gi == 0 || gi == nx - 1, yf = gj == 0 || gj == ny - 1;
        for (int u = lane; u < RK; u += 32) {
          const int gk = rk0 + u;
          const bool zf = nz > 1 && (gk == 0 || gk == nz - 1);
          if (!(xf || yf || zf)) continue;
          const int o = row * RK + u, b0 = r * SI + s * SJ;
          // Hx: y faces then z faces
          if (yf || zf) {
            float v;
            if (zf) {
              if (gk == 0)
                v = fadd(Ha[0][b0 + 1], fmul(mz, fsub(yface_hx(r, s, 1), Ha[0][b0])));
              else
                v = fadd(Ha[0][b0 + RK - 2],
                         fmul(mz, fsub(yface_hx(r, s, RK - 2), Ha[0][b0 + RK - 1])));
            } else {
              v = yface_hx(r, s, u);
            }
            Hb[0][o] = v;
          }
          // Hy: x faces then z faces
          if (xf || zf) {
            float v;
            if (zf) {
              if (gk == 0)
                v = fadd(Ha[1][b0 + 1], fmul(mz, fsub(xface(1, r, s, 1), Ha[1][b0])));
              else
                v = fadd(Ha[1][b0 + RK - 2],
                         fmul(mz, fsub(xface(1, r, s, RK - 2), Ha[1][b0 + RK - 1])));
            } else {
              v = xface(1, r, s, u);
            }
            Hb[1][o] = v;
          }
          // Hz: x faces then y faces
          if (xf || yf) {
            float v;
            if (yf) {
              const int base = r * SI + u;
              if (gj == 0)
                v = fadd(Ha[2][base + SJ], fmul(my, fsub(xface(2, r, 1, u), Ha[2][base])));
              else
                v = fadd(Ha[2][base + (RJ - 2) * SJ],
                         fmul(my, fsub(xface(2, r, RJ - 2, u), Ha[2][base + (RJ - 1) * SJ])));
            } else {
              v = xface(2, r, s, u);
            }
            Hb[2][o] = v;
          }
        }
      }
      __syncthreads();
    }
    // Ampere
    for (int row = warp; row < RI * RJ; row += nw) {
      const int r = row / RJ, s = row - r * RJ;
      const int gi = ri0 + r, gj = rj0 + s;
      for (int u = lane; u < RK; u += 32) {
        const int gk = rk0 + u;
        const int o = row * RK + u;
        if (gj >= 1 && gk >= 1 && s >= 1 && u >= 1) {
          const float c = fsub(dv<FDIV>(fsub(Hb[2][o], Hb[2][o - SJ]), dy, rdy),
                               dv<FDIV>(fsub(Hb[1][o], Hb[1][o - 1]), dz, rdz));
          E[0][o] = MAT ? fadd(fmul(ca[o], E[0][o]), fmul(cb[o], c)) : fadd(E[0][o], fmul(de, c));
        }
        if (gi >= 1 && gk >= 1 && r >= 1 && u >= 1) {
          const float c = fsub(dv<FDIV>(fsub(Hb[0][o], Hb[0][o - 1]), dz, rdz),
                               dv<FDIV>(fsub(Hb[2][o], Hb[2][o - SI]), dx, rdx));
          E[1][o] = MAT ? fadd(fmul(ca[o], E[1][o]), fmul(cb[o], c)) : fadd(E[1][o], fmul(de, c));
        }
        if (gi >= 1 && gj >= 1 && r >= 1 && s >= 1) {
          const float c = fsub(dv<FDIV>(fsub(Hb[1][o], Hb[1][o - SI]), dx, rdx),
                               dv<FDIV>(fsub(Hb[0][o], Hb[0][o - SJ]), dy, rdy));
          E[2][o] = MAT ? fadd(fmul(ca[o], E[2][o]), fmul(cb[o], c)) : fadd(E[2][o], fmul(de, c));
        }
      }
    }
    __syncthreads();
    for (int q = tid; q < np; q += blockDim.x) {
      const wf_probe& pr = P.prb[L.p[q]];
      const int o = (pr.i - ri0) * SI + (pr.j - rj0) * SJ + (pr.k - rk0);
      const float v = pr.comp < 3 ? E[pr.comp][o] : Hb[pr.comp - 3][o];
      P.traces[(long long)L.p[q] * P.trace_ld + (n - P.trace_step0)] = v;
    }
    if (P.check_max != nullptr && P.n_check > 0 && (n + 1) % P.n_check == 0) {
      unsigned m[6] = {0, 0, 0, 0, 0, 0};
      for (int row = warp; row < (ci1 - ci0) * (cj1 - cj0); row += nw) {
        const int a = row / (cj1 - cj0), bb = row - a * (cj1 - cj0);
        const int base = (ci0 + a - ri0) * SI + (cj0 + bb - rj0) * SJ - rk0;
        for (int k = ck0 + lane; k < ck1; k += 32) {
          const int o = base + k;
          m[0] = max(m[0], abs_bits(E[0][o]));
          m[1] = max(m[1], abs_bits(E[1][o]));
          m[2] = max(m[2], abs_bits(E[2][o]));
          m[3] = max(m[3], abs_bits(Hb[0][o]));
          m[4] = max(m[4], abs_bits(Hb[1][o]));
          m[5] = max(m[5], abs_bits(Hb[2][o]));
        }
      }
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        for (int sh = 16; sh > 0; sh >>= 1) m[c] = max(m[c], __shfl_xor_sync(0xffffffffu, m[c], sh));
        if (lane == 0) atomicMax(&L.bmax[c], m[c]);
      }
      __syncthreads();
      if (tid < 6) {
        const int idx = (n + 1) / P.n_check - P.check_base - 1;
        atomicMax(&P.check_max[idx * 6 + tid], L.bmax[tid]);
        L.bmax[tid] = 0u;
      }
    }
    for (int c = 0; c < 3; ++c) {
      float* tmp = Ha[c];
      Ha[c] = Hb[c];
      Hb[c] = tmp;
    }
    __syncthreads();
  }
  // store core
  for (int row = warp; row < (ci1 - ci0) * (cj1 - cj0); row += nw) {
    const int a = row / (cj1 - cj0), bb = row - a * (cj1 - cj0);
    const int i = ci0 + a, j = cj0 + bb;
    const long long g = ((long long)i * ny + j) * nz;
    const int base = (i - ri0) * SI + (j - rj0) * SJ - rk0;
    for (int k = ck0 + lane; k < ck1; k += 32) {
      P.out[0][g + k] = E[0][base + k];
      P.out[1][g + k] = E[1][base + k];
      P.out[2][g + k] = E[2][base + k];
      P.out[3][g + k] = Ha[0][base + k];
      P.out[4][g + k] = Ha[1][base + k];
      P.out[5][g + k] = Ha[2][base + k];
    }
  }
}

__global__ void k_copy6(Tile3D P, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    for (int c = 0; c < 6; ++c) P.out[c][i] = P.in[c][i];
}

template <bool MAT, bool FDIV>
static int launch3(const Tile3D& P, const wf_tune& t, int s0, int k, cudaStream_t st) {
  const int ti = t.tile_i, tj = t.tile_j, tk = t.tile_k;
  const int tiles_i = (P.nx + ti - 1) / ti, tiles_j = (P.ny + tj - 1) / tj,
            tiles_k = (P.nz + tk - 1) / tk;
  const size_t smem = tile3d_smem(std::min(ti + 2 * k, P.nx), std::min(tj + 2 * k, P.ny),
                                  std::min(tk + 2 * k, P.nz), MAT);
  cudaError_t e =
      cudaFuncSetAttribute(k3d_pass<MAT, FDIV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(k3d_pass)");
  const long long nblk = (long long)tiles_i * tiles_j * tiles_k;
  if (nblk > 0x7fffffffLL) return set_error(WF_E_LIMIT, "wf_fdtd3d_run: too many tiles");
  k3d_pass<MAT, FDIV><<<(unsigned)nblk, t.threads, smem, st>>>(P, ti, tj, tk, tiles_j, tiles_k, s0, k);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "launch k3d_pass");
  return WF_OK;
}

}  // namespace wf

using namespace wf;

extern "C" int32_t wf_fdtd3d_run(const wf_grid3d* g, float* const* f, float* const* s,
                                 const float* ca, const float* cb, const wf_source* src,
                                 int32_t nsrc, const wf_probe* probes, int32_t nprobe,
                                 float* traces, int64_t trace_ld, int32_t trace_step0,
                                 int32_t step0, int32_t nsteps, int32_t n_check,
                                 uint32_t* check_max, const wf_tune* tune, void* stream) {
  if (g == nullptr || f == nullptr || s == nullptr)
    return set_error(WF_E_ARG, "wf_fdtd3d_run: null grid/state/scratch array");
  for (int c = 0; c < 6; ++c)
    if (f[c] == nullptr || s[c] == nullptr)
      return set_error(WF_E_ARG, "wf_fdtd3d_run: null field pointer %d", c);
  if (g->nx < 4 || g->ny < 4 || !(g->nz == 1 || g->nz >= 4))
    return set_error(WF_E_ARG, "wf_fdtd3d_run: grid %dx%dx%d below the stencil minimum", g->nx,
                     g->ny, g->nz);
  if ((ca == nullptr) != (cb == nullptr))
    return set_error(WF_E_ARG, "wf_fdtd3d_run: Ca and Cb must be given together");
  if (nsteps < 0 || step0 < 0 || nsrc < 0 || nprobe < 0 || (nsrc > 0 && src == nullptr) ||
      (nprobe > 0 && (probes == nullptr || traces == nullptr)))
    return set_error(WF_E_ARG, "wf_fdtd3d_run: bad counts or null descriptor arrays");
  if (nsrc > 32767 || nprobe > 32767)
    return set_error(WF_E_LIMIT, "wf_fdtd3d_run: at most 32767 sources and probes");
  if (nsteps == 0) return WF_OK;
  wf_tune t{};
  if (tune) {
    t = *tune;
  } else {
    t.steps_per_pass = 1;
    t.tile_i = 4;
    t.tile_j = 8;
    t.tile_k = 30;
    t.threads = 256;
  }
  if (t.steps_per_pass < 1 || t.steps_per_pass > 8 || t.tile_i < 2 || t.tile_j < 2 ||
      t.tile_k < 2 || t.threads < 32 || t.threads > 512 || (t.threads & 31))
    return set_error(WF_E_ARG, "wf_fdtd3d_run: bad tune");
  cudaStream_t st = (cudaStream_t)stream;
  Tile3D P{};
  P.nx = g->nx;
  P.ny = g->ny;
  P.nz = g->nz;
  P.dh = g->dh;
  P.de = g->de;
  P.dx = g->dx;
  P.dy = g->dy;
  P.dz = g->dz;
  P.mx = g->mur_x;
  P.my = g->mur_y;
  P.mz = g->mur_z;
  P.ca = ca;
  P.cb = cb;
  P.src = src;
  P.nsrc = nsrc;
  P.prb = probes;
  P.nprb = nprobe;
  P.traces = traces;
  P.trace_ld = trace_ld;
  P.trace_step0 = trace_step0;
  P.n_check = n_check;
  P.check_max = check_max;
  P.check_base = n_check > 0 ? step0 / n_check : 0;
  const int all3 = WF_FASTDIV_X | WF_FASTDIV_Y | WF_FASTDIV_Z;
  const int all2 = WF_FASTDIV_X | WF_FASTDIV_Y;
  const bool fd = g->nz > 1 ? (g->flags & all3) == all3 : (g->flags & all2) == all2;
  const PassPlan plan(nsteps, t.steps_per_pass);
  for (int p = 0; p < plan.passes(); ++p) {
    float* const* in = (p & 1) ? s : f;
    float* const* out = (p & 1) ? f : s;
    for (int c = 0; c < 6; ++c) {
      P.in[c] = in[c];
      P.out[c] = out[c];
    }
    const int s0 = step0 + plan.offset(p), k = plan.len(p);
    const int rc = ca ? (fd ? launch3<true, true>(P, t, s0, k, st) : launch3<true, false>(P, t, s0, k, st))
                      : (fd ? launch3<false, true>(P, t, s0, k, st) : launch3<false, false>(P, t, s0, k, st));
    if (rc) return rc;
  }
  if (plan.needs_copy()) {
    for (int c = 0; c < 6; ++c) {
      P.in[c] = s[c];
      P.out[c] = f[c];
    }
    k_copy6<<<592, 256, 0, st>>>(P, (long long)g->nx * g->ny * g->nz);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "launch k_copy6");
  }
  return WF_OK;
}
