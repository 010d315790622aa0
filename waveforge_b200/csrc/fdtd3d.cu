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
#include <atomic>
#include <mutex>

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
  // batched instances (blockIdx.y; streaming kernel only): element strides
  // between instances of the fields, coefficients (0 = shared) and traces
  long long fstride, cstride, tstride;
  int sstride;  // wf_source elements between instances' source lists (0 = shared)
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

// ---------------------------------------------------------------------------
// k3d_stream: one full time step as a 2.5D stream along i.
//
// A CTA owns a 16 (j) x 32 (k) block of columns -- a 14 x 30 core with a
// one-cell halo on each side -- warp w = row j, lane = column k, one column
// per thread, and walks a segment [ia, ib) of i-planes.  Each column keeps
// its values in registers: old E of planes f..f+3 (prefetched two planes
// ahead), old and curl-updated H of planes f-1..f+1.  In-plane neighbours come
// from warp shuffles (k) and small shared exchange rows (j).
// Iteration f: (A) Faraday update of plane p = f+1 (needs old E of p, p+1);
// (B) Mur faces of plane f as pure functions of old and curl-updated H --
// x faces read plane 1 (f = 0) or plane Nx-2 (f = Nx-1), then y faces read
// row j=1 / Ny-2 through shared memory, then z faces read column k=1 / Nz-2
// through shuffles (src/core/boundaries.py:499-583 order); (C) Ampere update
// of plane f (needs final H of planes f and f-1) and the stores, detectors
// and maxima of its core.  A segment starts one plane early (f0 = ia-1) to
// have the final H of plane ia-1 without storing it.  Every float op is the
// same separately rounded op, in the same order, as k3d_pass, so both
// kernels are bit-identical to the reference.
// ---------------------------------------------------------------------------
constexpr int kSK = 32, kCK = kSK - 2;

struct F3 {
  float x, y, z;
};

template <int kSJ, bool DIRECT, bool MAT, bool FDIV>
__global__ void __launch_bounds__(kSJ * kSK, 512 / (kSJ * kSK)) k3d_stream(Tile3D P, int tiles_j,
                                                                          int tiles_k,
                                                                          int seg_len, int n) {
  constexpr int kCJ = kSJ - 2;
  if (blockIdx.y) {
    // this CTA's instance of a batched launch; sources: nsrc per instance
    const long long q = blockIdx.y;
    for (int c = 0; c < 6; ++c) {
      P.in[c] += q * P.fstride;
      P.out[c] += q * P.fstride;
    }
    if (P.ca) {
      P.ca += q * P.cstride;
      P.cb += q * P.cstride;
    }
    P.traces += q * P.tstride;
    P.src += q * P.sstride;
  }
  __shared__ float sA[kSJ][kSK], sB[kSJ][kSK], sC[kSJ][kSK], sD[kSJ][kSK];
  __shared__ Lists3D L;
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  int b = blockIdx.x;
  const int tk = b % tiles_k;
  b /= tiles_k;
  const int tj = b % tiles_j, seg = b / tiles_j;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, tid = threadIdx.x;
  const int gj = tj * kCJ - 1 + w, gk = tk * kCK - 1 + lane;
  const bool in = gj >= 0 && gj < ny && gk >= 0 && gk < nz;
  const bool core = in && w >= 1 && w <= kCJ && lane >= 1 && lane <= kCK;
  const int ia = seg * seg_len, ib = min(nx, ia + seg_len);
  if (ia >= ib) return;
  const int f0 = max(ia - 1, 0);
  const long long PS = (long long)ny * nz;
  const long long col = in ? (long long)gj * nz + gk : 0;
  const float dh = P.dh, de = P.de, dx = P.dx, dy = P.dy, dz = P.dz;
  const float mx = P.mx, my = P.my, mz = P.mz;
  const double rdx = __drcp_rn((double)dx), rdy = __drcp_rn((double)dy),
               rdz = __drcp_rn((double)dz);
  const int j0 = tj * kCJ - 1, k0 = tk * kCK - 1;
  const bool yfaces = (j0 <= 0) || (j0 + kSJ >= ny);   // CTA-uniform

  // ---- local source / probe lists -----------------------------------------
  if (tid == 0) {
    int nh = 0, ne = 0;
    for (int q = 0; q < P.nsrc; ++q) {
      const wf_source& S = P.src[q];
      if (S.i1 <= f0 || S.i0 >= ib + 2 || S.j1 <= j0 || S.j0 >= j0 + kSJ || S.k1 <= k0 ||
          S.k0 >= k0 + kSK)
        continue;
      if (S.comp >= WF_HX) {
        if (nh < kMaxLocalSrc3) L.h[nh++] = (short)q;
      } else {
        if (ne < kMaxLocalSrc3) L.e[ne++] = (short)q;
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
    if (pr.i >= ia && pr.i < ib && pr.j >= j0 + 1 && pr.j < j0 + 1 + kCJ && pr.k >= k0 + 1 &&
        pr.k < k0 + 1 + kCK) {
      const int slot = atomicAdd(&L.np, 1);
      if (slot < kMaxLocalProbe3) L.p[slot] = (short)q;
    }
  }
  __syncthreads();
  const int ne = L.ne, nh = L.nh, np = min(L.np, kMaxLocalProbe3);

  auto loadE = [&](int p) -> F3 {
    F3 v{0.f, 0.f, 0.f};
    if (in && p < nx) {
      const long long o = (long long)p * PS + col;
      v.x = P.in[0][o];
      v.y = P.in[1][o];
      v.z = P.in[2][o];
      for (int q = 0; q < ne; ++q) {
        const wf_source& S = P.src[L.e[q]];
        if (p >= S.i0 && p < S.i1 && gj >= S.j0 && gj < S.j1 && gk >= S.k0 && gk < S.k1) {
          const float s = src3_value(S, p, gj, gk, n);
          if (S.comp == WF_EX) v.x = fadd(v.x, s);
          else if (S.comp == WF_EY) v.y = fadd(v.y, s);
          else v.z = fadd(v.z, s);
        }
      }
    }
    return v;
  };
  auto loadH = [&](int p) -> F3 {
    F3 v{0.f, 0.f, 0.f};
    if (in && p < nx) {
      const long long o = (long long)p * PS + col;
      v.x = P.in[3][o];
      v.y = P.in[4][o];
      v.z = P.in[5][o];
    }
    return v;
  };
  // Old Ex, Ez of plane p at row j+1 (the Faraday update's j neighbour),
  // with the same source injection the neighbouring column applies.
  const bool in_j1 = gj + 1 >= 0 && gj + 1 < ny && gk >= 0 && gk < nz;
  auto loadJ1 = [&](int p) -> float2 {
    float2 v{0.f, 0.f};
    if (DIRECT && in_j1 && p < nx) {
      const long long o = (long long)p * PS + (long long)(gj + 1) * nz + gk;
      v.x = P.in[0][o];
      v.y = P.in[2][o];
      for (int q = 0; q < ne; ++q) {
        const wf_source& S = P.src[L.e[q]];
        if (p >= S.i0 && p < S.i1 && gj + 1 >= S.j0 && gj + 1 < S.j1 && gk >= S.k0 && gk < S.k1) {
          const float s = src3_value(S, p, gj + 1, gk, n);
          if (S.comp == WF_EX) v.x = fadd(v.x, s);
          else if (S.comp == WF_EZ) v.y = fadd(v.y, s);
        }
      }
    }
    return v;
  };
  // Faraday update of plane p from its old E (e; j neighbour ej1 when
  // DIRECT, else exchanged through sA/sB) and the old E of plane p+1 (en,
  // own column).
  auto curl = [&](int p, const F3& e, const F3& en, const F3& ho, const float2& ej1) -> F3 {
    float ez_j, ex_j;
    if (DIRECT) {
      ex_j = ej1.x;
      ez_j = ej1.y;
    } else {
      sA[w][lane] = e.x;
      sB[w][lane] = e.z;
      __syncthreads();
      ez_j = w + 1 < kSJ ? sB[w + 1][lane] : 0.f;
      ex_j = w + 1 < kSJ ? sA[w + 1][lane] : 0.f;
    }
    const float ey_k = __shfl_down_sync(0xffffffffu, e.y, 1);
    const float ex_k = __shfl_down_sync(0xffffffffu, e.x, 1);
    F3 v = ho;
    for (int q = 0; q < nh; ++q) {
      const wf_source& S = P.src[L.h[q]];
      if (p >= S.i0 && p < S.i1 && gj >= S.j0 && gj < S.j1 && gk >= S.k0 && gk < S.k1) {
        const float s = src3_value(S, p, gj, gk, n);
        if (S.comp == WF_HX) v.x = fadd(v.x, s);
        else if (S.comp == WF_HY) v.y = fadd(v.y, s);
        else v.z = fadd(v.z, s);
      }
    }
    if (gj < ny - 1 && gk < nz - 1) {
      const float t1 = dv<FDIV>(fsub(ey_k, e.y), dz, rdz);
      const float t2 = dv<FDIV>(fsub(ez_j, e.z), dy, rdy);
      v.x = fadd(v.x, fmul(dh, fsub(t1, t2)));
    }
    if (p < nx - 1 && gk < nz - 1) {
      const float t1 = dv<FDIV>(fsub(en.z, e.z), dx, rdx);
      const float t2 = dv<FDIV>(fsub(ex_k, e.x), dz, rdz);
      v.y = fadd(v.y, fmul(dh, fsub(t1, t2)));
    }
    if (p < nx - 1 && gj < ny - 1) {
      const float t1 = dv<FDIV>(fsub(ex_j, e.x), dy, rdy);
      const float t2 = dv<FDIV>(fsub(en.y, e.y), dx, rdx);
      v.z = fadd(v.z, fmul(dh, fsub(t1, t2)));
    }
    return v;
  };

  // ---- prologue: planes f0, f0+1 ------------------------------------------
  F3 e0 = loadE(f0), e1 = loadE(f0 + 1), e2 = loadE(f0 + 2), e3 = loadE(f0 + 3);
  F3 h0o = loadH(f0), h1o = loadH(f0 + 1), h2o = loadH(f0 + 2);
  float2 j0v = loadJ1(f0), j1v = loadJ1(f0 + 1), j2v = loadJ1(f0 + 2);
  F3 h0c = curl(f0, e0, e1, h0o, j0v);
  F3 h1c{0.f, 0.f, 0.f};
  float hmo_y = 0.f, hmo_z = 0.f, hmc_y = 0.f, hmc_z = 0.f;  // plane f-1
  F3 hprev{0.f, 0.f, 0.f};                                   // final H of plane f-1
  float cav = 0.f, cbv = 0.f;
  if (MAT && in) {
    cav = P.ca[(long long)f0 * PS + col];
    cbv = P.cb[(long long)f0 * PS + col];
  }
  unsigned mxb[6] = {0u, 0u, 0u, 0u, 0u, 0u};
  const bool check = P.check_max != nullptr && P.n_check > 0 && (n + 1) % P.n_check == 0;

  for (int f = f0; f < ib; ++f) {
    const int p = f + 1;
    if (!DIRECT) __syncthreads();  // previous iteration's readers of sA/sB are done
    // (A) Faraday update of plane p
    if (p < nx) h1c = curl(p, e1, e2, h1o, j1v);
    // (B) Mur faces of plane f
    float hyx = h0c.y, hzx = h0c.z;
    if (f == 0) {
      hyx = fadd(h1o.y, fmul(mx, fsub(h1c.y, h0o.y)));
      hzx = fadd(h1o.z, fmul(mx, fsub(h1c.z, h0o.z)));
    } else if (f == nx - 1) {
      hyx = fadd(hmo_y, fmul(mx, fsub(hmc_y, h0o.y)));
      hzx = fadd(hmo_z, fmul(mx, fsub(hmc_z, h0o.z)));
    }
    float hxy = h0c.x, hzy = hzx;
    if (yfaces) {
      __syncthreads();  // readers of sA/sB in (A) are done
      sA[w][lane] = h0c.x;
      sB[w][lane] = hzx;
      sC[w][lane] = h0o.x;
      sD[w][lane] = h0o.z;
      __syncthreads();
      if (in && gj == 0 && w + 1 < kSJ) {
        hxy = fadd(sC[w + 1][lane], fmul(my, fsub(sA[w + 1][lane], h0o.x)));
        hzy = fadd(sD[w + 1][lane], fmul(my, fsub(sB[w + 1][lane], h0o.z)));
      } else if (in && gj == ny - 1 && w >= 1) {
        hxy = fadd(sC[w - 1][lane], fmul(my, fsub(sA[w - 1][lane], h0o.x)));
        hzy = fadd(sD[w - 1][lane], fmul(my, fsub(sB[w - 1][lane], h0o.z)));
      }
    }
    float hxF = hxy, hyF = hyx;
    const float hx_dn = __shfl_down_sync(0xffffffffu, hxy, 1);
    const float hxo_dn = __shfl_down_sync(0xffffffffu, h0o.x, 1);
    const float hy_dn = __shfl_down_sync(0xffffffffu, hyx, 1);
    const float hyo_dn = __shfl_down_sync(0xffffffffu, h0o.y, 1);
    const float hx_up = __shfl_up_sync(0xffffffffu, hxy, 1);
    const float hxo_up = __shfl_up_sync(0xffffffffu, h0o.x, 1);
    const float hy_up = __shfl_up_sync(0xffffffffu, hyx, 1);
    const float hyo_up = __shfl_up_sync(0xffffffffu, h0o.y, 1);
    if (nz > 1 && in) {
      if (gk == 0 && lane < 31) {
        hxF = fadd(hxo_dn, fmul(mz, fsub(hx_dn, h0o.x)));
        hyF = fadd(hyo_dn, fmul(mz, fsub(hy_dn, h0o.y)));
      } else if (gk == nz - 1 && lane > 0) {
        hxF = fadd(hxo_up, fmul(mz, fsub(hx_up, h0o.x)));
        hyF = fadd(hyo_up, fmul(mz, fsub(hy_up, h0o.y)));
      }
    }
    const float hzF = hzy;
    // (C) Ampere update and outputs of plane f
    if (f >= ia) {
      __syncthreads();  // readers of sA/sB (A or B) are done
      sA[w][lane] = hzF;
      sB[w][lane] = hxF;
      __syncthreads();
      const float hy_k = __shfl_up_sync(0xffffffffu, hyF, 1);
      const float hx_k = __shfl_up_sync(0xffffffffu, hxF, 1);
      if (core) {
        const float hz_j = sA[w - 1][lane], hx_j = sB[w - 1][lane];
        float ex = e0.x, ey = e0.y, ez = e0.z;
        if (gj >= 1 && gk >= 1) {
          const float c = fsub(dv<FDIV>(fsub(hzF, hz_j), dy, rdy), dv<FDIV>(fsub(hyF, hy_k), dz, rdz));
          ex = MAT ? fadd(fmul(cav, ex), fmul(cbv, c)) : fadd(ex, fmul(de, c));
        }
        if (f >= 1 && gk >= 1) {
          const float c = fsub(dv<FDIV>(fsub(hxF, hx_k), dz, rdz), dv<FDIV>(fsub(hzF, hprev.z), dx, rdx));
          ey = MAT ? fadd(fmul(cav, ey), fmul(cbv, c)) : fadd(ey, fmul(de, c));
        }
        if (f >= 1 && gj >= 1) {
          const float c = fsub(dv<FDIV>(fsub(hyF, hprev.y), dx, rdx), dv<FDIV>(fsub(hxF, hx_j), dy, rdy));
          ez = MAT ? fadd(fmul(cav, ez), fmul(cbv, c)) : fadd(ez, fmul(de, c));
        }
        const long long o = (long long)f * PS + col;
        P.out[0][o] = ex;
        P.out[1][o] = ey;
        P.out[2][o] = ez;
        P.out[3][o] = hxF;
        P.out[4][o] = hyF;
        P.out[5][o] = hzF;
        for (int q = 0; q < np; ++q) {
          const wf_probe& pr = P.prb[L.p[q]];
          if (pr.i == f && pr.j == gj && pr.k == gk) {
            const float v = pr.comp == WF_EX ? ex : pr.comp == WF_EY ? ey : pr.comp == WF_EZ ? ez
                          : pr.comp == WF_HX ? hxF : pr.comp == WF_HY ? hyF : hzF;
            P.traces[(long long)L.p[q] * P.trace_ld + (n - P.trace_step0)] = v;
          }
        }
        if (check) {
          mxb[0] = max(mxb[0], abs_bits(ex));
          mxb[1] = max(mxb[1], abs_bits(ey));
          mxb[2] = max(mxb[2], abs_bits(ez));
          mxb[3] = max(mxb[3], abs_bits(hxF));
          mxb[4] = max(mxb[4], abs_bits(hyF));
          mxb[5] = max(mxb[5], abs_bits(hzF));
        }
      }
    }
    // (D) slide the plane window
    hprev = F3{hxF, hyF, hzF};
    hmo_y = h0o.y;
    hmo_z = h0o.z;
    hmc_y = h0c.y;
    hmc_z = h0c.z;
    h0o = h1o;
    h0c = h1c;
    h1o = h2o;
    h2o = loadH(f + 3);
    e0 = e1;
    e1 = e2;
    e2 = e3;
    e3 = loadE(f + 4);
    j1v = j2v;
    j2v = loadJ1(f + 3);
    if (MAT && in && f + 1 < nx) {
      cav = P.ca[(long long)(f + 1) * PS + col];
      cbv = P.cb[(long long)(f + 1) * PS + col];
    }
  }
  if (check) {
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      for (int sh = 16; sh > 0; sh >>= 1) mxb[c] = max(mxb[c], __shfl_xor_sync(0xffffffffu, mxb[c], sh));
      if (lane == 0) atomicMax(&L.bmax[c], mxb[c]);
    }
    __syncthreads();
    if (tid < 6) {
      const int idx = (n + 1) / P.n_check - P.check_base - 1;
      atomicMax(&P.check_max[idx * 6 + tid], L.bmax[tid]);
    }
  }
}

template <int kSJ, bool DIRECT, bool MAT, bool FDIV>
static int launch_stream_cfg(const Tile3D& P, int seg_len, int n, int nb, cudaStream_t st) {
  constexpr int kCJ = kSJ - 2;
  const int tiles_j = (P.ny + kCJ - 1) / kCJ, tiles_k = (P.nz + kCK - 1) / kCK;
  const int nseg = (P.nx + seg_len - 1) / seg_len;
  const long long nblk = (long long)tiles_j * tiles_k * nseg;
  if (nblk > 0x7fffffffLL) return set_error(WF_E_LIMIT, "wf_fdtd3d_run: too many column blocks");
  if (nb < 1 || nb > 65535) return set_error(WF_E_LIMIT, "wf_fdtd3d: 1..65535 instances");
  dim3 grid((unsigned)nblk, (unsigned)nb);
  k3d_stream<kSJ, DIRECT, MAT, FDIV><<<grid, kSJ * kSK, 0, st>>>(P, tiles_j, tiles_k, seg_len, n);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "launch k3d_stream");
  return WF_OK;
}

}  // namespace wf

#include "fdtd3d_tma.cuh"

namespace wf {

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library).
typedef CUresult (*TmaEncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static TmaEncodeFn tma_encoder() {
  static TmaEncodeFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<TmaEncodeFn>(ptr);
  }
  return fn;
}

// 4D map {k, j, i, instance} of one float32 array with a kBoxK x kBoxJ x 1 x 1
// box; false when the layout breaks a TMA rule (16-byte strides / base).
static bool tma_map(CUtensorMap* m, const float* base, int nx, int ny, int nz, int ninst,
                    long long istride) {
  TmaEncodeFn fn = tma_encoder();
  if (fn == nullptr || base == nullptr || (nz & 3) || (reinterpret_cast<uintptr_t>(base) & 15) ||
      (ninst > 1 && (istride & 3)))
    return false;
  const cuuint64_t dims[4] = {(cuuint64_t)nz, (cuuint64_t)ny, (cuuint64_t)nx, (cuuint64_t)ninst};
  const long long plane = (long long)nx * ny * nz;
  const cuuint64_t strides[3] = {(cuuint64_t)nz * 4, (cuuint64_t)ny * nz * 4,
                                 (cuuint64_t)(ninst > 1 ? istride : plane) * 4};
  const cuuint32_t box[4] = {(cuuint32_t)kBoxK, (cuuint32_t)kBoxJ, 1, 1};
  const cuuint32_t es[4] = {1, 1, 1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float*>(base), dims, strides, box,
            es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Status word of the TMA pass: a bounded mbarrier wait that gives up writes
// WF_E_TIMEOUT here (and its CTA stops); wf_fdtd3d_take_status reads and
// clears it.  Host code passes its device address, looked up once per device.
// The cached address is that of the current CUDA context of the device: it
// stays valid until cudaDeviceReset, after which this library must be
// reloaded (the same holds for every cached module address in it).
static __device__ int g_tma_status;
static std::mutex g_tma_mu;  // guards the caches below (host threads may race)

static int* tma_status_ptr() {
  static int* ptr[64] = {nullptr};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lock(g_tma_mu);
  if (ptr[dev] == nullptr) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_tma_status) != cudaSuccess) return nullptr;
    ptr[dev] = static_cast<int*>(p);
  }
  return ptr[dev];
}

// Suspended polls a TMA pipeline wait makes after its first non-blocking look
// (negative = kSpinLimit); see wf_fdtd3d_set_wait_limit.
static std::atomic<long long> g_tma_wait_limit{-1};

// Opt k3d_tma into its dynamic shared memory (once per instantiation and
// device: the attribute belongs to the device's context).
template <bool MAT, bool FDIV>
static int tma_attr() {
  static bool attr[64] = {false};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= 64) return set_error(WF_E_LIMIT, "k3d_tma: device %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_tma_mu);
  if (!attr[dev]) {
    e = cudaFuncSetAttribute(k3d_tma<MAT, FDIV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(TmaSmem));
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(k3d_tma)");
    attr[dev] = true;
  }
  return WF_OK;
}

template <bool MAT, bool FDIV>
static int launch_tma(const TmaMaps& maps, const Tile3D& P, int seg_len, int n, int nb,
                      cudaStream_t st) {
  const int tiles_j = (P.ny + kTCJ - 1) / kTCJ, tiles_k = (P.nz + kTCK - 1) / kTCK;
  const int nseg = (P.nx + seg_len - 1) / seg_len;
  const long long nblk = (long long)tiles_j * tiles_k * nseg;
  if (nblk > 0x7fffffffLL || nb < 1 || nb > 65535)
    return set_error(WF_E_LIMIT, "wf_fdtd3d: too many column blocks or instances");
  const size_t smem = sizeof(TmaSmem);
  const int rc = tma_attr<MAT, FDIV>();
  if (rc != WF_OK) return rc;
  dim3 grid((unsigned)nblk, (unsigned)nb);
  const long long lim = g_tma_wait_limit.load();
  k3d_tma<MAT, FDIV><<<grid, kTJ * kTK, smem, st>>>(
      maps, P, tiles_j, tiles_k, seg_len, n, tma_status_ptr(),
      lim < 0 ? kSpinLimit : (unsigned)std::min(lim, 0xffffffffLL));
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "launch k3d_tma");
  return WF_OK;
}

// Streaming variants: rows per column block (16 = 512 threads, one CTA per
// SM; 8 = 256 threads, two per SM) and whether the Faraday update reads its
// j neighbour directly (no shared exchange, one CTA barrier less per plane).
template <bool MAT, bool FDIV>
static int launch_stream(const Tile3D& P, int seg_len, int n, int rows, bool direct, int nb,
                         cudaStream_t st) {
  if (rows == 8)
    return direct ? launch_stream_cfg<8, true, MAT, FDIV>(P, seg_len, n, nb, st)
                  : launch_stream_cfg<8, false, MAT, FDIV>(P, seg_len, n, nb, st);
  return direct ? launch_stream_cfg<16, true, MAT, FDIV>(P, seg_len, n, nb, st)
                : launch_stream_cfg<16, false, MAT, FDIV>(P, seg_len, n, nb, st);
}

// Segment length along i: enough column blocks for ~4 per SM, at least 8
// planes per segment.
static int stream_seg_len(int nx, int ny, int nz, int rows) {
  int dev = 0, nsm = 148;
  if (cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const long long plane = (long long)((ny + rows - 3) / (rows - 2)) * ((nz + kCK - 1) / kCK);
  long long nseg = (4LL * nsm + plane - 1) / plane;
  nseg = std::max(1LL, std::min(nseg, (long long)std::max(1, nx / 8)));
  return (int)((nx + nseg - 1) / nseg);
}

// Segment length of the TMA kernel.  A column block costs about (planes + 2)
// plane-steps (each segment re-reads three planes, mostly from L2); a launch
// takes the total spread over the resident slots plus about one block's
// length of tail.  Pick the segment count that minimises
// blocks x (L + 2) / slots + (L + 2), with at least 22 planes per segment.
// It picks 26 on a 256^3 volume and on 8 x 128^3, within 0.2 % of the best
// length of a sweep over 16..64 on both; the former minimum of 16 planes lost
// 4 % at 256^3.
template <bool MAT, bool FDIV>
static int tma_seg_len(int nx, int ny, int nz, int nb) {
  int dev = 0, nsm = 148, per_sm = 2;
  if (cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (tma_attr<MAT, FDIV>() != WF_OK ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k3d_tma<MAT, FDIV>, kTJ * kTK,
                                                    sizeof(TmaSmem)) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  const long long slots = (long long)nsm * per_sm;
  const long long cols = (long long)((ny + kTCJ - 1) / kTCJ) * ((nz + kTCK - 1) / kTCK) * nb;
  const int max_seg = std::max(1, nx / 22);
  int best = 1;
  long long best_cost = -1;
  for (int ns = 1; ns <= max_seg; ++ns) {
    const long long len = (nx + ns - 1) / ns;
    const long long cost = cols * ns * (len + 2) + slots * (len + 2);  // x slots
    if (best_cost < 0 || cost < best_cost) {
      best_cost = cost;
      best = ns;
    }
  }
  return (nx + best - 1) / best;
}

}  // namespace wf

using namespace wf;

static int run3d(const wf_grid3d* g, int nb, long long fstride, long long cstride,
                 long long tstride, int sstride, float* const* f, float* const* s, const float* ca,
                 const float* cb, const wf_source* src, int32_t nsrc, const wf_probe* probes,
                 int32_t nprobe, float* traces, int64_t trace_ld, int32_t trace_step0,
                 int32_t step0, int32_t nsteps, int32_t n_check, uint32_t* check_max,
                 const wf_tune* tune, void* stream) {
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
  // Default: the single-step streaming kernel (k3d_stream) for volumes, the
  // tile kernel (k3d_pass) for Nz == 1.  An explicit tune with tile_i == 0
  // selects streaming with segments of tile_j planes (0 = automatic); any
  // other tune selects the tile kernel with that shape and depth.
  wf_tune t{};
  bool stream_k = false, direct = true;
  int seg_len = 0, rows = 16;
  int variant = 0;  // streaming: 0 = TMA ring when the layout allows, else 2
  if (tune && tune->tile_i == 0) {
    // streaming: tile_j = segment length (0 = automatic); threads selects the
    // variant: 0 TMA ring (register kernel when Nz % 4 != 0), 1 register
    // kernel with shared j exchange, 2 register kernel with direct j loads;
    // tile_k = rows per column block of the register kernel (8 or 16)
    stream_k = true;
    seg_len = tune->tile_j;
    rows = tune->tile_k == 8 ? 8 : 16;
    variant = tune->threads;
    direct = variant != 1;
    if (seg_len < 0) return set_error(WF_E_ARG, "wf_fdtd3d_run: negative segment length");
  } else if (tune) {
    t = *tune;
  } else if (g->nz > 1) {
    stream_k = true;
  } else {
    t.steps_per_pass = 1;
    t.tile_i = 4;
    t.tile_j = 8;
    t.tile_k = 30;
    t.threads = 256;
  }
  if (nb > 1 && !stream_k)
    return set_error(WF_E_ARG, "wf_fdtd3d_batch_run: batched instances need the streaming kernel");
  const bool auto_seg = seg_len == 0;
  if (stream_k) {
    t.steps_per_pass = 1;
    if (auto_seg) seg_len = stream_seg_len(g->nx, g->ny, g->nz, rows);
  } else if (t.steps_per_pass < 1 || t.steps_per_pass > 8 || t.tile_i < 2 || t.tile_j < 2 ||
             t.tile_k < 2 || t.threads < 32 || t.threads > 512 || (t.threads & 31)) {
    return set_error(WF_E_ARG, "wf_fdtd3d_run: bad tune");
  }
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
  P.fstride = fstride;
  P.cstride = cstride;
  P.tstride = tstride;
  P.sstride = sstride;
  const int all3 = WF_FASTDIV_X | WF_FASTDIV_Y | WF_FASTDIV_Z;
  const int all2 = WF_FASTDIV_X | WF_FASTDIV_Y;
  const bool fd = g->nz > 1 ? (g->flags & all3) == all3 : (g->flags & all2) == all2;
  // TMA tensor maps of both ping-pong sets (and Ca/Cb), encoded once per call
  TmaMaps mapsA{}, mapsB{};
  bool tma = stream_k && variant == 0;
  if (tma) {
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    for (int c = 0; c < 6 && tma; ++c)
      tma = tma_map(&mapsA.m[c], f[c], nx, ny, nz, nb, fstride) &&
            tma_map(&mapsB.m[c], s[c], nx, ny, nz, nb, fstride);
    if (tma && ca)
      tma = tma_map(&mapsA.m[6], ca, nx, ny, nz, cstride ? nb : 1, cstride) &&
            tma_map(&mapsA.m[7], cb, nx, ny, nz, cstride ? nb : 1, cstride);
    mapsB.m[6] = mapsA.m[6];
    mapsB.m[7] = mapsA.m[7];
    if (tma && auto_seg)
      seg_len = ca ? (fd ? tma_seg_len<true, true>(g->nx, g->ny, g->nz, nb)
                         : tma_seg_len<true, false>(g->nx, g->ny, g->nz, nb))
                   : (fd ? tma_seg_len<false, true>(g->nx, g->ny, g->nz, nb)
                         : tma_seg_len<false, false>(g->nx, g->ny, g->nz, nb));
  }
  const PassPlan plan(nsteps, t.steps_per_pass);
  for (int p = 0; p < plan.passes(); ++p) {
    float* const* in = (p & 1) ? s : f;
    float* const* out = (p & 1) ? f : s;
    for (int c = 0; c < 6; ++c) {
      P.in[c] = in[c];
      P.out[c] = out[c];
    }
    const int s0 = step0 + plan.offset(p), k = plan.len(p);
    int rc;
    if (tma) {
      const TmaMaps& m = (p & 1) ? mapsB : mapsA;
      rc = ca ? (fd ? launch_tma<true, true>(m, P, seg_len, s0, nb, st)
                    : launch_tma<true, false>(m, P, seg_len, s0, nb, st))
              : (fd ? launch_tma<false, true>(m, P, seg_len, s0, nb, st)
                    : launch_tma<false, false>(m, P, seg_len, s0, nb, st));
    } else if (stream_k)
      rc = ca ? (fd ? launch_stream<true, true>(P, seg_len, s0, rows, direct, nb, st)
                    : launch_stream<true, false>(P, seg_len, s0, rows, direct, nb, st))
              : (fd ? launch_stream<false, true>(P, seg_len, s0, rows, direct, nb, st)
                    : launch_stream<false, false>(P, seg_len, s0, rows, direct, nb, st));
    else
      rc = ca ? (fd ? launch3<true, true>(P, t, s0, k, st) : launch3<true, false>(P, t, s0, k, st))
              : (fd ? launch3<false, true>(P, t, s0, k, st) : launch3<false, false>(P, t, s0, k, st));
    if (rc) return rc;
  }
  if (plan.needs_copy()) {
    for (int c = 0; c < 6; ++c) {
      P.in[c] = s[c];
      P.out[c] = f[c];
    }
    for (int q = 0; q < nb; ++q) {
      k_copy6<<<592, 256, 0, st>>>(P, (long long)g->nx * g->ny * g->nz);
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) return cuda_fail(e, "launch k_copy6");
      for (int c = 0; c < 6; ++c) {
        P.in[c] += fstride;
        P.out[c] += fstride;
      }
    }
  }
  return WF_OK;
}

extern "C" int32_t wf_fdtd3d_run(const wf_grid3d* g, float* const* f, float* const* s,
                                 const float* ca, const float* cb, const wf_source* src,
                                 int32_t nsrc, const wf_probe* probes, int32_t nprobe,
                                 float* traces, int64_t trace_ld, int32_t trace_step0,
                                 int32_t step0, int32_t nsteps, int32_t n_check,
                                 uint32_t* check_max, const wf_tune* tune, void* stream) {
  return run3d(g, 1, 0, 0, 0, 0, f, s, ca, cb, src, nsrc, probes, nprobe, traces, trace_ld,
               trace_step0, step0, nsteps, n_check, check_max, tune, stream);
}

extern "C" int32_t wf_fdtd3d_batch_run(const wf_grid3d* g, int32_t ninst, int64_t field_stride,
                                       float* const* f, float* const* s, const float* ca,
                                       const float* cb, int64_t coef_stride,
                                       const wf_source* src, int32_t src_per_inst,
                                       int32_t src_stride,
                                       const wf_probe* probes, int32_t nprobe, float* traces,
                                       int64_t trace_ld, int64_t trace_stride,
                                       int32_t trace_step0, int32_t step0, int32_t nsteps,
                                       int32_t n_check, uint32_t* check_max,
                                       const wf_tune* tune, void* stream) {
  if (g == nullptr || ninst < 1 || ninst > 65535)
    return set_error(WF_E_ARG, "wf_fdtd3d_batch_run: null grid or instance count outside 1..65535");
  const long long n = (long long)g->nx * g->ny * g->nz;
  if (ninst > 1 && (field_stride < n || (ca != nullptr && coef_stride != 0 && coef_stride < n) ||
                    (nprobe > 0 && trace_stride < (long long)nprobe * trace_ld) ||
                    src_stride < 0 || (src_stride > 0 && src_stride < src_per_inst)))
    return set_error(WF_E_ARG, "wf_fdtd3d_batch_run: instance strides overlap");
  return run3d(g, ninst, field_stride, coef_stride, trace_stride, src_stride, f, s, ca, cb, src,
               src_per_inst, probes, nprobe, traces, trace_ld, trace_step0, step0, nsteps,
               n_check, check_max, tune, stream);
}

extern "C" int32_t wf_fdtd3d_set_wait_limit(int64_t polls) {
  g_tma_wait_limit.store(polls < 0 ? -1LL : (long long)polls);
  return WF_OK;
}

extern "C" int32_t wf_fdtd3d_take_status(int32_t* status) {
  if (status == nullptr) return set_error(WF_E_ARG, "wf_fdtd3d_take_status: null output");
  int v = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&v, wf::g_tma_status, sizeof(int));
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyFromSymbol(status)");
  if (v != 0) {
    const int zero = 0;
    e = cudaMemcpyToSymbol(wf::g_tma_status, &zero, sizeof(int));
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyToSymbol(status)");
  }
  *status = v;
  return WF_OK;
}
