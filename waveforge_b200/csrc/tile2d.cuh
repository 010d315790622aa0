// tile2d.cuh -- the 2D TM Yee tile routine shared by the plain and batched kernels.
//
// One CTA advances one rectangular tile of one solve by k time steps inside
// shared memory (overlapped temporal blocking): it loads the tile core plus a
// k-cell halo of Ex, Ey, Hz (and Ca, Cb) from the pass-input buffers, runs k
// complete leapfrog steps on that region, and stores the core to the
// pass-output buffers.  The valid region shrinks by one cell per step on every
// side that is not a domain edge, so after k steps the core is exact.
//
// Per step, in reference order (src/core/fdtd2d.py:187-266):
//   1. soft injection into Ex/Ey (src/core/sources.py:863-887); Hz injection is
//      folded into phase 2 so the Mur snapshot stays pre-injection
//      (boundaries.py:237 snapshot happens before sources.step);
//   2. Faraday update of Hz on i<Nx-1, j<Ny-1 (fdtd2d.py:232-235);
//   3. first-order Mur on the four Hz edges, x edges then y edges, evaluated as
//      a pure function of the pre-step Hz and the curl-updated Hz
//      (boundaries.py:259-274);
//   4. Ampere updates of Ex (j>=1) and Ey (i>=1), scalar or Ca/Cb path
//      (fdtd2d.py:244-257);
//   5. detector gather and (every n_check steps) the |field| maxima.
// Hz is double-buffered in shared memory (ha = previous step, hb = new), which
// also provides the Mur snapshot for free.
#pragma once

#include "wf_common.cuh"

namespace wf {

constexpr int kMaxLocalSrc = 64;
constexpr int kMaxLocalProbe = 256;

struct Tile2D {
  int nx, ny;
  float dh, de, dx, dy, mx, my;
  const float *ex_in, *ey_in, *hz_in;
  float *ex_out, *ey_out, *hz_out;
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
  int check_base;  // step0_of_run / n_check
  int* status;     // device status word (may be null)
};

struct Lists2D {
  int nh, ne, np;
  short h[kMaxLocalSrc];
  short e[kMaxLocalSrc];
  short p[kMaxLocalProbe];
  unsigned bmax[3];
};

// Value of wave * amp for cell (i,j) of source s (row-major box offset).
__device__ __forceinline__ float src_value(const wf_source& s, int i, int j, int n) {
  const float w = s.wave[n];
  if (s.amp == nullptr) return w;
  const int c = (i - s.i0) * (s.j1 - s.j0) + (j - s.j0);
  return fmul(w, s.amp[c]);
}

__device__ __forceinline__ bool src_hits(const wf_source& s, int i, int j) {
  return i >= s.i0 && i < s.i1 && j >= s.j0 && j < s.j1;
}

// Smem bytes needed for a region of rh x rw cells.
__host__ __device__ inline size_t tile2d_smem(int rh, int rw, bool mat) {
  return (size_t)rh * rw * (mat ? 6 : 4) * sizeof(float);
}

template <bool MAT>
__device__ void tile2d(const Tile2D& P, int ci0, int ci1, int cj0, int cj1,
                       int step0, int k, float* sm, Lists2D& L) {
  const int nx = P.nx, ny = P.ny;
  const int ri0 = max(ci0 - k, 0), ri1 = min(ci1 + k, nx);
  const int rj0 = max(cj0 - k, 0), rj1 = min(cj1 + k, ny);
  const int RH = ri1 - ri0, RW = rj1 - rj0, RN = RH * RW;
  float* ex = sm;
  float* ey = ex + RN;
  float* ha = ey + RN;
  float* hb = ha + RN;
  float* ca = hb + RN;
  float* cb = ca + RN;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  const float dh = P.dh, de = P.de, dx = P.dx, dy = P.dy, mx = P.mx, my = P.my;

  // ---- local source / probe lists (sources keep collection order) --------
  if (tid == 0) {
    int nh = 0, ne = 0;
    for (int s = 0; s < P.nsrc; ++s) {
      const wf_source& S = P.src[s];
      if (S.i1 <= ri0 || S.i0 >= ri1 || S.j1 <= rj0 || S.j0 >= rj1) continue;
      if (S.comp == WF_HZ) {
        if (nh < kMaxLocalSrc) L.h[nh++] = (short)s;
        else if (P.status) atomicExch(P.status, WF_E_LIMIT);
      } else {
        if (ne < kMaxLocalSrc) L.e[ne++] = (short)s;
        else if (P.status) atomicExch(P.status, WF_E_LIMIT);
      }
    }
    L.nh = nh;
    L.ne = ne;
    L.np = 0;
    L.bmax[0] = L.bmax[1] = L.bmax[2] = 0u;
  }
  __syncthreads();
  for (int q = tid; q < P.nprb; q += blockDim.x) {
    const wf_probe& pr = P.prb[q];
    if (pr.i >= ci0 && pr.i < ci1 && pr.j >= cj0 && pr.j < cj1) {
      const int slot = atomicAdd(&L.np, 1);
      if (slot < kMaxLocalProbe) L.p[slot] = (short)q;
      else if (P.status) atomicExch(P.status, WF_E_LIMIT);
    }
  }

  // ---- load region ---------------------------------------------------------
  for (int r = warp; r < RH; r += nw) {
    const long long g = (long long)(ri0 + r) * ny + rj0;
    for (int c = lane; c < RW; c += 32) {
      const int o = r * RW + c;
      ex[o] = P.ex_in[g + c];
      ey[o] = P.ey_in[g + c];
      ha[o] = P.hz_in[g + c];
      if (MAT) {
        ca[o] = P.ca[g + c];
        cb[o] = P.cb[g + c];
      }
    }
  }
  __syncthreads();
  const int np = min(L.np, kMaxLocalProbe);
  const int nh = L.nh, ne = L.ne;

  for (int t = 0; t < k; ++t) {
    const int n = step0 + t;

    // (1) E-field soft injection, sequential to keep source order exact.
    if (ne > 0) {
      if (tid == 0) {
        for (int q = 0; q < ne; ++q) {
          const wf_source& S = P.src[L.e[q]];
          float* f = (S.comp == WF_EX) ? ex : ey;
          const int a0 = max(S.i0, ri0), a1 = min(S.i1, ri1);
          const int b0 = max(S.j0, rj0), b1 = min(S.j1, rj1);
          for (int i = a0; i < a1; ++i)
            for (int j = b0; j < b1; ++j) {
              const int o = (i - ri0) * RW + (j - rj0);
              f[o] = fadd(f[o], src_value(S, i, j, n));
            }
        }
      }
      __syncthreads();
    }

    // (2) Hz injection + Faraday curl into hb.
    for (int r = warp; r < RH; r += nw) {
      const int gi = ri0 + r;
      for (int c = lane; c < RW; c += 32) {
        const int gj = rj0 + c;
        const int o = r * RW + c;
        float v = ha[o];
        if (nh > 0) {
          for (int q = 0; q < nh; ++q) {
            const wf_source& S = P.src[L.h[q]];
            if (src_hits(S, gi, gj)) v = fadd(v, src_value(S, gi, gj, n));
          }
        }
        if (gi < nx - 1 && gj < ny - 1 && r + 1 < RH && c + 1 < RW) {
          const float t2 = fdiv(fsub(ex[o + 1], ex[o]), dy);
          const float t4 = fdiv(fsub(ey[o + RW], ey[o]), dx);
          v = fadd(v, fmul(dh, fsub(t2, t4)));
        }
        hb[o] = v;
      }
    }
    __syncthreads();

    // (3) Mur edges.  X = value after the x-edge pass, F = after the y-edge
    // pass.  X is only ever evaluated on columns that are not y-edges, so both
    // read pre-step Hz (ha) and curl-updated Hz (hb) of NON-edge cells only:
    // the edge writes below cannot race with these reads (needs Nx, Ny >= 3).
    {
      const bool top = (ri0 == 0), bot = (ri1 == nx), lef = (rj0 == 0), rig = (rj1 == ny);
      auto X = [&](int r, int c) -> float {
        const int gi = ri0 + r;
        if (gi == 0) return fadd(ha[RW + c], fmul(mx, fsub(hb[RW + c], ha[c])));
        if (gi == nx - 1)
          return fadd(ha[(RH - 2) * RW + c],
                      fmul(mx, fsub(hb[(RH - 2) * RW + c], ha[(RH - 1) * RW + c])));
        return hb[r * RW + c];
      };
      auto F = [&](int r, int c) -> float {
        const int gj = rj0 + c;
        if (gj == 0) return fadd(ha[r * RW + 1], fmul(my, fsub(X(r, 1), ha[r * RW])));
        if (gj == ny - 1)
          return fadd(ha[r * RW + RW - 2], fmul(my, fsub(X(r, RW - 2), ha[r * RW + RW - 1])));
        return X(r, c);
      };
      const int nrow = (top ? RW : 0) + (bot ? RW : 0);
      const int cr0 = top ? 1 : 0, cr1 = bot ? RH - 1 : RH;
      const int ncolr = cr1 - cr0;
      const int ncol = (lef ? ncolr : 0) + (rig ? ncolr : 0);
      for (int e = tid; e < nrow + ncol; e += blockDim.x) {
        int r, c;
        if (e < nrow) {
          const bool first = top && e < RW;
          r = first ? 0 : RH - 1;
          c = first ? e : e - (top ? RW : 0);
        } else {
          const int e2 = e - nrow;
          const bool first = lef && e2 < ncolr;
          c = first ? 0 : RW - 1;
          r = cr0 + (first ? e2 : e2 - (lef ? ncolr : 0));
        }
        hb[r * RW + c] = F(r, c);
      }
    }
    __syncthreads();

    // (4) Ampere updates (in place; each reads only its own Ex/Ey and hb).
    for (int r = warp; r < RH; r += nw) {
      const int gi = ri0 + r;
      for (int c = lane; c < RW; c += 32) {
        const int gj = rj0 + c;
        const int o = r * RW + c;
        if (gj >= 1 && c >= 1) {
          const float d = fdiv(fsub(hb[o], hb[o - 1]), dy);
          ex[o] = MAT ? fadd(fmul(ca[o], ex[o]), fmul(cb[o], d)) : fadd(ex[o], fmul(de, d));
        }
        if (gi >= 1 && r >= 1) {
          const float d = fdiv(fsub(hb[o], hb[o - RW]), dx);
          ey[o] = MAT ? fsub(fmul(ca[o], ey[o]), fmul(cb[o], d)) : fsub(ey[o], fmul(de, d));
        }
      }
    }
    __syncthreads();

    // (5) detectors (cells of the core) and stability maxima.
    for (int q = tid; q < np; q += blockDim.x) {
      const wf_probe& pr = P.prb[L.p[q]];
      const int o = (pr.i - ri0) * RW + (pr.j - rj0);
      const float v = pr.comp == WF_EX ? ex[o] : pr.comp == WF_EY ? ey[o] : hb[o];
      P.traces[(long long)L.p[q] * P.trace_ld + (n - P.trace_step0)] = v;
    }
    if (P.check_max != nullptr && P.n_check > 0 && (n + 1) % P.n_check == 0) {
      unsigned m0 = 0, m1 = 0, m2 = 0;
      for (int i = ci0 + warp; i < ci1; i += nw)
        for (int j = cj0 + lane; j < cj1; j += 32) {
          const int o = (i - ri0) * RW + (j - rj0);
          m0 = max(m0, abs_bits(ex[o]));
          m1 = max(m1, abs_bits(ey[o]));
          m2 = max(m2, abs_bits(hb[o]));
        }
      for (int sh = 16; sh > 0; sh >>= 1) {
        m0 = max(m0, __shfl_xor_sync(0xffffffffu, m0, sh));
        m1 = max(m1, __shfl_xor_sync(0xffffffffu, m1, sh));
        m2 = max(m2, __shfl_xor_sync(0xffffffffu, m2, sh));
      }
      if (lane == 0) {
        atomicMax(&L.bmax[0], m0);
        atomicMax(&L.bmax[1], m1);
        atomicMax(&L.bmax[2], m2);
      }
      __syncthreads();
      if (tid < 3) {
        const int idx = (n + 1) / P.n_check - P.check_base - 1;
        atomicMax(&P.check_max[idx * 3 + tid], L.bmax[tid]);
        L.bmax[tid] = 0u;
      }
    }
    float* tmp = ha;
    ha = hb;
    hb = tmp;
    __syncthreads();
  }

  // ---- store core ------------------------------------------------------
  for (int i = ci0 + warp; i < ci1; i += nw) {
    const long long g = (long long)i * ny;
    for (int j = cj0 + lane; j < cj1; j += 32) {
      const int o = (i - ri0) * RW + (j - rj0);
      P.ex_out[g + j] = ex[o];
      P.ey_out[g + j] = ey[o];
      P.hz_out[g + j] = ha[o];
    }
  }
  __syncthreads();
}

}  // namespace wf
