// tile2d.cuh -- the 2D TM Yee tile routine shared by the plain and batched kernels.
//
// One CTA advances one tile of one solve by k time steps (overlapped temporal
// blocking): it loads a region = core + k-cell halo of Ex, Ey, Hz (and Ca,
// Cb) from the pass-input buffers, runs k complete leapfrog steps on it, and
// stores the core to the pass-output buffers.  The valid part of the region
// shrinks by one cell per step on every side that is not a domain edge, so
// after k steps the core is exact.
//
// Register-resident layout: the region is RH x RW cells (RH = R*WY rows,
// RW = 32*WX columns).  Warp (wx, wy) owns columns wx*32..wx*32+31 (one per
// lane, so every global access is a coalesced 128-byte row segment) and rows
// wy*R..wy*R+R-1; each thread keeps its R cells of Ex, Ey, Hz, Ca, Cb in
// registers for the whole pass.  Horizontal neighbours come from warp
// shuffles, and only the cells on warp boundaries go through small shared
// exchange rows: two CTA barriers per step.  Tiles whose region touches no
// domain edge run a specialisation without any boundary logic.
//
// Per step, in reference order (src/core/fdtd2d.py:187-266):
//   1. soft injection into Ex/Ey (src/core/sources.py:863-887); Hz injection
//      is folded into 2 so the Mur snapshot stays pre-injection
//      (boundaries.py:237 snapshots before sources.step);
//   2. Faraday update of Hz on i<Nx-1, j<Ny-1 (fdtd2d.py:232-235);
//   3. first-order Mur on the four Hz edges, x edges then y edges, as a pure
//      function of the pre-step and the curl-updated Hz (boundaries.py:
//      259-274), staged in shared memory by edge tiles only;
//   4. Ampere updates of Ex (j>=1) and Ey (i>=1), scalar or Ca/Cb path
//      (fdtd2d.py:244-257);
//   5. detector samples and, every n_check steps, the |field| maxima.
// Every float op is a separately rounded IEEE op in the reference order; the
// spacing divisions use the verified exact division of wf_common.cuh.
#pragma once

#include "wf_common.cuh"

namespace wf {

constexpr int kMaxLocalSrc = 64;
constexpr int kMaxLocalProbe = 256;

struct Tile2D {
  int nx, ny;
  float dh, de, dx, dy, mx, my;
  int fastdiv;  // WF_FASTDIV_* bits of the grid
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

// Region geometry of one launch configuration.
template <int R_, int WX_, int WY_>
struct TileCfg {
  static constexpr int R = R_, WX = WX_, WY = WY_;
  static constexpr int THREADS = 32 * WX * WY;
  static constexpr int RH = R * WY, RW = 32 * WX;
};

// Shared memory of the tile routine (sized for the configuration).
template <class C>
struct TileSmem {
  alignas(16) float xe[C::WX][C::RH];  // Ex of each warp column's lane 0 (for lane 31 of the left warp)
  float yr[C::WY][C::RW];   // Ey of each segment's first row (for the segment above)
  alignas(16) float hx[C::WX][C::RH];  // Hz of each warp column's lane 31 (for lane 0 of the right warp)
  float hr[C::WY][C::RW];   // Hz of each segment's last row (for the segment below)
  float sp[C::RH][C::RW];   // Mur staging: pre-step Hz
  float sc[C::RH][C::RW];   // Mur staging: curl-updated Hz
  int nh, ne, np;
  short h[kMaxLocalSrc];
  short e[kMaxLocalSrc];
  short p[kMaxLocalProbe];
  unsigned bmax[3];
};

// Store a thread's R consecutive rows into a shared row of R floats with the
// widest aligned vector stores (16-byte when R % 4 == 0, else 8-byte when R
// is even): one lane writes a warp column's boundary values in R/4 or R/2
// instructions instead of R.
template <int R>
__device__ __forceinline__ void store_rows(float* dst, const float (&v)[R]) {
  if constexpr (R % 4 == 0) {
#pragma unroll
    for (int q = 0; q < R; q += 4)
      *reinterpret_cast<float4*>(dst + q) = make_float4(v[q], v[q + 1], v[q + 2], v[q + 3]);
  } else if constexpr (R % 2 == 0) {
#pragma unroll
    for (int q = 0; q < R; q += 2) *reinterpret_cast<float2*>(dst + q) = make_float2(v[q], v[q + 1]);
  } else {
#pragma unroll
    for (int q = 0; q < R; ++q) dst[q] = v[q];
  }
}

// Value of wave * amp for cell (i,j) of source s (row-major box offset).
__device__ __forceinline__ float src_value(const wf_source& s, int i, int j, int n) {
  const float w = s.wave[n];
  if (s.amp == nullptr) return w;
  const int c = (i - s.i0) * (s.j1 - s.j0) + (j - s.j0);
  return fmul(w, s.amp[c]);
}

// Per-thread view of one tile: geometry and lists fixed for the pass.
struct TileCtx {
  int ri0, ri1, rj0, rj1, RHa, RWa;
  int ci0, ci1, cj0, cj1;
  int lane, wx, wy, c, r0, gj;
  int nh, ne, np;
  bool my_h, my_e, pslow;
  int pown0, pown1, pq0, pq1;
};

template <class C, bool MAT, bool FDIV, bool EDGE>
__device__ __forceinline__ void tile2d_steps(const Tile2D& P, const TileCtx& T, TileSmem<C>& S,
                                             float (&ex)[C::R], float (&ey)[C::R],
                                             float (&hz)[C::R], const float (&ca)[C::R],
                                             const float (&cb)[C::R], int step0, int k) {
  constexpr int R = C::R, WX = C::WX, WY = C::WY;
  const int nx = P.nx, ny = P.ny;
  const int lane = T.lane, wx = T.wx, wy = T.wy, c = T.c, r0 = T.r0, gj = T.gj, ri0 = T.ri0;
  const float dh = P.dh, de = P.de, dx = P.dx, dy = P.dy, mx = P.mx, my = P.my;
  const double rdx = __drcp_rn((double)dx), rdy = __drcp_rn((double)dy);
  auto divx = [&](float a) { return FDIV ? div_fast(a, rdx) : fdiv(a, dx); };
  auto divy = [&](float a) { return FDIV ? div_fast(a, rdy) : fdiv(a, dy); };
  // Boundary predicates (compile away for interior tiles).
  const bool colv = T.c < T.RWa;
  const bool curl_col = EDGE ? (gj < ny - 1) : true;
  const bool ex_col = EDGE ? (gj >= 1) : true;

  for (int t = 0; t < k; ++t) {
    const int n = step0 + t;

    // (1) E-field soft injection on own cells, in collection order.
    if (T.my_e) {
      for (int s = 0; s < T.ne; ++s) {
        const wf_source& Q = P.src[S.e[s]];
        if (gj < Q.j0 || gj >= Q.j1) continue;
#pragma unroll
        for (int q = 0; q < R; ++q) {
          const int gi = ri0 + r0 + q;
          if (gi >= Q.i0 && gi < Q.i1) {
            if (Q.comp == WF_EX) ex[q] = fadd(ex[q], src_value(Q, gi, gj, n));
            else ey[q] = fadd(ey[q], src_value(Q, gi, gj, n));
          }
        }
      }
    }
    // exchange for the Faraday update
    if (lane == 0) store_rows<R>(&S.xe[wx][r0], ex);
    S.yr[wy][c] = ey[0];
    __syncthreads();

    // (2) Hz injection + Faraday curl.
#pragma unroll
    for (int q = 0; q < R; ++q) {
      float exr = __shfl_down_sync(0xffffffffu, ex[q], 1);
      if (lane == 31) exr = (wx + 1 < WX) ? S.xe[wx + 1][r0 + q] : 0.f;
      float eyb;
      if (q + 1 < R) eyb = ey[q + 1];
      else eyb = (wy + 1 < WY) ? S.yr[wy + 1][c] : 0.f;
      const float t2 = divy(fsub(exr, ex[q]));
      const float t4 = divx(fsub(eyb, ey[q]));
      if (EDGE) S.sp[r0 + q][c] = hz[q];  // Mur snapshot (pre-injection)
      float v = hz[q];
      if (T.my_h) {
        const int gi = ri0 + r0 + q;
        for (int s = 0; s < T.nh; ++s) {
          const wf_source& Q = P.src[S.h[s]];
          if (gi >= Q.i0 && gi < Q.i1 && gj >= Q.j0 && gj < Q.j1) v = fadd(v, src_value(Q, gi, gj, n));
        }
      }
      const float vc = fadd(v, fmul(dh, fsub(t2, t4)));
      if (EDGE) {
        const int gi = ri0 + r0 + q;
        hz[q] = (curl_col && gi < nx - 1) ? vc : v;
      } else {
        hz[q] = vc;
      }
    }

    // (3) Mur edges.
    if (EDGE) {
#pragma unroll
      for (int q = 0; q < R; ++q) S.sc[r0 + q][c] = hz[q];
      __syncthreads();
      // X: value after the x-edge pass, F: after the y-edge pass.  Only
      // non-edge staged values are read, so the results can go straight back
      // into registers (Nx, Ny >= 3).
      const int RHa = T.RHa, RWa = T.RWa;
      auto X = [&](int r, int cc) -> float {
        const int gi = ri0 + r;
        if (gi == 0) return fadd(S.sp[1][cc], fmul(mx, fsub(S.sc[1][cc], S.sp[0][cc])));
        if (gi == nx - 1)
          return fadd(S.sp[RHa - 2][cc], fmul(mx, fsub(S.sc[RHa - 2][cc], S.sp[RHa - 1][cc])));
        return S.sc[r][cc];
      };
      if (colv) {
#pragma unroll
        for (int q = 0; q < R; ++q) {
          const int r = r0 + q, gi = ri0 + r;
          if (r >= RHa) continue;
          if (gj == 0) hz[q] = fadd(S.sp[r][1], fmul(my, fsub(X(r, 1), S.sp[r][0])));
          else if (gj == ny - 1)
            hz[q] = fadd(S.sp[r][RWa - 2], fmul(my, fsub(X(r, RWa - 2), S.sp[r][RWa - 1])));
          else if (gi == 0 || gi == nx - 1) hz[q] = X(r, c);
        }
      }
    }

    // exchange for the Ampere update
    if (lane == 31) store_rows<R>(&S.hx[wx][r0], hz);
    S.hr[wy][c] = hz[R - 1];
    __syncthreads();

    // (4) Ampere updates.
#pragma unroll
    for (int q = 0; q < R; ++q) {
      float hl = __shfl_up_sync(0xffffffffu, hz[q], 1);
      if (lane == 0) hl = (wx > 0) ? S.hx[wx - 1][r0 + q] : 0.f;
      float ha;
      if (q > 0) ha = hz[q - 1];
      else ha = (wy > 0) ? S.hr[wy - 1][c] : 0.f;
      const float d1 = divy(fsub(hz[q], hl));
      const float d2 = divx(fsub(hz[q], ha));
      const float nex = MAT ? fadd(fmul(ca[q], ex[q]), fmul(cb[q], d1)) : fadd(ex[q], fmul(de, d1));
      const float ney = MAT ? fsub(fmul(ca[q], ey[q]), fmul(cb[q], d2)) : fsub(ey[q], fmul(de, d2));
      if (EDGE) {
        const int gi = ri0 + r0 + q;
        ex[q] = ex_col ? nex : ex[q];
        ey[q] = (gi >= 1) ? ney : ey[q];
      } else {
        ex[q] = nex;
        ey[q] = ney;
      }
    }

    // (5) detectors and stability maxima.
    if (T.pown0 >= 0) {
      auto sample = [&](int code) -> float {
        const int rr = code / 3, cmp = code % 3;
        float v = 0.f;
#pragma unroll
        for (int q = 0; q < R; ++q)
          if (q == rr) v = cmp == 0 ? ex[q] : (cmp == 1 ? ey[q] : hz[q]);
        return v;
      };
      P.traces[(long long)T.pown0 * P.trace_ld + (n - P.trace_step0)] = sample(T.pq0);
      if (T.pown1 >= 0)
        P.traces[(long long)T.pown1 * P.trace_ld + (n - P.trace_step0)] = sample(T.pq1);
      if (T.pslow) {
        for (int s = 0; s < T.np; ++s) {
          const int id = S.p[s];
          if (id == T.pown0 || id == T.pown1) continue;
          const wf_probe& pr = P.prb[id];
          const int rr = pr.i - ri0 - r0;
          if (pr.j == gj && rr >= 0 && rr < R)
            P.traces[(long long)id * P.trace_ld + (n - P.trace_step0)] =
                sample(rr * 3 + (pr.comp == WF_HZ ? 2 : pr.comp));
        }
      }
    }
    if (P.check_max != nullptr && P.n_check > 0 && (n + 1) % P.n_check == 0) {
      unsigned m0 = 0, m1 = 0, m2 = 0;
      if (gj >= T.cj0 && gj < T.cj1) {
#pragma unroll
        for (int q = 0; q < R; ++q) {
          const int gi = ri0 + r0 + q;
          if (gi >= T.ci0 && gi < T.ci1) {
            m0 = max(m0, abs_bits(ex[q]));
            m1 = max(m1, abs_bits(ey[q]));
            m2 = max(m2, abs_bits(hz[q]));
          }
        }
      }
      for (int sh = 16; sh > 0; sh >>= 1) {
        m0 = max(m0, __shfl_xor_sync(0xffffffffu, m0, sh));
        m1 = max(m1, __shfl_xor_sync(0xffffffffu, m1, sh));
        m2 = max(m2, __shfl_xor_sync(0xffffffffu, m2, sh));
      }
      if (lane == 0) {
        atomicMax(&S.bmax[0], m0);
        atomicMax(&S.bmax[1], m1);
        atomicMax(&S.bmax[2], m2);
      }
      __syncthreads();
      if (threadIdx.x < 3) {
        const int idx = (n + 1) / P.n_check - P.check_base - 1;
        atomicMax(&P.check_max[idx * 3 + threadIdx.x], S.bmax[threadIdx.x]);
        S.bmax[threadIdx.x] = 0u;
      }
    }
  }
}

template <class C, bool MAT, bool FDIV>
__device__ void tile2d(const Tile2D& P, int ci0, int ci1, int cj0, int cj1, int step0, int k,
                       TileSmem<C>& S) {
  constexpr int R = C::R, WX = C::WX;
  const int nx = P.nx, ny = P.ny;
  TileCtx T;
  T.ci0 = ci0;
  T.ci1 = ci1;
  T.cj0 = cj0;
  T.cj1 = cj1;
  T.ri0 = max(ci0 - k, 0);
  T.ri1 = min(ci1 + k, nx);
  T.rj0 = max(cj0 - k, 0);
  T.rj1 = min(cj1 + k, ny);
  T.RHa = T.ri1 - T.ri0;
  T.RWa = T.rj1 - T.rj0;
  const int tid = threadIdx.x;
  T.lane = tid & 31;
  const int warp = tid >> 5;
  T.wx = warp % WX;
  T.wy = warp / WX;
  T.c = T.wx * 32 + T.lane;
  T.r0 = T.wy * R;
  T.gj = T.rj0 + T.c;
  const int ri0 = T.ri0, ri1 = T.ri1, rj0 = T.rj0, rj1 = T.rj1, r0 = T.r0, gj = T.gj;

  // ---- local source / probe lists ------------------------------------------
  if (tid == 0) {
    int nh = 0, ne = 0;
    for (int s = 0; s < P.nsrc; ++s) {
      const wf_source& Q = P.src[s];
      if (Q.i1 <= ri0 || Q.i0 >= ri1 || Q.j1 <= rj0 || Q.j0 >= rj1) continue;
      if (Q.comp == WF_HZ) {
        if (nh < kMaxLocalSrc) S.h[nh++] = (short)s;
        else if (P.status) atomicExch(P.status, WF_E_LIMIT);
      } else {
        if (ne < kMaxLocalSrc) S.e[ne++] = (short)s;
        else if (P.status) atomicExch(P.status, WF_E_LIMIT);
      }
    }
    S.nh = nh;
    S.ne = ne;
    S.np = 0;
    S.bmax[0] = S.bmax[1] = S.bmax[2] = 0u;
  }
  __syncthreads();
  for (int q = tid; q < P.nprb; q += C::THREADS) {
    const wf_probe& pr = P.prb[q];
    if (pr.i >= ci0 && pr.i < ci1 && pr.j >= cj0 && pr.j < cj1) {
      const int slot = atomicAdd(&S.np, 1);
      if (slot < kMaxLocalProbe) S.p[slot] = (short)q;
      else if (P.status) atomicExch(P.status, WF_E_LIMIT);
    }
  }

  // ---- load own cells ----------------------------------------------------
  float ex[R], ey[R], hz[R], ca[R], cb[R];
  const bool colv = T.c < T.RWa;
#pragma unroll
  for (int q = 0; q < R; ++q) {
    const int r = r0 + q;
    ex[q] = ey[q] = hz[q] = 0.f;
    ca[q] = cb[q] = 0.f;
    if (colv && r < T.RHa) {
      const long long g = (long long)(ri0 + r) * ny + gj;
      ex[q] = P.ex_in[g];
      ey[q] = P.ey_in[g];
      hz[q] = P.hz_in[g];
      if (MAT) {
        ca[q] = P.ca[g];
        cb[q] = P.cb[g];
      }
    }
  }
  __syncthreads();
  T.nh = S.nh;
  T.ne = S.ne;
  T.np = min(S.np, kMaxLocalProbe);
  // Does any local source touch this thread's column segment?
  T.my_h = false;
  T.my_e = false;
  for (int q = 0; q < T.nh; ++q) {
    const wf_source& Q = P.src[S.h[q]];
    T.my_h |= gj >= Q.j0 && gj < Q.j1 && ri0 + r0 < Q.i1 && ri0 + r0 + R > Q.i0;
  }
  for (int q = 0; q < T.ne; ++q) {
    const wf_source& Q = P.src[S.e[q]];
    T.my_e |= gj >= Q.j0 && gj < Q.j1 && ri0 + r0 < Q.i1 && ri0 + r0 + R > Q.i0;
  }
  // Probes owned by this thread (up to two in registers, else the slow path).
  T.pown0 = T.pown1 = -1;
  T.pq0 = T.pq1 = 0;
  T.pslow = false;
  for (int q = 0; q < T.np; ++q) {
    const wf_probe& pr = P.prb[S.p[q]];
    const int rr = pr.i - ri0 - r0;
    if (pr.j == gj && rr >= 0 && rr < R) {
      const int code = rr * 3 + (pr.comp == WF_HZ ? 2 : pr.comp);
      if (T.pown0 < 0) {
        T.pown0 = S.p[q];
        T.pq0 = code;
      } else if (T.pown1 < 0) {
        T.pown1 = S.p[q];
        T.pq1 = code;
      } else {
        T.pslow = true;
      }
    }
  }
  const bool edge_tile = (ri0 == 0) || (ri1 == nx) || (rj0 == 0) || (rj1 == ny);
  if (edge_tile) tile2d_steps<C, MAT, FDIV, true>(P, T, S, ex, ey, hz, ca, cb, step0, k);
  else tile2d_steps<C, MAT, FDIV, false>(P, T, S, ex, ey, hz, ca, cb, step0, k);

  // ---- store core ----------------------------------------------------------
  if (gj >= cj0 && gj < cj1) {
#pragma unroll
    for (int q = 0; q < R; ++q) {
      const int gi = ri0 + r0 + q;
      if (gi >= ci0 && gi < ci1) {
        const long long g = (long long)gi * ny + gj;
        P.ex_out[g] = ex[q];
        P.ey_out[g] = ey[q];
        P.hz_out[g] = hz[q];
      }
    }
  }
  __syncthreads();
}

}  // namespace wf
