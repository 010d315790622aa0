// fdtd3d_tma.cuh -- k3d_tma: the single-step 3D streaming pass with its
// i-planes staged in shared memory by the Tensor Memory Accelerator.
// Included by fdtd3d.cu (uses Tile3D, Lists3D, dv<>, src3_value).
//
// A CTA of 16 (j) x 32 (k) threads owns a block of columns -- a 15 x 30 core
// behind a one-cell halo at j - 1, k - 1 and k + 1 -- and walks an i-segment
// exactly like k3d_stream, with the same float ops in the same order (so the
// two are bit-identical).  What changes is data movement: one thread issues,
// per i-plane, one cp.async.bulk.tensor load per array (Ex, Ey, Ez, Hx, Hy, Hz
// and Ca, Cb) of a 17 x 36 box (one j-row more than the threads: the E of the
// last thread row's j + 1 neighbours) into a 4-slot shared-memory ring,
// completing on the slot's
// mbarrier.  A thread keeps E, Ca and Cb of its cell of plane f in registers
// from the Faraday step of that plane, so plane f's slot is refilled with
// plane f + 4 as soon as the plane-f step starts (after the Mur code on face
// planes): planes f + 3 and f + 4 are in flight while plane f is finished.  All
// neighbours (j +- 1, k +- 1, i +- 1) are read from shared memory, so no
// thread issues global loads, shuffles or address arithmetic for them.  The
// box starts at k = floor4(k0 - 1) (a TMA box must start on a 16-byte
// boundary); lanes read column lane + (k0 - 1 - floor4(k0 - 1)).
// Curl-updated H of planes f and f+1 live in shared rows for the Mur faces and
// the Ampere neighbours (the final H of plane f too, on x-face planes).
// Interior planes run with the ring slots fixed at compile time (halo threads
// compute and do not store): straight-line in column blocks that touch no
// domain face, with the neighbour tests as selects in blocks on a j or k face,
// whose face cells correct H in place between the Faraday and Ampere halves.  Every mbarrier wait is bounded: after the limit the CTA records
// WF_E_TIMEOUT, waits (bounded) for the copies it still has in flight, and
// stops.
#pragma once

#include <cuda.h>

#include <type_traits>

namespace wf {

// 16 thread rows (j) x 32 lanes (k); row 0 and lanes 0, 31 are halo.  The box
// holds one more row (16) than the threads: the E of row 16 completes the curl
// of row 15, which makes rows 1..15 core (15 per block instead of 14).
constexpr int kTJ = 16, kTK = 32, kTCJ = kTJ - 1, kTCK = kTK - 2;
constexpr int kBoxJ = kTJ + 1;                  // box height in j
constexpr int kBoxK = 36;                       // box width in k (>= 32 + 3 + 1)
constexpr int kRing = 4;                        // i-plane slots
constexpr int kBoxF = kBoxJ * kBoxK;            // floats one box load writes
constexpr int kTileF = (kBoxF + 31) / 32 * 32;  // floats per array per slot (128-byte aligned)
constexpr int kSlotF = 8 * kTileF;              // floats per slot
constexpr int kHcF = kTJ * kTK;                 // floats per H row set component
constexpr int kHcSetF = 3 * kHcF;               // floats per plane of hc
constexpr unsigned kSpinLimit = 1u << 22;       // bounded mbarrier wait

struct TmaMaps {
  CUtensorMap m[8];  // Ex, Ey, Ez, Hx, Hy, Hz (pass input), Ca, Cb
};

struct TmaSmem {
  float raw[kRing][8][kTileF];      // slot, array, row * kBoxK + column
  float hc[2][3][kTJ][kTK];         // curl-updated H of planes (p mod 2)
  float hf[3][kTJ][kTK];            // final H of plane f
  float hom[2][kTJ][kTK];           // old Hy, Hz of plane Nx-2 (x face at Nx-1)
  unsigned long long bar[kRing];
  Lists3D L;
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned long long* b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}

// One 4D tile load {k, j, i, instance} into shared memory, completing on b.
__device__ __forceinline__ void tma_load4(void* dst, const CUtensorMap* map, int c0, int c1,
                                          int c2, int c3, unsigned long long* b) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3),
      "r"(smem_u32(b))
      : "memory");
}

// Non-blocking look at the slot's phase (mbarrier.test_wait never suspends).
__device__ __forceinline__ bool mbar_test_wait(unsigned long long* b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Wait for the phase `parity` of mbarrier b: one non-blocking look, then at
// most `limit` hardware-suspended polls.  False = gave up (the copies it
// waits for may still be in flight).
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* b, unsigned parity,
                                                  unsigned limit) {
  if (mbar_test_wait(b, parity)) return true;
  for (unsigned spin = 0; spin < limit; ++spin)
    if (mbar_try_wait(b, parity)) return true;
  return false;
}

// wait_limit bounds every wait of the plane pipeline (kSpinLimit in normal
// use; a smaller value only makes the CTA give up sooner).  The final wait
// for the copies still in flight after a give-up always uses kSpinLimit.
template <bool MAT, bool FDIV>
__global__ void __launch_bounds__(kTJ * kTK, 2) k3d_tma(const __grid_constant__ TmaMaps maps,
                                                        Tile3D P, int tiles_j, int tiles_k,
                                                        int seg_len, int n, int* status,
                                                        unsigned wait_limit) {
  extern __shared__ __align__(128) unsigned char smraw3[];
  TmaSmem& S = *reinterpret_cast<TmaSmem*>(smraw3);
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  int b = blockIdx.x;
  const int tk = b % tiles_k;
  b /= tiles_k;
  const int tj = b % tiles_j, seg = b / tiles_j;
  const int inst = blockIdx.y;
  if (inst) {
    const long long q = inst;
    P.traces += q * P.tstride;
    P.src += q * P.sstride;
  }
  const int ci_inst = P.cstride ? inst : 0;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, tid = threadIdx.x;
  const int j0 = tj * kTCJ - 1, k0 = tk * kTCK - 1;  // region origin (halo included)
  const int kb = k0 >= 0 ? (k0 & ~3) : -(((-k0) + 3) & ~3);  // floor to a multiple of 4
  const int cofs = k0 - kb;                                   // 0..3
  const int gj = j0 + w, gk = k0 + lane;
  const bool in = gj >= 0 && gj < ny && gk >= 0 && gk < nz;
  const bool core = in && w >= 1 && w <= kTCJ && lane >= 1 && lane <= kTCK;
  const int col = lane + cofs;
  const int ia = seg * seg_len, ib = min(nx, ia + seg_len);
  if (ia >= ib) return;
  const int f0 = max(ia - 1, 0);
  const int plast = min(nx - 1, ib + 1);  // last plane the segment reads
  const long long PS = (long long)ny * nz;
  // output offset of this column, instance included (P.out stays unmodified)
  const long long colg = (in ? (long long)gj * nz + gk : 0) + (long long)inst * P.fstride;
  // element offsets fit 32 bits: an array of 2^32 floats (16 GiB) times the
  // 14 arrays a launch touches would exceed the device memory
  const unsigned colg32 = (unsigned)colg, PS32 = (unsigned)PS;
  const float dh = P.dh, de = P.de, dx = P.dx, dy = P.dy, dz = P.dz;
  const float mx = P.mx, my = P.my, mz = P.mz;
  const double rdx = __drcp_rn((double)dx), rdy = __drcp_rn((double)dy),
               rdz = __drcp_rn((double)dz);
  const int narr = MAT ? 8 : 6;
  const unsigned bytes = (unsigned)(narr * kBoxF * sizeof(float));  // what the loads deliver

  if (tid == 0) {
    for (int s = 0; s < kRing; ++s) mbar_init(&S.bar[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    int nh = 0, ne = 0;
    for (int q = 0; q < P.nsrc; ++q) {
      const wf_source& Q = P.src[q];
      if (Q.i1 <= f0 || Q.i0 > plast || Q.j1 <= j0 || Q.j0 >= j0 + kBoxJ || Q.k1 <= k0 ||
          Q.k0 >= k0 + kTK)
        continue;
      if (Q.comp >= WF_HX) {
        if (nh < kMaxLocalSrc3) S.L.h[nh++] = (short)q;
      } else {
        if (ne < kMaxLocalSrc3) S.L.e[ne++] = (short)q;
      }
    }
    S.L.nh = nh;
    S.L.ne = ne;
    S.L.np = 0;
    for (int c = 0; c < 6; ++c) S.L.bmax[c] = 0u;
  }
  __syncthreads();
  for (int q = tid; q < P.nprb; q += blockDim.x) {
    const wf_probe& pr = P.prb[q];
    if (pr.i >= ia && pr.i < ib && pr.j >= j0 + 1 && pr.j < j0 + 1 + kTCJ && pr.k >= k0 + 1 &&
        pr.k < k0 + 1 + kTCK) {
      const int slot = atomicAdd(&S.L.np, 1);
      if (slot < kMaxLocalProbe3) S.L.p[slot] = (short)q;
    }
  }
  const int ne = S.L.ne, nh = S.L.nh;
  const bool check = P.check_max != nullptr && P.n_check > 0 && (n + 1) % P.n_check == 0;
  __syncthreads();  // the probe list is complete
  // CTAs with no source, probe or stability check of their own (the vast
  // majority) run a specialisation without that code
  const bool lists = ne > 0 || nh > 0 || S.L.np > 0 || check;
  auto body = [&](auto lists_tag) {
  constexpr bool LISTS = decltype(lists_tag)::value;

  unsigned pending = 0u;  // thread 0: slots with copies issued and not yet landed
  auto issue = [&](int p) {  // thread 0 only
    const int s = p % kRing;
    pending |= 1u << s;
    // the slot may hold source values written by ordinary stores: order them
    // before the asynchronous-proxy overwrite
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(&S.bar[s], bytes);
    for (int c = 0; c < 6; ++c) tma_load4(&S.raw[s][c][0], &maps.m[c], kb, j0, p, inst, &S.bar[s]);
    if (MAT) {
      tma_load4(&S.raw[s][6][0], &maps.m[6], kb, j0, p, ci_inst, &S.bar[s]);
      tma_load4(&S.raw[s][7][0], &maps.m[7], kb, j0, p, ci_inst, &S.bar[s]);
    }
  };
  unsigned phase = 0u;  // parity bit per slot
  bool failed = false;
  // Wait for plane p, then add this CTA's E-source values into it: each
  // thread to its own cell, the last thread row also to the box's extra row.
  const bool in16 = w == kTJ - 1 && gj + 1 < ny && gk >= 0 && gk < nz;
  // A wait that gives up leaves the slot's phase bit unflipped (so the drain
  // below waits for the copy actually outstanding) and injects nothing.
  auto land = [&](int p) {
    const int s = p % kRing;
    if (failed) return;
    if (!mbar_wait_bounded(&S.bar[s], (phase >> s) & 1u, wait_limit)) {
      failed = true;
      if (status != nullptr) atomicExch(status, WF_E_TIMEOUT);
      return;
    }
    phase ^= 1u << s;
    pending &= ~(1u << s);
    if (LISTS && ne > 0 && (in || in16)) {
      for (int q = 0; q < ne; ++q) {
        const wf_source& Q = P.src[S.L.e[q]];
        if (p < Q.i0 || p >= Q.i1 || gk < Q.k0 || gk >= Q.k1) continue;
        if (in && gj >= Q.j0 && gj < Q.j1) {
          float& cell = S.raw[s][Q.comp][w * kBoxK + col];
          cell = fadd(cell, src3_value(Q, p, gj, gk, n));
        }
        if (in16 && gj + 1 >= Q.j0 && gj + 1 < Q.j1) {
          float& cell = S.raw[s][Q.comp][kTJ * kBoxK + col];
          cell = fadd(cell, src3_value(Q, p, gj + 1, gk, n));
        }
      }
    }
  };

  // Per-thread shared-memory bases: slot arrays are addressed as
  // R[c * kTileF] (+ kBoxK for j + 1, + 1 for k + 1), H rows as Hrow[c * kHcF].
  float* const raw0 = &S.raw[0][0][0] + (w * kBoxK + col);
  float* const hc0 = &S.hc[0][0][0][0] + (w * kTK + lane);
  const bool cjk = gj < ny - 1 && gk < nz - 1, ck = gk < nz - 1, cj = gj < ny - 1;
  // a block none of whose cells lies on a j or k face needs the Mur code only
  // on the planes i = 0 and i = Nx - 1
  const bool face_blk = !(j0 >= 1 && j0 + kTJ - 1 <= ny - 2 && k0 >= 1 && k0 + kTK - 1 <= nz - 2);
  // j/k face cells of this thread (the in-place face path needs the cells
  // next to a face to be off every face: ny, nz >= 4)
  const bool lite_ok = ny >= 4 && nz >= 4;
  const bool on_face = (gj == 0 || gj == ny - 1) || (nz > 1 && in && (gk == 0 || gk == nz - 1));
  // carried between planes: Ey, Ez of plane p (read as the i + 1 neighbours
  // of plane p - 1), E, Ca, Cb of the plane being finished, curl-updated H
  float cey = 0.f, cez = 0.f, cca = 0.f, ccb = 0.f;
  F3 ecur{0.f, 0.f, 0.f}, hcur{0.f, 0.f, 0.f};

  // Faraday update of plane p into S.hc[p % 2] (all region cells); E, Ca, Cb
  // of plane p are left in ecur, cca, ccb, the curl-updated H in hcur.
  auto curl = [&](int p, bool first) {
    const float* R = raw0 + (p & (kRing - 1)) * kSlotF;
    const float* R1 = raw0 + ((p + 1) & (kRing - 1)) * kSlotF;
    const float ex = R[0];
    const float ey = first ? R[kTileF] : cey;
    const float ez = first ? R[2 * kTileF] : cez;
    // row w + 1 of the last row and plane p + 1 of the last plane read
    // in-bounds values that only feed results nobody uses
    const float ex_j = R[kBoxK], ez_j = R[2 * kTileF + kBoxK];
    const float ex_k = R[1], ey_k = R[kTileF + 1];
    const float ey_i = R1[kTileF], ez_i = R1[2 * kTileF];
    float vx = R[3 * kTileF], vy = R[4 * kTileF], vz = R[5 * kTileF];
    for (int q = 0; LISTS && q < nh; ++q) {
      const wf_source& Q = P.src[S.L.h[q]];
      if (p >= Q.i0 && p < Q.i1 && gj >= Q.j0 && gj < Q.j1 && gk >= Q.k0 && gk < Q.k1) {
        const float v = src3_value(Q, p, gj, gk, n);
        if (Q.comp == WF_HX) vx = fadd(vx, v);
        else if (Q.comp == WF_HY) vy = fadd(vy, v);
        else vz = fadd(vz, v);
      }
    }
    // every operand read below lies inside the staged boxes, so the three
    // updates run unconditionally and cells without the neighbour keep the
    // old value (a select, no branch)
    const bool il = p < nx - 1;
    {
      const float t1 = dv<FDIV>(fsub(ey_k, ey), dz, rdz);
      const float t2 = dv<FDIV>(fsub(ez_j, ez), dy, rdy);
      const float v = fadd(vx, fmul(dh, fsub(t1, t2)));
      vx = cjk ? v : vx;
    }
    {
      const float t1 = dv<FDIV>(fsub(ez_i, ez), dx, rdx);
      const float t2 = dv<FDIV>(fsub(ex_k, ex), dz, rdz);
      const float v = fadd(vy, fmul(dh, fsub(t1, t2)));
      vy = (il && ck) ? v : vy;
    }
    {
      const float t1 = dv<FDIV>(fsub(ex_j, ex), dy, rdy);
      const float t2 = dv<FDIV>(fsub(ey_i, ey), dx, rdx);
      const float v = fadd(vz, fmul(dh, fsub(t1, t2)));
      vz = (il && cj) ? v : vz;
    }
    float* H = hc0 + (p & 1) * kHcSetF;
    H[0] = vx;
    H[kHcF] = vy;
    H[2 * kHcF] = vz;
    ecur = F3{ex, ey, ez};
    hcur = F3{vx, vy, vz};
    if (MAT) {
      cca = R[6 * kTileF];
      ccb = R[7 * kTileF];
    }
    cey = ey_i;
    cez = ez_i;
  };

  // ---- prologue ---------------------------------------------------------------
  if (tid == 0) {
    for (int p = f0; p <= min(f0 + kRing - 1, plast); ++p) issue(p);
  }
  land(f0);
  if (f0 + 1 <= plast) land(f0 + 1);
  failed = __syncthreads_or(failed) != 0;
  if (!failed) curl(f0, true);
  F3 hprev{0.f, 0.f, 0.f};
  unsigned mxb[6] = {0u, 0u, 0u, 0u, 0u, 0u};
  const bool chk = LISTS && check;
  const bool zf_on = nz > 1;

  for (int f = f0; f < ib && !failed; ++f) {
    const int p = f + 1;
    if (f + 2 <= plast) land(f + 2);
    // A: injections and hc(f) visible; a timed-out wait anywhere stops the
    // whole CTA
    failed = __syncthreads_or(failed) != 0;
    if (failed) break;
    const bool face = face_blk || f == 0 || f == nx - 1;  // uniform over the CTA
    // j/k faces only (no x face on this plane, and plane f is not the one the
    // x face at Nx-1 reads): face cells fix their H in place in hc(f)
    const bool face_lite = lite_ok && f >= 1 && f + 2 < nx;
    // plane f's slot takes plane f + 4 once nothing reads it: right after
    // barrier A (Ca, Cb and E of plane f are in registers; the old H of plane
    // Nx - 2 is read below, but no plane is issued then) unless the Mur code
    // reads plane f's old H, then after barrier C
    if (!face && tid == 0 && f + kRing <= plast) issue(f + kRing);
    // Interior plane, no sources / probes / check: the update runs with the
    // ring slots fixed at compile time; halo threads compute too and only
    // core threads store.  In a column block off every face (FB false) every
    // neighbour exists, so it is straight-line; a block on a j or k face (FB)
    // keeps each cell's neighbour tests as selects and corrects its face
    // cells in place between the Faraday and the Ampere halves.
    if (!LISTS && f >= ia && f >= 1 && f + 2 < nx && (!face_blk || lite_ok)) {
     auto fastp = [&](auto s_tag, auto fb_tag) {
      constexpr int SF = decltype(s_tag)::value;  // f & 3
      constexpr bool FB = decltype(fb_tag)::value;
      const float* R = raw0 + ((SF + 1) & (kRing - 1)) * kSlotF;
      const float* R1 = raw0 + ((SF + 2) & (kRing - 1)) * kSlotF;
      const float ex = R[0], ey = cey, ez = cez;
      const float ex_j = R[kBoxK], ez_j = R[2 * kTileF + kBoxK];
      const float ex_k = R[1], ey_k = R[kTileF + 1];
      const float ey_i = R1[kTileF], ez_i = R1[2 * kTileF];
      float vx = R[3 * kTileF], vy = R[4 * kTileF], vz = R[5 * kTileF];
      {
        const float nx_ = fadd(vx, fmul(dh, fsub(dv<FDIV>(fsub(ey_k, ey), dz, rdz), dv<FDIV>(fsub(ez_j, ez), dy, rdy))));
        const float ny_ = fadd(vy, fmul(dh, fsub(dv<FDIV>(fsub(ez_i, ez), dx, rdx), dv<FDIV>(fsub(ex_k, ex), dz, rdz))));
        const float nz_ = fadd(vz, fmul(dh, fsub(dv<FDIV>(fsub(ex_j, ex), dy, rdy), dv<FDIV>(fsub(ey_i, ey), dx, rdx))));
        vx = (!FB || cjk) ? nx_ : vx;
        vy = (!FB || ck) ? ny_ : vy;   // p < nx - 1 holds on these planes
        vz = (!FB || cj) ? nz_ : vz;
      }
      float* H = hc0 + ((SF + 1) & 1) * kHcSetF;
      H[0] = vx;
      H[kHcF] = vy;
      H[2 * kHcF] = vz;
      float hxF = hcur.x, hyF = hcur.y, hzF = hcur.z;
      if constexpr (FB) {
        // Mur y and z faces of plane f, in place (as the general face path):
        // face cells read hc(f) and plane f's old H, a barrier, then write
        // their final H over hc(f); plane f's slot is refilled after that
        auto Ho = [&](int c, int ww, int ll) -> float {
          return S.raw[SF][3 + c][ww * kBoxK + ll + cofs];
        };
        auto Hc = [&](int c, int ww, int ll) -> float { return S.hc[SF & 1][c][ww][ll]; };
        auto yfx = [&](int ww, int ll) -> float {
          const int g = j0 + ww;
          if (g == 0 && ww + 1 < kTJ) return fadd(Ho(0, ww + 1, ll), fmul(my, fsub(Hc(0, ww + 1, ll), Ho(0, ww, ll))));
          if (g == ny - 1 && ww >= 1) return fadd(Ho(0, ww - 1, ll), fmul(my, fsub(Hc(0, ww - 1, ll), Ho(0, ww, ll))));
          return Hc(0, ww, ll);
        };
        if (on_face) {
          if (gj == 0 && w + 1 < kTJ) {
            hxF = fadd(Ho(0, w + 1, lane), fmul(my, fsub(Hc(0, w + 1, lane), Ho(0, w, lane))));
            hzF = fadd(Ho(2, w + 1, lane), fmul(my, fsub(Hc(2, w + 1, lane), Ho(2, w, lane))));
          } else if (gj == ny - 1 && w >= 1) {
            hxF = fadd(Ho(0, w - 1, lane), fmul(my, fsub(Hc(0, w - 1, lane), Ho(0, w, lane))));
            hzF = fadd(Ho(2, w - 1, lane), fmul(my, fsub(Hc(2, w - 1, lane), Ho(2, w, lane))));
          }
          if (zf_on && in) {
            if (gk == 0 && lane + 1 < kTK) {
              hxF = fadd(Ho(0, w, lane + 1), fmul(mz, fsub(yfx(w, lane + 1), Ho(0, w, lane))));
              hyF = fadd(Ho(1, w, lane + 1), fmul(mz, fsub(Hc(1, w, lane + 1), Ho(1, w, lane))));
            } else if (gk == nz - 1 && lane >= 1) {
              hxF = fadd(Ho(0, w, lane - 1), fmul(mz, fsub(yfx(w, lane - 1), Ho(0, w, lane))));
              hyF = fadd(Ho(1, w, lane - 1), fmul(mz, fsub(Hc(1, w, lane - 1), Ho(1, w, lane))));
            }
          }
        }
        __syncthreads();  // every correction has read what it needs
        if (on_face) {
          S.hc[SF & 1][0][w][lane] = hxF;
          S.hc[SF & 1][1][w][lane] = hyF;
          S.hc[SF & 1][2][w][lane] = hzF;
        }
        __syncthreads();  // C: final H of plane f visible; plane f's slot unread
        if (tid == 0 && f + kRing <= plast) issue(f + kRing);
      }
      // Ampere of plane f from the final H of plane f
      const float* N = hc0 + (SF & 1) * kHcSetF;
      const float hz_j = N[2 * kHcF - kTK], hx_j = N[-kTK];
      const float hy_k = N[kHcF - 1], hx_k = N[-1];
      const float t1 = fsub(dv<FDIV>(fsub(hzF, hz_j), dy, rdy), dv<FDIV>(fsub(hyF, hy_k), dz, rdz));
      const float t2 = fsub(dv<FDIV>(fsub(hxF, hx_k), dz, rdz), dv<FDIV>(fsub(hzF, hprev.z), dx, rdx));
      const float t3 = fsub(dv<FDIV>(fsub(hyF, hprev.y), dx, rdx), dv<FDIV>(fsub(hxF, hx_j), dy, rdy));
      float exn = MAT ? fadd(fmul(cca, ecur.x), fmul(ccb, t1)) : fadd(ecur.x, fmul(de, t1));
      float eyn = MAT ? fadd(fmul(cca, ecur.y), fmul(ccb, t2)) : fadd(ecur.y, fmul(de, t2));
      const float ezn = MAT ? fadd(fmul(cca, ecur.z), fmul(ccb, t3)) : fadd(ecur.z, fmul(de, t3));
      if (FB) {  // f >= 1 here, so only the j and k tests remain
        exn = (gj >= 1 && gk >= 1) ? exn : ecur.x;
        eyn = gk >= 1 ? eyn : ecur.y;
      }
      const float ezf = (!FB || gj >= 1) ? ezn : ecur.z;
      if (core) {
        const unsigned o = (unsigned)f * PS32 + colg32;
        P.out[0][o] = exn;
        P.out[1][o] = eyn;
        P.out[2][o] = ezf;
        P.out[3][o] = hxF;
        P.out[4][o] = hyF;
        P.out[5][o] = hzF;
      }
      hprev = F3{hxF, hyF, hzF};
      ecur = F3{ex, ey, ez};
      hcur = F3{vx, vy, vz};
      if (MAT) {
        cca = R[6 * kTileF];
        ccb = R[7 * kTileF];
      }
      cey = ey_i;
      cez = ez_i;
     };
      if (face_blk) {
        switch (f & 3) {
          case 0: fastp(std::integral_constant<int, 0>{}, std::true_type{}); break;
          case 1: fastp(std::integral_constant<int, 1>{}, std::true_type{}); break;
          case 2: fastp(std::integral_constant<int, 2>{}, std::true_type{}); break;
          default: fastp(std::integral_constant<int, 3>{}, std::true_type{}); break;
        }
      } else {
        switch (f & 3) {
          case 0: fastp(std::integral_constant<int, 0>{}, std::false_type{}); break;
          case 1: fastp(std::integral_constant<int, 1>{}, std::false_type{}); break;
          case 2: fastp(std::integral_constant<int, 2>{}, std::false_type{}); break;
          default: fastp(std::integral_constant<int, 3>{}, std::false_type{}); break;
        }
      }
      continue;
    }
    const F3 ef = ecur;  // E of plane f (sources included)
    const float cav = cca, cbv = ccb;
    float hxF = hcur.x, hyF = hcur.y, hzF = hcur.z;
    if (p < nx) curl(p, false);
    const int sf = f & (kRing - 1), hf0 = f & 1;
    auto Ho = [&](int c, int ww, int ll) -> float { return S.raw[sf][3 + c][ww * kBoxK + ll + cofs]; };
    if (f == nx - 2) {
      S.hom[0][w][lane] = Ho(1, w, lane);
      S.hom[1][w][lane] = Ho(2, w, lane);
    }
    const float* Hn;  // final H of plane f, row-major [3][kTJ][kTK]
    if (face && !face_lite) {
      __syncthreads();  // B: hc(p) visible
      // ---- Mur faces of plane f, as pure functions of old and curl-updated H ----
      const int sp = p & (kRing - 1), hp = p & 1, hm = (f + 1) & 1;
      auto Hc = [&](int c, int ww, int ll) -> float { return S.hc[hf0][c][ww][ll]; };
      // Hy, Hz after the x faces
      auto xf = [&](int c, int ww, int ll) -> float {
        if (f == 0) return fadd(S.raw[sp][3 + c][ww * kBoxK + ll + cofs],
                                fmul(mx, fsub(S.hc[hp][c][ww][ll], Ho(c, ww, ll))));
        if (f == nx - 1) return fadd(S.hom[c - 1][ww][ll], fmul(mx, fsub(S.hc[hm][c][ww][ll], Ho(c, ww, ll))));
        return Hc(c, ww, ll);
      };
      // Hx after the y faces (Hx has no x face)
      auto yfx = [&](int ww, int ll) -> float {
        const int g = j0 + ww;
        if (g == 0 && ww + 1 < kTJ) return fadd(Ho(0, ww + 1, ll), fmul(my, fsub(Hc(0, ww + 1, ll), Ho(0, ww, ll))));
        if (g == ny - 1 && ww >= 1) return fadd(Ho(0, ww - 1, ll), fmul(my, fsub(Hc(0, ww - 1, ll), Ho(0, ww, ll))));
        return Hc(0, ww, ll);
      };
      hxF = yfx(w, lane);
      hyF = xf(1, w, lane);
      hzF = xf(2, w, lane);
      if (gj == 0 && w + 1 < kTJ)
        hzF = fadd(Ho(2, w + 1, lane), fmul(my, fsub(xf(2, w + 1, lane), Ho(2, w, lane))));
      else if (gj == ny - 1 && w >= 1)
        hzF = fadd(Ho(2, w - 1, lane), fmul(my, fsub(xf(2, w - 1, lane), Ho(2, w, lane))));
      if (zf_on && in) {
        if (gk == 0 && lane + 1 < kTK) {
          hxF = fadd(Ho(0, w, lane + 1), fmul(mz, fsub(yfx(w, lane + 1), Ho(0, w, lane))));
          hyF = fadd(Ho(1, w, lane + 1), fmul(mz, fsub(xf(1, w, lane + 1), Ho(1, w, lane))));
        } else if (gk == nz - 1 && lane >= 1) {
          hxF = fadd(Ho(0, w, lane - 1), fmul(mz, fsub(yfx(w, lane - 1), Ho(0, w, lane))));
          hyF = fadd(Ho(1, w, lane - 1), fmul(mz, fsub(xf(1, w, lane - 1), Ho(1, w, lane))));
        }
      }
      S.hf[0][w][lane] = hxF;
      S.hf[1][w][lane] = hyF;
      S.hf[2][w][lane] = hzF;
      __syncthreads();  // C: final H of plane f visible; plane f's slot unread
      if (tid == 0 && f + kRing <= plast) issue(f + kRing);
      Hn = &S.hf[0][0][0];
    } else if (face) {
      // Mur y and z faces of plane f, in place: the face cells read hc(f)
      // and plane f's old H, a barrier, then they write their final H over
      // hc(f).  Plane f is not the plane the x face at Nx-1 reads later
      // (f + 2 < nx), so its curl-updated values are not needed again.
      auto Hc = [&](int c, int ww, int ll) -> float { return S.hc[hf0][c][ww][ll]; };
      auto yfx = [&](int ww, int ll) -> float {
        const int g = j0 + ww;
        if (g == 0 && ww + 1 < kTJ) return fadd(Ho(0, ww + 1, ll), fmul(my, fsub(Hc(0, ww + 1, ll), Ho(0, ww, ll))));
        if (g == ny - 1 && ww >= 1) return fadd(Ho(0, ww - 1, ll), fmul(my, fsub(Hc(0, ww - 1, ll), Ho(0, ww, ll))));
        return Hc(0, ww, ll);
      };
      if (on_face) {
        if (gj == 0 && w + 1 < kTJ) {
          hxF = fadd(Ho(0, w + 1, lane), fmul(my, fsub(Hc(0, w + 1, lane), Ho(0, w, lane))));
          hzF = fadd(Ho(2, w + 1, lane), fmul(my, fsub(Hc(2, w + 1, lane), Ho(2, w, lane))));
        } else if (gj == ny - 1 && w >= 1) {
          hxF = fadd(Ho(0, w - 1, lane), fmul(my, fsub(Hc(0, w - 1, lane), Ho(0, w, lane))));
          hzF = fadd(Ho(2, w - 1, lane), fmul(my, fsub(Hc(2, w - 1, lane), Ho(2, w, lane))));
        }
        if (zf_on && in) {
          if (gk == 0 && lane + 1 < kTK) {
            hxF = fadd(Ho(0, w, lane + 1), fmul(mz, fsub(yfx(w, lane + 1), Ho(0, w, lane))));
            hyF = fadd(Ho(1, w, lane + 1), fmul(mz, fsub(Hc(1, w, lane + 1), Ho(1, w, lane))));
          } else if (gk == nz - 1 && lane >= 1) {
            hxF = fadd(Ho(0, w, lane - 1), fmul(mz, fsub(yfx(w, lane - 1), Ho(0, w, lane))));
            hyF = fadd(Ho(1, w, lane - 1), fmul(mz, fsub(Hc(1, w, lane - 1), Ho(1, w, lane))));
          }
        }
      }
      __syncthreads();  // every correction has read what it needs
      if (on_face) {
        S.hc[hf0][0][w][lane] = hxF;
        S.hc[hf0][1][w][lane] = hyF;
        S.hc[hf0][2][w][lane] = hzF;
      }
      __syncthreads();  // C: final H of plane f visible; plane f's slot unread
      if (tid == 0 && f + kRing <= plast) issue(f + kRing);
      Hn = &S.hc[hf0][0][0][0];
    } else {
      // no face touches this block on this plane: the final H is the
      // curl-updated H, already visible since barrier A
      Hn = &S.hc[hf0][0][0][0];
    }
    // ---- Ampere update and outputs of plane f ----
    {
      // halo threads read neighbours of the row / column before their own
      // (still inside shared memory) and store nothing
      const float* N = Hn + (w * kTK + lane);
      const float hz_j = N[2 * kHcF - kTK], hx_j = N[-kTK];
      const float hy_k = N[kHcF - 1], hx_k = N[-1];
      float ex = ef.x, ey = ef.y, ez = ef.z;
      {
        const float c = fsub(dv<FDIV>(fsub(hzF, hz_j), dy, rdy), dv<FDIV>(fsub(hyF, hy_k), dz, rdz));
        const float v = MAT ? fadd(fmul(cav, ex), fmul(cbv, c)) : fadd(ex, fmul(de, c));
        ex = (gj >= 1 && gk >= 1) ? v : ex;
      }
      {
        const float c = fsub(dv<FDIV>(fsub(hxF, hx_k), dz, rdz), dv<FDIV>(fsub(hzF, hprev.z), dx, rdx));
        const float v = MAT ? fadd(fmul(cav, ey), fmul(cbv, c)) : fadd(ey, fmul(de, c));
        ey = (f >= 1 && gk >= 1) ? v : ey;
      }
      {
        const float c = fsub(dv<FDIV>(fsub(hyF, hprev.y), dx, rdx), dv<FDIV>(fsub(hxF, hx_j), dy, rdy));
        const float v = MAT ? fadd(fmul(cav, ez), fmul(cbv, c)) : fadd(ez, fmul(de, c));
        ez = (f >= 1 && gj >= 1) ? v : ez;
      }
     if (f >= ia && core) {
      const unsigned o = (unsigned)f * PS32 + colg32;
      P.out[0][o] = ex;
      P.out[1][o] = ey;
      P.out[2][o] = ez;
      P.out[3][o] = hxF;
      P.out[4][o] = hyF;
      P.out[5][o] = hzF;
      const int np = LISTS ? min(S.L.np, kMaxLocalProbe3) : 0;
      for (int q = 0; q < np; ++q) {
        const wf_probe& pr = P.prb[S.L.p[q]];
        if (pr.i == f && pr.j == gj && pr.k == gk) {
          const float v = pr.comp == WF_EX ? ex : pr.comp == WF_EY ? ey : pr.comp == WF_EZ ? ez
                        : pr.comp == WF_HX ? hxF : pr.comp == WF_HY ? hyF : hzF;
          P.traces[(long long)S.L.p[q] * P.trace_ld + (n - P.trace_step0)] = v;
        }
      }
      if (chk) {
        mxb[0] = max(mxb[0], abs_bits(ex));
        mxb[1] = max(mxb[1], abs_bits(ey));
        mxb[2] = max(mxb[2], abs_bits(ez));
        mxb[3] = max(mxb[3], abs_bits(hxF));
        mxb[4] = max(mxb[4], abs_bits(hyF));
        mxb[5] = max(mxb[5], abs_bits(hzF));
      }
     }
    }
    hprev = F3{hxF, hyF, hzF};
  }
  // without a give-up every issued plane has been landed (planes up to plast
  // are landed in the loop); after one, thread 0 waits out the copies it
  // issued that have not landed (its phase bits still name their phases),
  // with the full bound, so no copy writes shared memory after the CTA exits
  if (failed && tid == 0) {
    for (int s = 0; s < kRing; ++s)
      if ((pending >> s) & 1u) mbar_wait_bounded(&S.bar[s], (phase >> s) & 1u, kSpinLimit);
  }
  if (chk) {
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      for (int sh = 16; sh > 0; sh >>= 1) mxb[c] = max(mxb[c], __shfl_xor_sync(0xffffffffu, mxb[c], sh));
      if (lane == 0) atomicMax(&S.L.bmax[c], mxb[c]);
    }
    __syncthreads();
    if (tid < 6) {
      const int idx = (n + 1) / P.n_check - P.check_base - 1;
      atomicMax(&P.check_max[idx * 6 + tid], S.L.bmax[tid]);
    }
  }
  };
  if (lists) body(std::true_type{});
  else body(std::false_type{});
}

}  // namespace wf
