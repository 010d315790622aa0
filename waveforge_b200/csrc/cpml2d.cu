// cpml2d.cu -- 2D TM leapfrog with a convolutional PML (CPML) in place of the
// Mur edges.
//
// The reference stores graded CPML coefficient profiles next to its Mur ABC
// (src/core/boundaries.py:32-112, MurABC(pml_depth=...)) but no engine uses
// them: this file gives them an update.  Recursive-convolution CPML (Roden
// and Gedney 2000) with the reference's profile: over a layer of D cells on
// every side, each spatial derivative d of the update becomes
//     psi <- b * psi + c * d          (the layer's memory, one per cell)
//     d   <- d * (1 / kappa) + psi
// with (b, c, 1/kappa) sampled at the derivative's position: integer cells
// for the E updates, half cells for the Hz update (the dual staggering of
// boundaries.py:51-112).  Depth of a position x in a PML of D cells on an
// axis of n cells: rho = (D - x) / D on the low side, (x - (n - 1 - D)) / D
// on the high side.  Behind the layer the outermost fields stay as the
// reference's update ranges leave them (Hz on i = Nx-1 / j = Ny-1, Ex on j = 0,
// Ey on i = 0 are never updated).  Outside the layers every op is the
// reference update in the reference order, bit for bit.
//
// One step = E-source injection, Faraday (Hz injection + curl + psi_hz),
// Ampere (Ex, Ey + psi_e, stability maxima), detector samples: four short
// launches, HBM-bound; temporal blocking is left to the Mur engine.
#include <algorithm>

#include "tile2d.cuh"

namespace wf {

struct Cpml2D {
  int nx, ny, D;
  float dh, de, dx, dy;
  double rdx, rdy;
  float *ex, *ey, *hz;
  const float *ca, *cb;
  // per-axis tables: [b_E, c_E, ik_E, b_H, c_H, ik_H] x n (x axis, then y)
  const float *tx, *ty;
  // psi slabs: hzx [2D][ny], eyx [2D][ny], hzy [nx][2D], exy [nx][2D]
  float *phzx, *peyx, *phzy, *pexy;
};

// slab index of a position on an axis of n cells with a D-cell layer on each
// side (E at integer i, H at i + 1/2), or -1 outside the layers
__device__ __forceinline__ int slab_e(int i, int n, int D) {
  return i < D ? i : (i >= n - D ? D + (i - (n - D)) : -1);
}
__device__ __forceinline__ int slab_h(int i, int n, int D) {
  return i < D ? i : (i >= n - 1 - D && i <= n - 2 ? D + (i - (n - 1 - D)) : -1);
}

template <bool FDIV>
__device__ __forceinline__ float cdiv(float a, float d, double r) {
  return FDIV ? div_fast(a, r) : fdiv(a, d);
}

// E-source injection of step n, in collection order (one block).
__global__ void k_cpml_inject_e(Cpml2D C, const wf_source* __restrict__ src, int nsrc, int n) {
  for (int s = 0; s < nsrc; ++s) {
    const wf_source& Q = src[s];
    if (Q.comp == WF_EX || Q.comp == WF_EY) {
      float* f = Q.comp == WF_EX ? C.ex : C.ey;
      const int w = Q.j1 - Q.j0, cells = (Q.i1 - Q.i0) * w;
      for (int q = threadIdx.x; q < cells; q += blockDim.x) {
        const int i = Q.i0 + q / w, j = Q.j0 + q % w;
        const long long g = (long long)i * C.ny + j;
        f[g] = fadd(f[g], src_value(Q, i, j, n));
      }
    }
    __syncthreads();  // overlapping boxes add in collection order
  }
}

// Hz: injection, then the curl with the CPML terms (i < Nx-1, j < Ny-1).
template <bool FDIV>
__global__ void k_cpml_h(Cpml2D C, const wf_source* __restrict__ src, int nsrc, int n) {
  const int nx = C.nx, ny = C.ny, D = C.D;
  const long long total = (long long)nx * ny;
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(g / ny), j = (int)(g - (long long)i * ny);
    float v = C.hz[g];
    for (int s = 0; s < nsrc; ++s) {
      const wf_source& Q = src[s];
      if (Q.comp == WF_HZ && i >= Q.i0 && i < Q.i1 && j >= Q.j0 && j < Q.j1)
        v = fadd(v, src_value(Q, i, j, n));
    }
    if (i < nx - 1 && j < ny - 1) {
      float t2 = cdiv<FDIV>(fsub(C.ex[g + 1], C.ex[g]), C.dy, C.rdy);   // dEx/dy
      float t4 = cdiv<FDIV>(fsub(C.ey[g + ny], C.ey[g]), C.dx, C.rdx);  // dEy/dx
      const int sx = slab_h(i, nx, D), sy = slab_h(j, ny, D);
      if (sx >= 0) {
        float& p = C.phzx[(long long)sx * ny + j];
        p = fadd(fmul(C.tx[3 * nx + i], p), fmul(C.tx[4 * nx + i], t4));
        t4 = fadd(fmul(t4, C.tx[5 * nx + i]), p);
      }
      if (sy >= 0) {
        float& p = C.phzy[(long long)i * (2 * D) + sy];
        p = fadd(fmul(C.ty[3 * ny + j], p), fmul(C.ty[4 * ny + j], t2));
        t2 = fadd(fmul(t2, C.ty[5 * ny + j]), p);
      }
      v = fadd(v, fmul(C.dh, fsub(t2, t4)));
    }
    C.hz[g] = v;
  }
}

// Ex (j >= 1), Ey (i >= 1) with the CPML terms; |field| maxima on check steps.
template <bool MAT, bool FDIV>
__global__ void k_cpml_e(Cpml2D C, int check_idx, unsigned* check_max) {
  __shared__ unsigned bm[3];
  const int nx = C.nx, ny = C.ny, D = C.D;
  const long long total = (long long)nx * ny;
  if (threadIdx.x < 3) bm[threadIdx.x] = 0u;
  __syncthreads();
  unsigned m0 = 0, m1 = 0, m2 = 0;
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(g / ny), j = (int)(g - (long long)i * ny);
    const float h = C.hz[g];
    float ex = C.ex[g], ey = C.ey[g];
    const float ca = MAT ? C.ca[g] : 0.f, cb = MAT ? C.cb[g] : 0.f;
    if (j >= 1) {
      float d1 = cdiv<FDIV>(fsub(h, C.hz[g - 1]), C.dy, C.rdy);
      const int sy = slab_e(j, ny, D);
      if (sy >= 0) {
        float& p = C.pexy[(long long)i * (2 * D) + sy];
        p = fadd(fmul(C.ty[j], p), fmul(C.ty[ny + j], d1));
        d1 = fadd(fmul(d1, C.ty[2 * ny + j]), p);
      }
      ex = MAT ? fadd(fmul(ca, ex), fmul(cb, d1)) : fadd(ex, fmul(C.de, d1));
      C.ex[g] = ex;
    }
    if (i >= 1) {
      float d2 = cdiv<FDIV>(fsub(h, C.hz[g - ny]), C.dx, C.rdx);
      const int sx = slab_e(i, nx, D);
      if (sx >= 0) {
        float& p = C.peyx[(long long)sx * ny + j];
        p = fadd(fmul(C.tx[i], p), fmul(C.tx[nx + i], d2));
        d2 = fadd(fmul(d2, C.tx[2 * nx + i]), p);
      }
      ey = MAT ? fsub(fmul(ca, ey), fmul(cb, d2)) : fsub(ey, fmul(C.de, d2));
      C.ey[g] = ey;
    }
    if (check_max != nullptr) {
      m0 = max(m0, abs_bits(ex));
      m1 = max(m1, abs_bits(ey));
      m2 = max(m2, abs_bits(h));
    }
  }
  if (check_max != nullptr) {
    for (int sh = 16; sh > 0; sh >>= 1) {
      m0 = max(m0, __shfl_xor_sync(0xffffffffu, m0, sh));
      m1 = max(m1, __shfl_xor_sync(0xffffffffu, m1, sh));
      m2 = max(m2, __shfl_xor_sync(0xffffffffu, m2, sh));
    }
    if ((threadIdx.x & 31) == 0) {
      atomicMax(&bm[0], m0);
      atomicMax(&bm[1], m1);
      atomicMax(&bm[2], m2);
    }
    __syncthreads();
    if (threadIdx.x < 3) atomicMax(&check_max[check_idx * 3 + threadIdx.x], bm[threadIdx.x]);
  }
}

// Detector samples of step n (after the full step).
__global__ void k_cpml_probe(Cpml2D C, const wf_probe* __restrict__ prb, int nprb, float* traces,
                             long long trace_ld, int col) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nprb) return;
  const wf_probe& q = prb[p];
  const long long g = (long long)q.i * C.ny + q.j;
  const float* f = q.comp == WF_EX ? C.ex : (q.comp == WF_EY ? C.ey : C.hz);
  traces[(long long)p * trace_ld + col] = f[g];
}

}  // namespace wf

using namespace wf;

extern "C" int32_t wf_cpml2d_run(const wf_grid2d* g, float* ex, float* ey, float* hz,
                                 const float* ca, const float* cb, int32_t depth,
                                 const float* tables, float* psi, const wf_source* src,
                                 int32_t nsrc, const wf_probe* probes, int32_t nprobe,
                                 float* traces, int64_t trace_ld, int32_t trace_step0,
                                 int32_t step0, int32_t nsteps, int32_t n_check,
                                 uint32_t* check_max, void* stream) {
  if (g == nullptr || ex == nullptr || ey == nullptr || hz == nullptr || tables == nullptr ||
      psi == nullptr)
    return set_error(WF_E_ARG, "wf_cpml2d_run: null grid, field, table or psi pointer");
  if ((ca == nullptr) != (cb == nullptr))
    return set_error(WF_E_ARG, "wf_cpml2d_run: Ca and Cb must be given together");
  if (g->nx < 4 || g->ny < 4 || depth < 1 || 2 * depth + 2 > g->nx || 2 * depth + 2 > g->ny)
    return set_error(WF_E_ARG, "wf_cpml2d_run: grid %dx%d cannot hold a %d-cell layer per side",
                     g->nx, g->ny, depth);
  if (nsteps < 0 || step0 < 0 || nsrc < 0 || nprobe < 0 || (nsrc > 0 && src == nullptr) ||
      (nprobe > 0 && (probes == nullptr || traces == nullptr)))
    return set_error(WF_E_ARG, "wf_cpml2d_run: bad counts or null descriptor arrays");
  if (nsteps == 0) return WF_OK;
  int dev = 0, nsm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
  Cpml2D C{};
  C.nx = g->nx;
  C.ny = g->ny;
  C.D = depth;
  C.dh = g->dh;
  C.de = g->de;
  C.dx = g->dx;
  C.dy = g->dy;
  C.rdx = 1.0 / (double)g->dx;
  C.rdy = 1.0 / (double)g->dy;
  C.ex = ex;
  C.ey = ey;
  C.hz = hz;
  C.ca = ca;
  C.cb = cb;
  C.tx = tables;
  C.ty = tables + 6LL * g->nx;
  const long long sx = 2LL * depth * g->ny, sy = 2LL * depth * g->nx;
  C.phzx = psi;
  C.peyx = psi + sx;
  C.phzy = psi + 2 * sx;
  C.pexy = psi + 2 * sx + sy;
  const bool fd = (g->flags & (WF_FASTDIV_X | WF_FASTDIV_Y)) == (WF_FASTDIV_X | WF_FASTDIV_Y);
  cudaStream_t st = (cudaStream_t)stream;
  const long long n = (long long)g->nx * g->ny;
  const int blocks = (int)std::min<long long>((n + 255) / 256, 8LL * nsm);
  const bool has_e = nsrc > 0;  // the injection kernel skips non-E sources itself
  const int check_base = n_check > 0 ? step0 / n_check : 0;
  for (int t = 0; t < nsteps; ++t) {
    const int step = step0 + t;
    if (has_e) k_cpml_inject_e<<<1, 256, 0, st>>>(C, src, nsrc, step);
    if (fd) k_cpml_h<true><<<blocks, 256, 0, st>>>(C, src, nsrc, step);
    else k_cpml_h<false><<<blocks, 256, 0, st>>>(C, src, nsrc, step);
    const bool chk = check_max != nullptr && n_check > 0 && (step + 1) % n_check == 0;
    const int idx = chk ? (step + 1) / n_check - check_base - 1 : 0;
    unsigned* cm = chk ? check_max : nullptr;
    if (ca != nullptr) {
      if (fd) k_cpml_e<true, true><<<blocks, 256, 0, st>>>(C, idx, cm);
      else k_cpml_e<true, false><<<blocks, 256, 0, st>>>(C, idx, cm);
    } else {
      if (fd) k_cpml_e<false, true><<<blocks, 256, 0, st>>>(C, idx, cm);
      else k_cpml_e<false, false><<<blocks, 256, 0, st>>>(C, idx, cm);
    }
    if (nprobe > 0)
      k_cpml_probe<<<(nprobe + 255) / 256, 256, 0, st>>>(C, probes, nprobe, traces, trace_ld,
                                                        step - trace_step0);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "launch CPML step");
  }
  return WF_OK;
}
