/*
 * waveforge_b200.h -- C ABI of the B200 (sm_100a) Yee-FDTD + DAS engine.
 *
 * The reference project (shahzaibshazoo/waveforge) is pure Python/PyTorch and
 * has no native interface; each entry point below replaces one Python call
 * path of the reference, cited next to it.  All pointers are DEVICE pointers
 * unless marked "host"; sizes are element counts; streams are cudaStream_t
 * passed as void*.  Every function returns 0 on success or a WF_E* code and
 * never aborts or traps; wf_last_error() gives a message for the calling
 * thread.  The library allocates no device memory on these paths: scratch
 * buffers (ping-pong partners, work queues) are passed in by the caller.
 *
 * Field layout: row-major (i, j[, k]) with the LAST index unit-stride, exactly
 * the layout of the reference FieldSet tensors (src/core/fields.py:156-168,
 * 2D tensors are (Nx, Ny, 1)).  Component codes follow
 * src/core/fields.py:24 FIELD_COMPONENTS order.
 */
#ifndef WAVEFORGE_B200_H
#define WAVEFORGE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WF_ABI_VERSION 1

/* status codes */
#define WF_OK            0
#define WF_E_ARG         1   /* bad argument (size, pointer, range) */
#define WF_E_CUDA        2   /* a CUDA runtime call failed */
#define WF_E_LIMIT       3   /* a compile-time capacity was exceeded */
#define WF_E_DIVERGED    4   /* stability threshold exceeded (host-side check) */
#define WF_E_TIMEOUT     5   /* a bounded device wait gave up */

/* field component codes, src/core/fields.py:24 */
#define WF_EX 0
#define WF_EY 1
#define WF_EZ 2
#define WF_HX 3
#define WF_HY 4
#define WF_HZ 5

/* 2D TM grid constants, all float32-rounded exactly as PyTorch rounds the
 * Python-float scalars of the reference update (src/core/fdtd2d.py:158-161,
 * src/core/boundaries.py:177-178). */
typedef struct wf_grid2d {
  int32_t nx, ny;
  float dh;      /* dt / MU0 */
  float de;      /* dt / EPS0 (vacuum scalar path) */
  float dx, dy;
  float mur_x, mur_y;
  int32_t flags; /* WF_FASTDIV_* bits: set only after wf_check_fastdiv passed */
} wf_grid2d;

/* wf_grid*.flags: divisions by this spacing may be computed as
 * float32(double(x) * double(1/d)) -- one float64 product rounded once to
 * float32 -- which wf_check_fastdiv proved identical to IEEE division for
 * every float32 input.  Without the bit the kernels use IEEE division. */
#define WF_FASTDIV_X 1
#define WF_FASTDIV_Y 2
#define WF_FASTDIV_Z 4

/* 3D grid constants (src/core/fdtd3d.py:206-211, boundaries.py:429-431). */
typedef struct wf_grid3d {
  int32_t nx, ny, nz;
  float dh, de;
  float dx, dy, dz;
  float mur_x, mur_y, mur_z;
  int32_t flags; /* WF_FASTDIV_* bits */
} wf_grid3d;

/* One soft source (src/core/sources.py: PointSource :863-887, LineSource
 * :1015-1035, PlaneSource :730-749).  Every cell of the half-open box
 * [i0,i1)x[j0,j1)x[k0,k1) of component `comp` gets, at step n (before the H
 * update), field += wave[n] (amp == NULL) or field += wave[n]*amp[c] where c
 * is the row-major offset of the cell inside the box.  Sources are applied in
 * array order, as SourceCollection.step does (:1060-1071). */
typedef struct wf_source {
  int32_t comp;
  int32_t i0, i1, j0, j1, k0, k1;
  int32_t n_wave;
  const float* wave;
  const float* amp;
} wf_source;

/* One detector sample point: records comp[i,j,k] after every full step
 * (examples/brain_mimo_imaging.py:193-201). */
typedef struct wf_probe {
  int32_t comp, i, j, k;
} wf_probe;

/* Launch shape of the temporally blocked kernels. steps_per_pass = temporal
 * block depth K.  2D: tile_i x tile_j = the on-chip REGION of one CTA
 * (core + K-cell halo on each side); it selects one of the compiled
 * register layouts, in which one warp spans the region's width (4 adjacent
 * columns per lane for 128-wide regions) and `threads` sets the rows per
 * thread: 64x128 on 1024 threads (2 rows; threads = 512: 4 rows), 48x128 on
 * 512 threads (3 rows; threads >= 768: 768 threads of 2 rows), 32x128 and
 * 32x64 on 256 threads, 8x32 on 64.
 * 3D: tile_i x tile_j x tile_k = core cells per CTA, threads per CTA; with
 * tile_i = 0 the streaming kernels (tile_j = segment length, threads = variant). */
typedef struct wf_tune {
  int32_t steps_per_pass;
  int32_t tile_i, tile_j, tile_k;
  int32_t threads;
} wf_tune;

/* Library identity and the last error message of the calling thread. */
int32_t     wf_abi_version(void);
const char* wf_last_error(void);

/* Count the float32 inputs x (all 2^32 patterns) for which the fast
 * division by d differs from IEEE x/d; adds the count to *mismatches
 * (device, zeroed by the caller).  No reference counterpart: it guards the
 * bit-exactness of the spacing divisions of src/core/fdtd2d.py:232-245. */
int32_t wf_check_fastdiv(float d, uint32_t* mismatches, void* stream);

/* Advance a 2D TM grid nsteps time steps.
 * Replaces FDTD2D.step/run (src/core/fdtd2d.py:187-359) together with
 * MurABC.snapshot/apply (src/core/boundaries.py:230-274), the source
 * injection of SourceCollection.step (src/core/sources.py:1060-1071) and the
 * per-step detector gather (examples/brain_mimo_imaging.py:193-201).
 *
 *  ex,ey,hz     state, nx*ny each, updated in place (result always lands here)
 *  sx,sy,sz     caller-owned scratch, nx*ny each (ping-pong partner)
 *  ca,cb        per-cell coefficients nx*ny each, or both NULL (vacuum path)
 *  src,nsrc     device array of sources; every wave must have n_wave > last step
 *  probes,nprobe  device array of detector points
 *  traces       nprobe rows of trace_ld floats; step n goes to column n-trace_step0
 *  step0        global index of the first step (waveform row, trace column)
 *  n_check      stability-check period (steps_completed % n_check == 0)
 *  check_max    per-check maxima of |Ex|,|Ey|,|Hz| as float bits, 3 per check,
 *               indexed by (n+1)/n_check - (step0/n_check) - 1; NULL = off.
 *               The caller zeroes it.
 *  tune         NULL = built-in default.
 */
int32_t wf_fdtd2d_run(const wf_grid2d* g,
                      float* ex, float* ey, float* hz,
                      float* sx, float* sy, float* sz,
                      const float* ca, const float* cb,
                      const wf_source* src, int32_t nsrc,
                      const wf_probe* probes, int32_t nprobe,
                      float* traces, int64_t trace_ld, int32_t trace_step0,
                      int32_t step0, int32_t nsteps,
                      int32_t n_check, uint32_t* check_max,
                      const wf_tune* tune, void* stream);

/* Same as wf_fdtd2d_run, for callers that cannot allocate device memory
 * (applications whose own pool allocator owns all GPU memory, or loops that
 * must not call cudaMalloc/cudaFree because those can synchronise the
 * device).  No counterpart in the reference: it only exists for such callers.
 * The ping-pong scratch is a file-scope device array built into the library
 * (3 x WF_NOALLOC_MAX_CELLS floats = 12 MiB, reserved on every GPU that loads
 * the library until the process exits); grids above WF_NOALLOC_MAX_CELLS
 * cells are rejected with WF_E_LIMIT.  Nothing is allocated.  The first call
 * on each device looks the array's device address up once, so make that
 * first call before any stream capture; the address is cached for the
 * device's CUDA context, so after cudaDeviceReset reload the library before
 * the next call.  All calls on a device share the array: calls that may
 * overlap on the GPU race and must be serialised by the caller.  Nothing in
 * the array needs to start at zero.  Negative sizes give WF_E_ARG. */
#define WF_NOALLOC_MAX_CELLS (1LL << 20)
int32_t wf_fdtd2d_run_noalloc(const wf_grid2d* g,
                              float* ex, float* ey, float* hz,
                              const float* ca, const float* cb,
                              const wf_source* src, int32_t nsrc,
                              const wf_probe* probes, int32_t nprobe,
                              float* traces, int64_t trace_ld, int32_t trace_step0,
                              int32_t step0, int32_t nsteps,
                              int32_t n_check, uint32_t* check_max,
                              const wf_tune* tune, void* stream);

/* 2D TM grid constants of a float64 run: the reference's Python floats
 * unrounded (src/core/fdtd2d.py:158-161, src/core/boundaries.py:177-178). */
typedef struct wf_grid2d_f64 {
  int32_t nx, ny;
  double dh, de;
  double dx, dy;
  double mur_x, mur_y;
} wf_grid2d_f64;

/* Advance a float64 2D TM grid nsteps time steps: FDTD2D.step on a float64
 * FieldSet (src/core/grid.py:226-239, src/core/fields.py:124-130), every
 * operation of src/core/fdtd2d.py:219-257 and src/core/boundaries.py:237-274
 * one IEEE float64 operation in the reference's order, one launch per
 * operation.  A verification path, not the fast one.
 *
 *  ex,ey,hz     float64 state, nx*ny each, updated in place
 *  hz_prev      caller-owned nx*ny float64 scratch (the Mur snapshot)
 *  ca,cb        float64 per-cell coefficients, or both NULL (vacuum path)
 *  src          as wf_fdtd2d_run, but wave and amp point at float64 tables
 *  traces       float64, nprobe rows of trace_ld; step n -> column n-trace_step0
 *  check_max    per-check maxima of |Ex|,|Ey|,|Hz| as float64 bits, 3 per
 *               check, indexed as in wf_fdtd2d_run; NULL = off.  Zeroed by
 *               the caller. */
int32_t wf_fdtd2d_run_f64(const wf_grid2d_f64* g,
                          double* ex, double* ey, double* hz, double* hz_prev,
                          const double* ca, const double* cb,
                          const wf_source* src, int32_t nsrc,
                          const wf_probe* probes, int32_t nprobe,
                          double* traces, int64_t trace_ld, int32_t trace_step0,
                          int32_t step0, int32_t nsteps,
                          int32_t n_check, uint64_t* check_max, void* stream);

/* Advance a 3D grid nsteps time steps.
 * Replaces FDTD3D.step/run (src/core/fdtd3d.py:261-516) with
 * MurABC3D.snapshot/apply (src/core/boundaries.py:488-583), source injection
 * and detector gather.  f[6] = Ex,Ey,Ez,Hx,Hy,Hz state (nx*ny*nz each);
 * s[6] = scratch partners; check_max holds 6 maxima per check. */
int32_t wf_fdtd3d_run(const wf_grid3d* g,
                      float* const* f, float* const* s,
                      const float* ca, const float* cb,
                      const wf_source* src, int32_t nsrc,
                      const wf_probe* probes, int32_t nprobe,
                      float* traces, int64_t trace_ld, int32_t trace_step0,
                      int32_t step0, int32_t nsteps,
                      int32_t n_check, uint32_t* check_max,
                      const wf_tune* tune, void* stream);

/* Advance ninst independent 3D instances of one grid shape in ONE launch
 * per step (the streaming kernel; tune NULL or tile_i == 0), e.g. a batched
 * FieldSet (src/core/fields.py:97-101, 156-168: fields (B, Nx, Ny, Nz)) run
 * by FDTD3D.step (src/core/fdtd3d.py:261-402, whose ellipsis updates act on
 * every batch member).  Instance q uses f[c] + q*field_stride (and the same
 * offset of s[c]), Ca/Cb + q*coef_stride (0 = shared), sources
 * src[q*src_stride .. q*src_stride + src_per_inst) (src_stride 0 = every
 * instance shares the list, as the reference's broadcast sources do,
 * src/core/sources.py:885-887), traces + q*trace_stride; probes are the same
 * points in every instance; check_max collects the maxima over all
 * instances.  Other arguments as wf_fdtd3d_run. */
int32_t wf_fdtd3d_batch_run(const wf_grid3d* g, int32_t ninst, int64_t field_stride,
                            float* const* f, float* const* s,
                            const float* ca, const float* cb, int64_t coef_stride,
                            const wf_source* src, int32_t src_per_inst, int32_t src_stride,
                            const wf_probe* probes, int32_t nprobe,
                            float* traces, int64_t trace_ld, int64_t trace_stride,
                            int32_t trace_step0, int32_t step0, int32_t nsteps,
                            int32_t n_check, uint32_t* check_max,
                            const wf_tune* tune, void* stream);

/* One solve of a batched launch: an independent 2D TM grid with its own
 * state, scratch, coefficients, sources, probes and trace buffer.
 * Batching many of these is new functionality: the reference runs MIMO
 * transmitters one FDTD2D at a time (examples/brain_mimo_imaging.py:176-204,
 * examples/10_breast_tumor_mimo.py:123-145). */
typedef struct wf_solve2d {
  wf_grid2d g;
  float *ex, *ey, *hz;
  float *sx, *sy, *sz;
  const float *ca, *cb;
  const wf_source* src;
  const wf_probe* probes;
  float* traces;
  int64_t trace_ld;
  int32_t nsrc, nprobe;
  int32_t trace_step0;
  int32_t step0, nsteps;      /* steps to advance in this launch */
  int32_t n_check;            /* stability-check period, as in wf_fdtd2d_run */
  int32_t status;             /* written by the device: 0 ok, else WF_E_* */
  uint32_t* check_max;        /* 3 maxima per check, or NULL */
} wf_solve2d;

/* Advance every solve of a device array of descriptors in ONE persistent
 * launch: resident CTAs pull solves from a device work queue (queue[0] is the
 * next-item counter, zeroed by the caller; order[] lists solve indices,
 * largest first) and run each through all its steps with the same tile
 * routine as wf_fdtd2d_run, so each solve's result is bit-identical to
 * running it alone.  Each solve's result lands in its ex/ey/hz.
 * fastdiv != 0 runs the verified fast-division code for the whole launch:
 * every solve must then carry both WF_FASTDIV_X|Y bits (a solve without
 * them is not computed and gets status WF_E_ARG); fastdiv == 0 uses IEEE
 * division for all solves. */
int32_t wf_batch2d_run(const wf_solve2d* solves, int32_t nsolve,
                       const int32_t* order, int32_t* queue,
                       const wf_tune* tune, int32_t ctas_per_sm,
                       int32_t fastdiv, void* stream);

/* One temporal pass of many solves, spread over the GPU by tiles.
 * items: nitems (solve index, ci0, cj0) int32 triplets on the device, one
 * CTA each: the core tile [ci0, ci0+tile_i-2k) x [cj0, cj0+tile_j-2k) of
 * solve `solves[index]` advances k steps from step solves[index].step0 +
 * step_offset, reading its state buffers (parity 0) or its scratch buffers
 * (parity 1) and writing the other set.  Same tile routine as wf_fdtd2d_run,
 * so a solve advanced by a sequence of these passes is bit-identical to its
 * plain run with the same pass plan.  tune: region shape only (tile_i,
 * tile_j; NULL = 48x128); fastdiv as in wf_batch2d_run.  Batching many
 * solves is new; the reference runs them one FDTD2D at a time
 * (examples/brain_mimo_imaging.py:176-204). */
int32_t wf_batch2d_pass(const wf_solve2d* solves, const int32_t* items, int32_t nitems,
                        int32_t parity, int32_t step_offset, int32_t k,
                        const wf_tune* tune, int32_t fastdiv, void* stream);

/* ALL temporal passes of many solves in ONE persistent launch, spread over
 * the GPU by tiles.  The pass plan is wf_fdtd2d_run's for nsteps steps at
 * depth K = tune->steps_per_pass (every solve advances nsteps steps from its
 * own step0; the result lands in its ex/ey/hz).  tiles: ntiles (solve index,
 * ci0, cj0) int32 triplets, cores of (tile_i-2K) x (tile_j-2K) cells, largest
 * solves first; nbr: 9 int32 per tile, the tile itself and the tiles of the
 * same solve whose cores touch its region (-1 = none); done: ntiles int32 and
 * queue[0]: zeroed by the caller.  Resident CTAs take items pass-major
 * (item i = pass i / ntiles of tile i % ntiles); an item first waits, for at
 * most wait_limit polls (negative = 2^24), until done[] of its 9 entries
 * reaches its pass, and after its stores sets done[tile] = pass + 1.  A wait
 * that gives up writes WF_E_TIMEOUT to the solve's status (the tile is not
 * computed).  Needs 3K <= tile_i and 3K <= tile_j.  Same tile routine as
 * wf_fdtd2d_run, so every solve is bit-identical to its plain run.  Batching
 * is new; the reference runs one FDTD2D per transmitter
 * (examples/brain_mimo_imaging.py:176-204). */
int32_t wf_batch2d_queue(wf_solve2d* solves, const int32_t* tiles, int32_t ntiles,
                         const int32_t* nbr, int32_t* done, int32_t* queue, int32_t nsteps,
                         const wf_tune* tune, int32_t fastdiv, int64_t wait_limit,
                         void* stream);

/* Recompute and keep every state of nsteps forward steps, for ntx runs that
 * share the grid and the coefficients (e.g. the transmitters of one
 * phantom).  Run t owns states + t*tx_stride: nsteps+1 slots of three planes
 * (Ex, Ey, Hz; 3*nx*ny floats per slot); slot 0 is its input, slot s+1 the
 * state after step step0+s; it uses sources [t*src_per_tx, (t+1)*src_per_tx).
 * One launch per step covers every run.  Same tile routine and arithmetic
 * as wf_fdtd2d_run, so each slot is bit-identical to the state
 * wf_fdtd2d_run reaches.  No reference counterpart: the adjoint needs E^n
 * and H^{n+1} of every step of a checkpoint segment (the reference has no
 * adjoint; its plan is docs/architecture/DIFFERENTIABLE_PHYSICS.md). */
int32_t wf_fdtd2d_states(const wf_grid2d* g, float* states, int64_t tx_stride, int32_t ntx,
                         int32_t nsteps, const float* ca, const float* cb,
                         const wf_source* src, int32_t src_per_tx, int32_t step0, void* stream);

/* Reverse (adjoint) steps of the 2D TM update for
 * L = 1/2 sum_{p,n} (trace_p[n] - target_p[n])^2, the traces being the
 * detector samples of src/core/fdtd2d.py:187-266 recorded after each step,
 * for ntx runs at once.  Runs steps n = step0+nsteps-1 down to step0:
 *  states   run t: states + t*states_stride, the nsteps+1 slots of
 *           wf_fdtd2d_states (slot s = state before step step0+s)
 *  lam      ntx x 3 planes (aEx, aEy, aHz per run).  In: dL/d(state after
 *           step step0+nsteps) without that step's residual; out: dL/d(state
 *           before step0).  lam_scratch: the same size, caller scratch.
 *  resid    run t: resid + t*resid_stride, nprobe rows of resid_ld floats
 *           (trace - target); column n - resid_step0 holds step n
 *  g_ca/g_cb  float64 accumulators of dL/dCa, dL/dCb, one nx*ny plane per run
 *           (ntx planes each), required with ca/cb.  No reference
 *           counterpart. */
int32_t wf_adjoint2d_run(const wf_grid2d* g, const float* states, int64_t states_stride,
                         int32_t ntx, int32_t nsteps, const float* ca, const float* cb,
                         const wf_probe* probes, int32_t nprobe,
                         const float* resid, int64_t resid_ld, int64_t resid_stride,
                         int32_t resid_step0, int32_t step0, float* lam, float* lam_scratch,
                         double* g_ca, double* g_cb, void* stream);

/* Per-cell lossy coefficients from float64 eps_r, sigma, evaluated as
 * Material.ca / Material.cb (src/core/materials.py:61-82) in float64 and
 * rounded to float32 as MaterialMap.build stores them (:200-252). */
int32_t wf_material_coeffs(const double* eps_r, const double* sigma, int64_t n, double dt,
                           float* ca, float* cb, void* stream);

/* Chain rule of wf_material_coeffs: g_eps = scale * dL/deps_r and
 * g_sigma = scale * dL/dsigma from `count` consecutive planes of dL/dCa,
 * dL/dCb accumulators (float64, summed in plane order).  No reference
 * counterpart. */
int32_t wf_material_grad(const double* eps_r, const double* sigma, int64_t n, double dt,
                         const double* g_ca, const double* g_cb, int32_t count, double scale,
                         double* g_eps, double* g_sigma, void* stream);

/* One region of a painted 2D material map (painter's order: later regions
 * win).  Parameters are the float32-rounded Python floats of the host
 * painter; `material` indexes the Ca/Cb table (0 = default material).
 *  WF_REGION_CIRCLE   p = ci, cj, r*r         (MaterialMap.add_circle,
 *                                              src/core/materials.py:143-163)
 *  WF_REGION_RECT     p = i0, i1, j0, j1      (add_rectangle, :165-185)
 *  WF_REGION_ELLIPSE  p = ci, cj, a, b        (axis-aligned ellipse)
 *  WF_REGION_SHELL    p = outer ci,cj,a,b, inner ci,cj,a,b (outer & ~inner) */
#define WF_REGION_CIRCLE  0
#define WF_REGION_RECT    1
#define WF_REGION_ELLIPSE 2
#define WF_REGION_SHELL   3
typedef struct wf_region2d {
  int32_t kind;
  int32_t material;
  float p[8];
} wf_region2d;

/* Paint Ca/Cb (nx*ny float32 each) on the device, bit-identical to
 * MaterialMap.build (src/core/materials.py:200-252) for the same regions.
 * regions: device array; table_ca/cb: nmat float32 on the device.  Optional
 * (both or neither): eps_r/sigma float64 planes painted from the float64
 * tables table_eps/table_sigma (the adjoint's chain rule needs them).  A
 * region whose material index is outside [0, nmat) paints the default and
 * sets *status (device, nullable) to WF_E_ARG.  At most 1024 regions. */
int32_t wf_paint2d(int32_t nx, int32_t ny, const wf_region2d* regions, int32_t nreg,
                   const float* table_ca, const float* table_cb,
                   const double* table_eps, const double* table_sigma, int32_t nmat,
                   float* ca, float* cb, double* eps_r, double* sigma,
                   int32_t* status, void* stream);

/* 2D TM leapfrog with a convolutional PML of `depth` cells on every side in
 * place of the Mur edges.  No reference counterpart: the reference only
 * stores the graded profiles (src/core/boundaries.py:32-112, MurABC
 * pml_depth) and never applies them.  Arguments as wf_fdtd2d_run (fields
 * updated in place, no scratch), plus
 *  tables  6*(nx+ny) float32 on the device: for the x axis (nx entries each)
 *          b_E, c_E, 1/kappa_E, b_H, c_H, 1/kappa_H, then the same for y;
 *          E samples at integer cells, H samples at half cells
 *  psi     4*depth*(nx+ny) float32 on the device (zero before the first
 *          step): Hz-x [2*depth][ny], Ey-x [2*depth][ny], Hz-y [nx][2*depth],
 *          Ex-y [nx][2*depth] layer memories, updated in place.
 * Outside the layers the update is the reference's, bit for bit. */
int32_t wf_cpml2d_run(const wf_grid2d* g, float* ex, float* ey, float* hz, const float* ca,
                      const float* cb, int32_t depth, const float* tables, float* psi,
                      const wf_source* src, int32_t nsrc, const wf_probe* probes,
                      int32_t nprobe, float* traces, int64_t trace_ld, int32_t trace_step0,
                      int32_t step0, int32_t nsteps, int32_t n_check, uint32_t* check_max,
                      void* stream);

/* Bound of the TMA pass's shared-memory pipeline waits, for every later 3D
 * launch of this process: each wait takes one non-blocking look, then at
 * most `polls` hardware-suspended polls before it gives up with WF_E_TIMEOUT
 * (see wf_fdtd3d_take_status).  polls < 0 restores the built-in bound
 * (2^22).  A small bound makes the pass give up on loads that do complete:
 * failure-handling tests use it to take the timeout path without any device
 * fault.  The wait for copies still in flight after a give-up always uses
 * the built-in bound.  No reference counterpart. */
int32_t wf_fdtd3d_set_wait_limit(int64_t polls);

/* Status of the 3D passes since the last call on this device, then cleared:
 * 0, or WF_E_TIMEOUT when a bounded shared-memory pipeline wait of the TMA
 * pass gave up (that column block stopped; its outputs are incomplete).
 * Synchronous (reads a device word).  No reference counterpart: the
 * reference has no device pipeline to wait on. */
int32_t wf_fdtd3d_take_status(int32_t* status);

/* One region of a painted 3D material map (painter's order: later regions
 * win), parameters float32-rounded as in wf_region2d
 * (MaterialMap3D, src/core/materials.py:297-423):
 *  WF_REGION3_SPHERE     p = ci, cj, ck, r*r                  (add_sphere)
 *  WF_REGION3_BOX        p = i0, i1, j0, j1, k0, k1           (add_box)
 *  WF_REGION3_ELLIPSOID  p = ci, cj, ck, a*a, b*b, c*c        (add_ellipsoid)
 *  WF_REGION3_CYL_X/Y/Z  p = ci, cj, ck, r*r, height/2        (add_cylinder) */
#define WF_REGION3_SPHERE    0
#define WF_REGION3_BOX       1
#define WF_REGION3_ELLIPSOID 2
#define WF_REGION3_CYL_X     3
#define WF_REGION3_CYL_Y     4
#define WF_REGION3_CYL_Z     5
typedef struct wf_region3d {
  int32_t kind;
  int32_t material;
  float p[8];
} wf_region3d;

/* Paint Ca/Cb (nx*ny*nz float32 each, [i][j][k]) on the device,
 * bit-identical to MaterialMap3D.build3d (src/core/materials.py:425-478)
 * for the same regions.  regions: device array; table_ca/cb: nmat float32 on
 * the device (index 0 = default material).  A region whose material index is
 * outside [0, nmat) paints the default and sets *status (device, nullable)
 * to WF_E_ARG.  At most 1024 regions. */
int32_t wf_paint3d(int32_t nx, int32_t ny, int32_t nz, const wf_region3d* regions, int32_t nreg,
                   const float* table_ca, const float* table_cb, int32_t nmat, float* ca,
                   float* cb, int32_t* status, void* stream);

/* Delay-and-sum backprojection on the device, bit-identical to the reference
 * NumPy float64 path of examples/brain_mimo_imaging.py:211-266 (and its
 * variants through px/py, gate_start, skip_self).
 *  traces   (nant, nant, n_steps) float32, [tx][rx][n]
 *  traces_ref  NULL, or a second array of the same shape: the samples are then
 *           traces - traces_ref in float32 (delta_S = S_tumor - S_healthy,
 *           examples/brain_mimo_imaging.py:314)
 *  ant_x/y  nant antenna coordinates in metres (float64)
 *  px, py   nxi / nyi pixel coordinates in metres (float64)
 *  image    nxi*nyi float64 output, row-major [ix][iy], squared sum. */
int32_t wf_das2d(const float* traces, const float* traces_ref, int32_t nant, int32_t n_steps,
                 const double* ant_x, const double* ant_y,
                 const double* px, int32_t nxi, const double* py, int32_t nyi,
                 double v_medium, double dt,
                 int32_t gate_start, int32_t skip_self,
                 double* image, void* stream);

/* Travel-time table of AntennaRing.compute_das_image
 * (src/datasets/brain/antenna.py:216-260, 300-333): tt[a][iy][ix] =
 * float32 of the one-way time in samples from antenna a (ant_x/y_mm, device)
 * to pixel (px_mm[ix], py_mm[iy]) (device), through nlayer concentric circles
 * about (cx_mm, cy_mm) of radius layer_r_mm[l] and permittivity layer_eps[l]
 * (HOST arrays, outermost first, at most 16; nlayer = 0: free space), c = 3e8. */
int32_t wf_das_travel_times(int32_t nant, const double* ant_x_mm, const double* ant_y_mm,
                            const double* px_mm, int32_t nxi, const double* py_mm, int32_t nyi,
                            double cx_mm, double cy_mm, const double* layer_r_mm,
                            const double* layer_eps, int32_t nlayer, double dt, float* tt,
                            void* stream);

/* DAS power image of AntennaRing.compute_das_image (antenna.py:335-341):
 * image[p] = float32((sum_{tx,rx} env[tx][rx][rint(tt[tx][p] + tt[rx][p])])^2),
 * samples outside [0, n_steps) skipped, float64 sum in tx-major order.
 * env: (nant, nant, n_steps) float32 envelope; tt: (nant, npix) float32. */
int32_t wf_das_envelope_image(const float* env, int32_t nant, int32_t n_steps, const float* tt,
                              int32_t npix, float* image, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* WAVEFORGE_B200_H */
