"""Batched execution of many independent, uneven 2D TM solves.

The reference runs a MIMO study one ``FDTD2D`` at a time, one transmitter
after another (examples/brain_mimo_imaging.py:149-204,
examples/10_breast_tumor_mimo.py:123-145; on two GPUs one Python thread per
GPU).  ``Batch2D`` places every solve's fields, scratch, coefficients,
sources and detector traces on the device once, and advances all of them in
ONE persistent launch of ``wf_batch2d_run``: resident CTAs pull solves from a
device work queue in largest-first order and run each through its steps with
the same tile routine as ``FDTD2D``, so every solve's traces are
bit-identical to running it alone.  Solves that share a phantom share its
``Ca``/``Cb`` tensors.  Two other schedules spread a large solve over many
SMs: one launch per temporal pass over every solve's tiles ("tiled"), and
one persistent launch whose CTAs pull (pass, tile) items from a device queue
and wait, bounded, for the neighbouring tiles of the previous pass
("queue").

``run_plain`` runs the same solves one after another through
``wf_fdtd2d_run`` (the plain per-solve path) for comparison.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np
import torch

from . import _native as nat
from .core._engine import ProbeTable, SourceTable, source_list, tune_struct
from .core.boundaries import _mur_coeff
from .core.grid import YeeGrid
from .detectors import Detectors

EPS0: float = 8.8541878128e-12
MU0: float = 1.2566370614e-6
_ALLOWED = ("Ex", "Ey", "Hz")


@dataclass
class BatchSolve:
    """One independent solve: grid, coefficients (None = vacuum), sources, detectors."""

    grid: YeeGrid
    sources: object
    detectors: Optional[Detectors] = None
    Ca: Optional[torch.Tensor] = None
    Cb: Optional[torch.Tensor] = None
    n_check: int = 0
    tag: object = None
    _state: dict = field(default_factory=dict, repr=False)


def grid_struct(grid: YeeGrid, device: Optional[torch.device] = None) -> nat.WfGrid2D:
    """Float32-rounded constants of a 2D grid, with the Mur coefficients and
    their (-1, 0) validation of ``MurABC`` (src/core/boundaries.py:177-190)."""
    dt = grid.dt
    cm = [_mur_coeff(dt, grid.dx), _mur_coeff(dt, grid.dy)]
    for ax, c in zip("xy", cm):
        if not (-1.0 < c < 0.0):
            raise ValueError(f"C_mur_{ax}={c!r} is not in the open interval (-1, 0). This "
                             f"indicates a CFL violation — reduce dt or increase d{ax}.")
    flags = 0 if device is None else nat.fastdiv_flags(device, grid.dx, grid.dy)
    return nat.WfGrid2D(grid.Nx, grid.Ny, nat.f32(dt / MU0), nat.f32(dt / EPS0), nat.f32(grid.dx),
                        nat.f32(grid.dy), nat.f32(cm[0]), nat.f32(cm[1]), flags)



class PassPlan:
    """Pass schedule of a temporally blocked run (the plan of wf_common.cuh
    PassPlan): ``nsteps`` split into passes of at most ``K`` steps, the first
    pass split in two when the pass count is odd so the ping-pong ends in the
    state buffers; only an odd run of single-step passes needs a copy-back."""

    def __init__(self, nsteps: int, K: int) -> None:
        self.nsteps, self.K = nsteps, K
        self.P0 = -(-nsteps // K)
        L0 = min(nsteps, K)
        self.split = 1 if (self.P0 % 2 == 1 and L0 >= 2) else 0
        self.a = L0 // 2

    @property
    def passes(self) -> int:
        return self.P0 + self.split

    def _unsplit(self, q: int) -> int:
        return self.K if q < self.P0 - 1 else self.nsteps - self.K * (self.P0 - 1)

    def length(self, p: int) -> int:
        if not self.split:
            return self._unsplit(p)
        if p == 0:
            return self.a
        if p == 1:
            return self._unsplit(0) - self.a
        return self._unsplit(p - 1)

    def offset(self, p: int) -> int:
        if not self.split:
            return p * self.K
        if p == 0:
            return 0
        if p == 1:
            return self.a
        return (p - 1) * self.K

    @property
    def needs_copy(self) -> bool:
        return self.passes % 2 == 1


def tile_items(shapes: Sequence[tuple[int, int]], k: int, region: tuple[int, int],
               index: Optional[Sequence[int]] = None) -> np.ndarray:
    """(solve index, ci0, cj0) int32 triplets of every core tile of every
    solve for a pass of ``k`` steps with an RH x RW region (core RH-2k x
    RW-2k), largest solves first."""
    rh, rw = region
    ci, cj = rh - 2 * k, rw - 2 * k
    out = []
    idx = list(range(len(shapes))) if index is None else list(index)
    for q, (nx, ny) in sorted(zip(idx, shapes), key=lambda t: -t[1][0] * t[1][1]):
        ii, jj = np.meshgrid(np.arange(0, nx, ci, dtype=np.int32),
                             np.arange(0, ny, cj, dtype=np.int32), indexing="ij")
        t = np.empty((ii.size, 3), dtype=np.int32)
        t[:, 0] = q
        t[:, 1] = ii.reshape(-1)
        t[:, 2] = jj.reshape(-1)
        out.append(t)
    return np.concatenate(out) if out else np.zeros((0, 3), dtype=np.int32)


def tile_neighbours(tiles: np.ndarray, k: int, region: tuple[int, int]) -> np.ndarray:
    """(ntiles, 9) int32: for every tile of ``tile_items(.., k, ..)``, itself
    and the tiles of the same solve whose cores touch its region (-1 = none):
    with a core of at least k cells per side those are its 8 neighbours."""
    rh, rw = region
    ci, cj = rh - 2 * k, rw - 2 * k
    index = {(int(q), int(a), int(b)): t for t, (q, a, b) in enumerate(tiles)}
    out = np.full((len(tiles), 9), -1, dtype=np.int32)
    for t, (q, a, b) in enumerate(tiles):
        m = 0
        for di in (0, -ci, ci):
            for dj in (0, -cj, cj):
                nb = index.get((int(q), int(a) + di, int(b) + dj))
                if nb is not None:
                    out[t, m] = nb
                    m += 1
    return out


def run_tiled_passes(desc_dev_ptr: int, items_by_k: dict, plan: PassPlan, tune, fastdiv: bool,
                     stream: int) -> None:
    """Launch every pass of ``plan`` as one wf_batch2d_pass over its items
    (``items_by_k[k]`` = (device pointer, count))."""
    lib = nat.load()
    for p in range(plan.passes):
        k = plan.length(p)
        ptr, n = items_by_k[k]
        nat.check(lib.wf_batch2d_pass(desc_dev_ptr, ptr, n, p & 1, plan.offset(p), k,
                                      None if tune is None else ctypes.byref(tune),
                                      1 if fastdiv else 0, stream))


class Batch2D:
    """Device-resident set of solves advanced by one persistent launch per call."""

    def __init__(self, solves: Sequence[BatchSolve], n_steps: int, *, tune=None,
                 ctas_per_sm: int = 0, device=None, mode: str = "persistent") -> None:
        if tune == "auto" or mode == "auto":
            # time every candidate launch shape on these solves, keep the fastest
            from .autotune import tune_batch
            mode, tune = tune_batch(solves, n_steps, device=device)
        if mode not in ("persistent", "tiled", "queue"):
            raise ValueError("mode is 'persistent' (one CTA per solve, one launch), 'tiled' "
                             "(one launch per pass over every solve's tiles), 'queue' (one "
                             "persistent launch pulling (pass, tile) items) or 'auto'")
        self.mode = mode
        self._graph = None
        if not solves:
            raise ValueError("Batch2D needs at least one solve")
        self.device = torch.device(device) if device is not None else solves[0].grid.device
        if self.device.type != "cuda":
            raise RuntimeError("Batch2D runs on a CUDA device only (no CPU fallback)")
        nat.load()
        self.solves = list(solves)
        self.n_steps = n_steps
        self.tune = tune_struct(tune)
        self.ctas_per_sm = ctas_per_sm
        self.step = 0
        n = len(self.solves)
        # one flat allocation per role keeps the descriptor upload simple
        sizes = [s.grid.Nx * s.grid.Ny for s in self.solves]
        offs = [0]
        for sz in sizes:
            offs.append(offs[-1] + sz)
        total = offs[-1]
        self._state = torch.zeros((3, total), dtype=torch.float32, device=self.device)
        self._scratch = torch.empty((3, total), dtype=torch.float32, device=self.device)
        self._offs = offs
        nprb = [len(s.detectors) if s.detectors is not None else 0 for s in self.solves]
        toffs = [0]
        for q in nprb:
            toffs.append(toffs[-1] + q * n_steps)
        self._traces = torch.zeros(max(1, toffs[-1]), dtype=torch.float32, device=self.device)
        self._toffs = toffs
        self._tables = []
        self._desc = (nat.WfSolve2D * n)()
        for q, s in enumerate(self.solves):
            g = s.grid
            if g.Nx < 4 or g.Ny < 4:
                raise ValueError(f"solve {q}: grid {g.Nx}x{g.Ny} below 4x4")
            st = SourceTable(source_list(s.sources), self.device, _ALLOWED, 2)
            st.check_range(0, n_steps)
            pt = (s.detectors.table(self.device, _ALLOWED, (g.Nx, g.Ny, 1))
                  if s.detectors is not None else None)
            ca = None if s.Ca is None else s.Ca.to(self.device, torch.float32).contiguous()
            cb = None if s.Cb is None else s.Cb.to(self.device, torch.float32).contiguous()
            if (ca is None) != (cb is None):
                raise ValueError(f"solve {q}: Ca and Cb must be given together")
            if ca is not None and ca.numel() != g.Nx * g.Ny:
                raise ValueError(f"solve {q}: Ca/Cb must have Nx*Ny elements")
            self._tables.append((st, pt, ca, cb))
            d = self._desc[q]
            d.g = grid_struct(g, self.device)
            o = offs[q]
            el = 4
            d.ex = self._state[0].data_ptr() + o * el
            d.ey = self._state[1].data_ptr() + o * el
            d.hz = self._state[2].data_ptr() + o * el
            d.sx = self._scratch[0].data_ptr() + o * el
            d.sy = self._scratch[1].data_ptr() + o * el
            d.sz = self._scratch[2].data_ptr() + o * el
            d.ca = nat.ptr(ca)
            d.cb = nat.ptr(cb)
            d.src = st.ptr
            d.nsrc = st.count
            d.probes = None if pt is None else pt.ptr
            d.nprobe = 0 if pt is None else pt.count
            d.traces = self._traces.data_ptr() + toffs[q] * el
            d.trace_ld = n_steps
            d.trace_step0 = 0
            d.n_check = 0
            d.check_max = None
        both = nat.WF_FASTDIV_X | nat.WF_FASTDIV_Y
        self._fastdiv = all((d.g.flags & both) == both for d in self._desc)
        order = sorted(range(n), key=lambda q: -sizes[q])
        self._order = torch.tensor(order, dtype=torch.int32, device=self.device)
        self._queue = torch.zeros(1, dtype=torch.int32, device=self.device)
        self._desc_dev = None

    # ------------------------------------------------------------------
    @property
    def cells(self) -> int:
        return self._offs[-1]

    def _upload(self, step0: int, nsteps: int) -> None:
        self._launch_nsteps = nsteps
        for d in self._desc:
            d.step0 = step0
            d.nsteps = nsteps
            d.status = 0
        raw = bytes(memoryview(self._desc).cast("B"))
        host = torch.frombuffer(bytearray(raw), dtype=torch.uint8)
        if self._desc_dev is None:
            self._desc_dev = torch.empty_like(host, device=self.device)
        self._desc_dev.copy_(host)

    def run(self, nsteps: Optional[int] = None) -> None:
        """Advance every solve ``nsteps`` (default: all remaining) in one launch."""
        nsteps = self.n_steps - self.step if nsteps is None else nsteps
        if nsteps <= 0:
            return
        if self.step + nsteps > self.n_steps:
            raise IndexError(f"batch was built for {self.n_steps} steps")
        self._upload(self.step, nsteps)
        self.launch()
        self.step += nsteps

    @property
    def region(self) -> tuple[int, int]:
        t = self.tune
        return (48, 128) if t is None else (t.tile_i, t.tile_j)

    @property
    def depth(self) -> int:
        return 6 if self.tune is None else self.tune.steps_per_pass

    @property
    def threads(self) -> int:
        """Threads per CTA of the register layout (1024: the 6-row layout of
        the 48 x 128 region; 0: the region's default layout)."""
        return 0 if self.tune is None else self.tune.threads

    def launches_per_run(self) -> int:
        """Kernel launches of one full ``run()``."""
        if self.mode in ("persistent", "queue"):
            return 1
        plan = PassPlan(self.n_steps, self.depth)
        return plan.passes

    def _items(self, k: int):
        cache = self.__dict__.setdefault("_item_cache", {})
        if k not in cache:
            shapes = [(s.grid.Nx, s.grid.Ny) for s in self.solves]
            it = torch.from_numpy(tile_items(shapes, k, self.region)).to(self.device)
            cache[k] = (it, it.shape[0])
        t, n = cache[k]
        return t.data_ptr(), n

    def _queue_tables(self):
        """Tiles (cores of the full depth), their neighbour lists and the
        per-tile pass counters of the tile-queue mode, built once."""
        if "_qt" not in self.__dict__:
            shapes = [(s.grid.Nx, s.grid.Ny) for s in self.solves]
            tiles = tile_items(shapes, self.depth, self.region)
            nbr = tile_neighbours(tiles, self.depth, self.region)
            self._qt = (torch.from_numpy(tiles).to(self.device),
                        torch.from_numpy(nbr).to(self.device),
                        torch.zeros(len(tiles), dtype=torch.int32, device=self.device))
        return self._qt

    def launch(self) -> None:
        """Advance every solve by the uploaded step count: one persistent
        launch ("persistent": a CTA per solve; "queue": CTAs pulling
        (pass, tile) items), or one launch per temporal pass over every
        solve's tiles ("tiled"); each can be captured in a CUDA graph."""
        if self.mode == "queue":
            tiles, nbr, done = self._queue_tables()
            done.zero_()
            self._queue.zero_()
            nat.check(nat.load().wf_batch2d_queue(
                self._desc_dev.data_ptr(), tiles.data_ptr(), tiles.shape[0], nbr.data_ptr(),
                done.data_ptr(), self._queue.data_ptr(), self._launch_nsteps,
                None if self.tune is None else ctypes.byref(self.tune),
                1 if self._fastdiv else 0, -1, nat.stream_handle(self.device)))
            if PassPlan(self._launch_nsteps, self.depth).needs_copy:
                self._state.copy_(self._scratch)
            return
        if self.mode == "tiled":
            plan = PassPlan(self._launch_nsteps, self.depth)
            items = {plan.length(p): self._items(plan.length(p)) for p in range(plan.passes)}
            run_tiled_passes(self._desc_dev.data_ptr(), items, plan, self.tune, self._fastdiv,
                             nat.stream_handle(self.device))
            if plan.needs_copy:
                self._state.copy_(self._scratch)
            return
        self._queue.zero_()
        lib = nat.load()
        nat.check(lib.wf_batch2d_run(self._desc_dev.data_ptr(), len(self.solves),
                                     self._order.data_ptr(), self._queue.data_ptr(),
                                     None if self.tune is None else ctypes.byref(self.tune),
                                     self.ctas_per_sm, 1 if self._fastdiv else 0,
                                     nat.stream_handle(self.device)))

    def capture(self) -> None:
        """Record a full run from step 0 (state reset, every launch of the
        run) in a CUDA graph; ``replay()`` then repeats it with one graph
        launch.  Descriptors are uploaded once here and stay fixed."""
        self.reset()
        self._upload(0, self.n_steps)
        self.launch()                      # sets kernel attributes before capture
        torch.cuda.synchronize(self.device)
        graph = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream(self.device)
        side.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(side):
            with torch.cuda.graph(graph, stream=side, capture_error_mode="relaxed"):
                self._state.zero_()
                self._traces.zero_()
                self.launch()
        torch.cuda.current_stream(self.device).wait_stream(side)
        self._graph = graph
        self.step = self.n_steps

    def replay(self) -> None:
        """Re-run the captured run (reset + all steps) on the current stream."""
        if self._graph is None:
            raise RuntimeError("capture() first")
        self._graph.replay()
        self.step = self.n_steps

    def statuses(self) -> list[int]:
        raw = self._desc_dev.cpu().numpy().tobytes()
        arr = (nat.WfSolve2D * len(self.solves)).from_buffer_copy(raw)
        return [d.status for d in arr]

    def traces(self, q: int) -> torch.Tensor:
        """``(N_rx, n_steps)`` traces of solve q."""
        s = self.solves[q]
        nr = 0 if s.detectors is None else len(s.detectors)
        return self._traces[self._toffs[q]:self._toffs[q] + nr * self.n_steps].view(nr, self.n_steps)

    def traces_block(self, q0: int, n: int) -> torch.Tensor:
        """Traces of solves q0..q0+n-1 as one ``(n, N_rx, n_steps)`` view (all
        must record the same number of receivers; their buffers are adjacent)."""
        nr = len(self.solves[q0].detectors)
        for q in range(q0, q0 + n):
            if self.solves[q].detectors is None or len(self.solves[q].detectors) != nr:
                raise ValueError("traces_block needs solves with equal receiver counts")
        base = self._toffs[q0]
        return self._traces[base:base + n * nr * self.n_steps].view(n, nr, self.n_steps)

    def fields(self, q: int) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
        g = self.solves[q].grid
        o0, o1 = self._offs[q], self._offs[q + 1]
        return tuple(self._state[c, o0:o1].view(g.Nx, g.Ny, 1) for c in range(3))

    def reset(self) -> None:
        self._state.zero_()
        self._traces.zero_()
        self.step = 0

    # ------------------------------------------------------------------
    def run_plain_one(self, q: int, nsteps: Optional[int] = None, tune=None) -> None:
        """Solve q alone through ``wf_fdtd2d_run`` (the plain per-solve path),
        from step ``self.step``; does not advance ``self.step``."""
        nsteps = self.n_steps - self.step if nsteps is None else nsteps
        lib = nat.load()
        d = self._desc[q]
        st, pt, ca, cb = self._tables[q]
        t = tune_struct(tune)
        nat.check(lib.wf_fdtd2d_run(
            ctypes.byref(d.g), d.ex, d.ey, d.hz, d.sx, d.sy, d.sz, d.ca, d.cb, st.ptr, st.count,
            None if pt is None else pt.ptr, 0 if pt is None else pt.count, d.traces, d.trace_ld,
            0, self.step, nsteps, 0, None, None if t is None else ctypes.byref(t),
            nat.stream_handle(self.device)))

    def run_plain(self, nsteps: Optional[int] = None, tune=None) -> None:
        """The same solves, one ``wf_fdtd2d_run`` each (plain per-solve path)."""
        nsteps = self.n_steps - self.step if nsteps is None else nsteps
        for q in range(len(self._desc)):
            self.run_plain_one(q, nsteps, tune)
        self.step += nsteps
