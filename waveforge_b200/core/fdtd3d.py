"""3D six-component time-stepper on the CUDA engine (drop-in for src/core/fdtd3d.py).

Same constructor, ``step``/``run``/``reset``/``compile_step`` surface and
telemetry as the reference ``FDTD3D`` (src/core/fdtd3d.py:116-580); each
call hands a block of steps to ``wf_fdtd3d_run``.
"""

from __future__ import annotations

import ctypes
import math
import time
import warnings
from typing import Optional

import torch

from .. import _native as nat
from ._engine import (EngineBase, ProbeTable, SimulationDivergedError, SourceTable,  # noqa: F401
                      source_list, tune_struct)
from .fields import FIELD_COMPONENTS, FieldSet
from .grid import YeeGrid

EPS0: float = 8.8541878128e-12
MU0: float = 1.2566370614e-6
_C0: float = 1.0 / math.sqrt(EPS0 * MU0)


class FDTD3D(EngineBase):
    """3D full-vector FDTD time-stepper (src/core/fdtd3d.py:116-255)."""

    _components = FIELD_COMPONENTS

    def __init__(self, grid: YeeGrid, fields: FieldSet, boundary: object, sources: Optional[object] = None,
                 *, Ca: Optional[torch.Tensor] = None, Cb: Optional[torch.Tensor] = None,
                 stability_threshold: float = 1e10, n_check: int = 100, tune=None,
                 member_sources: Optional[list] = None) -> None:
        """``member_sources`` (new; batched FieldSet only): one source object
        per batch member -- e.g. one transmitter per member -- instead of the
        reference's broadcast of ``sources`` to every member.  Every member
        must inject the same number of source boxes."""
        if grid.Nx < 4:
            raise ValueError(f"grid.Nx must be >= 4 for a valid 3D Yee stencil, got {grid.Nx}")
        if grid.Ny < 4:
            raise ValueError(f"grid.Ny must be >= 4 for a valid 3D Yee stencil, got {grid.Ny}")
        if grid.Nz > 1 and grid.Nz < 4:
            raise ValueError(f"grid.Nz must be >= 4 when using 3D mode, got {grid.Nz}. Use Nz=1 for "
                             "2D-equivalent mode.")
        self._grid, self._fields, self._boundary, self._sources = grid, fields, boundary, sources
        self._Dh = grid.dt / MU0
        self._De = grid.dt / EPS0
        self._dx, self._dy, self._dz = grid.dx, grid.dy, grid.dz
        if (Ca is None) != (Cb is None):
            raise ValueError("Ca and Cb must be provided together or both omitted.")
        self._Ca, self._Cb = Ca, Cb
        self._has_materials = Ca is not None
        dx, dy, dz = grid.dx, grid.dy, grid.dz
        lim = 0.99 / (_C0 * math.sqrt(1.0 / (dx * dx) + 1.0 / (dy * dy) + 1.0 / (dz * dz)))
        if grid.dt > lim:
            warnings.warn(f"grid.dt={grid.dt:.6e} exceeds 0.99 × CFL limit {lim:.6e}. Simulation "
                          "may be unstable.", UserWarning, stacklevel=2)
        self._init_common(stability_threshold, n_check)
        self._device = fields.Ex.device
        for name in FIELD_COMPONENTS:
            nat.require_cuda(getattr(fields, name), f"FieldSet.{name}")
        if fields.dtype != torch.float32:
            raise TypeError("the CUDA engine computes in float32 (the reference default dtype)")
        if Ca is not None:
            nat.require_cuda(Ca, "Ca")
            nat.require_cuda(Cb, "Cb")
        nat.load()
        mx = getattr(boundary, "C_mur_x", None)
        if mx is None:
            raise TypeError("FDTD3D needs a MurABC3D boundary")
        self._g = nat.WfGrid3D(grid.Nx, grid.Ny, grid.Nz, nat.f32(self._Dh), nat.f32(self._De),
                               nat.f32(dx), nat.f32(dy), nat.f32(dz), nat.f32(boundary.C_mur_x),
                               nat.f32(boundary.C_mur_y), nat.f32(boundary.C_mur_z),
                               nat.fastdiv_flags(self._device, dx, dy, dz))
        self._tune = tune_struct(tune)
        self._scratch: Optional[torch.Tensor] = None
        self._member_sources = None
        self._member_table = None
        if member_sources is not None:
            if not fields.is_batched or len(member_sources) != fields.batch_size:
                raise ValueError("member_sources needs a batched FieldSet and one entry per member")
            if sources is not None:
                raise ValueError("give either sources (broadcast) or member_sources, not both")
            if tune is not None or grid.Nz == 1:
                raise ValueError("member_sources runs on the default 3D streaming kernel")
            self._member_sources = list(member_sources)

    def _prepare(self) -> None:
        if self._member_sources is None:
            self._sources_table(FIELD_COMPONENTS, 3)
        else:
            self._members_table()
        g, f = self._grid, self._fields
        n = g.Nx * g.Ny * g.Nz
        stream_tune = self._tune is None or self._tune.tile_i == 0
        if f.is_batched and stream_tune and g.Nz > 1:
            if self._scratch is None or self._scratch.numel() != 6 * f.batch_size * n:
                self._scratch = torch.empty((6, f.batch_size, n), dtype=torch.float32,
                                            device=self._device)
        elif self._scratch is None:
            self._scratch = torch.empty((6, g.Nx, g.Ny, g.Nz), dtype=torch.float32,
                                        device=self._device)

    def _members(self):
        f = self._fields
        comps = [getattr(f, c) for c in FIELD_COMPONENTS]
        if not f.is_batched:
            return [(comps, self._Ca, self._Cb)]
        out = []
        for b in range(f.batch_size):
            ca = None if self._Ca is None else (self._Ca[b] if self._Ca.dim() == 4 else self._Ca)
            cb = None if self._Cb is None else (self._Cb[b] if self._Cb.dim() == 4 else self._Cb)
            out.append(([t[b] for t in comps], ca, cb))
        return out

    def _advance(self, nsteps: int, probes: Optional[ProbeTable] = None,
                 traces: Optional[torch.Tensor] = None) -> None:
        if nsteps <= 0:
            return
        src = self._sources_table(FIELD_COMPONENTS, 3) if self._member_sources is None \
            else self._members_table()
        step0 = self.steps_completed
        src.check_range(step0, nsteps)
        g = self._grid
        n = g.Nx * g.Ny * g.Nz
        if self._scratch is None:
            self._scratch = torch.empty((6, g.Nx, g.Ny, g.Nz), dtype=torch.float32, device=self._device)
        chk, count = self._check_buffer(step0, nsteps)
        lib = nat.load()
        stream = nat.stream_handle(self._device)
        f = self._fields
        stream_tune = self._tune is None or self._tune.tile_i == 0
        if f.is_batched and stream_tune and g.Nz > 1:
            self._advance_batched(nsteps, src, probes, traces, chk, step0)
            self.steps_completed += nsteps
            self._process_checks(chk, count, step0)
            return
        members = self._members()
        if probes is not None and len(members) > 1:
            raise ValueError("Detectors.record on a batched FieldSet needs the default 3D tune")
        sp = (ctypes.c_void_p * 6)(*[self._scratch[c].data_ptr() for c in range(6)])
        for comps, ca, cb in members:
            for t in comps + ([ca, cb] if ca is not None else []):
                if not t.is_contiguous() or t.numel() != n:
                    raise ValueError("field / coefficient tensors must be contiguous (Nx, Ny, Nz)")
            fp = (ctypes.c_void_p * 6)(*[t.data_ptr() for t in comps])
            nat.check(lib.wf_fdtd3d_run(
                ctypes.byref(self._g), fp, sp, nat.ptr(ca), nat.ptr(cb), src.ptr, src.count,
                None if probes is None else probes.ptr, 0 if probes is None else probes.count,
                None if traces is None else traces.data_ptr(),
                0 if traces is None else traces.stride(0), step0, step0, nsteps,
                self._n_check if chk is not None else 0, None if chk is None else chk.data_ptr(),
                None if self._tune is None else ctypes.byref(self._tune), stream))
        self.steps_completed += nsteps
        self._process_checks(chk, count, step0)

    def _members_table(self) -> SourceTable:
        """One table of every member's source boxes, member after member."""
        if self._member_table is None:
            per = [sum(len(s.native_boxes()) for s in source_list(m)) for m in self._member_sources]
            if len(set(per)) != 1:
                raise ValueError(f"member_sources inject different numbers of boxes: {per}")
            inj = [s for m in self._member_sources for s in source_list(m)]
            self._member_table = SourceTable(inj, self._device, FIELD_COMPONENTS, 3)
            self._member_per = per[0]
        return self._member_table

    def _advance_batched(self, nsteps, src, probes, traces, chk, step0) -> None:
        """All batch members in one launch per step (wf_fdtd3d_batch_run):
        every member gets the same sources, as the reference broadcasts them
        (src/core/sources.py:885-887); Ca/Cb may be per member (B, Nx, Ny, Nz)
        or shared (Nx, Ny, Nz)."""
        g, f = self._grid, self._fields
        n, B = g.Nx * g.Ny * g.Nz, f.batch_size
        comps = [getattr(f, c) for c in FIELD_COMPONENTS]
        for t in comps:
            if not t.is_contiguous():
                raise ValueError("batched field tensors must be contiguous (B, Nx, Ny, Nz)")
        if self._scratch is None or self._scratch.numel() != 6 * B * n:
            self._scratch = torch.empty((6, B, n), dtype=torch.float32, device=self._device)
        ca, cb = self._Ca, self._Cb
        cstride = 0
        if ca is not None:
            if not (ca.is_contiguous() and cb.is_contiguous()):
                raise ValueError("Ca / Cb must be contiguous")
            if ca.numel() == B * n:
                cstride = n
            elif ca.numel() != n:
                raise ValueError("Ca / Cb must be (Nx, Ny, Nz) or (B, Nx, Ny, Nz)")
        fp = (ctypes.c_void_p * 6)(*[t.data_ptr() for t in comps])
        sp = (ctypes.c_void_p * 6)(*[self._scratch[c].data_ptr() for c in range(6)])
        per, sstride = src.count, 0
        if self._member_sources is not None:
            per = sstride = self._member_per
        nat.check(nat.load().wf_fdtd3d_batch_run(
            ctypes.byref(self._g), B, n, fp, sp, nat.ptr(ca), nat.ptr(cb), cstride, src.ptr,
            per, sstride, None if probes is None else probes.ptr,
            0 if probes is None else probes.count, None if traces is None else traces.data_ptr(),
            0 if traces is None else traces.stride(-2),
            0 if traces is None else traces.stride(0), step0, step0, nsteps,
            self._n_check if chk is not None else 0, None if chk is None else chk.data_ptr(),
            None if self._tune is None else ctypes.byref(self._tune),
            nat.stream_handle(self._device)))

    def step(self) -> None:
        """Advance all six components one step in place (src/core/fdtd3d.py:261-402)."""
        self._advance(1)

    def run(self, n_steps: int, *, verbose: bool = False, record=None):
        """Run ``n_steps`` steps (src/core/fdtd3d.py:457-516); ``record`` as in FDTD2D.run."""
        g = self._grid
        cells = g.Nx * g.Ny * g.Nz
        torch.cuda.synchronize(self._device)
        t0 = time.perf_counter()
        start = self.steps_completed
        probes = traces = None
        shape = None
        if record is not None:
            probes = record.table(self._device, FIELD_COMPONENTS, (g.Nx, g.Ny, g.Nz))
            shape = ((self._fields.batch_size,) if self._fields.is_batched else ()) + (probes.count,
                                                                                     n_steps)
        graphed = self._graphs is not None and not verbose and n_steps > 0
        if graphed:
            # captured once per (start, length, detectors), replayed afterwards
            traces = self._graphed(n_steps, probes, lambda: None if shape is None else torch.zeros(
                shape, dtype=torch.float32, device=self._device))
            if traces is not None:
                traces = traces.clone()
        elif record is not None:
            traces = torch.zeros(shape, dtype=torch.float32, device=self._device)
        chunk = max(1, n_steps // 10) if verbose else n_steps
        done = n_steps if graphed else 0
        while done < n_steps:
            ns = min(chunk, n_steps - done)
            self._advance(ns, probes, None if traces is None else traces[..., done:])
            done += ns
            if verbose:
                torch.cuda.synchronize(self._device)
                el = time.perf_counter() - t0
                if el > 0:
                    self.mcells_per_second = done * cells / el / 1e6
                self.elapsed_time = el
                print(f"  {100 * done // n_steps:3d}%  step {self.steps_completed}  "
                      f"field_max={self.last_field_max:.3e}  {self.mcells_per_second:.1f} Mcells/s")
        torch.cuda.synchronize(self._device)
        el = time.perf_counter() - t0
        st = ctypes.c_int32(0)
        nat.check(nat.load().wf_fdtd3d_take_status(ctypes.byref(st)))
        if st.value:
            raise RuntimeError(f"FDTD3D: a device pipeline wait gave up (status {st.value}); "
                               "the fields of this run are incomplete")
        self.elapsed_time += el
        if el > 0:
            self.mcells_per_second = (self.steps_completed - start) * cells / el / 1e6
        if record is not None:
            record._store(traces)
            return traces
        return None

    def __repr__(self) -> str:
        g = self._grid
        return (f"FDTD3D(shape=({g.Nx}, {g.Ny}, {g.Nz}), steps={self.steps_completed}, "
                f"time={self.time:.4e} s, throughput={self.mcells_per_second:.2f} Mcells/s, "
                f"device={g.device})")
