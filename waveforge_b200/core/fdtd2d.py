"""2D TM {Ex, Ey, Hz} time-stepper on the CUDA engine (drop-in for src/core/fdtd2d.py).

Constructor, ``step``/``run``/``reset``, telemetry attributes and errors follow
the reference ``FDTD2D`` (src/core/fdtd2d.py:67-423).  Each call hands a block
of steps to ``wf_fdtd2d_run`` (fused H+Mur+injection+E+detector kernel,
temporally blocked); fields stay in the caller's FieldSet tensors.  ``run``
additionally accepts ``record=Detectors(...)`` to gather traces on the device
inside the same kernels.  A float64 FieldSet runs ``wf_fdtd2d_run_f64``
instead: the reference's operations one launch each, in float64, for
verification runs.
"""

from __future__ import annotations

import ctypes
import time
from typing import Optional

import torch

from .. import _native as nat
from ._engine import EngineBase, ProbeTable, SimulationDivergedError, tune_struct  # noqa: F401
from .boundaries import MurABC
from .fields import FieldSet
from .grid import YeeGrid

EPS0: float = 8.8541878128e-12
MU0: float = 1.2566370614e-6

_ALLOWED_2D = ("Ex", "Ey", "Hz")


class FDTD2D(EngineBase):
    """2D TM FDTD time-stepper (src/core/fdtd2d.py:67-181)."""

    _components = _ALLOWED_2D

    def __init__(self, grid: YeeGrid, fields: FieldSet, boundary: MurABC, sources=None, *,
                 Ca: Optional[torch.Tensor] = None, Cb: Optional[torch.Tensor] = None,
                 stability_threshold: float = 1e10, n_check: int = 100, tune=None) -> None:
        if grid.Nx < 4:
            raise ValueError(f"grid.Nx must be >= 4 for a valid Yee stencil, got {grid.Nx}")
        if grid.Ny < 4:
            raise ValueError(f"grid.Ny must be >= 4 for a valid Yee stencil, got {grid.Ny}")
        if boundary._Nx != grid.Nx or boundary._Ny != grid.Ny:
            raise ValueError(f"boundary was built for a grid of shape ({boundary._Nx}, "
                             f"{boundary._Ny}) but grid has shape ({grid.Nx}, {grid.Ny}). They "
                             "must match.")
        if (Ca is None) != (Cb is None):
            raise ValueError("Ca and Cb must be provided together or both omitted.")
        self._grid, self._fields, self._boundary, self._sources = grid, fields, boundary, sources
        self._Dh = grid.dt / MU0
        self._De = grid.dt / EPS0
        self._dx, self._dy = grid.dx, grid.dy
        self._Ca, self._Cb = Ca, Cb
        self._has_materials = Ca is not None
        self._init_common(stability_threshold, n_check)
        self._device = fields.Ex.device
        for name in _ALLOWED_2D:
            nat.require_cuda(getattr(fields, name), f"FieldSet.{name}")
        if fields.dtype not in (torch.float32, torch.float64):
            raise TypeError(f"the CUDA engine computes in float32 (the reference default dtype) "
                            f"or float64, not {fields.dtype}")
        self._dtype = fields.dtype
        if Ca is not None:
            nat.require_cuda(Ca, "Ca")
            nat.require_cuda(Cb, "Cb")
        nat.load()
        # a CPML boundary (new) replaces the Mur edges: the step runs wf_cpml2d_run
        self._cpml = bool(getattr(boundary, "is_cpml", False))
        if self._cpml and fields.is_batched:
            raise ValueError("the CPML engine runs unbatched FieldSets")
        self._f64 = self._dtype == torch.float64
        if self._f64 and self._cpml:
            raise TypeError("the CPML engine computes in float32")
        mx = 0.0 if self._cpml else boundary.C_mur_x
        my = 0.0 if self._cpml else boundary.C_mur_y
        if self._f64:
            # float64 verification path (wf_fdtd2d_run_f64): the reference's
            # Python-float scalars unrounded; float32 Ca/Cb widen exactly, as
            # the reference's float32 x float64 products promote them
            self._g = nat.WfGrid2DF64(grid.Nx, grid.Ny, self._Dh, self._De, grid.dx, grid.dy,
                                      mx, my)
            if Ca is not None and Ca.dtype != torch.float64:
                self._Ca, self._Cb = Ca.to(torch.float64), Cb.to(torch.float64)
        else:
            if Ca is not None and (Ca.dtype != torch.float32 or Cb.dtype != torch.float32):
                raise TypeError("Ca and Cb must be float32 for a float32 FieldSet")
            self._g = nat.WfGrid2D(grid.Nx, grid.Ny, nat.f32(self._Dh), nat.f32(self._De),
                                   nat.f32(grid.dx), nat.f32(grid.dy), nat.f32(mx), nat.f32(my),
                                   nat.fastdiv_flags(self._device, grid.dx, grid.dy))
        self._tune = tune_struct(tune)
        self._scratch: Optional[torch.Tensor] = None

    # ------------------------------------------------------------------
    def _members(self):
        """(Ex, Ey, Hz, Ca, Cb) per batch member (reference batches share sources)."""
        f = self._fields
        ca, cb = self._Ca, self._Cb
        if not f.is_batched:
            return [(f.Ex, f.Ey, f.Hz, ca, cb)]
        out = []
        for b in range(f.batch_size):
            cab = None if ca is None else (ca[b] if ca.dim() == 4 else ca)
            cbb = None if cb is None else (cb[b] if cb.dim() == 4 else cb)
            out.append((f.Ex[b], f.Ey[b], f.Hz[b], cab, cbb))
        return out

    def _advance(self, nsteps: int, probes: Optional[ProbeTable] = None,
                 traces: Optional[torch.Tensor] = None) -> None:
        if nsteps <= 0:
            return
        src = self._sources_table(_ALLOWED_2D, 2)
        step0 = self.steps_completed
        src.check_range(step0, nsteps)
        g = self._grid
        self._alloc_scratch()
        chk, count = self._check_buffer(step0, nsteps)
        lib = nat.load()
        stream = nat.stream_handle(self._device)
        members = self._members()
        if probes is not None and len(members) > 1:
            raise ValueError("Detectors.record supports unbatched FieldSets")
        for ex, ey, hz, ca, cb in members:
            for t in (ex, ey, hz) + ((ca, cb) if ca is not None else ()):
                if not t.is_contiguous() or t.numel() != g.Nx * g.Ny:
                    raise ValueError("field / coefficient tensors must be contiguous (Nx, Ny, 1)")
            if self._f64:
                nat.check(lib.wf_fdtd2d_run_f64(
                    ctypes.byref(self._g), ex.data_ptr(), ey.data_ptr(), hz.data_ptr(),
                    self._scratch.data_ptr(), nat.ptr(ca), nat.ptr(cb), src.ptr, src.count,
                    None if probes is None else probes.ptr, 0 if probes is None else probes.count,
                    None if traces is None else traces.data_ptr(),
                    0 if traces is None else traces.stride(0), step0, step0, nsteps,
                    self._n_check if chk is not None else 0,
                    None if chk is None else chk.data_ptr(), stream))
                continue
            if self._cpml:
                bd = self._boundary
                nat.check(lib.wf_cpml2d_run(
                    ctypes.byref(self._g), ex.data_ptr(), ey.data_ptr(), hz.data_ptr(),
                    nat.ptr(ca), nat.ptr(cb), bd.depth, bd.tables.data_ptr(), bd.psi.data_ptr(),
                    src.ptr, src.count, None if probes is None else probes.ptr,
                    0 if probes is None else probes.count,
                    None if traces is None else traces.data_ptr(),
                    0 if traces is None else traces.stride(0), step0, step0, nsteps,
                    self._n_check if chk is not None else 0,
                    None if chk is None else chk.data_ptr(), stream))
                continue
            s = self._scratch
            nat.check(lib.wf_fdtd2d_run(
                ctypes.byref(self._g), ex.data_ptr(), ey.data_ptr(), hz.data_ptr(),
                s[0].data_ptr(), s[1].data_ptr(), s[2].data_ptr(),
                nat.ptr(ca), nat.ptr(cb), src.ptr, src.count,
                None if probes is None else probes.ptr, 0 if probes is None else probes.count,
                None if traces is None else traces.data_ptr(),
                0 if traces is None else traces.stride(0), step0,
                step0, nsteps, self._n_check if chk is not None else 0,
                None if chk is None else chk.data_ptr(),
                None if self._tune is None else ctypes.byref(self._tune), stream))
        self.steps_completed += nsteps
        self._process_checks(chk, count, step0)

    def _alloc_scratch(self) -> None:
        """Ping-pong partners of the float32 passes, or the float64 path's Mur
        snapshot of Hz."""
        if self._scratch is None:
            g = self._grid
            shape = (g.Nx, g.Ny) if self._f64 else (3, g.Nx, g.Ny)
            self._scratch = torch.empty(shape, dtype=self._dtype, device=self._device)

    def _prepare(self) -> None:
        self._sources_table(_ALLOWED_2D, 2)
        self._alloc_scratch()

    def reset(self) -> None:
        """Zero fields and telemetry, and the CPML layer memories if any."""
        super().reset()
        if self._cpml:
            self._boundary.reset()

    # ------------------------------------------------------------------
    def step(self) -> None:
        """Advance one full leapfrog step in place (src/core/fdtd2d.py:187-266)."""
        self._advance(1)

    def run(self, n_steps: int, *, verbose: bool = False, record=None):
        """Run ``n_steps`` steps (src/core/fdtd2d.py:301-359).

        ``record``: optional ``Detectors``; its traces for these steps are
        gathered on the device and returned as a ``(N_rx, n_steps)`` tensor.
        """
        is_cuda = self._device.type == "cuda"
        report = max(1, n_steps // 10)
        if is_cuda:
            torch.cuda.synchronize(self._device)
        t0 = time.perf_counter()
        start = self.steps_completed
        traces = probes = None
        if record is not None:
            probes = record.table(self._device, _ALLOWED_2D, (self._grid.Nx, self._grid.Ny, 1))
        graphed = self._graphs is not None and not verbose and n_steps > 0 and not self._cpml
        if graphed:
            # captured once per (start, length, detectors), replayed afterwards
            count = 0 if probes is None else probes.count
            traces = self._graphed(n_steps, probes, lambda: None if probes is None else torch.zeros(
                (count, n_steps), dtype=self._dtype, device=self._device))
            if traces is not None:
                traces = traces.clone()
        elif record is not None:
            traces = torch.zeros((probes.count, n_steps), dtype=self._dtype, device=self._device)
        done = n_steps if graphed else 0
        chunk = report if verbose else n_steps
        while done < n_steps:
            ns = min(chunk, n_steps - done)
            tv = None if traces is None else traces[:, done:]
            self._advance(ns, probes, tv)
            done += ns
            if verbose:
                torch.cuda.synchronize(self._device)
                el = time.perf_counter() - t0
                if el > 0:
                    self.mcells_per_second = done * self._grid.Nx * self._grid.Ny / el / 1e6
                self.elapsed_time = el
                print(f"  {100 * done // n_steps:3d}%  step {self.steps_completed}  "
                      f"field_max={self.last_field_max:.3e}  {self.mcells_per_second:.1f} Mcells/s")
        if is_cuda:
            torch.cuda.synchronize(self._device)
        el = time.perf_counter() - t0
        self.elapsed_time += el
        if el > 0:
            self.mcells_per_second = (self.steps_completed - start) * self._grid.Nx * self._grid.Ny / el / 1e6
        if record is not None:
            record._store(traces)
            return traces
        return None

    def __repr__(self) -> str:
        g = self._grid
        return (f"FDTD2D(shape=({g.Nx}, {g.Ny}, {g.Nz}), steps={self.steps_completed}, "
                f"time={self.time:.4e} s, throughput={self.mcells_per_second:.2f} Mcells/s, "
                f"device={g.device})")

