"""Host side of the CUDA time loop shared by FDTD2D and FDTD3D.

Responsibilities: translate the reference objects (sources, detectors,
material tensors) into C-ABI descriptors once, own the ping-pong scratch
fields, call the C-ABI for a block of steps, and turn the device-side
stability maxima into the reference's telemetry and SimulationDivergedError
(src/core/fdtd2d.py:268-295).
"""

from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import torch

from .. import _native as nat


class SimulationDivergedError(RuntimeError):
    """Field magnitude above the stability threshold (src/core/fdtd2d.py:48-62)."""

    def __init__(self, message: str) -> None:
        super().__init__(message)


def source_list(sources) -> list:
    """Flatten a SourceCollection / single injector into injector objects."""
    if sources is None:
        return []
    if hasattr(sources, "sources"):
        return list(sources.sources)
    if hasattr(sources, "_sources"):
        return list(sources._sources)
    if hasattr(sources, "native_boxes"):
        return [sources]
    raise TypeError(f"unsupported source object {type(sources).__name__}: the CUDA engine needs "
                    "PointSource / LineSource / PlaneSource injectors (or a SourceCollection)")


class SourceTable:
    """Device array of wf_source boxes plus the tensors they point at."""

    def __init__(self, injectors: Sequence, device: torch.device, allowed: Sequence[str],
                 dims: int, dtype: torch.dtype = torch.float32) -> None:
        boxes = []
        for inj in injectors:
            if not hasattr(inj, "native_boxes"):
                raise TypeError(f"unsupported source {type(inj).__name__} for the CUDA engine")
            boxes.extend(inj.native_boxes())
        self.keep = []
        self.n_wave_min = None
        arr = (nat.WfSource * max(1, len(boxes)))()
        for q, (comp, i0, i1, j0, j1, k0, k1, wave, amp) in enumerate(boxes):
            if comp not in allowed:
                raise KeyError(f"source component {comp!r} is not a field of the {dims}D engine "
                               f"(allowed: {tuple(allowed)})")
            wave = wave.contiguous()
            if wave.dtype != dtype:
                raise TypeError(f"source waveforms must be {dtype} (the grid dtype) on the CUDA "
                                "engine")
            if wave.device != device:
                wave = wave.to(device)
            self.keep.append(wave)
            if amp is not None:
                amp = amp.to(device=device, dtype=dtype).contiguous()
                self.keep.append(amp)
            arr[q] = nat.WfSource(nat.COMP_CODE[comp], i0, i1, j0, j1, k0, k1, wave.numel(),
                                  wave.data_ptr(), None if amp is None else amp.data_ptr())
            n = wave.numel()
            self.n_wave_min = n if self.n_wave_min is None else min(self.n_wave_min, n)
        self.count = len(boxes)
        self.dev = nat.to_device_bytes(arr, device) if boxes else None

    def check_range(self, step0: int, nsteps: int) -> None:
        if self.count and step0 + nsteps > self.n_wave_min:
            raise IndexError(f"a source waveform holds {self.n_wave_min} steps but steps up to "
                             f"{step0 + nsteps - 1} were requested (build sources with a larger "
                             "N_steps)")

    @property
    def ptr(self) -> Optional[int]:
        return None if self.dev is None else self.dev.data_ptr()


class ProbeTable:
    """Device array of wf_probe points."""

    def __init__(self, probes: Sequence[tuple], device: torch.device, allowed: Sequence[str],
                 shape: tuple) -> None:
        arr = (nat.WfProbe * max(1, len(probes)))()
        for q, p in enumerate(probes):
            comp = p[0]
            idx = tuple(int(v) for v in p[1:]) + (0,) * (4 - len(p))
            if comp not in allowed:
                raise KeyError(f"probe component {comp!r} not allowed (allowed: {tuple(allowed)})")
            for ax, (v, n) in enumerate(zip(idx, shape)):
                if not (0 <= v < n):
                    raise ValueError(f"probe {p} index {v} out of range [0, {n}) on axis {ax}")
            arr[q] = nat.WfProbe(nat.COMP_CODE[comp], *idx[:3])
        self.count = len(probes)
        self.dev = nat.to_device_bytes(arr, device) if probes else None

    @property
    def ptr(self) -> Optional[int]:
        return None if self.dev is None else self.dev.data_ptr()


class EngineBase:
    """Shared telemetry / stability bookkeeping."""

    _components: tuple[str, ...] = ()
    _dtype: torch.dtype = torch.float32   # arithmetic type of fields, waves and traces

    def _init_common(self, stability_threshold: float, n_check: int) -> None:
        self._threshold = stability_threshold
        self._n_check = n_check
        self.steps_completed = 0
        self.elapsed_time = 0.0
        self.mcells_per_second = 0.0
        self.last_field_max = -1.0
        self.n_stability_checks = 0
        self._src_key = None
        self._src_table: Optional[SourceTable] = None
        self._graphs: Optional[dict] = None  # CUDA graphs of runs (compile_step)

    def _check_buffer(self, step0: int, nsteps: int):
        nc = self._n_check
        if nc <= 0:
            return None, 0
        count = (step0 + nsteps) // nc - step0 // nc
        if count == 0:
            return None, 0
        bits = torch.int64 if self._dtype == torch.float64 else torch.int32
        buf = torch.zeros(count * len(self._components), dtype=bits, device=self._device)
        return buf, count

    def _process_checks(self, buf: Optional[torch.Tensor], count: int, step0: int) -> None:
        if buf is None:
            return
        vals = buf.cpu().view(self._dtype).view(count, len(self._components)).tolist()
        first = step0 // self._n_check + 1
        for c in range(count):
            self.n_stability_checks += 1
            for name, v in zip(self._components, vals[c]):
                if v > self.last_field_max:
                    self.last_field_max = v
                if v > self._threshold:
                    raise SimulationDivergedError(
                        f"Simulation diverged at step {(first + c) * self._n_check}: {name} max = "
                        f"{v:.3e} exceeds threshold {self._threshold:.3e}. Check CFL condition "
                        f"(dt={self._grid.dt:.3e}) and source amplitude.")

    def _sources_table(self, allowed, dims) -> SourceTable:
        injectors = source_list(self._sources)
        key = (id(self._sources), tuple(id(s) for s in injectors))
        if self._src_table is None or self._src_key != key:
            self._src_table = SourceTable(injectors, self._device, allowed, dims, self._dtype)
            self._src_key = key
        return self._src_table

    # ---- CUDA-graph replay of runs -------------------------------------
    def compile_step(self, *, backend: str = "inductor", mode: str = "reduce-overhead") -> None:
        """Replay runs from CUDA graphs (the counterpart of the reference's
        ``torch.compile(mode='reduce-overhead')`` step, src/core/fdtd3d.py:
        404-419; ``backend`` and ``mode`` are accepted and ignored).  From now
        on the first ``run(n)`` from a given start step (with given detectors
        and sources) is captured -- every pass launch of it, the zeroing of its
        trace and stability buffers -- and replayed; later runs with the same
        start step and length (e.g. after ``reset()``) replay that graph, one
        launch instead of one per pass, with bit-identical results.  Returned
        traces are copies (the graph owns its buffer)."""
        self._graphs = {}

    def _prepare(self) -> None:
        """Build the device tables and scratch a run needs before it can be
        captured (their uploads and allocations cannot happen inside a graph)."""

    def _graphed(self, nsteps: int, probes, alloc_traces):
        """Run ``_advance(nsteps, probes, traces)`` through the cached graph of
        this (start step, length, detectors, sources); returns the traces
        buffer owned by the graph (or None)."""
        self._prepare()
        start = self.steps_completed
        key = (start, nsteps, None if probes is None else id(probes), id(self._src_table),
               None if self._scratch is None else self._scratch.data_ptr())
        ent = self._graphs.get(key)
        if ent is None:
            rec = []
            self._process_checks = lambda buf, count, step0: rec.append((buf, count, step0))
            graph = torch.cuda.CUDAGraph()
            side = torch.cuda.Stream(self._device)
            side.wait_stream(torch.cuda.current_stream(self._device))
            try:
                with torch.cuda.stream(side):
                    with torch.cuda.graph(graph, stream=side, capture_error_mode="relaxed"):
                        traces = alloc_traces()
                        self._advance(nsteps, probes, traces)
            finally:
                del self._process_checks
                self.steps_completed = start
            torch.cuda.current_stream(self._device).wait_stream(side)
            ent = (graph, traces, rec)
            self._graphs[key] = ent
        graph, traces, rec = ent
        graph.replay()
        self.steps_completed = start + nsteps
        for buf, count, step0 in rec:
            self._process_checks(buf, count, step0)
        return traces

    def reset(self) -> None:
        """Zero fields and telemetry (src/core/fdtd2d.py:365-378)."""
        self._fields.zero_()
        self.steps_completed = 0
        self.elapsed_time = 0.0
        self.mcells_per_second = 0.0
        self.last_field_max = -1.0
        self.n_stability_checks = 0

    @property
    def grid(self):
        return self._grid

    @property
    def fields(self):
        return self._fields

    @property
    def dt(self) -> float:
        return self._grid.dt

    @property
    def time(self) -> float:
        return self.steps_completed * self._grid.dt

    @property
    def throughput(self) -> float:
        return self.mcells_per_second


def tune_struct(tune) -> Optional[ctypes.Structure]:
    if tune is None:
        return None
    if isinstance(tune, nat.WfTune):
        return tune
    k, ti, tj, tk, th = tune
    return nat.WfTune(k, ti, tj, tk, th)
