"""Continuous-batching request loop for 2D TM imaging solves.

The reference serves nothing: its drivers run one ``FDTD2D`` per
transmitter, one after another (examples/brain_mimo_imaging.py:149-204), and
its dataset generator does the same per sample (src/datasets/generator.py:
162-248).  ``Server`` keeps every admitted request's fields, coefficients,
traces (and, for gradient requests, checkpoints) resident on the device and
advances ALL admitted solves together by one chunk of ``chunk_steps`` steps
at a time: in the default "tiled" mode each temporal pass of the chunk is one
``wf_batch2d_pass`` launch over the tiles of every admitted solve (a large
grid spreads over all SMs); the "persistent" mode runs the chunk as one
``wf_batch2d_run`` launch with one CTA per solve.  Between chunks it

* admits queued requests in arrival order while their HBM footprint fits the
  budget (their phantoms are painted on the device by ``wf_paint2d``; only
  the region list crosses PCIe),
* retires finished requests (traces copied to pinned host memory),
* starts the adjoint of finished gradient requests on a second stream, where
  it overlaps the following chunks of the others.

Chunking does not change any result: every solve runs the same tile routine
whatever else is in the launch, and split runs equal one run, so a request's
traces (and gradient) are bit-identical alone and in any mix.

Latency = device completion time of the request's last operation (CUDA event,
aligned to the host clock at start) minus its submit time.  An optional
``max_wait_s`` rejects a request at submit when the estimated wait for the
work already queued ahead of it exceeds the bound (explicit overload policy).
"""

from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np
import torch

from . import _native as nat
from .batch import PassPlan, grid_struct, run_tiled_passes, tile_items
from .core._engine import ProbeTable
from .core.materials import MaterialMap

_ALLOWED = ("Ex", "Ey", "Hz")


@dataclass
class ImagingRequest:
    """One request: a phantom (device-paintable ``MaterialMap`` on a CPU grid
    whose Nx, Ny, dx, dt define the solve), transmitters (soft Hz point
    sources, one solve each), receivers (Hz points) and the step count.
    ``target``: a second phantom whose traces are the measurement; the
    request then also returns dL/deps_r and dL/dsigma of
    L = 1/2 ||traces(material) - traces(target)||^2."""

    material: MaterialMap
    transmitters: Sequence[tuple]
    receivers: Sequence[tuple]
    n_steps: int
    waveform: object
    target: Optional[MaterialMap] = None
    tag: object = None


@dataclass
class Ticket:
    request: ImagingRequest
    id: int
    t_submit: float
    status: str = "queued"          # queued, running, adjoint, done, rejected
    t_admit: Optional[float] = None
    t_done: Optional[float] = None
    traces: Optional[torch.Tensor] = None       # host (n_tx, n_rx, n_steps)
    grad_eps: Optional[torch.Tensor] = None     # host (Nx, Ny) float64
    grad_sigma: Optional[torch.Tensor] = None
    loss: Optional[float] = None
    reason: str = ""

    @property
    def latency(self) -> Optional[float]:
        return None if self.t_done is None else self.t_done - self.t_submit


def request_cells(req: ImagingRequest) -> int:
    g = req.material._grid
    return g.Nx * g.Ny


def request_work(req: ImagingRequest) -> int:
    """Cell-updates of the request's forward solves."""
    n = len(req.transmitters) * (2 if req.target is not None else 1)
    return n * request_cells(req) * req.n_steps


def request_footprint(req: ImagingRequest, chunk: int) -> int:
    """Device bytes the request holds while admitted."""
    cells = request_cells(req)
    ntx, nrx = len(req.transmitters), len(req.receivers)
    grad = req.target is not None
    nsol = ntx * (2 if grad else 1)
    b = nsol * 6 * cells * 4                       # state + ping-pong scratch
    b += (2 if grad else 1) * 2 * cells * 4        # Ca, Cb (model, target)
    b += nsol * nrx * req.n_steps * 4              # traces
    if grad:
        nseg = -(-req.n_steps // chunk)
        from .adjoint import tx_group
        G = tx_group(ntx, min(chunk, req.n_steps), cells)
        b += ntx * nseg * 3 * cells * 4            # checkpoints
        b += G * (min(chunk, req.n_steps) + 1 + 2) * 3 * cells * 4   # segment states, adjoint
        b += 2 * ntx * cells * 8 + 4 * cells * 8   # dL/dCa, dL/dCb per run; eps, sigma, grads
        b += ntx * nrx * req.n_steps * 4           # residual
    return b


class _SrcView:
    """One transmitter's single source inside a request's source array (the
    SourceTable interface the adjoint driver reads: dev, count)."""

    def __init__(self, table: torch.Tensor, offset: int) -> None:
        self.dev = table[offset:offset + ctypes.sizeof(nat.WfSource)]
        self.count = 1


class _Live:
    """Device-side state of one admitted request."""

    def __init__(self, srv: "Server", t: Ticket) -> None:
        req = t.request
        dev = srv.device
        g = req.material._grid
        self.ticket = t
        self.grid = g
        self.nx, self.ny = g.Nx, g.Ny
        self.cells = g.Nx * g.Ny
        self.ntx, self.nrx = len(req.transmitters), len(req.receivers)
        self.grad = req.target is not None
        self.nsol = self.ntx * (2 if self.grad else 1)
        self.N = req.n_steps
        self.done = 0
        self.bytes = request_footprint(req, srv.chunk)
        cells = self.cells
        self.state = torch.zeros((self.nsol, 3, cells), dtype=torch.float32, device=dev)
        self.scratch = torch.empty((self.nsol, 3, cells), dtype=torch.float32, device=dev)
        nmap = 2 if self.grad else 1
        self.coef = torch.empty((nmap, 2, cells), dtype=torch.float32, device=dev)
        self.traces = torch.zeros((self.nsol, self.nrx, self.N), dtype=torch.float32, device=dev)
        self.eps = self.sig = None
        if self.grad:
            self.eps = torch.empty((g.Nx, g.Ny), dtype=torch.float64, device=dev)
            self.sig = torch.empty_like(self.eps)
            req.material.build_device(dev, out=(self.coef[0, 0], self.coef[0, 1]),
                                      eps_sigma=(self.eps, self.sig))
            req.target.build_device(dev, out=(self.coef[1, 0], self.coef[1, 1]))
            self.nseg = -(-self.N // srv.chunk)
            self.ckpt = torch.empty((self.ntx, self.nseg, 3, cells), dtype=torch.float32,
                                    device=dev)
        else:
            req.material.build_device(dev, out=(self.coef[0, 0], self.coef[0, 1]))
        wave = srv._wave(req.waveform, g.dt, self.N)
        self.wave = wave
        src = (nat.WfSource * self.ntx)()
        for q, (i, j) in enumerate(req.transmitters):
            src[q] = nat.WfSource(nat.COMP_CODE["Hz"], int(i), int(i) + 1, int(j), int(j) + 1, 0,
                                  1, wave.numel(), wave.data_ptr(), None)
        self.src_dev = nat.to_device_bytes(src, dev)
        self.probes = ProbeTable([("Hz", int(i), int(j)) for i, j in req.receivers], dev,
                                 _ALLOWED, (g.Nx, g.Ny, 1))
        self.g = grid_struct(g, dev)
        # host->device bytes of admission: region lists + material tables per
        # painted map, the source and probe descriptors
        maps = [req.material] + ([req.target] if self.grad else [])
        self.h2d = sum(len(m._prims) * ctypes.sizeof(nat.WfRegion2D) + 24 * (len(m._prims) + 1)
                       for m in maps)
        self.h2d += self.ntx * ctypes.sizeof(nat.WfSource) + self.nrx * ctypes.sizeof(nat.WfProbe)
        both = nat.WF_FASTDIV_X | nat.WF_FASTDIV_Y
        self.fast = (self.g.flags & both) == both
        self.desc = []
        ssz = ctypes.sizeof(nat.WfSource)
        for q in range(self.nsol):
            d = nat.WfSolve2D()
            d.g = self.g
            d.ex, d.ey, d.hz = (self.state[q, c].data_ptr() for c in range(3))
            d.sx, d.sy, d.sz = (self.scratch[q, c].data_ptr() for c in range(3))
            m = 0 if q < self.ntx else 1
            d.ca, d.cb = self.coef[m, 0].data_ptr(), self.coef[m, 1].data_ptr()
            d.src = self.src_dev.data_ptr() + (q % self.ntx) * ssz
            d.nsrc = 1
            d.probes = self.probes.ptr
            d.nprobe = self.probes.count
            d.traces = self.traces[q].data_ptr()
            d.trace_ld = self.N
            d.trace_step0 = 0
            d.n_check = 0
            d.check_max = None
            self.desc.append(d)
        # descriptor bytes of the request's solves, patched per chunk (step0,
        # nsteps, status) through an int32 view
        self.desc_np = np.frombuffer(bytearray(bytes(memoryview(
            (nat.WfSolve2D * self.nsol)(*self.desc)).cast("B"))), dtype=np.uint8).copy()
        self.items: dict = {}   # k -> (solve-local index, ci0, cj0) int32 rows
        self.event = None
        self.host_traces = None

    def tile_rows(self, k: int, region: tuple[int, int]) -> np.ndarray:
        if k not in self.items:
            self.items[k] = tile_items([(self.nx, self.ny)] * self.nsol, k, region)
        return self.items[k]


class Server:
    """Continuous-batching server on one device (see the module docstring)."""

    def __init__(self, device, *, hbm_budget: float = 60e9, chunk_steps: int = 128,
                 max_wait_s: Optional[float] = None, max_active_solves: Optional[int] = None,
                 max_active_cells: float = 3.2e7, mode: str = "tiled", tune=None,
                 ctas_per_sm: int = 0) -> None:
        if mode not in ("tiled", "persistent"):
            raise ValueError("mode is 'tiled' or 'persistent'")
        self.mode = mode
        # tiled: a pass spreads every solve's tiles over all SMs, so a few
        # requests already fill the GPU; the in-flight cell cap bounds how
        # many requests share it (and so each one's latency)
        self.max_cells = int(max_active_cells)
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise RuntimeError("Server runs on a CUDA device only (no CPU fallback)")
        nat.load()
        if chunk_steps < 1:
            raise ValueError("chunk_steps must be >= 1")
        self.budget = int(hbm_budget)
        # the persistent kernel runs one CTA per solve: a few solves per SM
        # fill the GPU; admitting more only stretches every request's latency
        nsm = torch.cuda.get_device_properties(self.device).multi_processor_count
        self.max_active = int(max_active_solves) if max_active_solves else 3 * nsm
        self.chunk = int(chunk_steps)
        self.max_wait_s = max_wait_s
        # default: tiled -- depth 4 on 64 x 128 regions of the 512-thread
        # layout (4 x 4 cells per thread); persistent -- depth 6 on 48 x 128
        if tune is None:
            tune = (4, 64, 128, 1, 512) if mode == "tiled" else (6, 48, 128, 1, 0)
        self.tune = nat.WfTune(*tune)
        self.depth = self.tune.steps_per_pass
        self.region = (self.tune.tile_i, self.tune.tile_j)
        self.ctas_per_sm = ctas_per_sm
        self.stream = torch.cuda.current_stream(self.device)
        self.side = torch.cuda.Stream(self.device)
        self.queue: list[Ticket] = []
        self.live: list[_Live] = []
        self.adjoint: list[_Live] = []
        self.retiring: list[_Live] = []
        self.completed: list[Ticket] = []
        self.used = 0
        self._ids = 0
        self._waves: dict = {}
        self._queue_ctr = torch.zeros(1, dtype=torch.int32, device=self.device)
        self._desc_dev: Optional[torch.Tensor] = None
        self._order_dev: Optional[torch.Tensor] = None
        self.rate = 5e10            # cell-updates/s estimate for the wait bound (updated live)
        self.launches = 0
        self.cell_updates = 0
        self.h2d_bytes = 0
        self.d2h_bytes = 0
        self._chunk_events: list = []
        torch.cuda.synchronize(self.device)
        self.t0 = time.perf_counter()
        self.ev0 = torch.cuda.Event(enable_timing=True)
        self.ev0.record(self.stream)

    # ------------------------------------------------------------------
    def now(self) -> float:
        return time.perf_counter() - self.t0

    def _wave(self, waveform, dt: float, n: int) -> torch.Tensor:
        key = (id(waveform), dt)
        w = self._waves.get(key)
        if w is None or w[1].numel() < n:
            t = waveform.build(n, dt, self.device)
            t = t.to(self.device, torch.float32).contiguous()
            self._waves[key] = (waveform, t)
            w = self._waves[key]
        return w[1]

    def backlog(self) -> int:
        """Cell-updates queued or still to run."""
        q = sum(request_work(t.request) for t in self.queue)
        a = sum(L.nsol * L.cells * (L.N - L.done) for L in self.live)
        return q + a

    def submit(self, req: ImagingRequest, t: Optional[float] = None) -> Ticket:
        mm = req.material
        if not mm.device_paintable or (req.target is not None and not req.target.device_paintable):
            raise ValueError("requests need device-paintable phantoms (circle/rectangle/ellipse/shell)")
        if req.target is not None and req.target._grid.Nx * req.target._grid.Ny != request_cells(req):
            raise ValueError("target phantom must be on the same grid")
        if not req.transmitters or not req.receivers or req.n_steps < 1:
            raise ValueError("a request needs transmitters, receivers and n_steps >= 1")
        tk = Ticket(req, self._ids, self.now() if t is None else t)
        self._ids += 1
        if request_footprint(req, self.chunk) > self.budget:
            tk.status, tk.reason = "rejected", "footprint above the HBM budget"
            self.completed.append(tk)
            return tk
        if self.max_wait_s is not None:
            wait = self.backlog() / self.rate
            if wait > self.max_wait_s:
                tk.status, tk.reason = "rejected", f"overloaded (estimated wait {wait:.2f} s)"
                self.completed.append(tk)
                return tk
        self.queue.append(tk)
        return tk

    # ------------------------------------------------------------------
    def _admit(self) -> None:
        active = sum(L.nsol for L in self.live)
        cells = sum(L.nsol * L.cells for L in self.live)
        while self.queue:
            tk = self.queue[0]
            fp = request_footprint(tk.request, self.chunk)
            nsol = len(tk.request.transmitters) * (2 if tk.request.target is not None else 1)
            ncell = nsol * request_cells(tk.request)
            if self.used + fp > self.budget:
                break   # arrival order: the head waits for memory
            full = (active + nsol > self.max_active if self.mode == "persistent"
                    else cells + ncell > self.max_cells)
            if self.live and full:
                break   # the GPU is full: the head waits for a slot
            active += nsol
            cells += ncell
            self.queue.pop(0)
            L = _Live(self, tk)
            self.used += L.bytes
            self.h2d_bytes += L.h2d
            tk.status, tk.t_admit = "running", self.now()
            self.live.append(L)

    def _host_buffer(self, nbytes: int) -> torch.Tensor:
        """One of two pinned staging buffers, alternating per chunk (the chunk
        that used a buffer two rounds ago has finished when step() returns)."""
        self._hb_turn = 1 - getattr(self, "_hb_turn", 0)
        bufs = self.__dict__.setdefault("_hb", [None, None])
        b = bufs[self._hb_turn]
        if b is None or b.numel() < nbytes:
            b = torch.empty(max(nbytes, 1 << 20) * 2, dtype=torch.uint8, pin_memory=True)
            bufs[self._hb_turn] = b
        return b

    def _launch_chunk(self) -> None:
        if not self.live:
            return
        dsz = ctypes.sizeof(nat.WfSolve2D)
        o_step0 = nat.WfSolve2D.step0.offset // 4
        groups: dict = {}        # steps of this chunk -> [(request, first descriptor index)]
        nsol = 0
        for L in self.live:
            ns = min(self.chunk, L.N - L.done)
            if L.grad:
                L.ckpt[:, L.done // self.chunk].copy_(L.state[:L.ntx])
            groups.setdefault(ns, []).append((L, nsol))
            v = L.desc_np.view(np.int32).reshape(L.nsol, dsz // 4)
            v[:, o_step0] = L.done
            v[:, o_step0 + 1] = ns
            v[:, o_step0 + 3] = 0
            nsol += L.nsol
            self.cell_updates += L.nsol * L.cells * ns
            L.done += ns
        chunks = [L.desc_np for L in self.live]
        offs, plans = {}, {}
        off = nsol * dsz
        if self.mode == "persistent":
            sizes = np.concatenate([np.full(L.nsol, L.cells) for L in self.live])
            chunks.append(np.argsort(-sizes, kind="stable").astype(np.int32).view(np.uint8))
        else:
            for ns, members in groups.items():
                plan = PassPlan(ns, self.depth)
                plans[ns] = plan
                for k in {plan.length(p) for p in range(plan.passes)}:
                    rows = []
                    for L, q0 in members:
                        r = L.tile_rows(k, self.region).copy()
                        r[:, 0] += q0
                        rows.append(r)
                    it = np.concatenate(rows)
                    offs[(ns, k)] = (off, it.shape[0])
                    b = it.view(np.uint8).reshape(-1)
                    chunks.append(b)
                    off += b.size
        blob = np.concatenate(chunks)
        host = self._host_buffer(blob.size)
        host[:blob.size].numpy()[:] = blob
        dev = host[:blob.size].to(self.device, non_blocking=True)
        self.h2d_bytes += blob.size
        self._keep = dev
        fast = all(L.fast for L in self.live)
        stream = nat.stream_handle(self.device)
        if self.mode == "persistent":
            self._queue_ctr.zero_()
            nat.check(nat.load().wf_batch2d_run(
                dev.data_ptr(), nsol, dev.data_ptr() + nsol * dsz, self._queue_ctr.data_ptr(),
                ctypes.byref(self.tune), self.ctas_per_sm,
                1 if fast else 0, stream))
            self.launches += 1
        else:
            for ns, plan in plans.items():
                items = {k: (dev.data_ptr() + o, c) for (g, k), (o, c) in offs.items() if g == ns}
                run_tiled_passes(dev.data_ptr(), items, plan, self.tune, fast, stream)
                self.launches += plan.passes
                if plan.needs_copy:
                    for L, _ in groups[ns]:
                        L.state.copy_(L.scratch)
        ev = torch.cuda.Event(enable_timing=True)
        ev.record(self.stream)
        self._chunk_events.append((ev, self.now(), self.cell_updates))
        finished = [L for L in self.live if L.done >= L.N]
        self.live = [L for L in self.live if L.done < L.N]
        for L in finished:
            self._finish_forward(L)

    def _finish_forward(self, L: _Live) -> None:
        tk = L.ticket
        if not L.grad:
            L.host_traces = torch.empty((L.ntx, L.nrx, L.N), dtype=torch.float32, pin_memory=True)
            L.host_traces.copy_(L.traces, non_blocking=True)
            self.d2h_bytes += L.host_traces.numel() * 4
            L.event = torch.cuda.Event(enable_timing=True)
            L.event.record(self.stream)
            self.retiring.append(L)
            return
        tk.status = "adjoint"
        ready = torch.cuda.Event()
        ready.record(self.stream)
        self.side.wait_event(ready)
        with torch.cuda.stream(self.side):
            self._adjoint(L)
        self.retiring.append(L)

    def _adjoint(self, L: _Live) -> None:
        """Adjoint of a finished gradient request, enqueued on the side stream."""
        from .adjoint import adjoint_runs
        lib = nat.load()
        st = self.side.cuda_stream
        dev, N, cells = self.device, L.N, L.cells
        model, target = L.traces[:L.ntx], L.traces[L.ntx:]
        resid = (model - target).contiguous()
        loss = 0.5 * ((model.double() - target.double()) ** 2).sum()
        gca = torch.zeros((L.ntx, cells), dtype=torch.float64, device=dev)
        gcb = torch.zeros_like(gca)
        ca, cb = L.coef[0, 0], L.coef[0, 1]
        keep: list = []
        ssz = ctypes.sizeof(nat.WfSource)
        srcs = [_SrcView(L.src_dev, t * ssz) for t in range(L.ntx)]
        adjoint_runs(L.g, cells, N, self.chunk, ca, cb, L.ckpt, resid, srcs, L.probes, gca, gcb,
                     dev, stream=st, keep=keep)
        geps = torch.empty(cells, dtype=torch.float64, device=dev)
        gsig = torch.empty_like(geps)
        nat.check(lib.wf_material_grad(L.eps.data_ptr(), L.sig.data_ptr(), cells, L.grid.dt,
                                       gca.data_ptr(), gcb.data_ptr(), L.ntx, 1.0,
                                       geps.data_ptr(), gsig.data_ptr(), st))
        L.host_traces = torch.empty((L.ntx, L.nrx, N), dtype=torch.float32, pin_memory=True)
        L.host_traces.copy_(model, non_blocking=True)
        L.host_grad = torch.empty((3, cells), dtype=torch.float64, pin_memory=True)
        L.host_grad[0].copy_(geps, non_blocking=True)
        L.host_grad[1].copy_(gsig, non_blocking=True)
        L.host_grad[2, :1].copy_(loss.reshape(1), non_blocking=True)
        self.d2h_bytes += L.host_traces.numel() * 4 + (2 * cells + 1) * 8
        L.adj_keep = (resid, gca, gcb, geps, gsig, keep)
        L.event = torch.cuda.Event(enable_timing=True)
        L.event.record(self.side)

    def _retire(self, block: bool = False) -> list[Ticket]:
        out, keep = [], []
        for L in self.retiring:
            if block:
                L.event.synchronize()
            if L.event.query():
                tk = L.ticket
                tk.t_done = self.ev0.elapsed_time(L.event) / 1e3
                tk.traces = L.host_traces
                if L.grad:
                    tk.grad_eps = L.host_grad[0].view(L.nx, L.ny)
                    tk.grad_sigma = L.host_grad[1].view(L.nx, L.ny)
                    tk.loss = float(L.host_grad[2, 0])
                tk.status = "done"
                self.used -= L.bytes
                out.append(tk)
            else:
                keep.append(L)
        self.retiring = keep
        self.completed.extend(out)
        return out

    # ------------------------------------------------------------------
    def step(self) -> list[Ticket]:
        """One scheduling round: admit, launch one chunk, retire what finished."""
        self._admit()
        self._launch_chunk()
        # at most two chunks in flight: wait for the previous one, then
        # refresh the throughput estimate used by the wait bound
        if len(self._chunk_events) >= 2:
            ev, _, _ = self._chunk_events[-2]
            ev.synchronize()
            if len(self._chunk_events) >= 3:
                e_a, _, c_a = self._chunk_events[-3]
                dt = e_a.elapsed_time(ev) / 1e3
                _, _, c_b = self._chunk_events[-2]
                if dt > 0 and c_b > c_a:
                    self.rate = 0.8 * self.rate + 0.2 * (c_b - c_a) / dt
            self._chunk_events = self._chunk_events[-2:]
        return self._retire()

    def busy(self) -> bool:
        return bool(self.queue or self.live or self.retiring)

    def drain(self) -> list[Ticket]:
        out = []
        while self.queue or self.live:
            out += self.step()
        torch.cuda.synchronize(self.device)
        out += self._retire(block=True)
        return out

    def serve(self, arrivals: Sequence[tuple[float, ImagingRequest]]) -> list[Ticket]:
        """Real-time loop: submit each (t, request) when the clock reaches t,
        step while there is work, return every ticket once all are finished."""
        arrivals = sorted(arrivals, key=lambda a: a[0])
        tickets = []
        i = 0
        while i < len(arrivals) or self.busy():
            now = self.now()
            while i < len(arrivals) and arrivals[i][0] <= now:
                tickets.append(self.submit(arrivals[i][1], arrivals[i][0]))
                i += 1
            if self.queue or self.live:
                self.step()
            elif self.retiring:
                self._retire()
                time.sleep(0.0005)
            elif i < len(arrivals):
                time.sleep(max(0.0, min(0.002, arrivals[i][0] - self.now())))
        torch.cuda.synchronize(self.device)
        self._retire(block=True)
        return tickets


def serve_one_at_a_time(device, arrivals: Sequence[tuple[float, ImagingRequest]], *,
                        max_wait_s: Optional[float] = None) -> list[Ticket]:
    """The same requests, one at a time in arrival order, each transmitter a
    separate plain ``wf_fdtd2d_run`` solve (the reference's per-solve pattern
    on the B200 kernel); gradient requests use ``fdtd_misfit``.  Latency
    includes the wait for earlier requests; ``max_wait_s`` rejects at arrival
    like ``Server``."""
    from .adjoint import MisfitProblem2D, fdtd_misfit
    from .core.sources import PointSource, SourceCollection, TabulatedWaveform
    from .core.grid import YeeGrid
    dev = torch.device(device)
    lib = nat.load()
    stream = nat.stream_handle(dev)
    tickets = [Ticket(req, q, ta)
               for q, (ta, req) in enumerate(sorted(arrivals, key=lambda a: a[0]))]
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    waves = {}
    for tk in tickets:
        req = tk.request
        now = time.perf_counter() - t0
        if now < tk.t_submit:
            time.sleep(tk.t_submit - now)
        now = time.perf_counter() - t0
        if max_wait_s is not None and now - tk.t_submit > max_wait_s:
            tk.status, tk.reason = "rejected", f"overloaded (waited {now - tk.t_submit:.2f} s)"
            continue
        g = req.material._grid
        key = (id(req.waveform), g.dt)
        if key not in waves or waves[key].numel() < req.n_steps:
            waves[key] = req.waveform.build(req.n_steps, g.dt, dev).to(dev, torch.float32).contiguous()
        w = waves[key]
        tk.t_admit = now
        if req.target is None:
            ca, cb = req.material.build_device(dev)
            gs = grid_struct(g, dev)
            probes = ProbeTable([("Hz", int(i), int(j)) for i, j in req.receivers], dev, _ALLOWED,
                                (g.Nx, g.Ny, 1))
            traces = torch.zeros((len(req.transmitters), len(req.receivers), req.n_steps),
                                 dtype=torch.float32, device=dev)
            f = torch.empty((3, g.Nx * g.Ny), dtype=torch.float32, device=dev)
            s = torch.empty_like(f)
            for q, (i, j) in enumerate(req.transmitters):
                src = nat.to_device_bytes((nat.WfSource * 1)(nat.WfSource(
                    nat.COMP_CODE["Hz"], int(i), int(i) + 1, int(j), int(j) + 1, 0, 1, w.numel(),
                    w.data_ptr(), None)), dev)
                f.zero_()
                nat.check(lib.wf_fdtd2d_run(
                    ctypes.byref(gs), f[0].data_ptr(), f[1].data_ptr(), f[2].data_ptr(),
                    s[0].data_ptr(), s[1].data_ptr(), s[2].data_ptr(), ca.data_ptr(), cb.data_ptr(),
                    src.data_ptr(), 1, probes.ptr, probes.count, traces[q].data_ptr(), req.n_steps,
                    0, 0, req.n_steps, 0, None, None, stream))
            tk.traces = traces.cpu()
        else:
            gd = YeeGrid(g.Nx, g.Ny, g.dx, g.dy, courant=g.courant, device=dev)
            wt = TabulatedWaveform(w[:req.n_steps])
            srcs = [SourceCollection([PointSource(wt, int(i), int(j), "Hz", grid=gd,
                                                  N_steps=req.n_steps)])
                    for i, j in req.transmitters]
            eps_t = torch.empty((g.Nx, g.Ny), dtype=torch.float64, device=dev)
            sig_t = torch.empty_like(eps_t)
            req.target.build_device(dev, eps_sigma=(eps_t, sig_t))
            zero_t = torch.zeros((len(srcs), len(req.receivers), req.n_steps), device=dev)
            tp = MisfitProblem2D(gd, srcs, list(req.receivers), zero_t, req.n_steps)
            with torch.no_grad():
                fdtd_misfit(eps_t, sig_t, tp)
            prob = MisfitProblem2D(gd, srcs, list(req.receivers), tp.traces, req.n_steps,
                                   checkpoint_every=None)
            eps = torch.empty_like(eps_t)
            sig = torch.empty_like(eps_t)
            req.material.build_device(dev, eps_sigma=(eps, sig))
            eps.requires_grad_(True)
            sig.requires_grad_(True)
            loss = fdtd_misfit(eps, sig, prob)
            loss.backward()
            tk.traces = prob.traces.cpu()
            tk.grad_eps, tk.grad_sigma = eps.grad.cpu(), sig.grad.cpu()
            tk.loss = float(loss.detach())
        torch.cuda.synchronize(dev)
        tk.t_done = time.perf_counter() - t0
        tk.status = "done"
    return tickets
