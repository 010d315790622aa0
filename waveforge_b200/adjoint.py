"""Differentiable detector-trace misfit of the 2D TM solver (hand-written adjoint).

The reference project has no gradient path: its differentiable-physics plan
is a design document only (docs/architecture/DIFFERENTIABLE_PHYSICS.md), and
torch autograd cannot run through its in-place update loop
(src/core/fdtd2d.py:254-257, src/core/boundaries.py:259-274).  Here

    L(eps_r, sigma) = 1/2 * sum_{tx, rx, n} (trace[tx, rx, n] - target[tx, rx, n])^2

is a ``torch.autograd.Function``: the forward runs every transmitter through
the fused CUDA step (``wf_fdtd2d_run``) with per-cell Ca/Cb built on the device
from eps_r, sigma (``wf_material_coeffs``, the formula of
src/core/materials.py:61-82), keeping a field checkpoint every K ~ sqrt(N)
steps.  The backward walks the checkpoint segments from last to first:
``wf_fdtd2d_states`` recomputes the segment's states (bit-identical to the
forward, same kernel), ``wf_adjoint2d_run`` runs the time-reversed Yee steps
that carry dL/dstate backwards and accumulate dL/dCa, dL/dCb in float64, and
``wf_material_grad`` applies the chain rule to dL/deps_r, dL/dsigma.

Memory: checkpoints take ceil(N/K) x 3 planes per transmitter; the reverse
pass runs transmitters in groups whose segment buffers ((K+1) x 3 planes each)
fit 2 GB, one launch per step for the whole group.
"""

from __future__ import annotations

import ctypes
import math
from typing import Optional, Sequence

import torch

from . import _native as nat
from .batch import PassPlan, grid_struct, run_tiled_passes, tile_items
from .core._engine import ProbeTable, SourceTable, source_list
from .core.grid import YeeGrid
from .detectors import Detectors

_ALLOWED = ("Ex", "Ey", "Hz")


class MisfitProblem2D:
    """Everything of the misfit except the material: grid, one source set per
    transmitter run, the receivers, the target traces and the step count.

    ``transmitters``: one source object per run (``PointSource``,
    ``SourceCollection``, ...).  ``receivers``: ``Detectors`` or a list of
    ``(i, j)`` Hz points.  ``targets``: ``(n_tx, n_rx, n_steps)`` float32.
    ``checkpoint_every``: segment length K (default ceil(sqrt(n_steps))).
    """

    def __init__(self, grid: YeeGrid, transmitters: Sequence, receivers, targets: torch.Tensor,
                 n_steps: int, *, checkpoint_every: Optional[int] = None) -> None:
        if grid.Nz != 1:
            raise ValueError("MisfitProblem2D needs a 2D grid (Nz == 1)")
        self.grid = grid
        self.device = torch.device(grid.device)
        if self.device.type != "cuda":
            raise RuntimeError("the misfit gradient runs on a CUDA device only (no CPU fallback)")
        nat.load()
        self.n_steps = int(n_steps)
        if self.n_steps < 1:
            raise ValueError("n_steps must be >= 1")
        self.K = int(checkpoint_every) if checkpoint_every else max(1, math.ceil(math.sqrt(n_steps)))
        if self.K < 1:
            raise ValueError("checkpoint_every must be >= 1")
        self.detectors = receivers if isinstance(receivers, Detectors) else Detectors(receivers)
        shape = (grid.Nx, grid.Ny, 1)
        self.probes: ProbeTable = self.detectors.table(self.device, _ALLOWED, shape)
        self.sources = []
        for tx in transmitters:
            injectors = source_list(tx)
            for inj in injectors:
                for box in inj.native_boxes():
                    if box[0] != "Hz":
                        raise ValueError("MisfitProblem2D supports soft Hz sources only (an E "
                                         f"source {box[0]!r} would shift the Ca term of the "
                                         "gradient)")
            st = SourceTable(injectors, self.device, _ALLOWED, 2)
            st.check_range(0, self.n_steps)
            self.sources.append(st)
        if not self.sources:
            raise ValueError("MisfitProblem2D needs at least one transmitter")
        n_tx, n_rx = len(self.sources), len(self.detectors)
        targets = torch.as_tensor(targets)
        if tuple(targets.shape) != (n_tx, n_rx, self.n_steps):
            raise ValueError(f"targets must have shape {(n_tx, n_rx, self.n_steps)}, "
                             f"got {tuple(targets.shape)}")
        self.targets = targets.to(self.device, torch.float32).contiguous()
        self.g = grid_struct(grid, self.device)
        self.traces: Optional[torch.Tensor] = None

    @property
    def n_segments(self) -> int:
        return -(-self.n_steps // self.K)

    # ------------------------------------------------------------------
    def coefficients(self, eps64: torch.Tensor, sig64: torch.Tensor):
        """Float32 Ca, Cb on the device from float64 eps_r, sigma planes."""
        g = self.grid
        ca = torch.empty((g.Nx, g.Ny), dtype=torch.float32, device=self.device)
        cb = torch.empty_like(ca)
        nat.check(nat.load().wf_material_coeffs(eps64.data_ptr(), sig64.data_ptr(), eps64.numel(),
                                                g.dt, ca.data_ptr(), cb.data_ptr(),
                                                nat.stream_handle(self.device)))
        return ca, cb

    def forward_runs(self, ca: torch.Tensor, cb: torch.Tensor, keep_checkpoints: bool):
        """Run every transmitter; returns (traces (n_tx, n_rx, N), checkpoints
        (n_tx, n_seg, 3, Nx, Ny) or None).  All transmitters advance together:
        each temporal pass of a segment is one wf_batch2d_pass over the tiles
        of every transmitter's grid (same tile routine as wf_fdtd2d_run, so
        the traces are those of the plain per-transmitter runs)."""
        g, dev, N, K = self.grid, self.device, self.n_steps, self.K
        n_tx, n_rx = len(self.sources), len(self.detectors)
        cells = g.Nx * g.Ny
        traces = torch.zeros((n_tx, n_rx, N), dtype=torch.float32, device=dev)
        state = torch.zeros((n_tx, 3, cells), dtype=torch.float32, device=dev)
        scratch = torch.empty_like(state)
        ckpt = (torch.empty((n_tx, self.n_segments, 3, g.Nx, g.Ny), dtype=torch.float32,
                            device=dev) if keep_checkpoints else None)
        desc = (nat.WfSolve2D * n_tx)()
        for t, st in enumerate(self.sources):
            d = desc[t]
            d.g = self.g
            d.ex, d.ey, d.hz = (state[t, c].data_ptr() for c in range(3))
            d.sx, d.sy, d.sz = (scratch[t, c].data_ptr() for c in range(3))
            d.ca, d.cb = ca.data_ptr(), cb.data_ptr()
            d.src, d.nsrc = st.ptr, st.count
            d.probes, d.nprobe = self.probes.ptr, self.probes.count
            d.traces, d.trace_ld, d.trace_step0 = traces[t].data_ptr(), N, 0
            d.n_check, d.check_max = 0, None
        both = nat.WF_FASTDIV_X | nat.WF_FASTDIV_Y
        fast = (self.g.flags & both) == both
        stream = nat.stream_handle(dev)
        seg_len = K if keep_checkpoints else N
        items: dict = {}
        keep = []
        for s0 in range(0, N, seg_len):
            if keep_checkpoints:
                ckpt[:, s0 // K].copy_(state.view(n_tx, 3, g.Nx, g.Ny))
            ns = min(seg_len, N - s0)
            for d in desc:
                d.step0, d.nsteps, d.status = s0, ns, 0
            dd = nat.to_device_bytes(desc, dev)
            keep.append(dd)
            plan = PassPlan(ns, 6)
            for q in range(plan.passes):
                k = plan.length(q)
                if k not in items:
                    it = torch.from_numpy(tile_items([(g.Nx, g.Ny)] * n_tx, k, (48, 128))).to(dev)
                    items[k] = (it, it.shape[0])
            run_tiled_passes(dd.data_ptr(), {k: (t.data_ptr(), c) for k, (t, c) in items.items()},
                             plan, None, fast, stream)
            if plan.needs_copy:
                state.copy_(scratch)
        return traces, ckpt

    def adjoint(self, ca, cb, ckpt, resid):
        """float64 dL/dCa, dL/dCb summed over the transmitters: (n_tx, Nx*Ny)
        accumulator planes, one per transmitter."""
        g, dev, N, K = self.grid, self.device, self.n_steps, self.K
        cells = g.Nx * g.Ny
        gca = torch.zeros((len(self.sources), cells), dtype=torch.float64, device=dev)
        gcb = torch.zeros_like(gca)
        adjoint_runs(self.g, cells, N, K, ca, cb, ckpt, resid, self.sources, self.probes,
                     gca, gcb, dev)
        return gca, gcb


def tx_group(n_tx: int, K: int, cells: int, budget: float = 2e9) -> int:
    """Transmitter runs whose segment buffers ((K+1) x 3 planes each) fit
    ``budget`` bytes, at least one."""
    return max(1, min(n_tx, int(budget // ((K + 1) * 3 * cells * 4))))


def adjoint_runs(g, cells: int, N: int, K: int, ca, cb, ckpt, resid, sources, probes,
                 gca, gcb, dev, stream=None, keep: Optional[list] = None) -> None:
    """Reverse pass of every transmitter run: for each group of runs and each
    checkpoint segment from last to first, recompute the segment's states
    (wf_fdtd2d_states) and run the adjoint steps (wf_adjoint2d_run), one
    launch per step for the whole group.  ``sources``: one SourceTable per
    run; ``ckpt``: (n_tx, n_seg, 3, cells); ``resid``: (n_tx, n_rx, N);
    ``gca``/``gcb``: (n_tx, cells) float64 accumulators."""
    lib = nat.load()
    st = nat.stream_handle(dev) if stream is None else stream
    n_tx = len(sources)
    nseg = -(-N // K)
    counts = {s.count for s in sources}
    G = tx_group(n_tx, min(K, N), cells) if len(counts) == 1 else 1
    states = torch.empty((G, min(K, N) + 1, 3, cells), dtype=torch.float32, device=dev)
    lam = torch.empty((G, 3, cells), dtype=torch.float32, device=dev)
    lam_s = torch.empty_like(lam)
    if keep is not None:
        keep.extend([states, lam, lam_s])
    for t0 in range(0, n_tx, G):
        grp = sources[t0:t0 + G]
        ng = len(grp)
        srcs = [s.dev for s in grp if s.dev is not None]
        src = torch.cat(srcs) if srcs else None
        if keep is not None and src is not None:
            keep.append(src)
        per = grp[0].count
        lam[:ng].zero_()
        for s in reversed(range(nseg)):
            s0 = s * K
            ns = min(K, N - s0)
            states[:ng, 0].copy_(ckpt[t0:t0 + ng, s].reshape(ng, 3, cells))
            nat.check(lib.wf_fdtd2d_states(ctypes.byref(g), states.data_ptr(), states.stride(0), ng,
                                           ns, ca.data_ptr(), cb.data_ptr(),
                                           None if src is None else src.data_ptr(), per, s0, st))
            nat.check(lib.wf_adjoint2d_run(ctypes.byref(g), states.data_ptr(), states.stride(0), ng,
                                           ns, ca.data_ptr(), cb.data_ptr(), probes.ptr,
                                           probes.count, resid[t0].data_ptr(), resid.stride(1),
                                           resid.stride(0), 0, s0, lam.data_ptr(),
                                           lam_s.data_ptr(), gca[t0].data_ptr(),
                                           gcb[t0].data_ptr(), st))


def _plane64(x: torch.Tensor, g: YeeGrid, device, what: str) -> torch.Tensor:
    if x.numel() != g.Nx * g.Ny:
        raise ValueError(f"{what} must have Nx*Ny = {g.Nx * g.Ny} elements, got {x.numel()}")
    return x.detach().to(device=device, dtype=torch.float64).reshape(g.Nx, g.Ny).contiguous()


class FDTDMisfit(torch.autograd.Function):
    """L(eps_r, sigma) with the hand-written adjoint as its backward."""

    @staticmethod
    def forward(ctx, eps_r: torch.Tensor, sigma: torch.Tensor, problem: MisfitProblem2D):
        g = problem.grid
        e64 = _plane64(eps_r, g, problem.device, "eps_r")
        s64 = _plane64(sigma, g, problem.device, "sigma")
        if bool((e64 < 1.0).any()) or bool((s64 < 0.0).any()):
            raise ValueError("eps_r must be >= 1 and sigma >= 0 (src/core/materials.py:54-57)")
        ca, cb = problem.coefficients(e64, s64)
        ca_min = float(ca.min())
        if ca_min <= 0.0:
            raise ValueError(f"Ca <= 0 detected (min={ca_min:.6f}). Check material conductivities "
                             "or reduce dt. Physical passive media require Ca in (0, 1].")
        need = any(ctx.needs_input_grad[:2])
        traces, ckpt = problem.forward_runs(ca, cb, keep_checkpoints=need)
        resid = traces - problem.targets
        problem.traces = traces
        ctx.problem = problem
        ctx.shapes = (eps_r.shape, eps_r.dtype, sigma.shape, sigma.dtype)
        if need:
            ctx.save_for_backward(e64, s64, ca, cb, ckpt, resid)
        loss = 0.5 * ((traces.double() - problem.targets.double()) ** 2).sum()
        return loss.to(eps_r.dtype)

    @staticmethod
    def backward(ctx, grad_out):
        problem = ctx.problem
        e64, s64, ca, cb, ckpt, resid = ctx.saved_tensors
        gca, gcb = problem.adjoint(ca, cb, ckpt, resid)
        geps = torch.empty_like(e64)
        gsig = torch.empty_like(s64)
        nat.check(nat.load().wf_material_grad(e64.data_ptr(), s64.data_ptr(), e64.numel(),
                                              problem.grid.dt, gca.data_ptr(), gcb.data_ptr(),
                                              gca.shape[0], 1.0, geps.data_ptr(), gsig.data_ptr(),
                                              nat.stream_handle(problem.device)))
        scale = grad_out.to(torch.float64)
        eshape, edtype, sshape, sdtype = ctx.shapes
        return ((geps * scale).to(edtype).reshape(eshape),
                (gsig * scale).to(sdtype).reshape(sshape), None)


def fdtd_misfit(eps_r: torch.Tensor, sigma: torch.Tensor, problem: MisfitProblem2D) -> torch.Tensor:
    """1/2 ||traces - targets||^2 of the problem's transmitters for per-cell
    eps_r, sigma (shape (Nx, Ny) or (Nx, Ny, 1)); differentiable in both."""
    return FDTDMisfit.apply(eps_r, sigma, problem)
