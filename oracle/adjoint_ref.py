"""Float64 gradient oracle of the detector-trace misfit (test infrastructure only).

The reference has no adjoint or autograd path, and autograd through its own
loop fails ("modified by an inplace operation": the slice assignments of
src/core/fdtd2d.py:254-257 and the in-place Mur edges of
src/core/boundaries.py:259-274).  This module restates the same 2D TM step
OUT OF PLACE in float64 so that torch autograd differentiates it:

* Ca/Cb from eps_r, sigma ...... src/core/materials.py:61-82
* soft point injection before H  src/core/sources.py:863-887 (fdtd2d.py:226-228)
* Faraday update ............... src/core/fdtd2d.py:232-235
* Mur snapshot + edges ......... src/core/boundaries.py:237, 259-274 (x then y)
* Ampere, material path ........ src/core/fdtd2d.py:244-257
* detector gather after the step examples/brain_mimo_imaging.py:193-201

``functional_traces`` is checked against the in-place ``Oracle2D`` (itself
pinned to the reference's goldens) before its gradients are trusted.
``fd_gradient`` takes central finite differences of the misfit through the
in-place oracle.
"""

from __future__ import annotations

from typing import Sequence

import torch

from .fdtd_ref import C0, EPS0, MU0, Oracle2D


def coeffs(eps_r: torch.Tensor, sigma: torch.Tensor, dt: float):
    """Ca, Cb of src/core/materials.py:61-82, elementwise and differentiable."""
    alpha = sigma * dt / (2.0 * EPS0 * eps_r)
    return (1.0 - alpha) / (1.0 + alpha), (dt / (EPS0 * eps_r)) / (1.0 + alpha)


def functional_traces(ca: torch.Tensor, cb: torch.Tensor, dx: float, dy: float, dt: float,
                      src: tuple, wave: torch.Tensor, probes: Sequence[tuple],
                      nsteps: int) -> torch.Tensor:
    """Traces (n_probe, nsteps) of one soft-Hz-source run, out of place.

    ``src`` = (i, j) of the Hz point source; ``probes`` = (i, j) Hz points."""
    nx, ny = ca.shape
    dt_ = ca.dtype
    dh = dt / MU0                                   # fdtd2d.py:158
    cx = (C0 * dt - dx) / (C0 * dt + dx)            # boundaries.py:177
    cy = (C0 * dt - dy) / (C0 * dt + dy)            # boundaries.py:178
    ex = torch.zeros(nx, ny, dtype=dt_)
    ey = torch.zeros(nx, ny, dtype=dt_)
    hz = torch.zeros(nx, ny, dtype=dt_)
    onehot = torch.zeros(nx, ny, dtype=dt_)
    onehot[src[0], src[1]] = 1.0
    pi = torch.tensor([p[0] for p in probes])
    pj = torch.tensor([p[1] for p in probes])
    out = []
    for n in range(nsteps):
        hp = hz                                                     # boundaries.py:237
        h = hz + wave[n] * onehot                                   # sources.py:882-887
        curl = dh * ((ex[:-1, 1:] - ex[:-1, :-1]) / dy - (ey[1:, :-1] - ey[:-1, :-1]) / dx)
        hc = h + torch.nn.functional.pad(curl, (0, 1, 0, 1))        # fdtd2d.py:232-235
        r0 = hp[1] + cx * (hc[1] - hp[0])                           # boundaries.py:259-266
        r1 = hp[nx - 2] + cx * (hc[nx - 2] - hp[nx - 1])
        hx = torch.cat([r0[None], hc[1:-1], r1[None]], 0)
        c0 = hp[:, 1] + cy * (hx[:, 1] - hp[:, 0])                  # boundaries.py:267-274
        c1 = hp[:, ny - 2] + cy * (hx[:, ny - 2] - hp[:, ny - 1])
        hz = torch.cat([c0[:, None], hx[:, 1:-1], c1[:, None]], 1)
        dhy = (hz[:, 1:] - hz[:, :-1]) / dy                         # fdtd2d.py:244-245
        dhx = (hz[1:, :] - hz[:-1, :]) / dx
        ex = torch.cat([ex[:, :1], ca[:, 1:] * ex[:, 1:] + cb[:, 1:] * dhy], 1)   # :254-255
        ey = torch.cat([ey[:1], ca[1:] * ey[1:] - cb[1:] * dhx], 0)               # :256-257
        out.append(hz[pi, pj])
    return torch.stack(out, 1)


def misfit(eps_r: torch.Tensor, sigma: torch.Tensor, dx: float, dy: float, dt: float,
           tx: Sequence[tuple], waves: Sequence[torch.Tensor], probes: Sequence[tuple],
           targets: torch.Tensor, nsteps: int) -> torch.Tensor:
    """L = 1/2 sum over TX, probes and steps of (trace - target)^2 (float64)."""
    ca, cb = coeffs(eps_r, sigma, dt)
    loss = torch.zeros((), dtype=eps_r.dtype)
    for t, (src, w) in enumerate(zip(tx, waves)):
        tr = functional_traces(ca, cb, dx, dy, dt, src, w, probes, nsteps)
        loss = loss + 0.5 * ((tr - targets[t]) ** 2).sum()
    return loss


def inplace_traces(ca, cb, dx, dy, dt, src, wave, probes, nsteps) -> torch.Tensor:
    """The same run through the in-place oracle (float64)."""
    nx, ny = ca.shape
    o = Oracle2D(nx, ny, dx, dy, dt, ca, cb, dtype=torch.float64)
    o.n_check = 10 ** 9
    o.add_point_source("Hz", src[0], src[1], wave)
    return o.run(nsteps, [("Hz", i, j) for i, j in probes])


def fd_gradient(eps_r, sigma, dx, dy, dt, tx, waves, probes, targets, nsteps, cells,
                which: str = "eps", h: float = 1e-3) -> list[float]:
    """Central differences (L(p+h) - L(p-h)) / 2h of the float64 misfit at
    ``cells`` for p = eps_r or sigma, through the in-place oracle."""
    out = []
    for (i, j) in cells:
        vals = []
        for sgn in (1.0, -1.0):
            e = eps_r.clone()
            s = sigma.clone()
            (e if which == "eps" else s)[i, j] += sgn * h
            ca, cb = coeffs(e, s, dt)
            loss = 0.0
            for t, (src, w) in enumerate(zip(tx, waves)):
                tr = inplace_traces(ca, cb, dx, dy, dt, src, w, probes, nsteps)
                loss += 0.5 * float(((tr - targets[t]) ** 2).sum())
            vals.append(loss)
        out.append((vals[0] - vals[1]) / (2.0 * h))
    return out
