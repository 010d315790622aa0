"""Adjoint gradient of the detector-trace misfit.

CPU (oracle pinning): the out-of-place float64 restatement used for autograd
equals the in-place oracle loop, and its autograd gradient matches central
finite differences.  GPU: the hand-written adjoint (wf_adjoint2d_run behind
``fdtd_misfit``) matches float64 autograd over the whole field and central
finite differences (h = 1e-3) on sampled cells within 1e-4 relative; the
result does not depend on the checkpoint segment length; the loss equals the
plain forward's misfit.
"""

from __future__ import annotations

import math

import pytest
import torch

from oracle import adjoint_ref as A
from oracle import gauss_deriv_wave, stable_dt

N, STEPS, DX, COURANT, FC = 64, 300, 1e-3, 0.5, 10e9
TOL_GRAD = 1e-4   # relative, adjoint (float32 forward) vs float64 references
TUMOR = 12.0


def phantom(tumor_eps: float):
    """eps_r, sigma planes (float64): matching medium, an adipose-like ellipse,
    a fibroglandular-like disc and a tumour disc (the MIMO phantom's layers,
    with permittivities scaled down so a 300-step run crosses the grid)."""
    I, J = torch.meshgrid(torch.arange(N, dtype=torch.float64),
                          torch.arange(N, dtype=torch.float64), indexing="ij")
    eps = torch.full((N, N), 2.0, dtype=torch.float64)
    sig = torch.zeros((N, N), dtype=torch.float64)
    ell = ((I - 32) / 20) ** 2 + ((J - 30) / 16) ** 2 <= 1.0
    eps[ell], sig[ell] = 3.0, 0.04
    fib = (I - 30) ** 2 + (J - 34) ** 2 <= 7 ** 2
    eps[fib], sig[fib] = 8.0, 0.8
    tum = (I - 36) ** 2 + (J - 26) ** 2 <= 4 ** 2
    eps[tum], sig[tum] = tumor_eps, 1.0
    return eps, sig


def ring(n_ant, radius=26.0):
    return [(int(round(32 + radius * math.cos(2 * math.pi * k / n_ant))),
             int(round(32 + radius * math.sin(2 * math.pi * k / n_ant)))) for k in range(n_ant)]


def setup(n_tx=2):
    dt = stable_dt(DX, DX, courant=COURANT)
    wave = gauss_deriv_wave(STEPS, dt, fc=FC, dtype=torch.float64)
    ants = ring(8)
    tx = [ants[0], ants[3]][:n_tx]
    waves = [wave] * len(tx)
    eps_t, sig_t = phantom(TUMOR + 15.0)   # "measured" phantom: tumour eps_r + 15
    ca, cb = A.coeffs(eps_t, sig_t, dt)
    targets = torch.stack([A.functional_traces(ca, cb, DX, DX, dt, s, w, ants, STEPS)
                           for s, w in zip(tx, waves)])
    targets = targets.to(torch.float32).to(torch.float64)   # what the float32 engine sees
    return dt, wave, ants, tx, waves, targets


def test_functional_restatement_equals_inplace_oracle():
    dt, wave, ants, tx, waves, _ = setup(1)
    eps, sig = phantom(TUMOR)
    ca, cb = A.coeffs(eps, sig, dt)
    f = A.functional_traces(ca, cb, DX, DX, dt, tx[0], wave, ants, STEPS)
    g = A.inplace_traces(ca, cb, DX, DX, dt, tx[0], wave, ants, STEPS)
    assert float(g.abs().max()) > 0
    assert float((f - g).norm() / g.norm()) <= 1e-13


def test_float64_autograd_matches_finite_differences():
    dt, wave, ants, tx, waves, targets = setup(1)
    eps, sig = phantom(TUMOR)
    e = eps.clone().requires_grad_(True)
    s = sig.clone().requires_grad_(True)
    loss = A.misfit(e, s, DX, DX, dt, tx, waves, ants, targets[:1], STEPS)
    ge, gs = torch.autograd.grad(loss, (e, s))
    cells = [(36, 26), (30, 34), (20, 40)]
    fd_e = A.fd_gradient(eps, sig, DX, DX, dt, tx, waves, ants, targets[:1], STEPS, cells, "eps")
    fd_s = A.fd_gradient(eps, sig, DX, DX, dt, tx, waves, ants, targets[:1], STEPS, cells, "sigma")
    ad_e = torch.tensor([float(ge[c]) for c in cells], dtype=torch.float64)
    ad_s = torch.tensor([float(gs[c]) for c in cells], dtype=torch.float64)
    fe = torch.tensor(fd_e, dtype=torch.float64)
    fs = torch.tensor(fd_s, dtype=torch.float64)
    assert float(fe.abs().min()) > 0 and float(fs.abs().min()) > 0
    assert float((ad_e - fe).norm() / fe.norm()) <= 1e-6
    assert float((ad_s - fs).norm() / fs.norm()) <= 1e-6


# ---------------------------------------------------------------------------
# GPU: the hand-written adjoint
# ---------------------------------------------------------------------------

def _gpu_problem(cuda, targets, tx, wave, ants, checkpoint_every=None):
    from waveforge_b200 import MisfitProblem2D, PointSource, SourceCollection, TabulatedWaveform, YeeGrid
    g = YeeGrid(N, N, DX, DX, courant=COURANT, device=cuda)
    w32 = TabulatedWaveform(wave.to(torch.float32))
    srcs = [SourceCollection([PointSource(w32, i, j, "Hz", grid=g, N_steps=STEPS)]) for i, j in tx]
    return MisfitProblem2D(g, srcs, ants, targets.to(torch.float32), STEPS,
                           checkpoint_every=checkpoint_every)


@pytest.mark.gpu
def test_adjoint_matches_float64_autograd_and_fd(cuda):
    from waveforge_b200 import fdtd_misfit
    dt, wave, ants, tx, waves, targets = setup(2)
    eps, sig = phantom(TUMOR)
    prob = _gpu_problem(cuda, targets, tx, wave, ants)
    e = eps.to(cuda).requires_grad_(True)
    s = sig.to(cuda).requires_grad_(True)
    loss = fdtd_misfit(e, s, prob)
    loss.backward()
    g_e, g_s = e.grad.cpu(), s.grad.cpu()
    # float64 autograd through the out-of-place restatement
    e64 = eps.clone().requires_grad_(True)
    s64 = sig.clone().requires_grad_(True)
    loss64 = A.misfit(e64, s64, DX, DX, dt, tx, waves, ants, targets, STEPS)
    r_e, r_s = torch.autograd.grad(loss64, (e64, s64))
    assert abs(float(loss.detach()) - float(loss64.detach())) <= 1e-4 * abs(float(loss64.detach()))
    assert float(r_e.abs().max()) > 0
    err_e = float((g_e - r_e).norm() / r_e.norm())
    err_s = float((g_s - r_s).norm() / r_s.norm())
    assert err_e <= TOL_GRAD, err_e
    assert err_s <= TOL_GRAD, err_s
    # central finite differences, h = 1e-3, at cells inside the phantom's layers
    cells = [(36, 26), (30, 34), (32, 30), (20, 40), (44, 20), (10, 32)]
    fd_e = torch.tensor(A.fd_gradient(eps, sig, DX, DX, dt, tx, waves, ants, targets, STEPS,
                                      cells, "eps"), dtype=torch.float64)
    fd_s = torch.tensor(A.fd_gradient(eps, sig, DX, DX, dt, tx, waves, ants, targets, STEPS,
                                      cells, "sigma"), dtype=torch.float64)
    ad_e = torch.tensor([float(g_e[c]) for c in cells], dtype=torch.float64)
    ad_s = torch.tensor([float(g_s[c]) for c in cells], dtype=torch.float64)
    assert float((ad_e - fd_e).norm() / fd_e.norm()) <= TOL_GRAD
    assert float((ad_s - fd_s).norm() / fd_s.norm()) <= TOL_GRAD


@pytest.mark.gpu
def test_adjoint_independent_of_checkpoint_interval(cuda):
    from waveforge_b200 import fdtd_misfit
    dt, wave, ants, tx, waves, targets = setup(1)
    eps, sig = phantom(TUMOR)
    grads = []
    for k in (None, 1, 7, STEPS, 1000):
        prob = _gpu_problem(cuda, targets[:1], tx[:1], wave, ants, checkpoint_every=k)
        e = eps.to(cuda).requires_grad_(True)
        s = sig.to(cuda).requires_grad_(True)
        fdtd_misfit(e, s, prob).backward()
        grads.append((e.grad.clone(), s.grad.clone()))
    for ge, gs in grads[1:]:
        assert torch.equal(ge, grads[0][0]) and torch.equal(gs, grads[0][1])


@pytest.mark.gpu
def test_misfit_equals_plain_forward(cuda):
    """The loss is 1/2||traces - target||^2 of the plain FDTD2D run with the
    same float32 Ca/Cb (MaterialMap-built coefficients are bit-identical)."""
    from waveforge_b200 import (FDTD2D, Detectors, FieldSet, MurABC, PointSource,
                                SourceCollection, TabulatedWaveform, YeeGrid, fdtd_misfit)
    dt, wave, ants, tx, waves, targets = setup(1)
    eps, sig = phantom(TUMOR)
    prob = _gpu_problem(cuda, targets[:1], tx[:1], wave, ants)
    loss = fdtd_misfit(eps.to(cuda), sig.to(cuda), prob)
    ca32, cb32 = (c.to(torch.float32) for c in A.coeffs(eps, sig, dt))
    g = YeeGrid(N, N, DX, DX, courant=COURANT, device=cuda)
    f = FieldSet(g)
    src = PointSource(TabulatedWaveform(wave.to(torch.float32)), *tx[0], "Hz", grid=g, N_steps=STEPS)
    sim = FDTD2D(g, f, MurABC(g, f.Hz), SourceCollection([src]),
                 Ca=ca32.reshape(N, N, 1).to(cuda), Cb=cb32.reshape(N, N, 1).to(cuda))
    tr = sim.run(STEPS, record=Detectors(ants))
    assert torch.equal(tr, prob.traces[0])
    ref = 0.5 * float(((tr.double().cpu() - targets[0]) ** 2).sum())
    assert abs(float(loss) - ref) <= 1e-12 * ref
