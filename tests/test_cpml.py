"""Convolutional PML (new: the reference stores the graded profiles but never
applies them, src/core/boundaries.py:32-112).

CPU: the profile tables (cubic grading of the reference's formula, dual
staggering, symmetric layers), validation, and the physics of the update on
the oracle -- a pulse leaving a CPML-bounded box reflects far less than with
the Mur edges, measured against a larger box whose edges the wave has not
reached.  GPU: the CUDA path equals the oracle bit for bit (traces, fields,
stability maxima, across a reset)."""

from __future__ import annotations

import math

import numpy as np
import pytest
import torch

import oracle
from oracle.cpml_ref import OracleCPML2D
from waveforge_b200.core.boundaries import CPML, ETA0, _pml_bsigma_at_rho
from waveforge_b200.core.grid import YeeGrid


def _grid(n, device="cpu"):
    return YeeGrid(n, n, 1e-3, 1e-3, courant=0.5, device=device)


def test_profile_tables():
    g = _grid(40)
    pml = CPML(g, 8)
    t = pml.tables.view(2, 6, 40)
    for ax in range(2):
        bE, cE, ikE, bH, cH, ikH = (t[ax, k] for k in range(6))
        assert torch.all((bE > 0) & (bE <= 1) & (bH > 0) & (bH <= 1))
        assert torch.all((cE <= 0) & (cH <= 0) & (ikE > 0) & (ikE <= 1) & (ikH > 0) & (ikH <= 1))
        # interior reads (1, 0, 1); the layers are mirror images
        # (E layer cells: i < 8 and i >= 32; H: i < 8 and 31 <= i <= 38)
        assert torch.all(bE[8:32] == 1) and torch.all(cE[8:32] == 0) and torch.all(ikE[8:32] == 1)
        assert torch.all(cH[8:31] == 0) and torch.all(cH[39:] == 0)
        assert torch.equal(cE[:8], cE[32:40].flip(0)) and torch.equal(cH[:8], cH[31:39].flip(0))
        # deeper -> stronger decay (b) and stretching (1/kappa)
        assert torch.all(bE[0:7] < bE[1:8]) and torch.all(ikE[0:7] < ikE[1:8])
    # the outermost E sample (rho = 1) follows the reference's formula
    m, R, D, dx, dt = 3, 1e-8, 8, 1e-3, g.dt
    smax = (m + 1) * math.log(1.0 / R) / (2.0 * ETA0 * D * dx)
    _, b, c = _pml_bsigma_at_rho(1.0, smax, 5.0, 0.05, m, dt)
    assert float(pml.tables[0]) == np.float32(b) and float(pml.tables[40]) == np.float32(c)
    assert float(pml.tables[80]) == np.float32(1.0 / 5.0)


def test_validation():
    with pytest.raises(ValueError):
        CPML(_grid(20), 10)
    with pytest.raises(ValueError):
        CPML(_grid(20), 0)
    with pytest.raises(ValueError):
        CPML(YeeGrid(20, 20, 1e-3, 1e-3, Nz=8, dz=1e-3, device="cpu"), 3)


def _pulse_run(o, steps, c, probe):
    w = oracle.gaussian_wave(steps, o.dt, 1.0, 12 * o.dt, 40 * o.dt)
    o.add_point_source("Hz", c, c, w)
    return o.run(steps, [("Hz", *probe)])[0].double()


def test_cpml_absorbs_better_than_mur_on_the_oracle():
    """Hz pulse at the centre of a 72^2 box; the probe sits near the edge.
    Reference: the same run in a 232^2 box (no reflection within the window).
    The CPML's reflected field is far below the Mur edges' one."""
    n, big, steps = 72, 232, 220
    dt = oracle.stable_dt(1e-3, 1e-3, courant=0.5)
    c, cb = n // 2, big // 2
    probe = (c + 22, c + 5)
    pml = CPML(_grid(n), 12)
    ref = _pulse_run(oracle.Oracle2D(big, big, 1e-3, 1e-3, dt), steps, cb,
                     (probe[0] - c + cb, probe[1] - c + cb))
    mur = _pulse_run(oracle.Oracle2D(n, n, 1e-3, 1e-3, dt), steps, c, probe)
    cp = _pulse_run(OracleCPML2D(n, n, 1e-3, 1e-3, dt, 12, pml.tables), steps, c, probe)
    e_mur = float(torch.linalg.norm(mur - ref) / torch.linalg.norm(ref))
    e_cpml = float(torch.linalg.norm(cp - ref) / torch.linalg.norm(ref))
    assert e_cpml < 0.1 * e_mur and e_cpml < 5e-3, (e_cpml, e_mur)


@pytest.mark.gpu
@pytest.mark.parametrize("n,depth,mat", [(48, 6, True), (61, 10, False), (33, 3, True)])
def test_cpml_bit_exact_vs_oracle(cuda, n, depth, mat):
    from waveforge_b200 import FDTD2D, Detectors, FieldSet, PointSource, SourceCollection
    from waveforge_b200.core.sources import TabulatedWaveform
    rng = np.random.default_rng(n + depth)
    steps = 90
    g = YeeGrid(n, n + 5, 1e-3, 1e-3, courant=0.5, device=cuda)
    pml = CPML(g, depth)
    ca = cb = None
    if mat:
        ca = torch.from_numpy(rng.uniform(0.4, 1.0, (n, n + 5)).astype(np.float32))
        cb = torch.from_numpy(rng.uniform(1e-3, 0.2, (n, n + 5)).astype(np.float32)) * g.dt / 8.85e-12 / 30
    o = OracleCPML2D(n, n + 5, 1e-3, 1e-3, g.dt, depth, pml.tables, ca, cb)
    o.n_check = 10
    f = FieldSet(g)
    srcs, waves = [], []
    spec = [("Hz", n // 2, (n + 5) // 2), ("Ex", 2, 3), ("Ey", n - 3, n), ("Hz", 1, n + 3)]
    for comp, i, j in spec:
        w = torch.from_numpy(rng.standard_normal(steps).astype(np.float32))
        waves.append(w)
        srcs.append(PointSource(TabulatedWaveform(w), i, j, comp, grid=g, N_steps=steps))
        o.add_point_source(comp, i, j, w)
    probes = [("Hz", n // 2 + 3, 7), ("Ex", 1, 1), ("Ey", n - 1, n + 4), ("Hz", depth, depth)]
    sim = FDTD2D(g, f, pml, SourceCollection(srcs),
                 Ca=None if ca is None else ca.unsqueeze(2).to(cuda),
                 Cb=None if cb is None else cb.unsqueeze(2).to(cuda), n_check=10)
    for rep in range(2):   # a reset clears the layer memories too
        if rep:
            sim.reset()
            o = OracleCPML2D(n, n + 5, 1e-3, 1e-3, g.dt, depth, pml.tables, ca, cb)
            o.n_check = 10
            for (comp, i, j), w in zip(spec, waves):
                o.add_point_source(comp, i, j, w)
        tr = sim.run(steps, record=Detectors(probes)).cpu()
        ref = o.run(steps, probes)
        assert torch.equal(tr, ref.to(torch.float32)), rep
        for name in ("Ex", "Ey", "Hz"):
            assert torch.equal(getattr(f, name).cpu().reshape(n, n + 5), getattr(o, name)), name
        assert sim.last_field_max == o.last_field_max


@pytest.mark.gpu
def test_cpml_rejects_batched_fields(cuda):
    from waveforge_b200 import FDTD2D, FieldSet
    g = _grid(32, cuda)
    with pytest.raises(ValueError):
        FDTD2D(g, FieldSet(g, batch_size=2), CPML(g, 4))


def test_profile_pinned_to_reference():
    """Every b, c sample of the CPML tables equals, after float32 rounding,
    the reference's ``_pml_bsigma_at_rho`` at the same depth
    (src/core/boundaries.py:32-48; fixture written by running it), and the
    ``MurABC(pml_depth=...)`` tables equal the reference's
    ``_compute_pml_coeffs`` (:51-112) bit for bit in float64."""
    from conftest import golden
    from waveforge_b200.core.boundaries import _compute_pml_coeffs
    g = golden("cpml_profile")
    for q in range(int(g["ncases"])):
        n, D, dx, courant, dt = g[f"c{q}_grid"]
        n, D = int(n), int(D)
        grid = YeeGrid(n, n, float(dx), float(dx), courant=float(courant), device="cpu")
        assert grid.dt == float(dt)
        t = CPML(grid, D).tables.view(2, 6, n)
        for ax in range(2):
            for k, name in ((0, "bE"), (1, "cE"), (3, "bH"), (4, "cH")):
                want = torch.from_numpy(g[f"c{q}_{name}"].astype(np.float32))
                assert torch.equal(t[ax, k], want), (q, ax, name)
            rho_e = torch.from_numpy(g[f"c{q}_rhoE"])
            ik = (1.0 / (1.0 + 4.0 * rho_e ** 3)).to(torch.float32)
            assert torch.equal(t[ax, 2], ik), (q, ax)
        mine = _compute_pml_coeffs(D, float(dx), float(dt), torch.device("cpu"), torch.float64)
        for name, v in zip(("bE", "cE", "bH", "cH", "sE", "sH"), mine):
            assert np.array_equal(v.numpy(), g[f"c{q}_ref_{name}"]), (q, name)
