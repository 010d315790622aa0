"""Pin the CPU oracle to golden vectors produced by the reference itself.

Every case re-runs the oracle on CPU and demands float32 results bit-identical
to the reference run recorded by ``tests/golden/make_golden.py`` (SHA-256 of
traces and final fields).  The same tests check that the product's host-side
pieces (MaterialMap painting, waveform tables) reproduce the reference's
inputs exactly.  No GPU is needed.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from _cases import (breast_coeffs, edge2d_sources, edge3d_sources, head_coeffs, load,
                    lossy_coeffs)
from conftest import rel_l2, sha
from waveforge_b200.core.sources import GaussianDerivativePulse


def _run_oracle_2d(nx, ny, dx, dt, steps, sources, probes, ca=None, cb=None):
    o = oracle.Oracle2D(nx, ny, dx, dx, dt, ca, cb)
    for comp, kind, box, wave, amp in sources:
        o.add_box_source(comp, box, wave, amp)
    tr = o.run(steps, probes)
    return o, tr


def test_oracle_stable_dt_matches_reference():
    g = load("vacuum_point_256")
    assert oracle.stable_dt(float(g["dx"]), float(g["dx"]), None, float(g["courant"])) == float(g["dt"])


def test_gauss_deriv_tables_match_reference():
    g = load("vacuum_point_256")
    steps, dt = int(g["steps"]), float(g["dt"])
    w_or = oracle.gauss_deriv_wave(steps, dt)
    w_pr = GaussianDerivativePulse(1e9).build(steps, dt, torch.device("cpu"))
    assert np.array_equal(w_or.numpy(), g["wave"])
    assert np.array_equal(w_pr.numpy(), g["wave"])


def test_oracle_vacuum_point_bit_exact():
    g = load("vacuum_point_256")
    n, steps, dt = int(g["n"]), int(g["steps"]), float(g["dt"])
    i, j = (int(v) for v in g["src"])
    wave = torch.from_numpy(g["wave"])
    probes = [("Hz", int(a), int(b)) for a, b in g["rx"]]
    o, tr = _run_oracle_2d(n, n, float(g["dx"]), dt, steps,
                           [("Hz", "point", (i, i + 1, j, j + 1), wave, None)], probes)
    assert sha(tr) == str(g["sha_traces"])
    assert sha(o.Ex) == str(g["sha_ex"]) and sha(o.Ey) == str(g["sha_ey"])
    assert sha(o.Hz) == str(g["sha_hz"])
    # the fp32 reference itself sits ~1e-6 from its fp64 run
    assert rel_l2(tr.numpy(), g["traces64"]) < 1e-5


def test_oracle_lossy_ellipses_bit_exact():
    g = load("lossy_ellipses_256")
    ca, cb = lossy_coeffs(g)
    assert sha(ca.contiguous()) == str(g["sha_ca"]) and sha(cb.contiguous()) == str(g["sha_cb"])
    n, steps = int(g["n"]), int(g["steps"])
    i, j = (int(v) for v in g["src"])
    probes = [("Hz", int(a), int(b)) for a, b in g["rx"]]
    o, tr = _run_oracle_2d(n, n, float(g["dx"]), float(g["dt"]), steps,
                           [("Hz", "point", (i, i + 1, j, j + 1), torch.from_numpy(g["wave"]), None)],
                           probes, ca, cb)
    assert sha(tr) == str(g["sha_traces"])
    assert sha(o.Hz) == str(g["sha_hz"]) and sha(o.Ex) == str(g["sha_ex"])


def test_oracle_breast_mimo_bit_exact():
    g = load("breast_mimo_small")
    steps = int(g["steps"])
    for p in range(len(g["sides"])):
        ph, ca, cb = breast_coeffs(g, p)
        assert sha(ca.contiguous()) == str(g[f"p{p}_sha_ca"])
        ant = [tuple(int(v) for v in a) for a in g[f"p{p}_ant"]]
        assert ant == ph.antennas(16)
        probes = [("Hz", i, j) for i, j in ant]
        for tx in range(int(g["n_tx"])):
            i, j = ant[tx]
            o, tr = _run_oracle_2d(ph.side, ph.side, float(g["dx"]), float(g["dt"]), steps,
                                   [("Hz", "point", (i, i + 1, j, j + 1),
                                     torch.from_numpy(g["wave"]), None)], probes, ca, cb)
            assert sha(tr) == str(g[f"p{p}_tx{tx}_sha_traces"])


@pytest.mark.parametrize("name", ["tiny7x5", "odd33x17", "min4x4"])
def test_oracle_edge_cases_2d_bit_exact(name):
    d = load(f"edges2d_{name}")
    nx, ny, steps = int(d["nx"]), int(d["ny"]), int(d["steps"])
    probes = [(("Ex", "Ey", "Hz")[c], i, j) for c, i, j in d["probes"]]
    ca = torch.from_numpy(d["ca"]) if "ca" in d else None
    cb = torch.from_numpy(d["cb"]) if "cb" in d else None
    o, tr = _run_oracle_2d(nx, ny, float(d["dx"]), float(d["dt"]), steps, edge2d_sources(d),
                           probes, ca, cb)
    assert np.array_equal(o.Ex.numpy(), d["ex32"])
    assert np.array_equal(o.Ey.numpy(), d["ey32"])
    assert np.array_equal(o.Hz.numpy(), d["hz32"])
    assert np.array_equal(tr.numpy(), d["traces32"])


def test_oracle_head3d_bit_exact():
    g = load("head3d_32")
    ca, cb = head_coeffs(g)
    assert sha(ca) == str(g["sha_ca"]) and sha(cb) == str(g["sha_cb"])
    n, steps = int(g["n"]), int(g["steps"])
    o = oracle.Oracle3D(n, n, n, float(g["dx"]), float(g["dx"]), float(g["dx"]), float(g["dt"]), ca, cb)
    i, j, k = (int(v) for v in g["src"])
    o.add_box_source("Ez", (i, i + 1, j, j + 1, k, k + 1), torch.from_numpy(g["wave"]))
    tr = o.run(steps, [("Ez", *(int(v) for v in r)) for r in g["rx"]])
    assert sha(tr) == str(g["sha_traces"])
    for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        assert sha(getattr(o, c)) == str(g[f"sha_{c.lower()}"]), c


@pytest.mark.parametrize("name", ["box9x7x6", "flat8x6x1"])
def test_oracle_edge_cases_3d_bit_exact(name):
    d = load(f"edges3d_{name}")
    nx, ny, nz = (int(v) for v in d["shape"])
    o = oracle.Oracle3D(nx, ny, nz, 1e-3, 1e-3, 1e-3, float(d["dt"]))
    for comp, box, wave in edge3d_sources(d):
        o.add_box_source(comp, box, wave)
    comps = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
    tr = o.run(int(d["steps"]), [(comps[c], i, j, k) for c, i, j, k in d["probes"]])
    for c in comps:
        assert np.array_equal(getattr(o, c).numpy(), d[c.lower() + "32"]), c
    assert np.array_equal(tr.numpy(), d["traces32"])


def test_oracle_das_bit_exact():
    d = load("das_breast96")
    ant = [tuple(int(v) for v in a) for a in d["ant"]]
    side, steps, dx, dt = int(d["side"]), int(d["steps"]), float(d["dx"]), float(d["dt"])
    v = 299_792_458.0 / np.sqrt(40.0)
    img = oracle.das_backprojection_ref(d["delta"], ant, side, side, dx, dt, steps, v,
                                        image_shape=(48, 40))
    assert np.array_equal(img, d["img_canonical_48x40"])
    img = oracle.das_backprojection_ref(d["delta"], ant, side, side, dx, dt, steps, v)
    assert np.array_equal(img, d["img_full"])
    img = oracle.das_backprojection_ref(d["delta"], ant, side, side, dx, dt, steps, v, pitch=dx,
                                        gate_start=int(d["gate_start"]))
    assert np.array_equal(img, d["img_gated"])
