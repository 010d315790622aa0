"""Parity at the benchmark shapes, pinned straight to the reference.

The fixtures were written by running the reference's own float32 (and
float64) PyTorch loop at the full sizes the benchmarks use
(``tests/golden/make_golden.py``: ``breast_full``, ``lossy_full``,
``head3d_full``, ``head3d_batch``):

* breast MIMO phantoms of sides 256, 384 and 512, 3000 steps (the benchmark's
  run length), 16 receivers: through the plain per-solve kernel, the three
  batched schedules (persistent solve queue, tile passes, persistent tile
  queue), two tuned shapes, and CUDA-graph replays of the whole batch;
* the 4096^2 lossy-ellipse scene, 100 steps from seeded random starting
  fields (every cell, edge and tile boundary is live from step one), ring
  receivers plus receivers near the source, two tile shapes;
* the 256^3 head phantom, 30 steps from random starting fields of all six
  components, through the multi-segment TMA pass and the register streaming
  kernel;
* 8 batched 128^3 head instances (one launch per step for all 8, a batched
  FieldSet, the source broadcast to every member as the reference does).

Bar: float32 traces and final fields bit-identical to the reference (SHA-256),
and the float32 traces within 1e-5 relative L2 of the reference's float64 run.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from _cases import breast_coeffs, load
from conftest import rel_l2, sha
from waveforge_b200 import (FDTD2D, FDTD3D, Batch2D, BatchSolve, Detectors, FieldSet, MurABC,
                            MurABC3D, PointSource, SourceCollection, TabulatedWaveform, YeeGrid)
from waveforge_b200 import workloads as W
from waveforge_b200.core.materials import Material, MaterialMap, MaterialMap3D

pytestmark = pytest.mark.gpu

COMP3 = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def test_breast_full_shapes_bit_exact_all_modes(cuda):
    g = load("breast_mimo_full")
    steps = int(g["steps"])
    assert steps == 3000 and sorted(int(s) for s in g["sides"]) == [256, 384, 512]
    wave = torch.from_numpy(g["wave"])
    dx, courant = float(g["dx"]), float(g["courant"])
    solves, keys = [], []
    for p in range(len(g["sides"])):
        ph, ca, cb = breast_coeffs(g, p)
        ant = ph.antennas(16)
        i, j = ant[0]
        key = f"p{p}_tx0"
        ca_d = ca.reshape(ph.side, ph.side, 1).to(cuda)
        cb_d = cb.reshape(ph.side, ph.side, 1).to(cuda)
        # the plain per-solve kernel through the reference-facing API
        grid = YeeGrid(ph.side, ph.side, dx, dx, courant=courant, device=cuda)
        f = FieldSet(grid)
        src = PointSource(TabulatedWaveform(wave), i, j, "Hz", grid=grid, N_steps=steps)
        sim = FDTD2D(grid, f, MurABC(grid, f.Hz), SourceCollection([src]), Ca=ca_d, Cb=cb_d,
                     n_check=10 ** 9)
        tr = sim.run(steps, record=Detectors(ant))
        assert sha(tr) == str(g[key + "_sha_traces"]), key
        assert sha(f.Hz) == str(g[key + "_sha_hz"]), key
        assert rel_l2(tr[:, ::5].cpu().numpy(), g[key + "_traces64_dec"]) < 1e-5
        src_b = PointSource(TabulatedWaveform(wave), i, j, "Hz", grid=grid, N_steps=steps)
        solves.append(BatchSolve(grid, SourceCollection([src_b]), Detectors(ant), ca_d, cb_d))
        keys.append(key)

    def check(batch, what):
        torch.cuda.synchronize()
        assert all(s == 0 for s in batch.statuses()), what
        for q, key in enumerate(keys):
            assert sha(batch.traces(q)) == str(g[key + "_sha_traces"]), (what, key)
            assert sha(batch.fields(q)[2]) == str(g[key + "_sha_hz"]), (what, key)

    for mode in ("persistent", "tiled", "queue"):
        for tune in (None, (6, 64, 128, 1, 1024), (6, 64, 128, 1, 512)):
            b = Batch2D(solves, steps, tune=tune, mode=mode)
            b.run()
            check(b, (mode, tune))
    for mode in ("tiled", "queue"):
        b = Batch2D(solves, steps, tune=(6, 64, 128, 1, 512), mode=mode)
        b.capture()
        for rep in range(2):
            b.replay()
            check(b, ("graph replay", mode, rep))


def _lossy_full_coeffs(g):
    n = int(g["n"])
    wl = W.LossyEllipses(n=n, steps=int(g["steps"]), seed=int(g["seed"]))
    grid = YeeGrid(n, n, wl.dx, wl.dx, courant=wl.courant, device="cpu")
    mm = MaterialMap(grid, default=wl.background(Material))
    wl.paint(mm, Material)
    return mm.build()


def test_lossy_4096_full_size_bit_exact(cuda):
    g = load("lossy_full_4096")
    n, steps = int(g["n"]), int(g["steps"])
    ca, cb = _lossy_full_coeffs(g)
    assert sha(ca) == str(g["sha_ca"]) and sha(cb) == str(g["sha_cb"])
    init = W.initial_fields(int(g["init_seed"]), (n, n), ("Ex", "Ey", "Hz"))
    probes = [(str(c), int(i), int(j)) for c, (i, j) in zip(g["rx_comp"], g["rx"])]
    i, j = (int(v) for v in g["src"])
    for tune in (None, (2, 32, 128, 1, 0)):
        grid = YeeGrid(n, n, float(g["dx"]), float(g["dx"]), courant=float(g["courant"]),
                       device=cuda)
        assert grid.dt == float(g["dt"])
        f = FieldSet(grid)
        for c, v in init.items():
            getattr(f, c).copy_(torch.from_numpy(v).reshape(n, n, 1))
        src = PointSource(TabulatedWaveform(torch.from_numpy(g["wave"])), i, j, "Hz", grid=grid,
                          N_steps=steps)
        sim = FDTD2D(grid, f, MurABC(grid, f.Hz), SourceCollection([src]), Ca=ca.to(cuda),
                     Cb=cb.to(cuda), n_check=10 ** 9, tune=tune)
        tr = sim.run(steps, record=Detectors(probes))
        assert sha(tr) == str(g["sha_traces"]), tune
        assert sha(f.Ex) == str(g["sha_ex"]), tune
        assert sha(f.Ey) == str(g["sha_ey"]), tune
        assert sha(f.Hz) == str(g["sha_hz"]), tune
        assert rel_l2(tr.cpu().numpy(), g["traces64"]) < 1e-5
        assert rel_l2(f.Hz[::37, ::41, 0].cpu().numpy(), g["hz64_dec"]) < 1e-5
        del sim, f
        torch.cuda.empty_cache()


def _head_full_sim(cuda, g, tune=None):
    n, batch, steps = int(g["n"]), int(g["batch"]), int(g["steps"])
    wl = W.Head3D(n=n, steps=steps, seed=int(g["seed"]))
    gc = YeeGrid(n, n, wl.dx, wl.dx, Nz=n, dz=wl.dx, courant=wl.courant, device="cpu")
    mm = MaterialMap3D(gc, default=wl.background(Material))
    wl.paint(mm, Material)
    ca, cb = mm.build3d()
    assert sha(ca) == str(g["sha_ca"]) and sha(cb) == str(g["sha_cb"])
    grid = YeeGrid(n, n, wl.dx, wl.dx, Nz=n, dz=wl.dx, courant=wl.courant, device=cuda)
    f = FieldSet(grid, batch_size=batch)
    shape = (n, n, n) if batch == 1 else (batch, n, n, n)
    for c, v in W.initial_fields(int(g["init_seed"]), shape, COMP3).items():
        getattr(f, c).copy_(torch.from_numpy(v))
    i, j, k = (int(v) for v in g["src"])
    src = PointSource(TabulatedWaveform(torch.from_numpy(g["wave"])), i, j, "Ez", k=k, grid=grid,
                      N_steps=steps)
    sim = FDTD3D(grid, f, MurABC3D(grid, f.Hx, f.Hy, f.Hz), SourceCollection([src]),
                 Ca=ca.to(cuda), Cb=cb.to(cuda), n_check=10 ** 9, tune=tune)
    probes = [(str(c), *(int(v) for v in r)) for c, r in zip(g["rx_comp"], g["rx"])]
    return sim, f, Detectors(probes), steps


@pytest.mark.parametrize("tune", [None, (1, 0, 0, 16, 2)])
def test_head3d_256_full_size_bit_exact(cuda, tune):
    """tune None = the TMA pass (16-plane i-segments over 2592 column blocks at
    256^3); (1, 0, 0, 16, 2) = the register streaming kernel."""
    g = load("head3d_full_256")
    sim, f, det, steps = _head_full_sim(cuda, g, tune)
    tr = sim.run(steps, record=det)
    assert sha(tr) == str(g["sha_traces"])
    for c in COMP3:
        assert sha(getattr(f, c)) == str(g[f"sha_{c.lower()}"]), c
    assert rel_l2(tr.cpu().numpy(), g["traces64"]) < 1e-5


def test_head3d_batched_8x128_bit_exact(cuda):
    g = load("head3d_batch8x128")
    sim, f, det, steps = _head_full_sim(cuda, g)
    tr = sim.run(steps, record=det)
    assert tuple(tr.shape) == tuple(g["traces32"].shape)
    assert sha(tr) == str(g["sha_traces"])
    for c in COMP3:
        assert sha(getattr(f, c)) == str(g[f"sha_{c.lower()}"]), c
    assert rel_l2(tr.cpu().numpy(), g["traces64"]) < 1e-5
