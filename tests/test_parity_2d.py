"""2D parity of the CUDA path (through the C-ABI) with the reference.

Bar: float32 traces and final fields BIT-IDENTICAL to the reference's float32
PyTorch path (golden SHA-256 digests, and the pinned oracle for random
cases), for every temporal-block depth and tile shape.  The error of the same
results against the reference's float64 run is asserted below 1e-5 relative
L2 (the stated tolerance for float32 physics).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from _cases import breast_coeffs, edge2d_sources, load, lossy_coeffs
from conftest import rel_l2, sha
from waveforge_b200 import (FDTD2D, Batch2D, BatchSolve, Detectors, FieldSet, LineSource, MurABC,
                            PointSource, SimulationDivergedError, SourceCollection,
                            TabulatedWaveform, YeeGrid)
from waveforge_b200 import workloads as W
from waveforge_b200.core.materials import Material, MaterialMap

pytestmark = pytest.mark.gpu

# (steps_per_pass k, region rows, region cols, -, -): every compiled register
# layout, with temporal-block depths from 1 to the largest that leaves a core
TUNES = [None, (1, 8, 32, 1, 0), (2, 8, 32, 1, 0), (3, 8, 32, 1, 0), (4, 32, 64, 1, 0),
         (7, 32, 64, 1, 0), (5, 32, 128, 1, 0), (6, 48, 128, 1, 0), (11, 48, 128, 1, 0),
         (4, 48, 128, 1, 1024), (1, 48, 128, 1, 1024), (9, 48, 128, 1, 1024),
         (6, 64, 128, 1, 1024), (13, 64, 128, 1, 1024)]


def sim2d(cuda, nx, ny, dx, courant, sources_spec, ca=None, cb=None, steps=None, tune=None,
          dt=None):
    g = YeeGrid(nx, ny, dx, dx, courant=courant, dt=dt, device=cuda)
    f = FieldSet(g)
    b = MurABC(g, f.Hz)
    srcs = []
    for comp, kind, box, wave, amp in sources_spec:
        w = TabulatedWaveform(wave)
        i0, i1, j0, j1 = box
        if kind == "point":
            srcs.append(PointSource(w, i0, j0, comp, grid=g, N_steps=steps))
        else:
            axis = "x" if i1 - i0 > 1 else "y"
            pos, start, stop = (j0, i0, i1) if axis == "x" else (i0, j0, j1)
            srcs.append(LineSource(w, axis, pos, start, stop, comp, grid=g, N_steps=steps,
                                   amplitude_profile=amp))
    sc = SourceCollection(srcs) if srcs else None
    ca_d = None if ca is None else ca.reshape(nx, ny, 1).to(cuda)
    cb_d = None if cb is None else cb.reshape(nx, ny, 1).to(cuda)
    return FDTD2D(g, f, b, sc, Ca=ca_d, Cb=cb_d, n_check=10 ** 9, tune=tune), f


@pytest.mark.parametrize("tune", [None, (1, 8, 32, 1, 0), (5, 32, 64, 1, 0)])
def test_vacuum_point_bit_exact_vs_reference(cuda, tune):
    g = load("vacuum_point_256")
    n, steps = int(g["n"]), int(g["steps"])
    i, j = (int(v) for v in g["src"])
    sim, f = sim2d(cuda, n, n, float(g["dx"]), float(g["courant"]),
                   [("Hz", "point", (i, i + 1, j, j + 1), torch.from_numpy(g["wave"]), None)],
                   steps=steps, tune=tune)
    assert sim.dt == float(g["dt"])
    det = Detectors([(int(a), int(b)) for a, b in g["rx"]], "Hz")
    tr = sim.run(steps, record=det)
    assert sha(tr) == str(g["sha_traces"])
    assert sha(f.Ex) == str(g["sha_ex"]) and sha(f.Ey) == str(g["sha_ey"])
    assert sha(f.Hz) == str(g["sha_hz"])
    assert rel_l2(tr.cpu().numpy(), g["traces64"]) < 1e-5
    assert rel_l2(f.Hz[::2, ::2, 0].cpu().numpy(), g["hz64_dec"]) < 1e-4


def test_vacuum_point_step_loop_bit_exact(cuda):
    """The reference call pattern: step() then a Python-side gather."""
    g = load("vacuum_point_256")
    n, steps = int(g["n"]), int(g["steps"])
    i, j = (int(v) for v in g["src"])
    sim, f = sim2d(cuda, n, n, float(g["dx"]), float(g["courant"]),
                   [("Hz", "point", (i, i + 1, j, j + 1), torch.from_numpy(g["wave"]), None)],
                   steps=steps)
    rx = torch.tensor(g["rx"], device=cuda).long()
    buf = torch.zeros(len(rx), steps, device=cuda)
    for s in range(steps):
        sim.step()
        buf[:, s] = f.Hz[rx[:, 0], rx[:, 1], 0]
    assert sha(buf) == str(g["sha_traces"])
    assert sha(f.Hz) == str(g["sha_hz"])


def test_lossy_ellipses_bit_exact_vs_reference(cuda):
    g = load("lossy_ellipses_256")
    ca, cb = lossy_coeffs(g)
    n, steps = int(g["n"]), int(g["steps"])
    i, j = (int(v) for v in g["src"])
    for tune in TUNES:
        sim, f = sim2d(cuda, n, n, float(g["dx"]), float(g["courant"]),
                       [("Hz", "point", (i, i + 1, j, j + 1), torch.from_numpy(g["wave"]), None)],
                       ca, cb, steps=steps, tune=tune)
        tr = sim.run(steps, record=Detectors([(int(a), int(b)) for a, b in g["rx"]]))
        assert sha(tr) == str(g["sha_traces"]), tune
        assert sha(f.Hz) == str(g["sha_hz"]), tune
        assert sha(f.Ex) == str(g["sha_ex"]) and sha(f.Ey) == str(g["sha_ey"]), tune
        assert rel_l2(tr.cpu().numpy(), g["traces64"]) < 1e-5


@pytest.mark.parametrize("name", ["tiny7x5", "odd33x17", "min4x4"])
def test_edge_cases_bit_exact_vs_reference(cuda, name):
    d = load(f"edges2d_{name}")
    nx, ny, steps = int(d["nx"]), int(d["ny"]), int(d["steps"])
    ca = torch.from_numpy(d["ca"]) if "ca" in d else None
    cb = torch.from_numpy(d["cb"]) if "cb" in d else None
    comps = ("Ex", "Ey", "Hz")
    for tune in TUNES:
        sim, f = sim2d(cuda, nx, ny, float(d["dx"]), float(d["courant"]), edge2d_sources(d), ca, cb,
                       steps=steps, tune=tune)
        tr = sim.run(steps, record=Detectors([(comps[c], i, j) for c, i, j in d["probes"]]))
        assert np.array_equal(f.Ex[..., 0].cpu().numpy(), d["ex32"]), tune
        assert np.array_equal(f.Ey[..., 0].cpu().numpy(), d["ey32"]), tune
        assert np.array_equal(f.Hz[..., 0].cpu().numpy(), d["hz32"]), tune
        assert np.array_equal(tr.cpu().numpy(), d["traces32"]), tune


def test_breast_mimo_alone_and_batched_bit_exact(cuda):
    g = load("breast_mimo_small")
    steps = int(g["steps"])
    solves, keys = [], []
    wave = torch.from_numpy(g["wave"])
    for p in range(len(g["sides"])):
        ph, ca, cb = breast_coeffs(g, p)
        ant = ph.antennas(16)
        for tx in range(int(g["n_tx"])):
            i, j = ant[tx]
            sim, f = sim2d(cuda, ph.side, ph.side, float(g["dx"]), float(g["courant"]),
                           [("Hz", "point", (i, i + 1, j, j + 1), wave, None)], ca, cb, steps=steps)
            tr = sim.run(steps, record=Detectors(ant))
            assert sha(tr) == str(g[f"p{p}_tx{tx}_sha_traces"])
            assert sha(f.Hz) == str(g[f"p{p}_tx{tx}_sha_hz"])
            assert rel_l2(tr[:, ::5].cpu().numpy(), g[f"p{p}_tx{tx}_traces64_dec"]) < 1e-5
            grid = YeeGrid(ph.side, ph.side, float(g["dx"]), float(g["dx"]),
                           courant=float(g["courant"]), device=cuda)
            src = PointSource(TabulatedWaveform(wave), i, j, "Hz", grid=grid, N_steps=steps)
            solves.append(BatchSolve(grid, SourceCollection([src]), Detectors(ant),
                                     ca.reshape(ph.side, ph.side, 1).to(cuda),
                                     cb.reshape(ph.side, ph.side, 1).to(cuda)))
            keys.append(f"p{p}_tx{tx}")
    for mode in ("persistent", "tiled", "queue"):
        for tune in (None, (3, 32, 64, 1, 0), (6, 48, 128, 1, 0), (2, 8, 32, 1, 0),
                     (4, 48, 128, 1, 1024), (5, 48, 128, 1, 1024), (7, 64, 128, 1, 1024),
                     (6, 64, 128, 1, 512)):
            batch = Batch2D(solves, steps, tune=tune, mode=mode)
            if mode != "persistent":
                for chunk in (7, 100, 1, steps - 108):   # uneven chunks, a single-step pass
                    batch.run(chunk)
            else:
                batch.run()
            torch.cuda.synchronize()
            assert all(s == 0 for s in batch.statuses())
            for q, key in enumerate(keys):
                assert sha(batch.traces(q)) == str(g[key + "_sha_traces"]), (mode, tune, key)
                assert sha(batch.fields(q)[2]) == str(g[key + "_sha_hz"]), (mode, tune, key)


def _random_case(rng, nx, ny, steps, material, n_src):
    kinds = []
    for _ in range(n_src):
        comp = ("Ex", "Ey", "Hz")[rng.integers(0, 3)]
        wave = torch.from_numpy(rng.standard_normal(steps).astype(np.float32))
        if rng.random() < 0.75:
            i, j = int(rng.integers(0, nx)), int(rng.integers(0, ny))
            kinds.append((comp, "point", (i, i + 1, j, j + 1), wave, None))
        else:
            if rng.random() < 0.5:
                a, b = sorted(rng.choice(nx + 1, 2, replace=False))
                j = int(rng.integers(0, ny))
                box = (int(a), int(b), j, j + 1)
                n = int(b - a)
            else:
                a, b = sorted(rng.choice(ny + 1, 2, replace=False))
                i = int(rng.integers(0, nx))
                box = (i, i + 1, int(a), int(b))
                n = int(b - a)
            amp = torch.from_numpy(rng.uniform(0.2, 2.0, n).astype(np.float32))
            kinds.append((comp, "line", box, wave, amp))
    ca = cb = None
    if material:
        grid = YeeGrid(nx, ny, 1e-3, 1e-3, courant=0.9, device="cpu")
        mm = MaterialMap(grid, default=Material("bg", float(rng.uniform(1, 5)), float(rng.uniform(0, 1))))
        for q in range(4):
            mm.add_circle((float(rng.uniform(0, nx)), float(rng.uniform(0, ny))),
                          float(rng.uniform(1, max(nx, ny) / 3)),
                          Material(f"m{q}", float(rng.uniform(1, 60)), float(rng.uniform(0, 3))))
        ca, cb = (t[..., 0] for t in mm.build())
    return kinds, ca, cb


@pytest.mark.parametrize("seed", range(6))
def test_random_cases_bit_exact_vs_oracle(cuda, seed):
    rng = np.random.default_rng(100 + seed)
    nx, ny = int(rng.integers(4, 70)), int(rng.integers(4, 70))
    steps = int(rng.integers(1, 90))
    spec, ca, cb = _random_case(rng, nx, ny, steps, material=bool(seed % 2), n_src=int(rng.integers(0, 5)))
    dt = oracle.stable_dt(1e-3, 1e-3, None, 0.9)
    o = oracle.Oracle2D(nx, ny, 1e-3, 1e-3, dt, ca, cb)
    for comp, kind, box, wave, amp in spec:
        o.add_box_source(comp, box, wave, amp)
    probes = [(("Ex", "Ey", "Hz")[rng.integers(0, 3)], int(rng.integers(0, nx)), int(rng.integers(0, ny)))
              for _ in range(7)]
    tr_o = o.run(steps, probes)
    for tune in TUNES:
        sim, f = sim2d(cuda, nx, ny, 1e-3, 0.9, spec, ca, cb, steps=steps, tune=tune)
        tr = sim.run(steps, record=Detectors(probes))
        assert np.array_equal(tr.cpu().numpy(), tr_o.numpy()), tune
        for c in ("Ex", "Ey", "Hz"):
            assert np.array_equal(getattr(f, c)[..., 0].cpu().numpy(), getattr(o, c).numpy()), (tune, c)


def test_split_runs_equal_one_run(cuda):
    """run(a); run(b) == run(a+b) bit for bit (pass plans and step offsets)."""
    rng = np.random.default_rng(7)
    spec, ca, cb = _random_case(rng, 41, 37, 120, True, 3)
    s1, f1 = sim2d(cuda, 41, 37, 1e-3, 0.9, spec, ca, cb, steps=120, tune=(3, 8, 32, 1, 0))
    s1.run(120)
    s2, f2 = sim2d(cuda, 41, 37, 1e-3, 0.9, spec, ca, cb, steps=120, tune=(3, 8, 32, 1, 0))
    for n in (1, 2, 3, 5, 7, 13, 89):
        s2.run(n)
    for c in ("Ex", "Ey", "Hz"):
        assert torch.equal(getattr(f1, c), getattr(f2, c))


def test_divergence_detection_matches_reference(cuda):
    """tests/test_fdtd2d.py:143-156 and the threshold bookkeeping."""
    g = YeeGrid(8, 8, 1e-3, 1e-3, device=cuda)
    f = FieldSet(g)
    sim = FDTD2D(g, f, MurABC(g, f.Hz), stability_threshold=1.0, n_check=1)
    f.Hz[:] = 2.0
    with pytest.raises(SimulationDivergedError):
        sim.step()
    # last_field_max tracks the largest checked |field| like the reference
    rng = np.random.default_rng(3)
    spec, ca, cb = _random_case(rng, 30, 22, 64, True, 2)
    sim, f = sim2d(cuda, 30, 22, 1e-3, 0.9, spec, ca, cb, steps=64)
    sim._n_check = 16
    o = oracle.Oracle2D(30, 22, 1e-3, 1e-3, oracle.stable_dt(1e-3, 1e-3, None, 0.9), ca, cb)
    o.n_check = 16
    for comp, kind, box, wave, amp in spec:
        o.add_box_source(comp, box, wave, amp)
    o.run(64)
    sim.run(64)
    assert sim.last_field_max == o.last_field_max
    assert sim.n_stability_checks == 4


def test_waveform_shorter_than_run_raises(cuda):
    g = YeeGrid(16, 16, 1e-3, 1e-3, device=cuda)
    f = FieldSet(g)
    src = PointSource(TabulatedWaveform(torch.ones(10)), 8, 8, "Hz", grid=g, N_steps=10)
    sim = FDTD2D(g, f, MurABC(g, f.Hz), SourceCollection([src]))
    sim.run(10)
    with pytest.raises(IndexError):
        sim.step()


def test_full_size_linearity_and_tune_independence(cuda):
    """4096^2 lossy-ellipse grid: doubling the source doubles every sample
    exactly (every op is linear and x2 is exact in float32), and different
    temporal-block depths / tiles give bit-identical results."""
    wl = W.LossyEllipses(n=4096, steps=200)
    grid_c = YeeGrid(4096, 4096, wl.dx, wl.dx, courant=wl.courant, device="cpu")
    mm = MaterialMap(grid_c, default=wl.background(Material))
    wl.paint(mm, Material)
    ca, cb = (t[..., 0] for t in mm.build())
    wave = oracle.gauss_deriv_wave(wl.steps, grid_c.dt)
    i, j = wl.source
    outs = []
    for scale, tune in ((1.0, None), (2.0, None), (1.0, (2, 32, 128, 1, 0))):
        sim, f = sim2d(cuda, 4096, 4096, wl.dx, wl.courant,
                       [("Hz", "point", (i, i + 1, j, j + 1), wave * scale, None)], ca, cb,
                       steps=wl.steps, tune=tune)
        tr = sim.run(wl.steps, record=Detectors(wl.receivers))
        outs.append((tr.clone(), f.Hz.clone()))
        del sim, f
    assert float(outs[0][0].abs().max()) > 0.0
    # exact except where a value fell into the subnormal range (< 1.2e-38),
    # whose coarser rounding does not commute with scaling
    assert torch.allclose(outs[1][0], 2.0 * outs[0][0], rtol=0.0, atol=1e-36)
    assert torch.allclose(outs[1][1], 2.0 * outs[0][1], rtol=0.0, atol=1e-36)
    assert torch.equal(outs[2][0], outs[0][0])
    assert torch.equal(outs[2][1], outs[0][1])


def test_batch_graph_replay_and_autotune_bit_exact(cuda):
    """A CUDA-graph capture of a full batched run replays to the same bits as
    the plain runs (both scheduling modes, two replays in a row), and the
    autotuned batch (whatever shape it picks) gives the same bits too."""
    g = load("breast_mimo_small")
    steps = 120
    wave = torch.from_numpy(g["wave"][:steps].copy())
    solves, refs = [], []
    for p in range(len(g["sides"])):
        ph, ca, cb = breast_coeffs(g, p)
        ant = ph.antennas(16)
        for tx in range(3):
            i, j = ant[tx]
            grid = YeeGrid(ph.side, ph.side, float(g["dx"]), float(g["dx"]),
                           courant=float(g["courant"]), device=cuda)
            src = PointSource(TabulatedWaveform(wave), i, j, "Hz", grid=grid, N_steps=steps)
            solves.append(BatchSolve(grid, SourceCollection([src]), Detectors(ant),
                                     ca.reshape(ph.side, ph.side, 1).to(cuda),
                                     cb.reshape(ph.side, ph.side, 1).to(cuda)))
            sim, f = sim2d(cuda, ph.side, ph.side, float(g["dx"]), float(g["courant"]),
                           [("Hz", "point", (i, i + 1, j, j + 1), wave, None)], ca, cb,
                           steps=steps)
            refs.append((sim.run(steps, record=Detectors(ant)).clone(), f.Hz.clone()))
    for mode in ("persistent", "tiled", "queue"):
        b = Batch2D(solves, steps, mode=mode)
        b.capture()
        for _ in range(2):
            b.replay()
            torch.cuda.synchronize()
            for q, (tr, hz) in enumerate(refs):
                assert torch.equal(b.traces(q), tr), (mode, q)
                assert torch.equal(b.fields(q)[2].reshape(hz.shape), hz), (mode, q)
    auto = Batch2D(solves, steps, tune="auto")
    assert auto.mode in ("persistent", "tiled", "queue")
    auto.run()
    torch.cuda.synchronize()
    for q, (tr, hz) in enumerate(refs):
        assert torch.equal(auto.traces(q), tr)
    from waveforge_b200.autotune import tune_plain2d
    t = tune_plain2d(300, 200, materials=True, device=cuda)
    assert len(t) == 5 and t[0] >= 1


def test_tile_queue_bounded_wait_reports_timeout_then_recovers(cuda):
    """The tile-queue kernel's neighbour waits are bounded: with every pass
    counter preset to -1 (as if no tile had finished the previous pass) and a
    bound of 64 polls, items give up instead of waiting for good, the solves
    report WF_E_TIMEOUT, and the next normal run of the same batch is
    bit-identical to the plain per-solve runs."""
    import ctypes
    from waveforge_b200 import _native as nat
    g = load("breast_mimo_small")
    steps = 60
    wave = torch.from_numpy(g["wave"][:steps].copy())
    solves, refs = [], []
    for p in range(len(g["sides"])):
        ph, ca, cb = breast_coeffs(g, p)
        ant = ph.antennas(16)
        i, j = ant[0]
        grid = YeeGrid(ph.side, ph.side, float(g["dx"]), float(g["dx"]),
                       courant=float(g["courant"]), device=cuda)
        src = PointSource(TabulatedWaveform(wave), i, j, "Hz", grid=grid, N_steps=steps)
        solves.append(BatchSolve(grid, SourceCollection([src]), Detectors(ant),
                                 ca.reshape(ph.side, ph.side, 1).to(cuda),
                                 cb.reshape(ph.side, ph.side, 1).to(cuda)))
        sim, f = sim2d(cuda, ph.side, ph.side, float(g["dx"]), float(g["courant"]),
                       [("Hz", "point", (i, i + 1, j, j + 1), wave, None)], ca, cb, steps=steps)
        refs.append(sim.run(steps, record=Detectors(ant)).clone())
    b = Batch2D(solves, steps, tune=(3, 32, 64, 1, 0), mode="queue")
    b._upload(0, steps)
    tiles, nbr, done = b._queue_tables()
    done.fill_(-1)
    b._queue.zero_()
    nat.check(nat.load().wf_batch2d_queue(
        b._desc_dev.data_ptr(), tiles.data_ptr(), tiles.shape[0], nbr.data_ptr(),
        done.data_ptr(), b._queue.data_ptr(), steps, ctypes.byref(b.tune),
        1 if b._fastdiv else 0, 64, nat.stream_handle(cuda)))
    torch.cuda.synchronize()
    assert nat.WF_E_TIMEOUT in b.statuses()
    b.reset()
    b.run()
    torch.cuda.synchronize()
    assert all(s == 0 for s in b.statuses())
    for q, tr in enumerate(refs):
        assert torch.equal(b.traces(q), tr), q
