"""float64 runs of the 2D engine (``wf_fdtd2d_run_f64``) against the
reference's own float64 runs.

The reference's YeeGrid / FieldSet take ``dtype=torch.float64``
(src/core/grid.py:226-239, src/core/fields.py:124-130) and FDTD2D then steps
in float64.  The fixture ``f64_2d`` was written by running that loop
(``tests/golden/make_golden.py``, case ``f64``) with the float64 waveform and
amplitude tables stored; the ``edges2d_*`` fixtures hold the final float64 Hz
of the edge-semantics cases (float32 tables widened, float32 Ca/Cb widened).

Bar: float64 traces, final fields and stability telemetry bit-identical to
the reference (SHA-256 / array equality).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from _cases import edge2d_sources, load
from conftest import sha
from waveforge_b200 import (FDTD2D, Detectors, FieldSet, LineSource, MurABC, PointSource,
                            SourceCollection, TabulatedWaveform, YeeGrid)
from waveforge_b200 import workloads as W
from waveforge_b200.core.materials import Material, MaterialMap

F64 = torch.float64
COMP2 = ("Ex", "Ey", "Hz")


def _vac_sim(dev, g):
    grid = YeeGrid(160, 192, 1e-3, 1e-3, courant=0.6, device=dev, dtype=F64)
    assert grid.dt == float(g["vac_dt"])
    f = FieldSet(grid)
    w = torch.from_numpy(g["vac_waves"])
    steps = w.shape[1]
    tab = [TabulatedWaveform(w[q]) for q in range(4)]
    srcs = [PointSource(tab[0], 80, 96, "Hz", grid=grid, N_steps=steps),
            LineSource(tab[1], "x", 30, 60, 100, "Ex", grid=grid, N_steps=steps,
                       amplitude_profile=torch.from_numpy(g["vac_amp"])),
            PointSource(tab[2], 120, 50, "Ey", grid=grid, N_steps=steps),
            PointSource(tab[2], 120, 50, "Ey", grid=grid, N_steps=steps),
            PointSource(tab[3], 0, 140, "Hz", grid=grid, N_steps=steps)]
    sim = FDTD2D(grid, f, MurABC(grid, f.Hz), SourceCollection(srcs), n_check=50)
    det = Detectors([(COMP2[c], int(i), int(j)) for c, i, j in g["vac_probes"]])
    return sim, f, det, steps


def _check_vac(g, sim, f, tr):
    assert tr.dtype == F64
    assert sha(tr) == str(g["vac_sha_traces"])
    assert sha(f.Ex) == str(g["vac_sha_ex"])
    assert sha(f.Ey) == str(g["vac_sha_ey"])
    assert sha(f.Hz) == str(g["vac_sha_hz"])
    assert sim.last_field_max == float(g["vac_last_max"])
    assert sim.n_stability_checks == int(g["vac_checks"])


@pytest.mark.gpu
def test_f64_vacuum_sources_probes_bit_exact(cuda):
    """Overlapping, weighted and edge sources; probes on every edge; one run,
    uneven chunks and single steps all land on the reference's bits."""
    g = load("f64_2d")
    sim, f, det, steps = _vac_sim(cuda, g)
    _check_vac(g, sim, f, sim.run(steps, record=det))

    sim, f, det, steps = _vac_sim(cuda, g)
    parts = [sim.run(n, record=det) for n in (1, 123, 50, steps - 174)]
    _check_vac(g, sim, f, torch.cat(parts, dim=1))

    sim, f, det, steps = _vac_sim(cuda, g)
    for _ in range(steps):
        sim.step()
    assert sha(f.Hz) == str(g["vac_sha_hz"]) and sha(f.Ex) == str(g["vac_sha_ex"])


@pytest.mark.gpu
def test_f64_graph_replay_bit_exact(cuda):
    g = load("f64_2d")
    sim, f, det, steps = _vac_sim(cuda, g)
    sim.compile_step()
    for rep in range(2):
        sim.reset()
        _check_vac(g, sim, f, sim.run(steps, record=det))


@pytest.mark.gpu
def test_f64_lossy_materials_random_start_bit_exact(cuda):
    g = load("f64_2d")
    n, steps = int(g["mat_n"]), int(g["mat_steps"])
    wl = W.LossyEllipses(n=n, steps=steps, seed=int(g["mat_seed"]))
    gc = YeeGrid(n, n, wl.dx, wl.dx, courant=wl.courant, device="cpu", dtype=F64)
    mm = MaterialMap(gc, default=wl.background(Material))
    wl.paint(mm, Material)
    ca, cb = mm.build()
    assert ca.dtype == F64 and sha(ca) == str(g["mat_sha_ca"]) and sha(cb) == str(g["mat_sha_cb"])
    grid = YeeGrid(n, n, wl.dx, wl.dx, courant=wl.courant, device=cuda, dtype=F64)
    assert grid.dt == float(g["mat_dt"])
    f = FieldSet(grid)
    for c, v in W.initial_fields(int(g["mat_init_seed"]), (n, n), COMP2).items():
        getattr(f, c).copy_(torch.from_numpy(v).to(F64).reshape(n, n, 1))
    i, j = (int(v) for v in g["mat_src"])
    src = PointSource(TabulatedWaveform(torch.from_numpy(g["mat_wave"])), i, j, "Hz", grid=grid,
                      N_steps=steps)
    sim = FDTD2D(grid, f, MurABC(grid, f.Hz), SourceCollection([src]), Ca=ca.to(cuda),
                 Cb=cb.to(cuda), n_check=10 ** 9)
    tr = sim.run(steps, record=Detectors([(int(a), int(b)) for a, b in g["mat_rx"]]))
    assert sha(tr) == str(g["mat_sha_traces"])
    for c in COMP2:
        assert sha(getattr(f, c)) == str(g[f"mat_sha_{c.lower()}"]), c


@pytest.mark.gpu
def test_f64_batched_fieldset_bit_exact(cuda):
    g = load("f64_2d")
    nx, ny, B = 64, 48, 3
    wave = torch.from_numpy(g["batch_wave"])
    steps = wave.numel()
    gc = YeeGrid(nx, ny, 2e-3, 2e-3, courant=0.7, device="cpu", dtype=F64)
    mm = MaterialMap(gc, default=Material("bg", 3.0, 0.05))
    mm.add_circle((30.0, 20.0), 9.0, Material("c", 20.0, 0.8))
    ca, cb = mm.build()
    assert sha(ca) == str(g["batch_sha_ca"])
    grid = YeeGrid(nx, ny, 2e-3, 2e-3, courant=0.7, device=cuda, dtype=F64)
    f = FieldSet(grid, batch_size=B)
    for c, v in W.initial_fields(66, (B, nx, ny), COMP2).items():
        getattr(f, c).copy_(torch.from_numpy(v).to(F64).reshape(B, nx, ny, 1))
    src = PointSource(TabulatedWaveform(wave), 20, 30, "Hz", grid=grid, N_steps=steps)
    sim = FDTD2D(grid, f, MurABC(grid, f.Hz), SourceCollection([src]), Ca=ca.to(cuda),
                 Cb=cb.to(cuda), n_check=25)
    sim.run(steps)
    for c in COMP2:
        assert sha(getattr(f, c)) == str(g[f"batch_sha_{c.lower()}"]), c
    assert sim.last_field_max == float(g["batch_last_max"])
    assert sim.n_stability_checks == int(g["batch_checks"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["tiny7x5", "odd33x17", "min4x4"])
def test_f64_edge_cases_bit_exact(cuda, name):
    """float32 waveform / amplitude tables and float32 Ca/Cb widened to
    float64, as the reference's float64 run of the same case widens them."""
    d = load(f"edges2d_{name}")
    nx, ny, steps = int(d["nx"]), int(d["ny"]), int(d["steps"])
    grid = YeeGrid(nx, ny, float(d["dx"]), float(d["dx"]), courant=float(d["courant"]),
                   device=cuda, dtype=F64)
    f = FieldSet(grid)
    srcs = []
    for comp, kind, (i0, i1, j0, j1), wave, amp in edge2d_sources(d):
        w = TabulatedWaveform(wave)
        if kind == "point":
            srcs.append(PointSource(w, i0, j0, comp, grid=grid, N_steps=steps))
        else:
            axis = "x" if i1 - i0 > 1 else "y"
            pos, start, stop = (j0, i0, i1) if axis == "x" else (i0, j0, j1)
            srcs.append(LineSource(w, axis, pos, start, stop, comp, grid=grid, N_steps=steps,
                                   amplitude_profile=None if amp is None else amp.to(F64)))
    ca = cb = None
    if "ca" in d:   # float32 coefficients: the engine widens them
        ca = torch.from_numpy(d["ca"]).reshape(nx, ny, 1).to(cuda)
        cb = torch.from_numpy(d["cb"]).reshape(nx, ny, 1).to(cuda)
    sim = FDTD2D(grid, f, MurABC(grid, f.Hz), SourceCollection(srcs), Ca=ca, Cb=cb,
                 n_check=10 ** 9)
    sim.run(steps)
    assert np.array_equal(f.Hz[..., 0].cpu().numpy(), d["hz64"])


def test_f64_host_validation_needs_no_gpu():
    """Argument checks of the float64 path run before any device work."""
    grid = YeeGrid(16, 16, 1e-3, 1e-3, courant=0.5, device="cpu", dtype=F64)
    f = FieldSet(grid)
    with pytest.raises((TypeError, ValueError, RuntimeError)):
        FDTD2D(grid, f, MurABC(grid, f.Hz))   # host tensors: the engine needs CUDA fields
    g16 = YeeGrid(16, 16, 1e-3, 1e-3, courant=0.5, device="cpu", dtype=torch.float16)
    f16 = FieldSet(g16)
    with pytest.raises((TypeError, RuntimeError)):
        FDTD2D(g16, f16, MurABC(g16, f16.Hz))
