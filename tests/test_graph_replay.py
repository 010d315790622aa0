"""CUDA-graph replay of single-solve runs (``compile_step``).

The reference's ``FDTD3D.compile_step`` hands the step to
``torch.compile(mode='reduce-overhead')`` (src/core/fdtd3d.py:404-419).
Here ``compile_step()`` makes ``run(n)`` record its pass launches in a CUDA
graph the first time a (start step, length, detectors) combination occurs and
replay it afterwards.  Replayed runs must equal the reference's goldens bit
for bit, repeatedly, and keep the stability bookkeeping."""

from __future__ import annotations

import pytest
import torch

from _cases import head_coeffs, load
from conftest import sha
from test_parity_2d import sim2d
from test_parity_3d import COMPS, sim3d
from waveforge_b200 import Detectors, FDTD2D, FieldSet, MurABC, SimulationDivergedError, YeeGrid

pytestmark = pytest.mark.gpu


def test_plain2d_graph_replay_bit_exact(cuda):
    g = load("vacuum_point_256")
    n, steps = int(g["n"]), int(g["steps"])
    i, j = (int(v) for v in g["src"])
    sim, f = sim2d(cuda, n, n, float(g["dx"]), float(g["courant"]),
                   [("Hz", "point", (i, i + 1, j, j + 1), torch.from_numpy(g["wave"]), None)],
                   steps=steps)
    sim.compile_step()
    det = Detectors([(int(a), int(b)) for a, b in g["rx"]], "Hz")
    for rep in range(3):           # capture, then two replays
        sim.reset()
        tr = sim.run(steps, record=det)
        assert sim.steps_completed == steps
        assert sha(tr) == str(g["sha_traces"]), rep
        assert sha(f.Hz) == str(g["sha_hz"]) and sha(f.Ex) == str(g["sha_ex"]), rep
    assert len(sim._graphs) == 1
    # a run split in two chunks: two graphs, same result
    for rep in range(2):
        sim.reset()
        a = sim.run(400, record=det)
        b = sim.run(steps - 400, record=det)
        assert sha(torch.cat([a, b], dim=1)) == str(g["sha_traces"]), rep
    assert len(sim._graphs) == 3


def test_head3d_graph_replay_bit_exact(cuda):
    g = load("head3d_32")
    ca, cb = head_coeffs(g)
    n, steps = int(g["n"]), int(g["steps"])
    i, j, k = (int(v) for v in g["src"])
    sim, f = sim3d(cuda, (n, n, n), float(g["dx"]), float(g["courant"]),
                   [("Ez", (i, i + 1, j, j + 1, k, k + 1), torch.from_numpy(g["wave"]))],
                   ca, cb, steps=steps)
    sim.compile_step()
    det = Detectors([("Ez", *(int(v) for v in r)) for r in g["rx"]])
    for rep in range(3):
        sim.reset()
        tr = sim.run(steps, record=det)
        assert sha(tr) == str(g["sha_traces"]), rep
        for c in COMPS:
            assert sha(getattr(f, c)) == str(g[f"sha_{c.lower()}"]), (rep, c)


def test_graph_replay_keeps_stability_checks(cuda):
    """Divergence is still detected from the device maxima after a replay."""
    grid = YeeGrid(16, 16, 1e-3, 1e-3, device=cuda)
    f = FieldSet(grid)
    sim = FDTD2D(grid, f, MurABC(grid, f.Hz), stability_threshold=1.0, n_check=2)
    sim.compile_step()
    sim.run(4)                      # captured and replayed: fields stay zero
    assert sim.n_stability_checks == 2 and sim.last_field_max == 0.0
    sim.reset()
    f.Hz[:] = 2.0
    with pytest.raises(SimulationDivergedError):
        sim.run(4)                  # replay of the same graph sees the large field
