"""Host-side logic that needs no GPU: pass plans, tile coverage, typed
material regions, request generation, argument validation, and that every
compute entry refuses CPU tensors (there is no CPU fallback)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from waveforge_b200 import workloads as W
from waveforge_b200.batch import PassPlan, tile_items
from waveforge_b200.core.grid import YeeGrid, compute_stable_dt
from waveforge_b200.core.materials import Material, MaterialMap
from waveforge_b200.serving import request_footprint, request_work


@pytest.mark.parametrize("K", [1, 2, 3, 4, 6, 8])
def test_pass_plan_covers_steps_and_lands_in_state(K):
    for n in range(1, 80):
        pl = PassPlan(n, K)
        lens = [pl.length(p) for p in range(pl.passes)]
        offs = [pl.offset(p) for p in range(pl.passes)]
        assert sum(lens) == n and all(1 <= x <= K for x in lens)
        assert offs == [sum(lens[:p]) for p in range(pl.passes)]
        # an even pass count ends in the state buffers; only odd runs of
        # single-step passes need the copy-back
        assert pl.needs_copy == (pl.passes % 2 == 1)
        if pl.needs_copy:
            assert all(x == 1 for x in lens)


@pytest.mark.parametrize("region,k", [((48, 128), 6), ((64, 128), 8), ((32, 64), 3), ((8, 32), 1),
                                      ((32, 128), 4)])
def test_tile_items_partition_every_grid(region, k):
    rng = np.random.default_rng(3)
    shapes = [tuple(int(v) for v in rng.integers(4, 300, 2)) for _ in range(5)]
    it = tile_items(shapes, k, region)
    ci, cj = region[0] - 2 * k, region[1] - 2 * k
    for q, (nx, ny) in enumerate(shapes):
        cover = np.zeros((nx, ny), np.int32)
        for s, i0, j0 in it[it[:, 0] == q]:
            cover[i0:i0 + ci, j0:j0 + cj] += 1
        assert (cover == 1).all()
    # largest grids first
    firsts = [int(it[it[:, 0] == q][0, 0]) for q in range(len(shapes))]
    order = [int(x) for x in dict.fromkeys(it[:, 0].tolist())]
    assert sorted(order, key=lambda q: -shapes[q][0] * shapes[q][1]) == order and len(firsts) == 5


def test_typed_regions_equal_custom_masks_on_host():
    g = YeeGrid(90, 70, 1e-3, 1e-3, courant=0.5, device="cpu")
    a = MaterialMap(g, default=Material("bg", 3.0, 0.1))
    b = MaterialMap(g, default=Material("bg", 3.0, 0.1))
    m1, m2 = Material("e", 11.0, 0.4), Material("s", 30.0, 0.9)
    a.add_ellipse((44.3, 30.7), (21.5, 13.25), m1)
    b.add_custom(W.ellipse_mask(44.3, 30.7, 21.5, 13.25), m1)
    outer, inner = W.ellipse_mask(40.0, 35.0, 30.0, 25.0), W.ellipse_mask(40.0, 35.0, 27.0, 22.0)
    a.add_shell((40.0, 35.0), (30.0, 25.0), (27.0, 22.0), m2)
    b.add_custom(lambda I, J: outer(I, J) & ~inner(I, J), m2)
    for x, y in zip(a.build(), b.build()):
        assert torch.equal(x, y)
    assert a.device_paintable and not b.device_paintable


def test_serving_requests_are_seeded_and_accounted():
    r1 = W.serving_request(200, 500, 17, n_ant=8)
    r2 = W.serving_request(200, 500, 17, n_ant=8)
    c1, _ = r1.material.build()
    c2, _ = r2.material.build()
    assert torch.equal(c1, c2)
    assert request_work(r1) == 8 * 200 * 200 * 500
    g = W.serving_request(200, 500, 17, n_ant=8, gradient=True)
    assert g.target is not None and request_work(g) == 2 * request_work(r1)
    assert request_footprint(g, 64) > request_footprint(r1, 64)
    arr = W.ServingStream(rate=50.0, duration=0.4, seed=2).arrivals()
    assert all(0 <= t < 0.4 for t, _ in arr) and [t for t, _ in arr] == sorted(t for t, _ in arr)
    assert all(128 <= r.tag[0] <= 1024 and 1000 <= r.tag[1] <= 5000 for _, r in arr)


def test_grid_cfl_and_validation():
    dt = compute_stable_dt(1e-3, 1e-3, courant=0.5)
    assert dt == oracle.stable_dt(1e-3, 1e-3, courant=0.5)
    with pytest.raises(ValueError):
        YeeGrid(32, 32, 1e-3, 1e-3, dt=compute_stable_dt(1e-3, 1e-3, courant=0.99) * 1.5,
                device="cpu")
    with pytest.raises(ValueError):
        compute_stable_dt(1e-3, 1e-3, courant=1.2)


def test_antenna_ring_validation_and_geometry():
    from waveforge_b200 import AntennaRing
    g = YeeGrid(64, 64, 1e-3, 1e-3, courant=0.5, device="cpu")
    with pytest.raises(ValueError):
        AntennaRing(1, 10, 0, g)
    with pytest.raises(ValueError):
        AntennaRing(8, 40, 0, g)
    with pytest.raises(ValueError):
        AntennaRing(8, 10, 3, g)
    ring = AntennaRing(16, 30, 0, g)
    assert len(ring.positions) == 16
    assert all(1 <= i <= 62 and 1 <= j <= 62 for i, j, _ in ring.positions)
    assert ring.positions_mm[0] == (ring.positions[0][0] * 1.0, ring.positions[0][1] * 1.0, 0.0)


def test_detectors_validation():
    from waveforge_b200 import Detectors
    with pytest.raises(ValueError):
        Detectors([])
    with pytest.raises(ValueError):
        Detectors([(1, 2, 3, 4)])
    d = Detectors([(1, 2), ("Ex", 3, 4)])
    assert d.points == [("Hz", 1, 2, 0), ("Ex", 3, 4, 0)]


def test_no_cpu_fallback():
    """Every engine refuses CPU tensors with an explicit error."""
    from waveforge_b200 import FDTD2D, FieldSet, MurABC
    from waveforge_b200.serving import Server
    g = YeeGrid(16, 16, 1e-3, 1e-3, courant=0.5, device="cpu")
    f = FieldSet(g)
    with pytest.raises(RuntimeError, match="CUDA"):
        FDTD2D(g, f, MurABC(g, f.Hz))
    with pytest.raises(RuntimeError, match="CUDA"):
        Server("cpu")
    mm = MaterialMap(g).add_circle((8.0, 8.0), 3.0, Material("d", 4.0, 0.0))
    with pytest.raises(RuntimeError, match="CUDA"):
        mm.build_device("cpu")


def test_dataset_cli_dry_run_and_arguments(capsys):
    """The generator's command line keeps the reference's arguments
    (datasets/generate_brain_dataset.py:60-108); --dry_run exits 0 without a GPU."""
    from waveforge_b200.datasets import generate_brain_dataset as cli
    a = cli.parse_args(["--n_samples", "8", "--output_dir", "/tmp/x", "--phantom", "B",
                        "--freq_low_ghz", "1", "--freq_high_ghz", "3", "--grid_size", "48"])
    assert (a.n_samples, a.phantom, a.grid_size, a.n_tx, a.ring_radius, a.n_steps) == (8, "B", 48, 8, 30, 300)
    assert cli.main(["--n_samples", "4", "--output_dir", "/tmp/x", "--dry_run"]) == 0
    assert "DRY RUN" in capsys.readouterr().out


def test_cole_cole_spectrum_matches_pointwise():
    from waveforge_b200.datasets.brain import TISSUES, cole_cole_spectrum, cole_cole_to_fdtd
    f, e, s = cole_cole_spectrum(TISSUES["gray_matter"], 1e8, 1e10, 7)
    for x, ee, ss in zip(f, e, s):
        assert (ee, ss) == cole_cole_to_fdtd(TISSUES["gray_matter"], float(x))
    assert e[0] > e[-1] and s[0] < s[-1]   # dispersion: permittivity falls, loss rises
