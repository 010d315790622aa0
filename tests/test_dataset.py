"""Brain dataset path against the reference (golden brain_dataset40.npz, made
by tests/golden/make_golden.py from the reference's src/datasets).

CPU: Cole-Cole tissue values, seeded head geometries and bleed placement are
exactly equal; a phantom's painted Ca/Cb are bit-identical.  GPU: whole
generator samples -- both MIMO acquisitions run as one batched solve -- give
bit-identical target/reference/scattered signals, the same metadata and .npz
key set, and the DAS image within rel-L2 1e-5 (the Hilbert envelope is a
float64 device FFT instead of scipy's)."""

from __future__ import annotations

import hashlib
import json

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from waveforge_b200.core.grid import YeeGrid
from waveforge_b200.datasets.brain import (BrainPhantom3D, all_tissues_at_freq,
                                           sample_random_geometry)

G = np.load(GOLDEN / "brain_dataset40.npz")


def _sha(a) -> str:
    a = a.detach().cpu().contiguous().numpy() if torch.is_tensor(a) else np.ascontiguousarray(a)
    return hashlib.sha256(a.tobytes()).hexdigest()


@pytest.mark.parametrize("freq", [0.5e9, 1e9, 2e9, 6.5e9])
def test_tissue_values_equal_reference(freq):
    t = all_tissues_at_freq(freq)
    got = np.array([t[str(n)] for n in G["tissue_names"]], dtype=np.float64)
    assert np.array_equal(got, G[f"tissue_{int(freq)}"])


def test_random_geometries_equal_reference():
    for row in G["geoms"]:
        n, dx10, seed = (int(v) for v in row[:3])
        g = sample_random_geometry(seed, n, dx10 / 10)
        got = [*g.center, g.scalp_outer_r, g.skull_outer_r, g.skull_inner_r, g.dura_inner_r,
               g.csf_inner_r, g.gray_matter_r, g.white_matter_r]
        assert got == [int(v) for v in row[3:]], (n, dx10, seed)


def test_bleed_placement_equals_reference():
    grid = YeeGrid(64, 64, 3e-3, 3e-3, Nz=64, dz=3e-3, device="cpu")
    for case, row in zip(G["bleed_cases"], G["bleeds"]):
        btype, age, size = str(case).split("/")
        ph = BrainPhantom3D(grid, 1e9, geometry=sample_random_geometry(int(row[0]), 64, 3.0),
                            seed=int(row[1]))
        b = ph.add_random_bleed(btype, age, size)
        if row[2] < 0:
            assert b is None, case
        else:
            assert b is not None and list(b.center) == [int(v) for v in row[2:5]], case
            assert b.radius == int(row[5]) and b.eps_r == row[6] and b.sigma == row[7], case


def test_phantom_coefficients_bit_exact():
    grid = YeeGrid(64, 64, 3e-3, 3e-3, Nz=64, dz=3e-3, device="cpu")
    ph = BrainPhantom3D(grid, 1e9, geometry=sample_random_geometry(7, 64, 3.0), seed=9)
    ph.add_bleed_at((40, 30, 28), 4, "intracerebral", "subacute")
    ca, cb = ph.build()
    assert _sha(ca) == str(G["phantom64_ca_sha"]) and _sha(cb) == str(G["phantom64_cb_sha"])
    assert ph.get_label() == 3 and ph.get_metadata()["n_bleeds"] == 1


def test_generator_needs_cuda(tmp_path):
    from waveforge_b200.datasets import BrainDatasetGenerator
    with pytest.raises(RuntimeError, match="CUDA"):
        BrainDatasetGenerator(tmp_path, grid_size=40, dx_mm=6.0, n_tx=4, ring_radius_cells=18,
                              device="cpu", verbose=False)


def _gen(tmp_path, **kw):
    from waveforge_b200.datasets import BrainDatasetGenerator
    return BrainDatasetGenerator(tmp_path, grid_size=40, dx_mm=6.0, n_tx=4, ring_radius_cells=18,
                                 n_steps=700, device="cuda", seed=0, verbose=False, **kw)


@pytest.mark.gpu
@pytest.mark.parametrize("tag,kw", [("nb", {}), ("nb0", {}),
                                    ("uwb", {"freq_low_hz": 1e9, "freq_high_hz": 3e9})])
def test_generate_sample_equals_reference(cuda, tmp_path, tag, kw):
    gen = _gen(tmp_path, **kw)
    smp = gen.generate_sample(label=int(G[f"{tag}_label"]), seed=int(G[f"{tag}_seed"]))
    assert smp is not None
    assert _sha(smp["signals_total"]) == str(G[f"{tag}_sha_total"])
    assert _sha(smp["signals_reference"]) == str(G[f"{tag}_sha_reference"])
    assert np.array_equal(smp["signals_scattered"], G[f"{tag}_signals_scattered"])
    for k in ("bleed_center_cells", "bleed_radius_cells", "phantom_skull_inner_r", "phantom_gray_r",
              "phantom_scalp_outer_r", "dt_s", "freq_hz"):
        assert np.array_equal(np.asarray(smp[k]), G[f"{tag}_{k}"]), k
    assert [smp["bleed_type"], smp["bleed_age"]] == [str(v) for v in G[f"{tag}_bleed"]]
    ref_img = G[f"{tag}_das_image"].astype(np.float64)
    img = np.asarray(smp["das_image"], dtype=np.float64)
    assert img.shape == ref_img.shape
    if np.abs(ref_img).max() > 0:
        rel = np.linalg.norm(img - ref_img) / np.linalg.norm(ref_img)
        assert rel <= 1e-5, rel
        assert np.argmax(img) == np.argmax(ref_img)
    else:
        assert np.abs(img).max() == 0
    path = gen.save_sample(smp, 0)
    assert sorted(np.load(path, allow_pickle=True).files) == [str(k) for k in G[f"{tag}_npz_keys"]]


@pytest.mark.gpu
def test_single_and_full_mimo_equal_pair(cuda, tmp_path):
    """One transmitter alone, all transmitters of one phantom, and the
    target/reference pair give the same bits for the same solve."""
    gen = _gen(tmp_path)
    geom = sample_random_geometry(11, 40, 6.0)
    ph = BrainPhantom3D(gen.grid, 1e9, geometry=geom, seed=3)
    ph.add_bleed_at((20, 21, 20), 3, "intracerebral", "acute")
    healthy = BrainPhantom3D(gen.grid, 1e9, geometry=geom, seed=4)
    full, _ = gen._run_full_mimo(ph)
    one, _ = gen._run_simulation(ph, 2)
    tgt, ref, _ = gen._run_pair(ph, healthy)
    assert np.array_equal(one, full[2]) and np.array_equal(full, tgt)
    assert not np.array_equal(tgt, ref)
    full_h, _ = gen._run_full_mimo(healthy)
    assert np.array_equal(full_h, ref)


@pytest.mark.gpu
def test_balanced_dataset_writes_samples_and_manifest(cuda, tmp_path):
    from waveforge_b200.datasets import BrainDatasetGenerator
    gen = BrainDatasetGenerator(tmp_path, grid_size=32, dx_mm=6.0, n_tx=4, ring_radius_cells=14,
                                n_steps=60, device="cuda", seed=0, verbose=False)
    man = gen.generate_balanced_dataset(6, base_seed=3, show_progress=False)
    assert man["n_completed"] + man["n_failed"] == 6
    disk = json.loads((tmp_path / "manifest.json").read_text())
    assert disk["n_completed"] == man["n_completed"] and len(disk["sample_paths"]) == man["n_completed"]
    for p, label in zip(man["sample_paths"], man["labels"]):
        z = np.load(p, allow_pickle=True)
        assert int(z["label"]) == label and z["signals_total"].shape == (4, 4, 60)


@pytest.mark.gpu
def test_samples_batched_together_equal_reference(cuda, tmp_path):
    """Two samples (a bleed and a healthy head) advanced in one batched
    solve give each sample's reference signals bit for bit."""
    gen = _gen(tmp_path)
    out = gen.generate_samples([(int(G["nb_label"]), int(G["nb_seed"])),
                                (int(G["nb0_label"]), int(G["nb0_seed"]))])
    for tag, smp in zip(("nb", "nb0"), out):
        assert smp is not None
        assert _sha(smp["signals_total"]) == str(G[f"{tag}_sha_total"])
        assert _sha(smp["signals_reference"]) == str(G[f"{tag}_sha_reference"])
        assert np.array_equal(smp["signals_scattered"], G[f"{tag}_signals_scattered"])
