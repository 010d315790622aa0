"""AntennaRing (src/datasets/brain/antenna.py): ring geometry, device
recording, and compute_das_image against golden images that
tests/golden/make_golden.py produced by running the reference.

CPU: the oracle restatement reproduces the golden images bit for bit and the
ring positions match.  GPU: with the reference's (scipy) envelope the device
travel-time table + DAS give the golden image bit for bit (free space and
layered, even and odd trace lengths); the full path with the device envelope
agrees to rel-L2 <= 1e-5 with the same peak pixel; recording through the
step kernels equals the per-step record() gather.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from conftest import golden, rel_l2
from waveforge_b200.core.grid import YeeGrid

HEAD = {"cx_cells": 48, "cy_cells": 47, "layers": [(41, 10.0), (33, 5.0), (14, 40.0)]}


def _ring(device, n_steps):
    from waveforge_b200 import AntennaRing, TabulatedWaveform
    g = YeeGrid(96, 96, 0.5e-3, 0.5e-3, courant=0.5, device=device)
    ring = AntennaRing(8, 40, 0, g)
    if device != "cpu":
        ring.build_sources(TabulatedWaveform(torch.zeros(n_steps)), 0, N_steps=n_steps)
    return ring, g


def test_oracle_and_positions_match_reference_golden():
    d = golden("antenna_ring96")
    ring, g = _ring("cpu", 600)
    assert [tuple(p) for p in ring.positions] == [tuple(int(v) for v in p) for p in d["positions"]]
    for n in (600, 599):
        env = d[f"env_{n}"]
        a = oracle.antenna_das_image_ref(None, d["positions"], 96, 96, float(d["dx"]),
                                         float(d["dt"]), n, 40, env=env)
        b = oracle.antenna_das_image_ref(None, d["positions"], 96, 96, float(d["dx"]),
                                         float(d["dt"]), n, 33, HEAD, env=env)
        assert np.array_equal(a, d[f"img_free_{n}"])
        assert np.array_equal(b, d[f"img_head_{n}"])


@pytest.mark.gpu
@pytest.mark.parametrize("n", [600, 599])
def test_device_das_bit_exact_given_reference_envelope(cuda, n):
    d = golden("antenna_ring96")
    ring, _ = _ring(cuda, n)
    env = torch.from_numpy(d[f"env_{n}"])
    img_f = ring.compute_das_image_from_envelope(env, 40).cpu().numpy()
    img_h = ring.compute_das_image_from_envelope(env, 33, HEAD).cpu().numpy()
    assert np.array_equal(img_f, d[f"img_free_{n}"])
    assert np.array_equal(img_h, d[f"img_head_{n}"])


@pytest.mark.gpu
@pytest.mark.parametrize("n", [600, 599])
def test_full_das_image_matches_reference(cuda, n):
    d = golden("antenna_ring96")
    sig = golden("das_breast96")["delta"][:, :, :n]
    ring, _ = _ring(cuda, n)
    env = ring.envelope(sig).cpu().numpy()
    assert rel_l2(env, d[f"env_{n}"]) < 1e-6
    for size, head, key in ((40, None, f"img_free_{n}"), (33, HEAD, f"img_head_{n}")):
        img = ring.compute_das_image(sig, size, head)
        ref = d[key]
        assert img.dtype == np.float32 and img.shape == ref.shape
        assert rel_l2(img, ref) <= 1e-5
        assert np.unravel_index(img.argmax(), img.shape) == np.unravel_index(ref.argmax(), ref.shape)


@pytest.mark.gpu
def test_kernel_recording_equals_per_step_record(cuda):
    from waveforge_b200 import (FDTD2D, AntennaRing, FieldSet, GaussianDerivativePulse, MurABC)
    steps = 150
    g = YeeGrid(64, 64, 1e-3, 1e-3, courant=0.5, device=cuda)
    a = AntennaRing(6, 25, 0, g, component="Hz")
    b = AntennaRing(6, 25, 0, g, component="Hz")
    w = GaussianDerivativePulse(10e9)
    for tx in (0, 3):
        f1 = FieldSet(g)
        s1 = FDTD2D(g, f1, MurABC(g, f1.Hz), a.build_sources(w, tx, steps))
        for n in range(steps):
            s1.step()
            a.record(f1.Hz, n, tx)
        f2 = FieldSet(g)
        s2 = FDTD2D(g, f2, MurABC(g, f2.Hz), b.build_sources(w, tx, steps))
        b.store(tx, s2.run(steps, record=b.detectors()))
    sa, sb = a.get_signals(), b.get_signals()
    assert sa.shape == (6, 6, steps)
    assert np.array_equal(sa, sb)
    assert np.abs(sa[3]).max() > 0
