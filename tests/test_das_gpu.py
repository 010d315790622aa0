"""DAS backprojection on the GPU: bit-identical float64 images to the
reference NumPy functions (golden images), and to the oracle for the
variants (gate, self-pair skip, pixel pitch, image shape)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from _cases import load
from waveforge_b200 import YeeGrid, das_backprojection

pytestmark = pytest.mark.gpu

C0 = 299_792_458.0


def _grid(d, cuda):
    side = int(d["side"])
    g = YeeGrid(side, side, float(d["dx"]), float(d["dx"]), courant=0.5, device=cuda)
    assert g.dt == float(d["dt"])
    return g


def test_das_canonical_bit_exact(cuda):
    d = load("das_breast96")
    g = _grid(d, cuda)
    ant = [tuple(int(v) for v in a) for a in d["ant"]]
    steps = int(d["steps"])
    img = das_backprojection(d["delta"], ant, g, steps, image_shape=(48, 40))
    assert np.array_equal(img, d["img_canonical_48x40"])
    img = das_backprojection(d["delta"], ant, g, steps)
    assert np.array_equal(img, d["img_full"])
    assert np.unravel_index(img.argmax(), img.shape) == np.unravel_index(
        d["img_full"].argmax(), d["img_full"].shape)


def test_das_gated_variant_bit_exact(cuda):
    d = load("das_breast96")
    g = _grid(d, cuda)
    ant = [tuple(int(v) for v in a) for a in d["ant"]]
    img = das_backprojection(d["delta"], ant, g, int(d["steps"]), pitch=g.dx,
                             gate_start=int(d["gate_start"]))
    assert np.array_equal(img, d["img_gated"])


@pytest.mark.parametrize("seed", range(3))
def test_das_variants_vs_oracle(cuda, seed):
    rng = np.random.default_rng(50 + seed)
    n_ant, steps, nx, ny = int(rng.integers(2, 20)), int(rng.integers(10, 400)), 60, 44
    dx = 1e-3
    g = YeeGrid(nx, ny, dx, dx, courant=0.5, device=cuda)
    ant = [(int(rng.integers(0, nx)), int(rng.integers(0, ny))) for _ in range(n_ant)]
    delta = rng.standard_normal((n_ant, n_ant, steps)).astype(np.float32)
    eps = float(rng.uniform(1, 50))
    v = C0 / np.sqrt(eps)
    kw = dict(image_shape=(int(rng.integers(5, 70)), int(rng.integers(5, 70))),
              gate_start=int(rng.integers(0, steps // 2)), skip_self=bool(seed % 2))
    ref = oracle.das_backprojection_ref(delta, ant, nx, ny, dx, g.dt, steps, v, **kw)
    img = das_backprojection(delta, ant, g, steps, eps_eff=eps, **kw)
    assert np.array_equal(img, ref)
    ref = oracle.das_backprojection_ref(delta, ant, nx, ny, dx, g.dt, steps, v, pitch=dx)
    img = das_backprojection(torch.from_numpy(delta).to(cuda), ant, g, steps, v_medium=v, pitch=dx)
    assert np.array_equal(img, ref)
