"""Device painter (wf_paint2d) against the host MaterialMap.build.

The host painter reproduces the reference's Ca/Cb bit for bit (pinned by the
golden digests); the device painter must give the same bits for the same
regions: the benchmark's lossy-ellipse maps, breast phantoms of every size,
and circle/rectangle/shell corner cases with parameters on cell boundaries.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from waveforge_b200 import workloads as W
from waveforge_b200.core.grid import YeeGrid
from waveforge_b200.core.materials import Material, MaterialMap

pytestmark = pytest.mark.gpu


def _both(mm, cuda):
    ca, cb = mm.build()
    nx, ny = ca.shape[0], ca.shape[1]
    eps = torch.empty((nx, ny), dtype=torch.float64, device=cuda)
    sig = torch.empty_like(eps)
    cad, cbd = mm.build_device(cuda, eps_sigma=(eps, sig))
    e_h, s_h = mm.build_eps_sigma()
    return (ca, cb, e_h, s_h), (cad.cpu(), cbd.cpu(), eps.cpu(), sig.cpu())


@pytest.mark.parametrize("n", [256, 1024])
def test_device_painter_lossy_ellipses(cuda, n):
    wl = W.LossyEllipses(n=n, steps=10)
    g = YeeGrid(n, n, wl.dx, wl.dx, courant=wl.courant, device="cpu")
    mm = MaterialMap(g, default=wl.background(Material))
    wl.paint(mm, Material)
    host, dev = _both(mm, cuda)
    for a, b in zip(host, dev):
        assert torch.equal(a.reshape(b.shape), b)


def test_device_painter_breast_phantoms(cuda):
    rng = np.random.default_rng(11)
    for side in W.BREAST_SIDES:
        ph = W.BreastPhantom.draw(rng, side)
        g = YeeGrid(side, side, 0.5e-3, 0.5e-3, courant=0.5, device="cpu")
        for tumor in (True, False):
            mm = MaterialMap(g, default=ph.background(Material))
            ph.paint(mm, Material, with_tumor=tumor)
            host, dev = _both(mm, cuda)
            for a, b in zip(host, dev):
                assert torch.equal(a.reshape(b.shape), b)


def test_device_painter_primitives_on_cell_boundaries(cuda):
    g = YeeGrid(37, 29, 1e-3, 1e-3, courant=0.5, device="cpu")
    mm = MaterialMap(g, default=Material("bg", 2.0, 0.0))
    mm.add_rectangle((3, 20), (0, 28), Material("slab", 4.0, 0.01))
    mm.add_circle((18.0, 14.0), 7.0, Material("disc", 9.0, 0.3))      # r*r = 49 hits cells exactly
    mm.add_ellipse((10.5, 9.25), (6.5, 3.0), Material("ell", 12.0, 0.5))
    mm.add_shell((25.0, 15.0), (10.0, 8.0), (7.0, 5.0), Material("shell", 30.0, 1.1))
    mm.add_circle((0.1, 0.1), 0.3, Material("speck", 50.0, 0.0))
    host, dev = _both(mm, cuda)
    for a, b in zip(host, dev):
        assert torch.equal(a.reshape(b.shape), b)
    labels = torch.unique(dev[0])
    assert labels.numel() >= 5


def test_device_painter_rejects_custom_masks(cuda):
    g = YeeGrid(16, 16, 1e-3, 1e-3, courant=0.5, device="cpu")
    mm = MaterialMap(g).add_custom(lambda I, J: I > J, Material("tri", 3.0, 0.0))
    with pytest.raises(ValueError):
        mm.build_device(cuda)
