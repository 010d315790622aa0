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


# ---- 3D painter (wf_paint3d) against MaterialMap3D.build3d -------------------

def _both3d(mm, cuda):
    ca, cb = mm.build3d()
    cad, cbd = mm.build3d_device(cuda)
    return (ca, cb), (cad.cpu(), cbd.cpu())


def test_device_painter_3d_random_primitives(cuda):
    """Spheres, boxes, ellipsoids and cylinders on all three axes, with
    centres on and between cells, overlapping in painter's order."""
    from waveforge_b200.core.materials import MaterialMap3D
    rng = np.random.default_rng(8)
    g = YeeGrid(37, 29, 1e-3, 1e-3, Nz=44, dz=1e-3, courant=0.5, device="cpu")
    mm = MaterialMap3D(g, default=Material("bg", 2.0, 0.01))
    for q in range(40):
        m = Material(f"m{q}", float(rng.uniform(1, 60)), float(rng.uniform(0, 1.5)))
        c = tuple(float(v) for v in rng.uniform(-3, 45, 3).round(1 if q % 2 else 0))
        kind = q % 6
        if kind == 0:
            mm.add_sphere(c, float(rng.uniform(1, 12)), m)
        elif kind == 1:
            lo = rng.uniform(-2, 30, 3).round(1)
            mm.add_box(tuple(lo), tuple(lo + rng.uniform(1, 15, 3).round(1)), m)
        elif kind == 2:
            mm.add_ellipsoid(c, tuple(rng.uniform(1.5, 14, 3)), m)
        else:
            mm.add_cylinder(c, "xyz"[kind - 3], float(rng.uniform(1, 9)),
                            float(rng.uniform(2, 30)), m)
    (ca, cb), (cad, cbd) = _both3d(mm, cuda)
    assert torch.equal(ca, cad) and torch.equal(cb, cbd)


def test_device_painter_3d_brain_phantom_golden(cuda):
    """The head phantom painted on the device gives the reference's Ca/Cb
    digests (golden brain_dataset40.npz)."""
    import hashlib
    from conftest import GOLDEN
    from waveforge_b200.datasets.brain import BrainPhantom3D, sample_random_geometry
    d = np.load(GOLDEN / "brain_dataset40.npz")
    g = YeeGrid(64, 64, 3e-3, 3e-3, Nz=64, dz=3e-3, device=cuda)
    ph = BrainPhantom3D(g, 1e9, geometry=sample_random_geometry(7, 64, 3.0), seed=9)
    ph.add_bleed_at((40, 30, 28), 4, "intracerebral", "subacute")
    ca, cb = ph.build_device(cuda)
    h = lambda t: hashlib.sha256(t.cpu().contiguous().numpy().tobytes()).hexdigest()
    assert h(ca) == str(d["phantom64_ca_sha"]) and h(cb) == str(d["phantom64_cb_sha"])


def test_device_painter_3d_rejects_custom_masks(cuda):
    from waveforge_b200.core.materials import MaterialMap3D
    g = YeeGrid(8, 8, 1e-3, 1e-3, Nz=8, dz=1e-3, device="cpu")
    mm = MaterialMap3D(g).add_custom3d(lambda I, J, K: I > 3, Material("x", 3.0, 0.0))
    assert not mm.device_paintable3d
    with pytest.raises(ValueError):
        mm.build3d_device(cuda)


def test_device_painter_3d_reports_bad_material_index(cuda):
    """A region whose material index is outside the table paints the default
    and sets the status word (no fault)."""
    import ctypes
    from waveforge_b200 import _native as nat
    lib = nat.load()
    regs = (nat.WfRegion3D * 1)()
    regs[0].kind, regs[0].material = 0, 5          # table holds 2 materials
    for t, v in enumerate((3.0, 3.0, 3.0, 4.0)):
        regs[0].p[t] = v
    host = torch.frombuffer(bytearray(bytes(memoryview(regs).cast("B"))), dtype=torch.uint8)
    dreg = host.to(cuda)
    tca = torch.tensor([0.5, 0.25], device=cuda)
    tcb = torch.tensor([1.0, 2.0], device=cuda)
    ca = torch.zeros((6, 6, 6), device=cuda)
    cb = torch.zeros_like(ca)
    st = torch.zeros(1, dtype=torch.int32, device=cuda)
    nat.check(lib.wf_paint3d(6, 6, 6, dreg.data_ptr(), 1, tca.data_ptr(), tcb.data_ptr(), 2,
                             ca.data_ptr(), cb.data_ptr(), st.data_ptr(), nat.stream_handle(cuda)))
    assert int(st.item()) == nat.WF_E_ARG
    assert torch.all(ca == 0.5) and torch.all(cb == 1.0)
