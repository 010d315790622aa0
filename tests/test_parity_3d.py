"""3D parity of the CUDA path with the reference: bit-identical float32
traces and final fields (golden digests, pinned oracle), for several tile
shapes and temporal-block depths."""

from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from _cases import edge3d_sources, head_coeffs, load
from conftest import rel_l2, sha
from waveforge_b200 import (FDTD3D, Detectors, FieldSet, MurABC3D, PlaneSource, PointSource,
                            SourceCollection, TabulatedWaveform, YeeGrid)

pytestmark = pytest.mark.gpu

COMPS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
# None = default (streaming kernel for Nz > 1); tile_i == 0 = streaming with
# segments of tile_j planes; the rest select the tile kernel
TUNES3 = [None, (1, 4, 4, 4, 64), (2, 3, 5, 7, 96), (3, 6, 6, 10, 128), (1, 8, 8, 30, 256),
          (1, 0, 1, 0, 0), (1, 0, 3, 8, 2), (1, 0, 2, 16, 1), (1, 0, 0, 8, 1), (1, 0, 0, 16, 2)]


def sim3d(cuda, shape, dx, courant, srcs, ca=None, cb=None, steps=None, tune=None):
    nx, ny, nz = shape
    g = YeeGrid(nx, ny, dx, dx, Nz=nz, dz=dx, courant=courant, device=cuda)
    f = FieldSet(g)
    b = MurABC3D(g, f.Hx, f.Hy, f.Hz)
    objs = []
    for comp, box, wave in srcs:
        w = TabulatedWaveform(wave)
        i0, i1, j0, j1, k0, k1 = box
        if (i1 - i0, j1 - j0, k1 - k0) == (1, 1, 1):
            objs.append(PointSource(w, i0, j0, comp, k=k0, grid=g, N_steps=steps))
        else:
            if i1 - i0 == 1 and (j1 - j0, k1 - k0) == (ny, nz):
                objs.append(PlaneSource(w, "yz", i0, comp, grid=g, N_steps=steps))
            elif j1 - j0 == 1 and (i1 - i0, k1 - k0) == (nx, nz):
                objs.append(PlaneSource(w, "xz", j0, comp, grid=g, N_steps=steps))
            else:
                objs.append(PlaneSource(w, "xy", k0, comp, grid=g, N_steps=steps))
    sc = SourceCollection(objs) if objs else None
    return FDTD3D(g, f, b, sc, Ca=None if ca is None else ca.to(cuda),
                  Cb=None if cb is None else cb.to(cuda), n_check=10 ** 9, tune=tune), f


def test_head3d_bit_exact_vs_reference(cuda):
    g = load("head3d_32")
    ca, cb = head_coeffs(g)
    n, steps = int(g["n"]), int(g["steps"])
    i, j, k = (int(v) for v in g["src"])
    for tune in TUNES3:
        sim, f = sim3d(cuda, (n, n, n), float(g["dx"]), float(g["courant"]),
                       [("Ez", (i, i + 1, j, j + 1, k, k + 1), torch.from_numpy(g["wave"]))],
                       ca, cb, steps=steps, tune=tune)
        tr = sim.run(steps, record=Detectors([("Ez", *(int(v) for v in r)) for r in g["rx"]]))
        assert sha(tr) == str(g["sha_traces"]), tune
        for c in COMPS:
            assert sha(getattr(f, c)) == str(g[f"sha_{c.lower()}"]), (tune, c)
        assert rel_l2(tr.cpu().numpy(), g["traces64"]) < 1e-5


@pytest.mark.parametrize("name", ["box9x7x6", "flat8x6x1"])
def test_edge_cases_3d_bit_exact_vs_reference(cuda, name):
    d = load(f"edges3d_{name}")
    shape = tuple(int(v) for v in d["shape"])
    steps = int(d["steps"])
    probes = [(COMPS[c], i, j, k) for c, i, j, k in d["probes"]]
    for tune in TUNES3:
        sim, f = sim3d(cuda, shape, 1e-3, float(d["courant"]), edge3d_sources(d), steps=steps,
                       tune=tune)
        tr = sim.run(steps, record=Detectors(probes))
        for c in COMPS:
            assert np.array_equal(getattr(f, c).cpu().numpy(), d[c.lower() + "32"]), (tune, c)
        assert np.array_equal(tr.cpu().numpy(), d["traces32"]), tune


@pytest.mark.parametrize("seed", range(4))
def test_random_3d_bit_exact_vs_oracle(cuda, seed):
    rng = np.random.default_rng(300 + seed)
    shape = tuple(int(v) for v in rng.integers(4, 19, 3))
    steps = int(rng.integers(1, 30))
    nx, ny, nz = shape
    srcs = []
    for _ in range(int(rng.integers(1, 5))):
        c = COMPS[rng.integers(0, 6)]
        i, j, k = int(rng.integers(0, nx)), int(rng.integers(0, ny)), int(rng.integers(0, nz))
        srcs.append((c, (i, i + 1, j, j + 1, k, k + 1),
                     torch.from_numpy(rng.standard_normal(steps).astype(np.float32))))
    ca = cb = None
    if seed % 2:
        ca = torch.from_numpy(rng.uniform(0.3, 1.0, shape).astype(np.float32))
        cb = torch.from_numpy(rng.uniform(0.001, 0.1, shape).astype(np.float32))
    dt = oracle.stable_dt(1e-3, 1e-3, 1e-3, 0.9)
    o = oracle.Oracle3D(nx, ny, nz, 1e-3, 1e-3, 1e-3, dt, ca, cb)
    for c, box, w in srcs:
        o.add_box_source(c, box, w)
    probes = [(COMPS[rng.integers(0, 6)], int(rng.integers(0, nx)), int(rng.integers(0, ny)),
               int(rng.integers(0, nz))) for _ in range(6)]
    tr_o = o.run(steps, probes)
    for tune in TUNES3:
        sim, f = sim3d(cuda, shape, 1e-3, 0.9, srcs, ca, cb, steps=steps, tune=tune)
        tr = sim.run(steps, record=Detectors(probes))
        assert np.array_equal(tr.cpu().numpy(), tr_o.numpy()), tune
        for c in COMPS:
            assert np.array_equal(getattr(f, c).cpu().numpy(), getattr(o, c).numpy()), (tune, c)


@pytest.mark.parametrize("tma_shape", [True, False])
@pytest.mark.parametrize("mat", [False, True])
def test_streaming_kernel_equals_tile_kernel_multi_block(cuda, mat, tma_shape):
    """A volume spanning several 14 x 30 column blocks in j and k and several
    i-segments: the streaming kernel (automatic and forced segment lengths)
    equals the tile kernel bit for bit in traces, final fields and the
    stability maxima, with E and H sources inside and across block edges."""
    rng = np.random.default_rng(77 + mat)
    shape = (23, 37, 72) if tma_shape else (23, 37, 71)
    nx, ny, nz = shape
    steps = 17
    srcs = []
    for c, (i, j, k) in (("Ez", (11, 14, 30)), ("Hy", (5, 15, 31)), ("Ex", (0, 0, 0)),
                         ("Hx", (22, 36, nz - 1)), ("Ey", (12, 28, 59)), ("Ez", (20, 13, 29)),
                         ("Ex", (3, 27, 60)),
                         # E sources on the extra box row of the TMA blocks (15 core rows)
                         ("Ex", (7, 15, 20)), ("Ez", (9, 30, 44)), ("Ey", (13, 30, 2))):
        srcs.append((c, (i, i + 1, j, j + 1, k, k + 1),
                     torch.from_numpy(rng.standard_normal(steps).astype(np.float32))))
    ca = cb = None
    if mat:
        ca = torch.from_numpy(rng.uniform(0.3, 1.0, shape).astype(np.float32))
        cb = torch.from_numpy(rng.uniform(0.001, 0.1, shape).astype(np.float32))
    probes = [(COMPS[q % 6], int(rng.integers(0, nx)), int(rng.integers(0, ny)),
               int(rng.integers(0, nz))) for q in range(24)]
    probes += [("Hx", 0, 14, 30), ("Hz", 22, 0, 0), ("Ey", 11, 15, 29), ("Hy", 3, 36, nz - 1)]
    outs = []
    for tune in ((1, 8, 8, 30, 256), None, (1, 0, 2, 0, 0), (1, 0, 7, 8, 2), (1, 0, 5, 16, 1),
                 (1, 0, 0, 8, 1), (1, 0, 0, 16, 2), (1, 0, 1, 0, 0)):
        sim, f = sim3d(cuda, shape, 1e-3, 0.9, srcs, ca, cb, steps=steps, tune=tune)
        sim._n_check = 4
        tr = sim.run(steps, record=Detectors(probes))
        outs.append((tr.cpu(), [getattr(f, c).cpu() for c in COMPS], sim.last_field_max,
                     sim.n_stability_checks))
    ref = outs[0]
    assert float(ref[0].abs().max()) > 0
    for o in outs[1:]:
        assert torch.equal(o[0], ref[0])
        for a, b in zip(o[1], ref[1]):
            assert torch.equal(a, b)
        assert o[2] == ref[2] and o[3] == ref[3]


def test_batched_instances_equal_separate_runs(cuda):
    """A batched FieldSet (B, Nx, Ny, Nz) with per-member Ca/Cb runs in one
    launch per step and equals B separate runs bit for bit (traces, fields,
    stability maxima); sources reach every member, as the reference's
    broadcast injection does."""
    from waveforge_b200 import FieldSet as FS
    rng = np.random.default_rng(909)
    B, shape, steps = 3, (19, 33, 40), 12
    nx, ny, nz = shape
    ca = torch.from_numpy(rng.uniform(0.3, 1.0, (B,) + shape).astype(np.float32))
    cb = torch.from_numpy(rng.uniform(0.001, 0.1, (B,) + shape).astype(np.float32))
    wave = torch.from_numpy(rng.standard_normal(steps).astype(np.float32))
    probes = [("Ez", 9, 16, 20), ("Hx", 0, 5, 39), ("Hy", 18, 32, 0), ("Ex", 4, 30, 31)]
    g = YeeGrid(nx, ny, 1e-3, 1e-3, Nz=nz, dz=1e-3, courant=0.9, device=cuda)
    f = FS(g, batch_size=B)
    src = SourceCollection([PointSource(TabulatedWaveform(wave), 9, 16, "Ez", k=20, grid=g,
                                        N_steps=steps)])
    sim = FDTD3D(g, f, MurABC3D(g, f.Hx, f.Hy, f.Hz), src, Ca=ca.to(cuda), Cb=cb.to(cuda),
                 n_check=5)
    tr = sim.run(steps, record=Detectors(probes)).cpu()
    assert tr.shape == (B, len(probes), steps)
    maxima = []
    for b in range(B):
        s1, f1 = sim3d(cuda, shape, 1e-3, 0.9, [("Ez", (9, 10, 16, 17, 20, 21), wave)], ca[b],
                       cb[b], steps=steps)
        s1._n_check = 5
        t1 = s1.run(steps, record=Detectors(probes)).cpu()
        assert torch.equal(t1, tr[b])
        for c in COMPS:
            assert torch.equal(getattr(f1, c).cpu(), getattr(f, c)[b].cpu()), (b, c)
        maxima.append(s1.last_field_max)
    assert sim.last_field_max == max(maxima)
    assert float(tr.abs().max()) > 0


@pytest.mark.parametrize("nz", [40, 39])
def test_member_sources_equal_separate_runs(cuda, nz):
    """FDTD3D(member_sources=...): each batch member injects its own sources
    (here a different transmitter and waveform per member) and equals the
    separate single run bit for bit -- on the TMA pass (Nz % 4 == 0) and on
    the register streaming kernel it falls back to otherwise."""
    from waveforge_b200 import FieldSet as FS
    rng = np.random.default_rng(31 + nz)
    B, steps = 4, 14
    shape = (21, 30, nz)
    ca = torch.from_numpy(rng.uniform(0.3, 1.0, shape).astype(np.float32))
    cb = torch.from_numpy(rng.uniform(0.001, 0.1, shape).astype(np.float32))
    waves = [torch.from_numpy(rng.standard_normal(steps).astype(np.float32)) for _ in range(B)]
    pos = [(5, 7, 9), (15, 20, 30), (10, 3, 2), (19, 28, nz - 2)]
    probes = [("Ez", 10, 15, 20), ("Hy", 3, 28, 1), ("Ex", 20, 1, nz - 1)]
    g = YeeGrid(*shape[:2], 1e-3, 1e-3, Nz=nz, dz=1e-3, courant=0.9, device=cuda)
    f = FS(g, batch_size=B)
    members = [SourceCollection([PointSource(TabulatedWaveform(waves[b]), *pos[b][:2], "Ez",
                                             k=pos[b][2], grid=g, N_steps=steps)]) for b in range(B)]
    sim = FDTD3D(g, f, MurABC3D(g, f.Hx, f.Hy, f.Hz), Ca=ca.to(cuda), Cb=cb.to(cuda),
                 member_sources=members)
    tr = sim.run(steps, record=Detectors(probes)).cpu()
    for b in range(B):
        i, j, k = pos[b]
        s1, f1 = sim3d(cuda, shape, 1e-3, 0.9, [("Ez", (i, i + 1, j, j + 1, k, k + 1), waves[b])],
                       ca, cb, steps=steps)
        assert torch.equal(s1.run(steps, record=Detectors(probes)).cpu(), tr[b]), b
        for c in COMPS:
            assert torch.equal(getattr(f1, c).cpu(), getattr(f, c)[b].cpu()), (b, c)


def test_member_sources_validation(cuda):
    from waveforge_b200 import FieldSet as FS, LineSource
    g = YeeGrid(12, 12, 1e-3, 1e-3, Nz=12, dz=1e-3, courant=0.9, device=cuda)
    w = TabulatedWaveform(torch.ones(4))
    one = SourceCollection([PointSource(w, 3, 3, "Ez", k=3, grid=g, N_steps=4)])
    two = SourceCollection([PointSource(w, 3, 3, "Ez", k=3, grid=g, N_steps=4),
                            PointSource(w, 5, 5, "Ez", k=5, grid=g, N_steps=4)])
    f = FS(g, batch_size=2)
    b = MurABC3D(g, f.Hx, f.Hy, f.Hz)
    with pytest.raises(ValueError):
        FDTD3D(g, FS(g), MurABC3D(g, f.Hx, f.Hy, f.Hz), member_sources=[one])  # not batched
    with pytest.raises(ValueError):
        FDTD3D(g, f, b, member_sources=[one])                                  # wrong count
    with pytest.raises(ValueError):
        FDTD3D(g, f, b, one, member_sources=[one, one])                        # both kinds
    sim = FDTD3D(g, f, b, member_sources=[one, two])                           # box counts differ
    with pytest.raises(ValueError):
        sim.run(2)


@pytest.mark.parametrize("shape", [(40, 48, 64), (50, 33, 68), (34, 4, 8), (21, 5, 12),
                                   (17, 21, 4)])
def test_tma_pass_paths_bit_exact_vs_oracle(cuda, shape):
    """Shapes that reach every path of the TMA pass: column blocks off every
    face (straight-line interior planes; (40, 48, 64) and (50, 33, 68) have
    them), blocks on j / k faces (in-place face corrections, down to the
    smallest ny and nz the engine takes), x-face planes (final-H copy),
    several i-segments (segments of 16 and of 5
    planes besides the automatic length), sources and probes inside an
    interior block and on faces (the list path), and stability checks every
    3 steps (the list path on every block)."""
    nx, ny, nz = shape
    rng = np.random.default_rng(nx * 10000 + ny * 100 + nz)
    steps = 14
    ca = torch.from_numpy(rng.uniform(0.3, 1.0, shape).astype(np.float32))
    cb = torch.from_numpy(rng.uniform(0.001, 0.1, shape).astype(np.float32))
    pts = [(nx // 2, ny // 2, nz // 2), (nx // 2, min(20, ny - 1), min(40, nz - 1)),
           (0, ny - 1, 0), (nx - 1, 0, nz - 1), (1, 1, nz - 2)]
    srcs = [(COMPS[q % 6], (i, i + 1, j, j + 1, k, k + 1),
             torch.from_numpy(rng.standard_normal(steps).astype(np.float32)))
            for q, (i, j, k) in enumerate(pts)]
    init = {c: rng.standard_normal(shape).astype(np.float32) * (1.0 if c[0] == "E" else 2.7e-3)
            for c in COMPS}
    dt = oracle.stable_dt(1e-3, 1e-3, 1e-3, 0.9)
    o = oracle.Oracle3D(nx, ny, nz, 1e-3, 1e-3, 1e-3, dt, ca, cb)
    for c, v in init.items():
        getattr(o, c).copy_(torch.from_numpy(v))
    for c, box, w in srcs:
        o.add_box_source(c, box, w)
    probes = [(COMPS[q % 6], min(nx - 1, int(a)), min(ny - 1, int(b)), min(nz - 1, int(d)))
              for q, (a, b, d) in enumerate(pts + [(nx // 3, ny - 2, 1), (nx - 2, 2, nz // 3)])]
    tr_o = o.run(steps, probes)
    for tune in (None, (1, 0, 16, 0, 0), (1, 0, 5, 0, 0)):
        g = YeeGrid(nx, ny, 1e-3, 1e-3, Nz=nz, dz=1e-3, courant=0.9, device=cuda)
        f = FieldSet(g)
        for c, v in init.items():
            getattr(f, c).copy_(torch.from_numpy(v))
        sc = SourceCollection([PointSource(TabulatedWaveform(w), box[0], box[2], c, k=box[4], grid=g,
                                           N_steps=steps) for c, box, w in srcs])
        sim = FDTD3D(g, f, MurABC3D(g, f.Hx, f.Hy, f.Hz), sc, Ca=ca.to(cuda), Cb=cb.to(cuda),
                     n_check=3, tune=tune)
        tr = sim.run(steps, record=Detectors(probes))
        assert np.array_equal(tr.cpu().numpy(), tr_o.numpy()), tune
        for c in COMPS:
            assert np.array_equal(getattr(f, c).cpu().numpy(), getattr(o, c).numpy()), (tune, c)
        assert sim.n_stability_checks == steps // 3
