"""Generate the golden vectors of the parity tests by running the REFERENCE.

Run in a container that holds the read-only reference checkout:
    python tests/golden/make_golden.py --ref /root/reference [--only case,...]

It imports the reference's own ``core`` package and example DAS functions
(pure Python + PyTorch, CPU), runs each case in float32 and float64, and
writes ``tests/golden/<case>.npz`` with:
  * the exact inputs the product needs to rebuild the case (waveform table,
    source / receiver positions, grid constants),
  * SHA-256 digests of the float32 outputs (traces, final fields, Ca/Cb),
    so tests can demand bit-identical results,
  * decimated float32 and float64 samples of the same outputs for
    relative-L2 error statements.
Nothing on the GPU box reads the reference; only these fixtures travel.
"""

from __future__ import annotations

import argparse
import hashlib
import importlib.util
import math
import sys
import warnings
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from waveforge_b200 import workloads as W  # noqa: E402  (recipes only; no compute)

warnings.filterwarnings("ignore", category=UserWarning)


def sha(t) -> str:
    a = t.detach().cpu().contiguous().numpy() if torch.is_tensor(t) else np.ascontiguousarray(t)
    return hashlib.sha256(a.tobytes()).hexdigest()


def load_ref(ref: Path):
    sys.path.insert(0, str(ref / "src"))
    import core  # noqa: F401  the reference package
    from core import grid, fields, materials, sources, boundaries, fdtd2d, fdtd3d
    return dict(grid=grid, fields=fields, materials=materials, sources=sources,
                boundaries=boundaries, fdtd2d=fdtd2d, fdtd3d=fdtd3d)


def load_example(ref: Path, rel: str, name: str):
    spec = importlib.util.spec_from_file_location(name, ref / "examples" / rel)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def gauss_deriv_class(R):
    Waveform = R["sources"].Waveform

    class GaussDeriv(Waveform):
        """Benchmark pulse on the reference Waveform base (same expression as
        waveforge_b200.core.sources.GaussianDerivativePulse)."""

        def __init__(self, fc=1e9, amplitude=1.0):
            self.fc, self.A = fc, amplitude
            self.tau = 1.0 / (2.0 * math.pi * fc)
            self.t0 = 3.0 * self.tau

        def _compute(self, t):
            u = (t - self.t0) / self.tau
            return self.A * (-u) * torch.exp(-0.5 * (u * u))

        peak_time = property(lambda s: s.t0 - s.tau)
        bandwidth = property(lambda s: s.fc)
        amplitude = property(lambda s: s.A)

    return GaussDeriv


def run_2d(R, nx, ny, dx, courant, steps, dtype, paint=None, default=None, sources=(), probes=(),
           n_check=10 ** 9, init=None):
    """sources: (comp, kind, args, wave_tensor) ; probes: (comp, i, j);
    init: {component: float32 (nx, ny) array} of starting values."""
    grid = R["grid"].YeeGrid(nx, ny, dx, dx, courant=courant, device="cpu", dtype=dtype)
    f = R["fields"].FieldSet(grid)
    for c, v in (init or {}).items():
        getattr(f, c).copy_(torch.from_numpy(v).to(dtype).reshape(getattr(f, c).shape))
    b = R["boundaries"].MurABC(grid, f.Hz)
    Ca = Cb = None
    if paint is not None:
        mm = R["materials"].MaterialMap(grid, default=default)
        paint(mm, R["materials"].Material)
        Ca, Cb = mm.build()
    TW = tab_class(R)
    srcs = []
    for comp, kind, args, wave in sources:
        w = TW(wave)
        if kind == "point":
            srcs.append(R["sources"].PointSource(w, *args, comp, grid=grid, N_steps=steps))
        elif kind == "line":
            axis, pos, start, stop, amp = args
            srcs.append(R["sources"].LineSource(w, axis, pos, start, stop, comp, grid=grid,
                                                N_steps=steps, amplitude_profile=amp))
    sc = R["sources"].SourceCollection(srcs) if srcs else None
    sim = R["fdtd2d"].FDTD2D(grid, f, b, sc, Ca=Ca, Cb=Cb, n_check=n_check)
    tr = torch.zeros(len(probes), steps, dtype=dtype)
    for s in range(steps):
        sim.step()
        for r, (comp, i, j) in enumerate(probes):
            tr[r, s] = getattr(f, comp)[i, j, 0]
    return grid, f, tr, Ca, Cb


def tab_class(R):
    Waveform = R["sources"].Waveform

    class Tab(Waveform):
        def __init__(self, table):
            self.table = table

        def build(self, N_steps, dt, device, dtype=torch.float32):
            return self.table[:N_steps].to(dtype).to(device)

        def _compute(self, t):
            raise NotImplementedError

        peak_time = property(lambda s: -1.0)
        bandwidth = property(lambda s: 0.0)
        amplitude = property(lambda s: 1.0)

    return Tab


def dec(a, k):
    return np.ascontiguousarray(np.asarray(a)[..., ::k])


def case_vacuum_point(R, out):
    """256^2 vacuum, Hz point source at (128,128), 4 receivers at 60 cells, 1000 steps."""
    GD = gauss_deriv_class(R)
    n, steps = 256, 1000
    rx = [("Hz", 188, 128), ("Hz", 128, 188), ("Hz", 68, 128), ("Hz", 128, 68)]
    res = {}
    for dt_name, dtype in (("32", torch.float32), ("64", torch.float64)):
        grid = R["grid"].YeeGrid(n, n, 1e-3, 1e-3, courant=0.5, device="cpu", dtype=dtype)
        wave = GD().build(steps, grid.dt, torch.device("cpu"), dtype)
        if dtype == torch.float32:
            wave32 = wave.clone()
        g, f, tr, _, _ = run_2d(R, n, n, 1e-3, 0.5, steps, dtype,
                                sources=[("Hz", "point", (128, 128), wave)], probes=rx)
        res[dt_name] = (g, f, tr)
    g32, f32, tr32 = res["32"]
    _, f64, tr64 = res["64"]
    np.savez_compressed(
        out / "vacuum_point_256.npz", n=n, steps=steps, dx=1e-3, courant=0.5, dt=g32.dt,
        src=np.array([128, 128]), rx=np.array([r[1:] for r in rx]), wave=wave32.numpy(),
        traces32=tr32.numpy(), traces64=tr64.numpy(),
        sha_traces=sha(tr32), sha_ex=sha(f32.Ex), sha_ey=sha(f32.Ey), sha_hz=sha(f32.Hz),
        hz32=f32.Hz[..., 0].numpy(), hz64_dec=dec(f64.Hz[::2, :, 0].numpy(), 2))


def case_lossy_ellipses(R, out, n=256, steps=600):
    wl = W.LossyEllipses(n=n, steps=steps)
    GD = gauss_deriv_class(R)
    M = R["materials"].Material
    rx = [("Hz", i, j) for i, j in wl.receivers]
    res = {}
    for dt_name, dtype in (("32", torch.float32), ("64", torch.float64)):
        grid = R["grid"].YeeGrid(n, n, wl.dx, wl.dx, courant=wl.courant, device="cpu", dtype=dtype)
        wave = GD().build(steps, grid.dt, torch.device("cpu"), dtype)
        if dtype == torch.float32:
            wave32 = wave.clone()
        res[dt_name] = run_2d(R, n, n, wl.dx, wl.courant, steps, dtype, paint=wl.paint,
                              default=wl.background(M),
                              sources=[("Hz", "point", wl.source, wave)], probes=rx)
    g32, f32, tr32, ca, cb = res["32"]
    _, f64, tr64, _, _ = res["64"]
    np.savez_compressed(
        out / f"lossy_ellipses_{n}.npz", n=n, steps=steps, dx=wl.dx, courant=wl.courant,
        dt=g32.dt, seed=wl.seed, src=np.array(wl.source), rx=np.array([r[1:] for r in rx]),
        wave=wave32.numpy(), sha_ca=sha(ca), sha_cb=sha(cb), traces32=tr32.numpy(),
        traces64=tr64.numpy(), sha_traces=sha(tr32), sha_ex=sha(f32.Ex), sha_ey=sha(f32.Ey),
        sha_hz=sha(f32.Hz), hz32_dec=dec(f32.Hz[::4, :, 0].numpy(), 4),
        hz64_dec=dec(f64.Hz[::4, :, 0].numpy(), 4))


def case_breast_mimo(R, out, sides=(150, 200), n_tx=2, steps=1500, name="breast_mimo_small"):
    """Breast phantoms of the given sides (drawn in order from the workload's
    seed), first n_tx transmitters each, 16 receivers."""
    wl = W.BreastMIMO(n_phantoms=len(sides), steps=steps)
    rng = np.random.default_rng(wl.seed)
    phantoms = [W.BreastPhantom.draw(rng, side=s) for s in sides]
    GD = gauss_deriv_class(R)
    M = R["materials"].Material
    data = dict(steps=steps, dx=wl.dx, courant=wl.courant, seed=wl.seed, sides=np.array(sides),
                n_tx=n_tx)
    for p_idx, ph in enumerate(phantoms):
        ant = ph.antennas(16)
        rx = [("Hz", i, j) for i, j in ant]
        data[f"p{p_idx}_geom"] = np.array([ph.side, ph.A, ph.B, *ph.tumor_center, ph.tumor_r])
        data[f"p{p_idx}_ant"] = np.array(ant)
        for tx in range(n_tx):
            res = {}
            for dt_name, dtype in (("32", torch.float32), ("64", torch.float64)):
                grid = R["grid"].YeeGrid(ph.side, ph.side, wl.dx, wl.dx, courant=wl.courant,
                                         device="cpu", dtype=dtype)
                wave = GD().build(steps, grid.dt, torch.device("cpu"), dtype)
                if dtype == torch.float32:
                    data["wave"] = wave.numpy()
                    data["dt"] = grid.dt
                res[dt_name] = run_2d(R, ph.side, ph.side, wl.dx, wl.courant, steps, dtype,
                                      paint=lambda mm, Mat, ph=ph: ph.paint(mm, Mat),
                                      default=ph.background(M),
                                      sources=[("Hz", "point", ant[tx], wave)], probes=rx)
            _, f32, tr32, ca, cb = res["32"]
            _, f64, tr64, _, _ = res["64"]
            key = f"p{p_idx}_tx{tx}"
            data[key + "_sha_traces"] = sha(tr32)
            data[key + "_sha_hz"] = sha(f32.Hz)
            data[key + "_traces32_dec"] = dec(tr32.numpy(), 5)
            data[key + "_traces64_dec"] = dec(tr64.numpy(), 5)
            data[f"p{p_idx}_sha_ca"] = sha(ca)
            data[f"p{p_idx}_sha_cb"] = sha(cb)
    np.savez_compressed(out / f"{name}.npz", **data)


def case_edges_2d(R, out):
    """Tiny grids exercising edge semantics: sources on edges/corners, E
    sources, overlapping sources, a weighted line source, odd sizes."""
    rng = np.random.default_rng(11)
    cases = {}
    specs = [
        ("tiny7x5", 7, 5, 60, None,
         [("Hz", "point", (0, 0)), ("Hz", "point", (1, 1)), ("Ex", "point", (3, 0)),
          ("Ey", "point", (0, 2)), ("Hz", "line", ("x", 4, 0, 7, True)),
          ("Hz", "point", (6, 4)), ("Hz", "point", (6, 4)), ("Hz", "point", (1, 3))]),
        ("odd33x17", 33, 17, 150, "circles",
         [("Hz", "point", (1, 8)), ("Hz", "point", (32, 16)), ("Ey", "line", ("y", 20, 2, 15, False))]),
        ("min4x4", 4, 4, 40, None, [("Hz", "point", (1, 2)), ("Ex", "point", (2, 1))]),
    ]
    for name, nx, ny, steps, mat, srcs in specs:
        waves = [torch.from_numpy(rng.standard_normal(steps).astype(np.float32)) for _ in srcs]
        amps = {}
        full = []
        for q, ((comp, kind, args), w) in enumerate(zip(srcs, waves)):
            if kind == "line":
                axis, pos, start, stop, weighted = args
                amp = (torch.from_numpy(rng.uniform(0.5, 2.0, stop - start).astype(np.float32))
                       if weighted else None)
                amps[q] = amp
                full.append((comp, "line", (axis, pos, start, stop, amp), w))
            else:
                full.append((comp, "point", args, w))
        probes = [(c, i, j) for c in ("Ex", "Ey", "Hz") for i in range(nx) for j in range(ny)
                  if (i in (0, 1, nx - 2, nx - 1) or j in (0, 1, ny - 2, ny - 1))][:200]
        paint = None
        default = None
        if mat == "circles":
            M = R["materials"].Material
            default = M("bg", 4.0, 0.1)
            circ = [(float(a), float(b), float(c), float(e), float(s)) for a, b, c, e, s in
                    zip(rng.uniform(0, nx, 4), rng.uniform(0, ny, 4), rng.uniform(2, 8, 4),
                        rng.uniform(1, 50, 4), rng.uniform(0, 2, 4))]

            def paint(mm, Mat, circ=circ):
                for q, (ci, cj, r, e, s) in enumerate(circ):
                    mm.add_circle((ci, cj), r, Mat(f"c{q}", e, s))
        for dt_name, dtype in (("32", torch.float32), ("64", torch.float64)):
            ws = [(c, k, a if k == "point" else (a[0], a[1], a[2], a[3], None if a[4] is None
                   else a[4].to(dtype)), w.to(dtype)) for c, k, a, w in full]
            g, f, tr, ca, cb = run_2d(R, nx, ny, 1e-3, 0.7, steps, dtype, paint=paint,
                                      default=default, sources=ws, probes=probes)
            if dtype == torch.float32:
                d = dict(nx=nx, ny=ny, steps=steps, dx=1e-3, courant=0.7, dt=g.dt,
                         ex32=f.Ex[..., 0].numpy(), ey32=f.Ey[..., 0].numpy(),
                         hz32=f.Hz[..., 0].numpy(), traces32=tr.numpy(),
                         probes=np.array([(("Ex", "Ey", "Hz").index(c), i, j) for c, i, j in probes]))
                if ca is not None:
                    d["ca"] = ca[..., 0].numpy()
                    d["cb"] = cb[..., 0].numpy()
                for q, ((comp, kind, args), w) in enumerate(zip(srcs, waves)):
                    d[f"src{q}_comp"] = comp
                    d[f"src{q}_kind"] = kind
                    d[f"src{q}_args"] = np.array([v for v in (args if kind == "point" else args[1:4])])
                    if kind == "line":
                        d[f"src{q}_axis"] = args[0]
                        if amps.get(q) is not None:
                            d[f"src{q}_amp"] = amps[q].numpy()
                    d[f"src{q}_wave"] = w.numpy()
                d["nsrc"] = len(srcs)
            else:
                d["hz64"] = f.Hz[..., 0].numpy()
        cases[name] = d
    for name, d in cases.items():
        np.savez_compressed(out / f"edges2d_{name}.npz", **d)


def run_3d(R, shape, dx, courant, steps, dtype, paint=None, default=None, sources=(), probes=(),
           init=None, batch=1):
    """probes: (comp, i, j, k), recorded for every batch member (rows
    member-major when batch > 1); init: {component: float32 array of the
    field shape, (batch, nx, ny, nz) when batched}."""
    nx, ny, nz = shape
    grid = R["grid"].YeeGrid(nx, ny, dx, dx, Nz=nz, dz=dx, courant=courant, device="cpu", dtype=dtype)
    f = R["fields"].FieldSet(grid, batch_size=batch)
    for c, v in (init or {}).items():
        getattr(f, c).copy_(torch.from_numpy(v).to(dtype).reshape(getattr(f, c).shape))
    b = R["boundaries"].MurABC3D(grid, f.Hx, f.Hy, f.Hz)
    Ca = Cb = None
    if paint is not None:
        mm = R["materials"].MaterialMap3D(grid, default=default)
        paint(mm, R["materials"].Material)
        Ca, Cb = mm.build3d()
    TW = tab_class(R)
    srcs = []
    for comp, kind, args, wave in sources:
        w = TW(wave)
        if kind == "point":
            i, j, k = args
            srcs.append(R["sources"].PointSource(w, i, j, comp, k=k, grid=grid, N_steps=steps))
        elif kind == "plane":
            plane, pos = args
            srcs.append(R["sources"].PlaneSource(w, plane, pos, comp, grid=grid, N_steps=steps))
    sc = R["sources"].SourceCollection(srcs) if srcs else None
    sim = R["fdtd3d"].FDTD3D(grid, f, b, sc, Ca=Ca, Cb=Cb, n_check=10 ** 9)
    if batch == 1:
        tr = torch.zeros(len(probes), steps, dtype=dtype)
    else:
        tr = torch.zeros(batch, len(probes), steps, dtype=dtype)
    with torch.no_grad():
        for s in range(steps):
            sim.step()
            for r, (comp, i, j, k) in enumerate(probes):
                tr[..., r, s] = getattr(f, comp)[..., i, j, k]
    return grid, f, tr, Ca, Cb


def case_head3d(R, out, n=32, steps=200):
    wl = W.Head3D(n=n, steps=steps)
    GD = gauss_deriv_class(R)
    M = R["materials"].Material
    rx = [("Ez", *p) for p in wl.receivers()]
    res = {}
    for dt_name, dtype in (("32", torch.float32), ("64", torch.float64)):
        dxx = wl.dx
        stable = R["grid"].compute_stable_dt(dxx, dxx, dxx, wl.courant)
        wave = GD().build(steps, stable, torch.device("cpu"), dtype)
        if dtype == torch.float32:
            wave32 = wave.clone()
        res[dt_name] = run_3d(R, (n, n, n), dxx, wl.courant, steps, dtype, paint=wl.paint,
                              default=wl.background(M),
                              sources=[("Ez", "point", wl.source, wave)], probes=rx)
    g, f32, tr32, ca, cb = res["32"]
    _, f64, tr64, _, _ = res["64"]
    np.savez_compressed(
        out / f"head3d_{n}.npz", n=n, steps=steps, dx=wl.dx, courant=wl.courant, dt=g.dt,
        seed=wl.seed, src=np.array(wl.source), rx=np.array([r[1:] for r in rx]),
        wave=wave32.numpy(), sha_ca=sha(ca), sha_cb=sha(cb), traces32=tr32.numpy(),
        traces64=tr64.numpy(), sha_traces=sha(tr32),
        **{f"sha_{c.lower()}": sha(getattr(f32, c)) for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")})


def case_edges_3d(R, out):
    rng = np.random.default_rng(12)
    specs = [
        ("box9x7x6", (9, 7, 6), 40, [("Hx", "point", (0, 3, 2)), ("Hy", "point", (4, 0, 5)),
                                     ("Ez", "point", (4, 3, 0)), ("Hz", "point", (8, 6, 3)),
                                     ("Ex", "plane", ("yz", 2)), ("Hz", "point", (1, 1, 1))]),
        ("flat8x6x1", (8, 6, 1), 50, [("Hz", "point", (3, 2, 0)), ("Ez", "point", (5, 4, 0))]),
    ]
    for name, shape, steps, srcs in specs:
        waves = [torch.from_numpy(rng.standard_normal(steps).astype(np.float32)) for _ in srcs]
        nx, ny, nz = shape
        probes = [(c, i, j, k) for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
                  for i, j, k in [(0, 0, 0), (nx - 1, ny - 1, nz - 1), (1, 2, min(1, nz - 1)),
                                  (nx // 2, ny // 2, nz // 2)]]
        d = {}
        for dt_name, dtype in (("32", torch.float32), ("64", torch.float64)):
            ws = [(c, k, a, w.to(dtype)) for (c, k, a), w in zip(srcs, waves)]
            g, f, tr, _, _ = run_3d(R, shape, 1e-3, 0.5, steps, dtype, sources=ws, probes=probes)
            if dtype == torch.float32:
                d.update(shape=np.array(shape), steps=steps, dx=1e-3, courant=0.5, dt=g.dt,
                         traces32=tr.numpy(), nsrc=len(srcs),
                         probes=np.array([(("Ex", "Ey", "Ez", "Hx", "Hy", "Hz").index(c), i, j, k)
                                          for c, i, j, k in probes]))
                for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
                    d[c.lower() + "32"] = getattr(f, c).numpy()
                for q, ((comp, kind, args), w) in enumerate(zip(srcs, waves)):
                    d[f"src{q}_comp"] = comp
                    d[f"src{q}_kind"] = kind
                    d[f"src{q}_args"] = np.array(args if kind == "point" else [("xy", "xz", "yz").index(args[0]), args[1]])
                    d[f"src{q}_wave"] = w.numpy()
            else:
                d["hz64"] = f.Hz.numpy()
        np.savez_compressed(out / f"edges3d_{name}.npz", **d)


def case_das(R, ref: Path, out):
    """DAS on a 96^2 breast-like phantom, 8 antennas, healthy vs tumour."""
    bm = load_example(ref, "brain_mimo_imaging.py", "ref_brain_mimo")
    bc = load_example(ref, "09_brain_clot_dataset_sample.py", "ref_brain_clot")
    GD = gauss_deriv_class(R)
    M = R["materials"].Material
    side, steps = 96, 600
    rng = np.random.default_rng(21)
    ph = W.BreastPhantom.draw(rng, side=side)
    ph = W.BreastPhantom(side, ph.A, ph.B, ph.tumor_center, max(6.0, ph.tumor_r / 2), ph.skin)
    ant = ph.antennas(8)
    grid = R["grid"].YeeGrid(side, side, 0.5e-3, 0.5e-3, courant=0.5, device="cpu")
    wave = GD().build(steps, grid.dt, torch.device("cpu"), torch.float32)
    S = {}
    for tumor in (False, True):
        sig = np.zeros((8, 8, steps), np.float32)
        for tx in range(8):
            _, _, tr, _, _ = run_2d(R, side, side, 0.5e-3, 0.5, steps, torch.float32,
                                    paint=lambda mm, Mat, t=tumor: ph.paint(mm, Mat, with_tumor=t),
                                    default=ph.background(M),
                                    sources=[("Hz", "point", ant[tx], wave)],
                                    probes=[("Hz", i, j) for i, j in ant])
            sig[tx] = tr.numpy()
        S[tumor] = sig
    delta = S[True] - S[False]
    img_c = bm.das_backprojection(delta, ant, grid, steps, image_shape=(48, 40))
    img_f = bm.das_backprojection(delta, ant, grid, steps)
    img_g = bc.das_backprojection(delta, ant, grid, steps)
    np.savez_compressed(out / "das_breast96.npz", delta=delta, ant=np.array(ant), side=side,
                        steps=steps, dx=0.5e-3, dt=grid.dt, img_canonical_48x40=img_c,
                        img_full=img_f, img_gated=img_g, gate_start=max(0, int(0.9e-9 / grid.dt)),
                        tumor=np.array([*ph.tumor_center, ph.tumor_r]))


def case_antenna(R, ref: Path, out):
    """AntennaRing.compute_das_image (src/datasets/brain/antenna.py:262-341) on the
    breast DAS signals: free-space and layered (ray-circle chord) delays, even and
    odd trace lengths; the scipy Hilbert envelope is stored for the bit-exact DAS
    stage."""
    from scipy.signal import hilbert
    from datasets.brain.antenna import AntennaRing
    d = np.load(out / "das_breast96.npz")
    delta = d["delta"]
    side = int(d["side"])
    grid = R["grid"].YeeGrid(side, side, 0.5e-3, 0.5e-3, courant=0.5, device="cpu")
    GD = gauss_deriv_class(R)
    res = {}
    for n_steps in (600, 599):
        sig = np.ascontiguousarray(delta[:, :, :n_steps])
        ring = AntennaRing(8, 40, 0, grid)
        ring.build_sources(GD(), 0, N_steps=n_steps)
        head = {"cx_cells": 48, "cy_cells": 47, "layers": [(41, 10.0), (33, 5.0), (14, 40.0)]}
        res[f"img_free_{n_steps}"] = ring.compute_das_image(sig, image_size=40)
        res[f"img_head_{n_steps}"] = ring.compute_das_image(sig, image_size=33, head_geometry=head)
        res[f"env_{n_steps}"] = np.abs(hilbert(sig, axis=-1)).astype(np.float32)
    res["positions"] = np.array(ring.positions)
    np.savez_compressed(out / "antenna_ring96.npz", dt=grid.dt, dx=grid.dx, side=side,
                        head_cx=48, head_cy=47, head_layers=np.array([[41, 10.0], [33, 5.0], [14, 40.0]]),
                        **res)


def case_brain_dataset(R, ref: Path, out):
    """The brain dataset path (src/datasets): Cole-Cole tissue values, seeded
    head geometries, seeded bleed placement, a phantom's Ca/Cb digests, and
    whole generator samples (both MIMO acquisitions, scattered signals, DAS
    image, metadata, saved .npz key set) at 40^3 / 6 mm / 4 antennas."""
    import tempfile
    from datasets.brain import tissue_library as TL
    from datasets.brain.phantom import BrainPhantom3D, sample_random_geometry
    from datasets.generator import BrainDatasetGenerator
    res = {}
    names = sorted(TL.TISSUES) + [f"blood_{a}" for a in ("acute", "subacute", "chronic")]
    res["tissue_names"] = np.array(names)
    for f in (0.5e9, 1e9, 2e9, 6.5e9):
        t = TL.all_tissues_at_freq(f)
        res[f"tissue_{int(f)}"] = np.array([t[n] for n in names], dtype=np.float64)
    geoms = []
    for grid_size, dx_mm in ((64, 3.0), (48, 4.0), (40, 6.0)):
        for seed in range(12):
            g = sample_random_geometry(seed * 37 + 5, grid_size, dx_mm)
            geoms.append([grid_size, int(dx_mm * 10), seed * 37 + 5, *g.center, g.scalp_outer_r,
                          g.skull_outer_r, g.skull_inner_r, g.dura_inner_r, g.csf_inner_r,
                          g.gray_matter_r, g.white_matter_r])
    res["geoms"] = np.array(geoms, dtype=np.int64)
    grid64 = R["grid"].YeeGrid(64, 64, dx=3e-3, dy=3e-3, Nz=64, dz=3e-3, device="cpu")
    bleeds = []
    for q, (btype, age, size) in enumerate([(b, a, z) for b in ("epidural", "subdural", "intracerebral")
                                            for a in ("acute", "chronic") for z in ("small", "large")]):
        geom = sample_random_geometry(100 + q, 64, 3.0)
        ph = BrainPhantom3D(grid64, 1e9, geometry=geom, seed=200 + q)
        b = ph.add_random_bleed(btype, age, size)
        bleeds.append([100 + q, 200 + q] + ([-1, -1, -1, -1, 0, 0] if b is None else
                                            [*b.center, b.radius, b.eps_r, b.sigma]))
    res["bleeds"] = np.array(bleeds, dtype=np.float64)
    res["bleed_cases"] = np.array([f"{b}/{a}/{z}" for b in ("epidural", "subdural", "intracerebral")
                                   for a in ("acute", "chronic") for z in ("small", "large")])
    geom = sample_random_geometry(7, 64, 3.0)
    ph = BrainPhantom3D(grid64, 1e9, geometry=geom, seed=9)
    ph.add_bleed_at((40, 30, 28), 4, "intracerebral", "subacute")
    ca, cb = ph.build()
    res["phantom64_ca_sha"], res["phantom64_cb_sha"] = sha(ca), sha(cb)
    with tempfile.TemporaryDirectory() as tmp:
        for tag, kw, label, seed in (("nb", {}, 3, 11), ("nb0", {}, 0, 4),
                                     ("uwb", {"freq_low_hz": 1e9, "freq_high_hz": 3e9}, 1, 23)):
            gen = BrainDatasetGenerator(tmp, grid_size=40, dx_mm=6.0, n_tx=4, ring_radius_cells=18,
                                        n_steps=700, device="cpu", seed=0, **kw)
            smp = gen.generate_sample(label=label, seed=seed)
            path = gen.save_sample(smp, 0)
            res[f"{tag}_label"], res[f"{tag}_seed"] = label, seed
            for k in ("signals_total", "signals_reference", "signals_scattered", "das_image",
                      "bleed_center_cells", "bleed_radius_cells", "phantom_skull_inner_r",
                      "phantom_gray_r", "phantom_scalp_outer_r", "dt_s", "freq_hz"):
                res[f"{tag}_{k}"] = np.asarray(smp[k])
            res[f"{tag}_bleed"] = np.array([smp["bleed_type"], smp["bleed_age"]])
            res[f"{tag}_sha_total"] = sha(smp["signals_total"])
            res[f"{tag}_sha_reference"] = sha(smp["signals_reference"])
            res[f"{tag}_npz_keys"] = np.array(sorted(np.load(path, allow_pickle=True).files))
    np.savez_compressed(out / "brain_dataset40.npz", **res)


def case_lossy_full(R, out, n=4096, steps=100, init_seed=41):
    """The 4096^2 lossy-ellipse scene at its full size, from seeded random
    starting fields (so the short run reaches every cell, edge and tile
    boundary), the ring receivers plus 8 near the source, float32 and
    float64."""
    wl = W.LossyEllipses(n=n, steps=steps)
    GD = gauss_deriv_class(R)
    M = R["materials"].Material
    si, sj = wl.source
    rx = [("Hz", i, j) for i, j in wl.receivers] + [
        (c, si + di, sj + dj) for c, di, dj in (("Hz", 12, 0), ("Hz", 0, -17), ("Ex", -9, 9),
                                                ("Ey", 20, 20), ("Hz", 0, 0), ("Ex", 3, -30),
                                                ("Ey", -25, 4), ("Hz", -30, -30))]
    init = W.initial_fields(init_seed, (n, n), ("Ex", "Ey", "Hz"))
    res = {}
    for dt_name, dtype in (("32", torch.float32), ("64", torch.float64)):
        grid = R["grid"].YeeGrid(n, n, wl.dx, wl.dx, courant=wl.courant, device="cpu", dtype=dtype)
        wave = GD().build(steps, grid.dt, torch.device("cpu"), dtype)
        if dtype == torch.float32:
            wave32 = wave.clone()
        res[dt_name] = run_2d(R, n, n, wl.dx, wl.courant, steps, dtype, paint=wl.paint,
                              default=wl.background(M),
                              sources=[("Hz", "point", wl.source, wave)], probes=rx, init=init)
        print("  lossy", n, dt_name, "done", flush=True)
    g32, f32, tr32, ca, cb = res["32"]
    _, f64, tr64, _, _ = res["64"]
    np.savez_compressed(
        out / f"lossy_full_{n}.npz", n=n, steps=steps, dx=wl.dx, courant=wl.courant,
        dt=g32.dt, seed=wl.seed, init_seed=init_seed, src=np.array(wl.source),
        rx_comp=np.array([r[0] for r in rx]), rx=np.array([r[1:] for r in rx]),
        wave=wave32.numpy(), sha_ca=sha(ca), sha_cb=sha(cb), traces32=tr32.numpy(),
        traces64=tr64.numpy(), sha_traces=sha(tr32), sha_ex=sha(f32.Ex), sha_ey=sha(f32.Ey),
        sha_hz=sha(f32.Hz), hz32_dec=np.ascontiguousarray(f32.Hz[::37, ::41, 0].numpy()),
        hz64_dec=np.ascontiguousarray(f64.Hz[::37, ::41, 0].numpy()))


def case_head3d_full(R, out, n=256, steps=30, init_seed=43, batch=1):
    """The head phantom at a full benchmark size (256^3, or batch x 128^3)
    from seeded random starting fields of all six components, Ez source at
    the centre, the ring receivers plus 8 near the source, float32 only
    (plus float64 traces for the error statement)."""
    wl = W.Head3D(n=n, steps=steps)
    GD = gauss_deriv_class(R)
    M = R["materials"].Material
    si, sj, sk = wl.source
    rx = [("Ez", *p) for p in wl.receivers()] + [
        (c, si + di, sj + dj, sk + dk) for c, di, dj, dk in (
            ("Ez", 0, 0, 0), ("Ex", 5, -3, 2), ("Ey", -4, 6, 0), ("Hx", 2, 2, -7),
            ("Hy", -6, 0, 5), ("Hz", 3, -5, 3), ("Ez", 9, 9, -9), ("Ez", 0, 0, 1))]
    shape = (n, n, n) if batch == 1 else (batch, n, n, n)
    init = W.initial_fields(init_seed, shape, ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"))
    res = {}
    for dt_name, dtype in (("32", torch.float32), ("64", torch.float64)):
        stable = R["grid"].compute_stable_dt(wl.dx, wl.dx, wl.dx, wl.courant)
        wave = GD().build(steps, stable, torch.device("cpu"), dtype)
        if dtype == torch.float32:
            wave32 = wave.clone()
        res[dt_name] = run_3d(R, (n, n, n), wl.dx, wl.courant, steps, dtype, paint=wl.paint,
                              default=wl.background(M),
                              sources=[("Ez", "point", wl.source, wave)], probes=rx, init=init,
                              batch=batch)
        print("  head3d", n, batch, dt_name, "done", flush=True)
    g, f32, tr32, ca, cb = res["32"]
    _, f64, tr64, _, _ = res["64"]
    name = f"head3d_full_{n}" if batch == 1 else f"head3d_batch{batch}x{n}"
    np.savez_compressed(
        out / f"{name}.npz", n=n, batch=batch, steps=steps, dx=wl.dx, courant=wl.courant,
        dt=g.dt, seed=wl.seed, init_seed=init_seed, src=np.array(wl.source),
        rx_comp=np.array([r[0] for r in rx]), rx=np.array([r[1:] for r in rx]),
        wave=wave32.numpy(), sha_ca=sha(ca), sha_cb=sha(cb), traces32=tr32.numpy(),
        traces64=tr64.numpy(), sha_traces=sha(tr32),
        **{f"sha_{c.lower()}": sha(getattr(f32, c)) for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")})


def case_cpml_profile(R, out):
    """The CPML profile at every sample position the product's CPML uses,
    evaluated by the reference's own ``_pml_bsigma_at_rho`` (and its
    ``_compute_pml_coeffs`` tables), for three grids.  The position -> depth
    mapping (low side (D - x) / D, high side (x - (n - 1 - D)) / D, E at
    integer cells, Hz at half cells, the last half cell outside the grid) is
    the product's; the profile values are the reference's."""
    B = R["boundaries"]
    res = {}
    for q, (n, D, dx, courant) in enumerate(((40, 8, 1e-3, 0.5), (64, 10, 0.5e-3, 0.5),
                                             (33, 6, 2e-3, 0.9))):
        dt = R["grid"].compute_stable_dt(dx, dx, None, courant)
        m, Rt, kmax, amax = 3, 1e-8, 5.0, 0.05
        smax = (m + 1) * math.log(1.0 / Rt) / (2.0 * B.ETA0 * D * dx)
        cols = {k: [] for k in ("bE", "cE", "bH", "cH", "rhoE", "rhoH")}
        for half, tag in ((0.0, "E"), (0.5, "H")):
            for i in range(n):
                x = i + half
                rho = max((D - x) / D, (x - (n - 1 - D)) / D, 0.0)
                if rho <= 0.0 or (half and i > n - 2):
                    b, c, rho = 1.0, 0.0, 0.0
                else:
                    rho = min(rho, 1.0)
                    _, b, c = B._pml_bsigma_at_rho(rho, smax, kmax, amax, m, dt)
                cols["b" + tag].append(b)
                cols["c" + tag].append(c)
                cols["rho" + tag].append(rho)
        for k, v in cols.items():
            res[f"c{q}_{k}"] = np.array(v, dtype=np.float64)
        res[f"c{q}_grid"] = np.array([n, D, dx, courant, dt])
        ref = B._compute_pml_coeffs(D, dx, dt, torch.device("cpu"), torch.float64)
        for name, t in zip(("bE", "cE", "bH", "cH", "sE", "sH"), ref):
            res[f"c{q}_ref_{name}"] = t.numpy()
    res["ncases"] = 3
    np.savez_compressed(out / "cpml_profile.npz", **res)


def case_f64_2d(R, out):
    """float64 FieldSets run by the reference's FDTD2D, with the float64
    waveform and amplitude tables stored so the float64 engine can replay them:
      vac   -- 160x192 vacuum; a Gaussian-derivative Hz point source, a
               weighted Ex line source, two coincident Ey point sources and an
               Hz point on the i=0 edge; 60 probes of all three components
               (edges included); 700 steps; stability checks every 50 steps;
      mat   -- the lossy-ellipse scene at 256^2, 500 steps, seeded random
               starting fields;
      batch -- a batched FieldSet (3 members, 64x48, different random starting
               fields, shared Ca/Cb, one broadcast Hz point source), 300 steps.
    Digests (SHA-256) cover the float64 traces and final fields."""
    F = R["fields"]
    S = R["sources"]
    Tab = tab_class(R)
    GD = gauss_deriv_class(R)
    M = R["materials"].Material
    rng = np.random.default_rng(64)
    res = {}

    # --- vac
    nx, ny, steps = 160, 192, 700
    grid = R["grid"].YeeGrid(nx, ny, 1e-3, 1e-3, courant=0.6, device="cpu", dtype=torch.float64)
    f = F.FieldSet(grid)
    b = R["boundaries"].MurABC(grid, f.Hz)
    w0 = GD().build(steps, grid.dt, torch.device("cpu"), torch.float64)
    w1 = torch.from_numpy(rng.standard_normal(steps))
    w2 = torch.from_numpy(rng.standard_normal(steps))
    w3 = torch.from_numpy(rng.standard_normal(steps))
    amp = torch.from_numpy(rng.uniform(0.5, 2.0, 40))
    srcs = [S.PointSource(Tab(w0), 80, 96, "Hz", grid=grid, N_steps=steps),
            S.LineSource(Tab(w1), "x", 30, 60, 100, "Ex", grid=grid, N_steps=steps,
                         amplitude_profile=amp),
            S.PointSource(Tab(w2), 120, 50, "Ey", grid=grid, N_steps=steps),
            S.PointSource(Tab(w2), 120, 50, "Ey", grid=grid, N_steps=steps),
            S.PointSource(Tab(w3), 0, 140, "Hz", grid=grid, N_steps=steps)]
    sim = R["fdtd2d"].FDTD2D(grid, f, b, S.SourceCollection(srcs), n_check=50)
    pts = [(0, 0), (0, 191), (159, 0), (159, 191), (1, 96), (158, 96), (80, 0), (80, 191),
           (80, 96), (30, 80), (120, 50), (100, 140), (0, 140), (1, 140), (45, 20),
           (140, 170), (80, 1), (80, 190), (2, 2), (157, 189)]
    probes = [(c, i, j) for c in ("Ex", "Ey", "Hz") for i, j in pts]
    tr = torch.zeros(len(probes), steps, dtype=torch.float64)
    for s in range(steps):
        sim.step()
        for r, (c, i, j) in enumerate(probes):
            tr[r, s] = getattr(f, c)[i, j, 0]
    res.update(vac_waves=torch.stack([w0, w1, w2, w3]).numpy(), vac_amp=amp.numpy(),
               vac_probes=np.array([(("Ex", "Ey", "Hz").index(c), i, j) for c, i, j in probes]),
               vac_sha_traces=sha(tr), vac_sha_ex=sha(f.Ex), vac_sha_ey=sha(f.Ey),
               vac_sha_hz=sha(f.Hz), vac_traces_dec=dec(tr.numpy(), 7),
               vac_last_max=sim.last_field_max, vac_checks=sim.n_stability_checks,
               vac_dt=grid.dt)

    # --- mat
    n, steps = 256, 500
    wl = W.LossyEllipses(n=n, steps=steps)
    grid = R["grid"].YeeGrid(n, n, wl.dx, wl.dx, courant=wl.courant, device="cpu",
                             dtype=torch.float64)
    f = F.FieldSet(grid)
    init = W.initial_fields(65, (n, n), ("Ex", "Ey", "Hz"))
    for c, v in init.items():
        getattr(f, c).copy_(torch.from_numpy(v).to(torch.float64).reshape(n, n, 1))
    b = R["boundaries"].MurABC(grid, f.Hz)
    mm = R["materials"].MaterialMap(grid, default=wl.background(M))
    wl.paint(mm, M)
    ca, cb = mm.build()
    wave = GD().build(steps, grid.dt, torch.device("cpu"), torch.float64)
    src = S.PointSource(Tab(wave), *wl.source, "Hz", grid=grid, N_steps=steps)
    sim = R["fdtd2d"].FDTD2D(grid, f, b, S.SourceCollection([src]), Ca=ca, Cb=cb,
                             n_check=10 ** 9)
    rx = [("Hz", i, j) for i, j in wl.receivers]
    tr = torch.zeros(len(rx), steps, dtype=torch.float64)
    for s in range(steps):
        sim.step()
        for r, (c, i, j) in enumerate(rx):
            tr[r, s] = getattr(f, c)[i, j, 0]
    res.update(mat_n=n, mat_steps=steps, mat_seed=wl.seed, mat_init_seed=65,
               mat_wave=wave.numpy(), mat_src=np.array(wl.source),
               mat_rx=np.array([r[1:] for r in rx]), mat_sha_ca=sha(ca), mat_sha_cb=sha(cb),
               mat_sha_traces=sha(tr), mat_sha_ex=sha(f.Ex), mat_sha_ey=sha(f.Ey),
               mat_sha_hz=sha(f.Hz), mat_dt=grid.dt)

    # --- batch
    nx, ny, B, steps = 64, 48, 3, 300
    grid = R["grid"].YeeGrid(nx, ny, 2e-3, 2e-3, courant=0.7, device="cpu", dtype=torch.float64)
    f = F.FieldSet(grid, batch_size=B)
    for c, v in W.initial_fields(66, (B, nx, ny), ("Ex", "Ey", "Hz")).items():
        getattr(f, c).copy_(torch.from_numpy(v).to(torch.float64).reshape(B, nx, ny, 1))
    b = R["boundaries"].MurABC(grid, f.Hz)
    mm = R["materials"].MaterialMap(grid, default=M("bg", 3.0, 0.05))
    mm.add_circle((30.0, 20.0), 9.0, M("c", 20.0, 0.8))
    ca, cb = mm.build()
    wave = torch.from_numpy(rng.standard_normal(steps))
    src = S.PointSource(Tab(wave), 20, 30, "Hz", grid=grid, N_steps=steps)
    sim = R["fdtd2d"].FDTD2D(grid, f, b, S.SourceCollection([src]), Ca=ca, Cb=cb, n_check=25)
    for s in range(steps):
        sim.step()
    res.update(batch_wave=wave.numpy(), batch_sha_ca=sha(ca), batch_sha_ex=sha(f.Ex),
               batch_sha_ey=sha(f.Ey), batch_sha_hz=sha(f.Hz), batch_last_max=sim.last_field_max,
               batch_checks=sim.n_stability_checks)
    np.savez_compressed(out / "f64_2d.npz", **res)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="root of the reference project checkout")
    ap.add_argument("--only", default="")
    a = ap.parse_args()
    ref = Path(a.ref)
    R = load_ref(ref)
    torch.set_num_threads(8)
    out = HERE
    todo = {
        "vacuum": lambda: case_vacuum_point(R, out),
        "lossy": lambda: case_lossy_ellipses(R, out),
        "breast": lambda: case_breast_mimo(R, out),
        "breast_full": lambda: case_breast_mimo(R, out, sides=(256, 384, 512), n_tx=1, steps=3000,
                                                name="breast_mimo_full"),
        "lossy_full": lambda: case_lossy_full(R, out),
        "head3d_full": lambda: case_head3d_full(R, out),
        "head3d_batch": lambda: case_head3d_full(R, out, n=128, batch=8, init_seed=47),
        "cpml": lambda: case_cpml_profile(R, out),
        "f64": lambda: case_f64_2d(R, out),
        "edges2d": lambda: case_edges_2d(R, out),
        "head3d": lambda: case_head3d(R, out),
        "edges3d": lambda: case_edges_3d(R, out),
        "das": lambda: case_das(R, ref, out),
        "antenna": lambda: case_antenna(R, ref, out),
        "brain": lambda: case_brain_dataset(R, ref, out),
    }
    for k, fn in todo.items():
        if a.only and k not in a.only.split(","):
            continue
        print("golden:", k, flush=True)
        fn()


if __name__ == "__main__":
    main()
