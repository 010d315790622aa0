"""Rebuild the golden cases for the oracle (CPU) and for the CUDA engine (GPU).

Coefficients are painted with the product's host-side MaterialMap on a CPU
grid (pure host code, checked against the reference's Ca/Cb digests), the
waveform tables come from the fixtures, and the same source / probe
descriptions feed both the oracle and the engine.
"""

from __future__ import annotations

import numpy as np
import torch

from conftest import golden
from waveforge_b200 import workloads as W
from waveforge_b200.core.grid import YeeGrid
from waveforge_b200.core.materials import Material, MaterialMap, MaterialMap3D

COMP2 = ("Ex", "Ey", "Hz")
COMP3 = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def cpu_grid(nx, ny, dx, courant, nz=1):
    if nz > 1:
        return YeeGrid(nx, ny, dx, dx, Nz=nz, dz=dx, courant=courant, device="cpu")
    return YeeGrid(nx, ny, dx, dx, courant=courant, device="cpu")


def lossy_coeffs(g: dict):
    n = int(g["n"])
    wl = W.LossyEllipses(n=n, steps=int(g["steps"]), seed=int(g["seed"]))
    grid = cpu_grid(n, n, float(g["dx"]), float(g["courant"]))
    mm = MaterialMap(grid, default=wl.background(Material))
    wl.paint(mm, Material)
    ca, cb = mm.build()
    return ca[..., 0], cb[..., 0]


def breast_coeffs(g: dict, p: int, with_tumor=True):
    side, A, B, ti, tj, r = (float(v) for v in g[f"p{p}_geom"])
    ph = W.BreastPhantom(int(side), A, B, (ti, tj), r)
    grid = cpu_grid(ph.side, ph.side, float(g["dx"]), float(g["courant"]))
    mm = MaterialMap(grid, default=ph.background(Material))
    ph.paint(mm, Material, with_tumor=with_tumor)
    ca, cb = mm.build()
    return ph, ca[..., 0], cb[..., 0]


def head_coeffs(g: dict):
    n = int(g["n"])
    wl = W.Head3D(n=n, steps=int(g["steps"]), seed=int(g["seed"]))
    grid = cpu_grid(n, n, float(g["dx"]), float(g["courant"]), nz=n)
    mm = MaterialMap3D(grid, default=wl.background(Material))
    wl.paint(mm, Material)
    return mm.build3d()


def edge2d_sources(d: dict):
    """[(comp, kind, (i0,i1,j0,j1), wave, amp)] from an edges2d fixture."""
    out = []
    for q in range(int(d["nsrc"])):
        comp = str(d[f"src{q}_comp"])
        kind = str(d[f"src{q}_kind"])
        wave = torch.from_numpy(d[f"src{q}_wave"])
        args = [int(v) for v in d[f"src{q}_args"]]
        amp = torch.from_numpy(d[f"src{q}_amp"]) if f"src{q}_amp" in d else None
        if kind == "point":
            i, j = args
            out.append((comp, "point", (i, i + 1, j, j + 1), wave, None))
        else:
            pos, start, stop = args
            axis = str(d[f"src{q}_axis"])
            box = (start, stop, pos, pos + 1) if axis == "x" else (pos, pos + 1, start, stop)
            out.append((comp, "line", box, wave, amp))
    return out


def edge3d_sources(d: dict):
    out = []
    nx, ny, nz = (int(v) for v in d["shape"])
    for q in range(int(d["nsrc"])):
        comp = str(d[f"src{q}_comp"])
        kind = str(d[f"src{q}_kind"])
        wave = torch.from_numpy(d[f"src{q}_wave"])
        a = [int(v) for v in d[f"src{q}_args"]]
        if kind == "point":
            i, j, k = a
            out.append((comp, (i, i + 1, j, j + 1, k, k + 1), wave))
        else:
            plane, pos = ("xy", "xz", "yz")[a[0]], a[1]
            box = {"xy": (0, nx, 0, ny, pos, pos + 1), "xz": (0, nx, pos, pos + 1, 0, nz),
                   "yz": (pos, pos + 1, 0, ny, 0, nz)}[plane]
            out.append((comp, box, wave))
    return out


def load(name):
    return golden(name)
