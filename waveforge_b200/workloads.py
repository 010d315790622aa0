"""Seeded synthetic workloads used by the benchmark and the parity tests.

No public dataset is involved: every phantom is drawn from
``numpy.random.default_rng(seed)``.  The builders take the MaterialMap
instance and the Material class as arguments, so the same recipe paints a
``waveforge_b200.core.MaterialMap`` or the reference's own ``MaterialMap``
(the golden-vector generator does the latter) with identical masks.

Workloads (sizes as in the benchmark configurations):
* ``vacuum_point`` : 256^2 vacuum, Hz point source at the centre, 4 receivers
  at 60 cells on the axes, 1000 steps.
* ``lossy_ellipses``: 4096^2, background eps_r 10, 64 random axis-aligned
  ellipses (semi-axes U[20,400] cells, eps_r U[1,60], sigma U[0,1.5] S/m),
  Hz source at (512, 2048), 16 receivers on a 1500-cell ring, 2000 steps;
  ``scale`` shrinks every length for test-size versions.
* ``breast_mimo``  : elliptical breast phantoms (skin 36/0.8, adipose
  5/0.04, fibroglandular 40/0.8, tumour disc 55/1.0 of radius U[8,24]) in a
  matching medium eps_r 10, 16-antenna ring at 0.85 x half-width, each
  antenna a separate Hz-source solve, dx = 0.5 mm, 3000 steps.
* ``head_3d``      : nested ellipsoids (skull 12/0.2, 6 cells thick; brain
  45/0.7; clot sphere r=6 60/1.2) in eps_r 10, Ez dipole at the centre,
  32 Ez receivers on a ring in the mid plane, 1500 steps.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


def ellipse_mask(ci: float, cj: float, a: float, b: float):
    return lambda I, J: ((I - ci) / a) ** 2 + ((J - cj) / b) ** 2 <= 1.0


def _add_ellipse(mm, center, axes, material) -> None:
    """An axis-aligned ellipse: the product map's primitive (which its device
    painter also knows), or the same mask through ``add_custom`` on a map that
    lacks it (the reference's MaterialMap, src/core/materials.py:183-198)."""
    if hasattr(mm, "add_ellipse"):
        mm.add_ellipse(center, axes, material)
    else:
        mm.add_custom(ellipse_mask(center[0], center[1], axes[0], axes[1]), material)


def _add_shell(mm, center, outer, inner, material) -> None:
    """Cells inside the outer ellipse and outside the inner one, as
    ``_add_ellipse`` chooses between the primitive and ``add_custom``."""
    if hasattr(mm, "add_shell"):
        mm.add_shell(center, outer, inner, material)
    else:
        o = ellipse_mask(center[0], center[1], outer[0], outer[1])
        i = ellipse_mask(center[0], center[1], inner[0], inner[1])
        mm.add_custom(lambda I, J: o(I, J) & ~i(I, J), material)


def ring_positions(n: int, radius: float, ci: float, cj: float, nx: int, ny: int,
                   margin: int = 1) -> list[tuple[int, int]]:
    """``n`` cells on a circle, rounded and clamped to [margin, N-1-margin]."""
    out = []
    for k in range(n):
        a = 2.0 * math.pi * k / n
        i = int(round(ci + radius * math.cos(a)))
        j = int(round(cj + radius * math.sin(a)))
        out.append((max(margin, min(nx - 1 - margin, i)), max(margin, min(ny - 1 - margin, j))))
    return out


# ---------------------------------------------------------------------------
# 2D lossy ellipses (HBM-roofline workload)
# ---------------------------------------------------------------------------

@dataclass
class LossyEllipses:
    n: int = 4096
    steps: int = 2000
    seed: int = 2
    n_ellipses: int = 64
    dx: float = 1e-3
    courant: float = 0.5

    @property
    def scale(self) -> float:
        return self.n / 4096.0

    @property
    def source(self) -> tuple[int, int]:
        return (int(round(512 * self.scale)), int(round(2048 * self.scale)))

    @property
    def receivers(self) -> list[tuple[int, int]]:
        c = self.n / 2.0
        return ring_positions(16, 1500 * self.scale, c, c, self.n, self.n)

    def paint(self, mm, Material) -> None:
        rng = np.random.default_rng(self.seed)
        s = self.scale
        for e in range(self.n_ellipses):
            ci, cj = (float(v) for v in rng.uniform(0, self.n, 2))
            a, b = (float(v) for v in rng.uniform(20 * s, 400 * s, 2))
            er = float(rng.uniform(1.0, 60.0))
            sg = float(rng.uniform(0.0, 1.5))
            _add_ellipse(mm, (ci, cj), (a, b), Material(f"ellipse{e}", er, sg))

    @staticmethod
    def background(Material):
        return Material("background", 10.0, 0.0)


# ---------------------------------------------------------------------------
# 2D breast MIMO (batched workload)
# ---------------------------------------------------------------------------

BREAST_SIDES = (150, 200, 256, 384, 512)


@dataclass
class BreastPhantom:
    side: int
    A: float
    B: float
    tumor_center: tuple[float, float]
    tumor_r: float
    skin: int = 2

    @staticmethod
    def draw(rng: np.random.Generator, side: int | None = None) -> "BreastPhantom":
        if side is None:
            side = int(rng.choice(BREAST_SIDES))
        else:
            rng.integers(0, len(BREAST_SIDES))  # keep the draw sequence aligned
        A = float(rng.uniform(0.35, 0.45)) * side
        B = float(rng.uniform(0.35, 0.45)) * side
        r = float(rng.uniform(8.0, 24.0))
        th = float(rng.uniform(0.0, 2.0 * math.pi))
        rho = float(rng.uniform(0.0, 0.5))
        c = side / 2.0
        tc = (c + rho * (A - 2 - r) * math.cos(th), c + rho * (B - 2 - r) * math.sin(th))
        return BreastPhantom(side, A, B, tc, r)

    def paint(self, mm, Material, with_tumor: bool = True) -> None:
        c = self.side / 2.0
        A, B, sk = self.A, self.B, self.skin
        _add_shell(mm, (c, c), (A, B), (A - sk, B - sk), Material("skin", 36.0, 0.8))
        _add_ellipse(mm, (c, c), (A - sk, B - sk), Material("adipose", 5.0, 0.04))
        _add_ellipse(mm, (c, c), (A / 2.0, B / 2.0), Material("fibroglandular", 40.0, 0.8))
        if with_tumor:
            mm.add_circle(self.tumor_center, self.tumor_r, Material("tumor", 55.0, 1.0))

    def antennas(self, n: int = 16) -> list[tuple[int, int]]:
        c = self.side / 2.0
        return ring_positions(n, 0.85 * c, c, c, self.side, self.side)

    @staticmethod
    def background(Material):
        return Material("matching", 10.0, 0.0)


@dataclass
class BreastMIMO:
    n_phantoms: int = 64
    n_tx: int = 16
    steps: int = 3000
    seed: int = 3
    dx: float = 0.5e-3
    courant: float = 0.5

    def phantoms(self) -> list[BreastPhantom]:
        rng = np.random.default_rng(self.seed)
        return [BreastPhantom.draw(rng) for _ in range(self.n_phantoms)]

    def cell_updates(self) -> int:
        return sum(p.side * p.side for p in self.phantoms()) * self.n_tx * self.steps


# ---------------------------------------------------------------------------
# 3D head (3D workload)
# ---------------------------------------------------------------------------

@dataclass
class Head3D:
    n: int = 256
    steps: int = 1500
    seed: int = 4
    dx: float = 1e-3
    courant: float = 0.5
    n_rx: int = 32

    def geometry(self):
        rng = np.random.default_rng(self.seed)
        c = self.n / 2.0
        outer = tuple(float(v) * self.n for v in (0.36, 0.42, 0.34))
        t = 6.0 * self.n / 256.0 if self.n < 256 else 6.0
        inner = tuple(a - t for a in outer)
        u = rng.uniform(-0.45, 0.45, 3)
        clot_r = 6.0 * min(1.0, self.n / 256.0) if self.n < 256 else 6.0
        clot = tuple(c + float(u[q]) * (inner[q] - clot_r) for q in range(3))
        return (c, c, c), outer, inner, clot, max(1.0, clot_r)

    def paint(self, mm3, Material) -> None:
        ctr, outer, inner, clot, cr = self.geometry()
        mm3.add_ellipsoid(ctr, outer, Material("skull", 12.0, 0.2))
        mm3.add_ellipsoid(ctr, inner, Material("brain", 45.0, 0.7))
        mm3.add_sphere(clot, cr, Material("clot", 60.0, 1.2))

    def receivers(self) -> list[tuple[int, int, int]]:
        c = self.n / 2.0
        k = self.n // 2
        return [(i, j, k) for i, j in ring_positions(self.n_rx, 0.45 * self.n, c, c, self.n, self.n)]

    @property
    def source(self) -> tuple[int, int, int]:
        return (self.n // 2, self.n // 2, self.n // 2)

    @staticmethod
    def background(Material):
        return Material("background", 10.0, 0.0)


# ---------------------------------------------------------------------------
# seeded initial fields (full-size parity cases)
# ---------------------------------------------------------------------------

def initial_fields(seed: int, shape: tuple, comps: tuple) -> dict:
    """Seeded float32 white-noise starting values for the named components
    (E components with unit variance, H components scaled by 1/377 ohm), so
    that a short run touches every cell of a full-size grid, its edges and
    every internal block boundary of the kernels from the first step."""
    rng = np.random.default_rng(seed)
    out = {}
    for c in comps:
        v = rng.standard_normal(shape, dtype=np.float32)
        out[c] = v if c.startswith("E") else (v * np.float32(1.0 / 377.0)).astype(np.float32)
    return out


# ---------------------------------------------------------------------------
# serving stream (Poisson requests of lossy phantoms, some with gradients)
# ---------------------------------------------------------------------------

_GD_PULSE = None


def _pulse():
    global _GD_PULSE
    if _GD_PULSE is None:
        from .core.sources import GaussianDerivativePulse
        _GD_PULSE = GaussianDerivativePulse(1e9)
    return _GD_PULSE


def serving_request(side: int, steps: int, seed: int, *, n_ant: int = 16, gradient: bool = False,
                    dx: float = 1e-3, courant: float = 0.5, n_ellipses: int = 64):
    """One imaging request of the serving workload: a lossy-ellipse phantom
    (the 4096^2 workload's generator scaled to ``side``) with a tumour disc,
    ``n_ant`` antennas on a ring of radius 0.4*side (each one a transmitter
    run, all of them receivers), a 1 GHz Gaussian-derivative Hz pulse.  With
    ``gradient`` the request also carries the measured phantom: the same
    with the tumour's eps_r + 15."""
    from .core.grid import YeeGrid
    from .core.materials import Material, MaterialMap
    from .serving import ImagingRequest
    grid = YeeGrid(side, side, dx, dx, courant=courant, device="cpu")
    wl = LossyEllipses(n=side, steps=steps, seed=seed, n_ellipses=n_ellipses, dx=dx,
                       courant=courant)
    rng = np.random.default_rng(seed + 7919)
    r = max(2.0, 0.03 * side)
    c = side / 2.0
    ti, tj = (float(v) for v in c + rng.uniform(-0.25, 0.25, 2) * side)

    def phantom(tumor_eps: float):
        mm = MaterialMap(grid, default=wl.background(Material))
        wl.paint(mm, Material)
        mm.add_circle((ti, tj), r, Material("tumor", tumor_eps, 1.0))
        return mm

    ant = ring_positions(n_ant, 0.4 * side, c, c, side, side)
    return ImagingRequest(phantom(55.0), ant, ant, steps, _pulse(),
                          target=phantom(70.0) if gradient else None, tag=(side, steps, seed))


@dataclass
class ServingStream:
    """Poisson arrivals at ``rate``/s for ``duration`` s; side log-uniform in
    [side_min, side_max], steps uniform in [steps_min, steps_max], ``n_ant``
    transmitters each, a ``grad_fraction`` of them gradient requests."""
    rate: float = 200.0
    duration: float = 60.0
    seed: int = 5
    side_min: int = 128
    side_max: int = 1024
    steps_min: int = 1000
    steps_max: int = 5000
    n_ant: int = 16
    grad_fraction: float = 0.1

    def arrivals(self):
        rng = np.random.default_rng(self.seed)
        t, out, q = 0.0, [], 0
        while True:
            t += float(rng.exponential(1.0 / self.rate))
            if t >= self.duration:
                return out
            side = int(round(math.exp(rng.uniform(math.log(self.side_min), math.log(self.side_max)))))
            steps = int(rng.integers(self.steps_min, self.steps_max + 1))
            grad = bool(rng.uniform() < self.grad_fraction)
            out.append((t, serving_request(side, steps, self.seed * 100003 + q, n_ant=self.n_ant,
                                           gradient=grad)))
            q += 1
