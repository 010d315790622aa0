"""Multi-shell 3D head phantom with anatomically constrained haemorrhages
(drop-in for src/datasets/brain/phantom.py).

Concentric spheres, outside in: scalp, skull, dura, CSF, gray matter, white
matter, painted in that order, then any bleeds on top.  Geometry and bleed
placement are drawn from ``random.Random(seed)`` with the same sequence of
draws as the reference (phantom.py:86-179 and :285-372), so a seed gives the
same phantom -- and, through ``MaterialMap3D.build3d``, bit-identical Ca/Cb;
``build_device`` paints the same coefficients on the GPU.
"""

from __future__ import annotations

import math
import random
from dataclasses import dataclass
from typing import Optional

import numpy as np
import torch

from ...core.grid import YeeGrid
from ...core.materials import Material, MaterialMap3D
from .tissue_library import tissue_at_freq


@dataclass
class BleedConfig:
    """One haemorrhage (phantom.py:37-45): type, age, centre cell, radius in
    cells and its (eps_r, sigma) at the phantom frequency."""
    bleed_type: str
    age: str
    center: tuple[int, int, int]
    radius: int
    eps_r: float
    sigma: float


@dataclass
class PhantomGeometry:
    """Shell radii in cells about ``center`` (phantom.py:48-58)."""
    center: tuple[int, int, int]
    scalp_outer_r: int
    skull_outer_r: int
    skull_inner_r: int
    dura_inner_r: int
    csf_inner_r: int
    gray_matter_r: int
    white_matter_r: int


# Fixed adult proportions at 3 mm cells: training (A) and test (B) phantoms
# (phantom.py:61-83).
PHANTOM_A = PhantomGeometry((32, 32, 32), 28, 26, 23, 20, 17, 17, 10)
PHANTOM_B = PhantomGeometry((32, 32, 32), 27, 25, 21, 18, 15, 15, 9)

# Bleed radius ranges in cells by size class (phantom.py:182-186)
BLEED_SIZES = {"small": (2, 4), "medium": (4, 7), "large": (7, 12)}

# Shells painted outside in: (tissue, geometry field holding its outer radius)
_LAYERS = (("scalp", "scalp_outer_r"), ("skull_cortical", "skull_outer_r"),
           ("dura", "skull_inner_r"), ("csf", "csf_inner_r"),
           ("gray_matter", "gray_matter_r"), ("white_matter", "white_matter_r"))


def sample_random_geometry(seed: int, grid_size: int = 64, dx_mm: float = 3.0) -> PhantomGeometry:
    """A head drawn from adult population statistics (phantom.py:86-179):
    outer radius N(94, 4) mm clamped to [80, 110], skull N(7, 1.5) mm
    clamped to [3, 12], ~2 mm scalp, epidural and CSF spaces of 3-6 cells,
    white matter at 60-75 % of the brain radius; then minimum widths and the
    radius ordering are enforced.  Draw order: gauss, gauss, randint,
    randint, uniform."""
    rng = random.Random(seed)
    half = grid_size // 2
    head_mm = min(110.0, max(80.0, rng.gauss(94.0, 4.0)))
    scalp = min(max(int(head_mm / dx_mm), half - 4), half - 2)
    skull_mm = min(12.0, max(3.0, rng.gauss(7.0, 1.5)))
    skull_cells = max(1, round(skull_mm / dx_mm))
    skull_out = scalp - max(1, round(2.0 / dx_mm))
    skull_in = skull_out - skull_cells
    dura_in = skull_in - rng.randint(3, 6)
    csf_in = dura_in - rng.randint(3, 6)
    white = max(4, round(csf_in * rng.uniform(0.60, 0.75)))
    # minimum widths (epidural and subdural zones of 3 cells) and ordering
    skull_in = max(skull_in, 6)
    dura_in = max(min(dura_in, skull_in - 3), 4)
    csf_in = max(min(csf_in, dura_in - 3), 4)
    if white >= csf_in:
        white = max(3, csf_in - 2)
    return PhantomGeometry((half, half, half), scalp, skull_out, skull_in, dura_in, csf_in,
                           csf_in, white)


class BrainPhantom3D:
    """Head phantom whose tissues take their Cole-Cole (eps_r, sigma) at
    ``freq_hz`` (phantom.py:189-513).  ``seed`` drives bleed placement."""

    _TISSUE_NAMES = ("scalp", "skull_cortical", "csf", "gray_matter", "white_matter", "dura")

    def __init__(self, grid: YeeGrid, freq_hz: float, geometry: Optional[PhantomGeometry] = None,
                 seed: Optional[int] = None) -> None:
        self._grid = grid
        self._freq_hz = freq_hz
        self._geom = geometry or PHANTOM_A
        self._rng = random.Random(seed)
        self._np_rng = np.random.default_rng(seed)
        self._bleeds: list[BleedConfig] = []
        self._tissue_params = {n: tissue_at_freq(n, freq_hz) for n in self._TISSUE_NAMES}

    freq_hz = property(lambda s: s._freq_hz)
    geometry = property(lambda s: s._geom)
    bleeds = property(lambda s: list(s._bleeds))
    has_bleed = property(lambda s: bool(s._bleeds))

    # -- placement ---------------------------------------------------------
    def _distance_from_center(self, i: int, j: int, k: int) -> float:
        c = self._geom.center
        return math.sqrt((i - c[0]) ** 2 + (j - c[1]) ** 2 + (k - c[2]) ** 2)

    def _get_zone_bounds(self, bleed_type: str) -> tuple[float, float]:
        """(inner, outer) radii of the shell a bleed centre may lie in
        (phantom.py:243-268): epidural between dura and skull, subdural
        between brain surface and dura, intracerebral inside the brain."""
        g = self._geom
        zones = {"epidural": (g.dura_inner_r, g.skull_inner_r),
                 "subdural": (g.csf_inner_r, g.dura_inner_r),
                 "intracerebral": (0, g.gray_matter_r)}
        if bleed_type not in zones:
            raise ValueError("bleed_type must be 'epidural', 'subdural', or 'intracerebral', "
                             f"got '{bleed_type}'")
        return zones[bleed_type]

    def _is_in_zone(self, i: int, j: int, k: int, bleed_type: str) -> bool:
        inner, outer = self._get_zone_bounds(bleed_type)
        return inner < self._distance_from_center(i, j, k) < outer

    def _bleed_fits(self, i: int, j: int, k: int, radius: int, bleed_type: str) -> bool:
        """Never into bone; an intracerebral bleed stays inside the brain
        surface (phantom.py:276-290)."""
        limit = self._geom.gray_matter_r if bleed_type == "intracerebral" else self._geom.skull_inner_r
        return self._distance_from_center(i, j, k) + radius <= limit

    def sample_bleed_position(self, bleed_type: str, radius: int,
                              max_attempts: int = 1000) -> Optional[tuple[int, int, int]]:
        """Rejection-sample a centre: radius U(r_min, r_max), polar angle
        U(0, pi), azimuth U(0, 2 pi), truncated to cells; kept if the sphere
        stays off the grid edge and out of bone (phantom.py:292-346)."""
        cx, cy, cz = self._geom.center
        g = self._grid
        inner, outer = self._get_zone_bounds(bleed_type)
        r_min, r_max = (0, outer - radius) if bleed_type == "intracerebral" else (inner, outer)
        if r_min >= r_max:
            return None
        for _ in range(max_attempts):
            r = self._rng.uniform(r_min, r_max)
            theta = self._rng.uniform(0, math.pi)
            phi = self._rng.uniform(0, 2 * math.pi)
            i = int(cx + r * math.sin(theta) * math.cos(phi))
            j = int(cy + r * math.sin(theta) * math.sin(phi))
            k = int(cz + r * math.cos(theta))
            inside = (radius < i < g.Nx - radius and radius < j < g.Ny - radius
                      and radius < k < g.Nz - radius)
            if inside and self._bleed_fits(i, j, k, radius, bleed_type):
                return (i, j, k)
        return None

    def add_random_bleed(self, bleed_type: str = "intracerebral", age: str = "acute",
                         size: str = "medium") -> Optional[BleedConfig]:
        """Radius ~ randint over the size class, then a sampled centre; None
        when no valid centre was found (phantom.py:348-390)."""
        if age not in ("acute", "subacute", "chronic"):
            raise ValueError(f"age must be 'acute', 'subacute', or 'chronic', got '{age}'")
        if size not in BLEED_SIZES:
            raise ValueError(f"size must be one of {list(BLEED_SIZES.keys())}, got '{size}'")
        radius = self._rng.randint(*BLEED_SIZES[size])
        pos = self.sample_bleed_position(bleed_type, radius)
        if pos is None:
            return None
        return self._add(bleed_type, age, pos, radius)

    def add_bleed_at(self, position: tuple[int, int, int], radius: int,
                     bleed_type: str = "intracerebral", age: str = "acute") -> BleedConfig:
        """A bleed at a given cell; ValueError if it would not fit
        (phantom.py:392-418)."""
        if not self._bleed_fits(position[0], position[1], position[2], radius, bleed_type):
            raise ValueError(f"Position {position} with radius {radius} does not fit in "
                             f"'{bleed_type}' zone for the current phantom geometry.")
        return self._add(bleed_type, age, position, radius)

    def _add(self, bleed_type, age, pos, radius) -> BleedConfig:
        eps_r, sigma = tissue_at_freq(age, self._freq_hz)
        b = BleedConfig(bleed_type, age, pos, radius, eps_r, sigma)
        self._bleeds.append(b)
        return b

    # -- coefficients -------------------------------------------------------
    def material_map(self) -> MaterialMap3D:
        """The painter's list: shells outside in, then the bleeds
        (phantom.py:420-455)."""
        mm = MaterialMap3D(self._grid)
        g = self._geom
        for tissue, field in _LAYERS:
            eps_r, sigma = self._tissue_params[tissue]
            mm.add_sphere(center=g.center, radius=getattr(g, field),
                          material=Material(tissue, eps_r=eps_r, sigma=sigma))
        for b in self._bleeds:
            mm.add_sphere(center=b.center, radius=b.radius,
                          material=Material(f"bleed_{b.bleed_type}_{b.age}", eps_r=b.eps_r,
                                            sigma=b.sigma))
        return mm

    def build(self) -> tuple[torch.Tensor, torch.Tensor]:
        """(Ca, Cb), each (Nx, Ny, Nz) float32 on the grid's device."""
        return self.material_map().build3d()

    def build_device(self, device=None) -> tuple[torch.Tensor, torch.Tensor]:
        """The same (Ca, Cb) painted on a CUDA device (``wf_paint3d``),
        bit-identical to ``build()``: only the shell and bleed spheres cross
        to the device."""
        return self.material_map().build3d_device(device)

    def get_label(self) -> int:
        """0 healthy, 1 epidural, 2 subdural, 3 intracerebral (first bleed)."""
        if not self._bleeds:
            return 0
        return {"epidural": 1, "subdural": 2, "intracerebral": 3}.get(self._bleeds[0].bleed_type, 0)

    def get_metadata(self) -> dict:
        """Frequency, label, bleeds and tissue parameters (phantom.py:472-505)."""
        dx = self._grid.dx
        return {
            "freq_hz": self._freq_hz,
            "has_bleed": self.has_bleed,
            "label": self.get_label(),
            "n_bleeds": len(self._bleeds),
            "phantom_type": "A" if self._geom is PHANTOM_A else "B",
            "bleeds": [{"type": b.bleed_type, "age": b.age, "center_cells": b.center,
                        "radius_cells": b.radius, "center_mm": tuple(c * dx * 1e3 for c in b.center),
                        "radius_mm": b.radius * dx * 1e3, "eps_r": b.eps_r, "sigma": b.sigma}
                       for b in self._bleeds],
            "tissue_params": {n: {"eps_r": p[0], "sigma": p[1]}
                              for n, p in self._tissue_params.items()},
        }

    def __repr__(self) -> str:
        g = self._grid
        extra = f", bleeds={len(self._bleeds)}" if self._bleeds else ""
        return (f"BrainPhantom3D(freq={self._freq_hz / 1e9:.2f}GHz, "
                f"grid={g.Nx}x{g.Ny}x{g.Nz}{extra})")
