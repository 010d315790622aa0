"""Per-cell material coefficients (mirror of src/core/materials.py).

``MaterialMap.build()`` paints regions in insertion order (painter's
algorithm) on host float32 index grids and returns ``(Ca, Cb)`` on
``grid.device``, with the same arithmetic as the reference so the
coefficient tensors are bit-identical (src/core/materials.py:200-252,
425-478).  ``build_eps_sigma()`` additionally returns the per-cell
(eps_r, sigma) maps that the adjoint needs.
"""

from __future__ import annotations

import math
import warnings
from dataclasses import dataclass
from typing import Callable

import torch

from .grid import YeeGrid

EPS0: float = 8.8541878128e-12
MU0: float = 1.2566370614e-6


@dataclass
class Material:
    """eps_r, sigma (S/m), mu_r of one medium (src/core/materials.py:33-94)."""

    name: str
    eps_r: float
    sigma: float
    mu_r: float = 1.0

    def __post_init__(self) -> None:
        if self.eps_r < 1.0:
            raise ValueError(f"eps_r must be >= 1, got {self.eps_r} for '{self.name}'")
        if self.sigma < 0.0:
            raise ValueError(f"sigma must be >= 0, got {self.sigma} for '{self.name}'")
        if self.mu_r <= 0.0:
            raise ValueError(f"mu_r must be > 0, got {self.mu_r} for '{self.name}'")

    def _alpha(self, dt: float) -> float:
        return self.sigma * dt / (2.0 * EPS0 * self.eps_r)

    def ca(self, dt: float) -> float:
        """Ca = (1 - a)/(1 + a), a = sigma*dt/(2*eps0*eps_r)."""
        a = self._alpha(dt)
        return (1.0 - a) / (1.0 + a)

    def cb(self, dt: float) -> float:
        """Cb = (dt/(eps0*eps_r))/(1 + a)."""
        a = self._alpha(dt)
        return (dt / (EPS0 * self.eps_r)) / (1.0 + a)

    def skin_depth(self, freq: float) -> float:
        if self.sigma == 0.0:
            return float("inf")
        return math.sqrt(2.0 / (2.0 * math.pi * freq * MU0 * self.sigma))

    def wavelength(self, freq: float) -> float:
        return (1.0 / math.sqrt(EPS0 * MU0)) / (freq * math.sqrt(self.eps_r * self.mu_r))


TISSUE_LIBRARY: dict[str, Material] = {
    "free_space": Material("free_space", eps_r=1.0, sigma=0.000),
    "skull": Material("skull", eps_r=8.0, sigma=0.100),
    "brain": Material("brain", eps_r=40.0, sigma=1.500),
    "tumor": Material("tumor", eps_r=55.0, sigma=2.100),
    "blood": Material("blood", eps_r=55.0, sigma=2.100),
    "saline": Material("saline", eps_r=70.0, sigma=2.000),
}


def _check_ca(ca_arr: torch.Tensor, three_d: bool) -> None:
    ca_min = float(ca_arr.min().item())
    if ca_min <= 0.0:
        extra = "" if three_d else " Physical passive media require Ca in (0, 1]."
        raise ValueError(f"Ca <= 0 detected (min={ca_min:.6f}). Check material conductivities "
                         f"or reduce dt.{extra}")
    if ca_min < 0.5:
        warnings.warn(f"Some Ca values are below 0.5 (min={ca_min:.4f}). Very high "
                      "conductivity — verify material parameters.", UserWarning, stacklevel=3)


class MaterialMap:
    """Region painter for 2D grids (src/core/materials.py:115-290)."""

    def __init__(self, grid: YeeGrid, default: Material | None = None) -> None:
        self._grid = grid
        self._default = default or TISSUE_LIBRARY["free_space"]
        self._regions: list[Callable[[torch.Tensor, torch.Tensor], torch.Tensor]] = []
        self._materials: list[Material] = []
        # typed description of each region for the device painter (None = custom mask)
        self._prims: list = []

    def add_circle(self, center: tuple[float, float], radius: float, material: Material) -> "MaterialMap":
        ci, cj = float(center[0]), float(center[1])
        r2 = radius * radius
        self._regions.append(lambda I, J: ((I - ci) ** 2 + (J - cj) ** 2) <= r2)
        self._materials.append(material)
        self._prims.append(("circle", (ci, cj, r2)))
        return self

    def add_ellipse(self, center: tuple[float, float], semi_axes: tuple[float, float],
                    material: Material) -> "MaterialMap":
        """Axis-aligned ellipse ((I-ci)/a)**2 + ((J-cj)/b)**2 <= 1 (the mask the
        reference's phantom examples paint with add_custom)."""
        ci, cj = float(center[0]), float(center[1])
        a, b = float(semi_axes[0]), float(semi_axes[1])
        self._regions.append(lambda I, J: ((I - ci) / a) ** 2 + ((J - cj) / b) ** 2 <= 1.0)
        self._materials.append(material)
        self._prims.append(("ellipse", (ci, cj, a, b)))
        return self

    def add_shell(self, center: tuple[float, float], outer: tuple[float, float],
                  inner: tuple[float, float], material: Material,
                  inner_center: tuple[float, float] | None = None) -> "MaterialMap":
        """Cells inside the outer ellipse and outside the inner one (a skin or
        skull layer)."""
        ci, cj = float(center[0]), float(center[1])
        ki, kj = (ci, cj) if inner_center is None else (float(inner_center[0]), float(inner_center[1]))
        a, b = float(outer[0]), float(outer[1])
        a2, b2 = float(inner[0]), float(inner[1])

        def fn(I, J):
            out = ((I - ci) / a) ** 2 + ((J - cj) / b) ** 2 <= 1.0
            inn = ((I - ki) / a2) ** 2 + ((J - kj) / b2) ** 2 <= 1.0
            return out & ~inn
        self._regions.append(fn)
        self._materials.append(material)
        self._prims.append(("shell", (ci, cj, a, b, ki, kj, a2, b2)))
        return self

    def add_rectangle(self, i_range: tuple[int, int], j_range: tuple[int, int],
                      material: Material) -> "MaterialMap":
        i0, i1 = i_range
        j0, j1 = j_range
        self._regions.append(lambda I, J: (I >= i0) & (I <= i1) & (J >= j0) & (J <= j1))
        self._materials.append(material)
        self._prims.append(("rect", (float(i0), float(i1), float(j0), float(j1))))
        return self

    def add_custom(self, mask_fn: Callable[[torch.Tensor, torch.Tensor], torch.Tensor],
                   material: Material) -> "MaterialMap":
        self._regions.append(mask_fn)
        self._materials.append(material)
        self._prims.append(None)
        return self

    @property
    def device_paintable(self) -> bool:
        """True when every region is a circle, rectangle, ellipse or shell."""
        return all(p is not None for p in self._prims)

    def build_device(self, device=None, out: tuple | None = None,
                     eps_sigma: tuple | None = None) -> tuple[torch.Tensor, torch.Tensor]:
        """``(Ca, Cb)`` painted by the CUDA painter (``wf_paint2d``), each
        ``(Nx, Ny, 1)`` float32 on ``device`` (default ``grid.device``),
        bit-identical to ``build()``.  Only the region list and the material
        tables cross to the device.  ``out``: optional (Ca, Cb) tensors to
        fill; ``eps_sigma``: optional float64 (eps_r, sigma) planes to fill
        too.  The Ca <= 0 check runs on the material table (no device sync)."""
        from .. import _native as nat
        if not self.device_paintable:
            raise ValueError("build_device needs circle/rectangle/ellipse/shell regions only "
                             "(add_custom masks are host-only: use build())")
        dev = torch.device(device if device is not None else self._grid.device)
        if dev.type != "cuda":
            raise RuntimeError("build_device paints on a CUDA device only (use build() on the host)")
        nx, ny = self._grid.Nx, self._grid.Ny
        dt = self._grid.dt
        mats = [self._default, *self._materials]
        tca = torch.tensor([m.ca(dt) for m in mats], dtype=torch.float32)
        tcb = torch.tensor([m.cb(dt) for m in mats], dtype=torch.float32)
        teps = torch.tensor([m.eps_r for m in mats], dtype=torch.float64)
        tsig = torch.tensor([m.sigma for m in mats], dtype=torch.float64)
        _check_ca(tca, three_d=False)
        kinds = {"circle": 0, "rect": 1, "ellipse": 2, "shell": 3}
        regs = (nat.WfRegion2D * max(1, len(self._prims)))()
        for q, (kind, params) in enumerate(self._prims):
            r = regs[q]
            r.kind = kinds[kind]
            r.material = q + 1
            for t, v in enumerate(params):
                r.p[t] = nat.f32(v)
        rb = bytes(memoryview(regs).cast("B"))
        nm = len(mats)
        parts = [torch.frombuffer(bytearray(rb), dtype=torch.uint8), teps.view(torch.uint8),
                 tsig.view(torch.uint8), tca.view(torch.uint8), tcb.view(torch.uint8)]
        host = torch.cat(parts).pin_memory()
        blob = host.to(dev, non_blocking=True)
        base = blob.data_ptr()
        o_eps = len(rb)                 # a multiple of 8 (40-byte regions)
        o_sig = o_eps + 8 * nm
        o_ca = o_sig + 8 * nm
        o_cb = o_ca + 4 * nm
        if out is None:
            ca = torch.empty((nx, ny, 1), dtype=torch.float32, device=dev)
            cb = torch.empty((nx, ny, 1), dtype=torch.float32, device=dev)
        else:
            ca, cb = out
        e_ptr = s_ptr = None
        if eps_sigma is not None:
            e_ptr, s_ptr = eps_sigma[0].data_ptr(), eps_sigma[1].data_ptr()
        lib = nat.load()
        nat.check(lib.wf_paint2d(nx, ny, base, len(self._prims), base + o_ca, base + o_cb,
                                 base + o_eps, base + o_sig, nm, ca.data_ptr(), cb.data_ptr(),
                                 e_ptr, s_ptr, None, nat.stream_handle(dev)))
        return ca, cb

    def _paint2d(self):
        nx, ny = self._grid.Nx, self._grid.Ny
        I = torch.arange(nx, dtype=torch.float32).unsqueeze(1).expand(nx, ny)
        J = torch.arange(ny, dtype=torch.float32).unsqueeze(0).expand(nx, ny)
        label = torch.zeros((nx, ny), dtype=torch.int16)  # 0 = default material
        for r, mask_fn in enumerate(self._regions, start=1):
            label[mask_fn(I, J)] = r
        return label

    def _coeffs_from_label(self, label: torch.Tensor, mats: list[Material]):
        dt = self._grid.dt
        table_ca = torch.tensor([m.ca(dt) for m in mats], dtype=torch.float32)
        table_cb = torch.tensor([m.cb(dt) for m in mats], dtype=torch.float32)
        lab = label.long()
        return table_ca[lab], table_cb[lab]

    def build(self) -> tuple[torch.Tensor, torch.Tensor]:
        """(Ca, Cb), each ``(Nx, Ny, 1)`` on ``grid.device`` (materials.py:200-252)."""
        label = self._paint2d()
        ca_arr, cb_arr = self._coeffs_from_label(label, [self._default, *self._materials])
        _check_ca(ca_arr, three_d=False)
        dev, dt = self._grid.device, self._grid.dtype
        return (ca_arr.unsqueeze(2).to(device=dev, dtype=dt),
                cb_arr.unsqueeze(2).to(device=dev, dtype=dt))

    def build_eps_sigma(self) -> tuple[torch.Tensor, torch.Tensor]:
        """Per-cell (eps_r, sigma), float64, shape ``(Nx, Ny)`` on the host."""
        label = self._paint2d().long()
        mats = [self._default, *self._materials]
        eps = torch.tensor([m.eps_r for m in mats], dtype=torch.float64)[label]
        sig = torch.tensor([m.sigma for m in mats], dtype=torch.float64)[label]
        return eps, sig

    def summary(self) -> str:
        dt = self._grid.dt
        lines = [f"MaterialMap — grid ({self._grid.Nx}×{self._grid.Ny}), dt={dt:.3e} s",
                 f"  Default: {self._default.name} (eps_r={self._default.eps_r}, "
                 f"σ={self._default.sigma})"]
        for i, m in enumerate(self._materials):
            lines.append(f"  Region {i}: {m.name} — eps_r={m.eps_r}, σ={m.sigma} S/m, "
                         f"Ca={m.ca(dt):.6f}, Cb={m.cb(dt):.3e}")
        return "\n".join(lines)

    def __repr__(self) -> str:
        return (f"MaterialMap(grid=({self._grid.Nx},{self._grid.Ny}), "
                f"n_regions={len(self._regions)}, default={self._default.name})")


class MaterialMap3D(MaterialMap):
    """3D primitives + ``build3d`` (src/core/materials.py:297-484)."""

    def __init__(self, grid: YeeGrid, default: Material | None = None) -> None:
        super().__init__(grid, default)
        self._regions3d: list = []
        self._materials3d: list[Material] = []
        # typed description of each 3D region for the device painter (None = custom mask)
        self._prims3d: list = []

    def add_sphere(self, center: tuple, radius: float, material: Material) -> "MaterialMap3D":
        ci, cj, ck = (float(c) for c in center)
        r2 = radius * radius
        self._regions3d.append(lambda I, J, K: (I - ci) ** 2 + (J - cj) ** 2 + (K - ck) ** 2 <= r2)
        self._materials3d.append(material)
        self._prims3d.append((0, (ci, cj, ck, r2)))
        return self

    def add_cylinder(self, center: tuple, axis: str, radius: float, height: float,
                     material: Material) -> "MaterialMap3D":
        ci, cj, ck = (float(c) for c in center)
        r2, h2 = radius * radius, height / 2.0
        if axis == "x":
            fn = lambda I, J, K: ((J - cj) ** 2 + (K - ck) ** 2 <= r2) & ((I - ci).abs() <= h2)
        elif axis == "y":
            fn = lambda I, J, K: ((I - ci) ** 2 + (K - ck) ** 2 <= r2) & ((J - cj).abs() <= h2)
        else:
            fn = lambda I, J, K: ((I - ci) ** 2 + (J - cj) ** 2 <= r2) & ((K - ck).abs() <= h2)
        self._regions3d.append(fn)
        self._materials3d.append(material)
        self._prims3d.append(({"x": 3, "y": 4}.get(axis, 5), (ci, cj, ck, r2, h2)))
        return self

    def add_box(self, corner_min: tuple, corner_max: tuple, material: Material) -> "MaterialMap3D":
        i0, j0, k0 = (float(c) for c in corner_min)
        i1, j1, k1 = (float(c) for c in corner_max)
        self._regions3d.append(lambda I, J, K: (I >= i0) & (I <= i1) & (J >= j0) & (J <= j1)
                               & (K >= k0) & (K <= k1))
        self._materials3d.append(material)
        self._prims3d.append((1, (i0, i1, j0, j1, k0, k1)))
        return self

    def add_ellipsoid(self, center: tuple, semi_axes: tuple, material: Material) -> "MaterialMap3D":
        ci, cj, ck = (float(c) for c in center)
        a2, b2, c2 = (float(s) ** 2 for s in semi_axes)
        self._regions3d.append(
            lambda I, J, K: (I - ci) ** 2 / a2 + (J - cj) ** 2 / b2 + (K - ck) ** 2 / c2 <= 1.0)
        self._materials3d.append(material)
        self._prims3d.append((2, (ci, cj, ck, a2, b2, c2)))
        return self

    def add_custom3d(self, mask_fn, material: Material) -> "MaterialMap3D":
        self._regions3d.append(mask_fn)
        self._materials3d.append(material)
        self._prims3d.append(None)
        return self

    @property
    def device_paintable3d(self) -> bool:
        """True when every 3D region is a sphere, box, ellipsoid or cylinder."""
        return all(p is not None for p in self._prims3d)

    def build3d_device(self, device=None, out: tuple | None = None) -> tuple[torch.Tensor, torch.Tensor]:
        """``(Ca, Cb)``, each ``(Nx, Ny, Nz)`` float32 painted on ``device``
        (default ``grid.device``) by ``wf_paint3d``, bit-identical to
        ``build3d()``.  Only the region list and the material table cross to
        the device.  ``out``: optional (Ca, Cb) tensors to fill.  The
        Ca <= 0 check runs on the material table (no device sync)."""
        from .. import _native as nat
        if not self.device_paintable3d:
            raise ValueError("build3d_device needs sphere/box/ellipsoid/cylinder regions only "
                             "(add_custom3d masks are host-only: use build3d())")
        dev = torch.device(device if device is not None else self._grid.device)
        if dev.type != "cuda":
            raise RuntimeError("build3d_device paints on a CUDA device only (use build3d())")
        g = self._grid
        dt = g.dt
        mats = [self._default, *self._materials3d]
        tca = torch.tensor([m.ca(dt) for m in mats], dtype=torch.float32)
        tcb = torch.tensor([m.cb(dt) for m in mats], dtype=torch.float32)
        _check_ca(tca, three_d=True)
        regs = (nat.WfRegion3D * max(1, len(self._prims3d)))()
        for q, (kind, params) in enumerate(self._prims3d):
            regs[q].kind = kind
            regs[q].material = q + 1
            for t, v in enumerate(params):
                regs[q].p[t] = nat.f32(v)
        rb = bytes(memoryview(regs).cast("B"))
        host = torch.cat([torch.frombuffer(bytearray(rb), dtype=torch.uint8),
                          tca.view(torch.uint8), tcb.view(torch.uint8)]).pin_memory()
        blob = host.to(dev, non_blocking=True)
        base, nm = blob.data_ptr(), len(mats)
        shape = (g.Nx, g.Ny, g.Nz)
        if out is None:
            ca = torch.empty(shape, dtype=torch.float32, device=dev)
            cb = torch.empty(shape, dtype=torch.float32, device=dev)
        else:
            ca, cb = out
            for t in (ca, cb):
                if t.dtype != torch.float32 or not t.is_contiguous() or t.numel() != g.Nx * g.Ny * g.Nz:
                    raise ValueError("out tensors must be contiguous float32 with Nx*Ny*Nz cells")
        nat.check(nat.load().wf_paint3d(g.Nx, g.Ny, g.Nz, base, len(self._prims3d),
                                        base + len(rb), base + len(rb) + 4 * nm, nm,
                                        ca.data_ptr(), cb.data_ptr(), None,
                                        nat.stream_handle(dev)))
        self._keep = (host, blob)
        return ca, cb

    def _paint3d(self):
        nx, ny, nz = self._grid.Nx, self._grid.Ny, self._grid.Nz
        I = torch.arange(nx, dtype=torch.float32).view(-1, 1, 1).expand(nx, ny, nz)
        J = torch.arange(ny, dtype=torch.float32).view(1, -1, 1).expand(nx, ny, nz)
        K = torch.arange(nz, dtype=torch.float32).view(1, 1, -1).expand(nx, ny, nz)
        label = torch.zeros((nx, ny, nz), dtype=torch.int16)
        for r, fn in enumerate(self._regions3d, start=1):
            label[fn(I, J, K)] = r
        return label

    def build3d(self) -> tuple[torch.Tensor, torch.Tensor]:
        """(Ca, Cb), each ``(Nx, Ny, Nz)`` on ``grid.device`` (materials.py:425-478)."""
        label = self._paint3d()
        ca_arr, cb_arr = self._coeffs_from_label(label, [self._default, *self._materials3d])
        _check_ca(ca_arr, three_d=True)
        dev, dt = self._grid.device, self._grid.dtype
        return ca_arr.to(device=dev, dtype=dt), cb_arr.to(device=dev, dtype=dt)

    def __repr__(self) -> str:
        g = self._grid
        return (f"MaterialMap3D(grid=({g.Nx},{g.Ny},{g.Nz}), n_regions2d={len(self._regions)}, "
                f"n_regions3d={len(self._regions3d)}, default={self._default.name})")
