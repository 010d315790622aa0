"""Yee grid geometry and CFL time step (mirror of src/core/grid.py).

Same public surface as the reference ``YeeGrid``/``compute_stable_dt``/
``GridMetadata`` (src/core/grid.py:30-665), with one deliberate difference:
a CUDA device that is requested but unavailable raises instead of silently
falling back to CPU (src/core/grid.py:350-356), because every compute path of
this package runs on the GPU.
"""

from __future__ import annotations

import math
import warnings
from dataclasses import dataclass, field

import torch

C0: float = 299_792_458.0


@dataclass
class GridMetadata:
    """Grid summary (src/core/grid.py:30-113)."""

    Nx: int
    Ny: int
    Nz: int
    dx: float
    dy: float
    dz: float
    dt: float
    courant: float
    device: torch.device
    dtype: torch.dtype = field(default=torch.float32)
    is_3d: bool = field(default=False)

    def cells_total(self) -> int:
        return self.Nx * self.Ny * self.Nz

    def vram_estimate_bytes(self, n_field_tensors: int = 6) -> int:
        return n_field_tensors * self.cells_total() * (torch.finfo(self.dtype).bits // 8)

    def __repr__(self) -> str:
        mode = "3D" if self.is_3d else "2D"
        return (f"GridMetadata(mode={mode}, shape=({self.Nx}, {self.Ny}, {self.Nz}), "
                f"spacing=({self.dx:.3g}, {self.dy:.3g}, {self.dz:.3g}) m, dt={self.dt:.6e} s, "
                f"courant={self.courant}, device={self.device}, dtype={self.dtype}, "
                f"cells={self.cells_total():,}, "
                f"VRAM~{self.vram_estimate_bytes() / 2**20:.2f} MB)")


def compute_stable_dt(dx: float, dy: float, dz: float | None = None, courant: float = 0.98) -> float:
    """dt = courant / (c0 * sqrt(1/dx^2 + 1/dy^2 [+ 1/dz^2])), src/core/grid.py:120-169."""
    if not (0.0 < courant < 1.0):
        raise ValueError(f"courant must satisfy 0 < courant < 1, got {courant!r}")
    for name, v in (("dx", dx), ("dy", dy)):
        if v <= 0.0:
            raise ValueError(f"{name} must be > 0, got {v!r}")
    if dz is not None and dz <= 0.0:
        raise ValueError(f"dz must be > 0 when provided, got {dz!r}")
    s = (1.0 / dx) ** 2 + (1.0 / dy) ** 2
    if dz is not None:
        s += (1.0 / dz) ** 2
    return courant / (C0 * math.sqrt(s))


class YeeGrid:
    """Yee lattice (src/core/grid.py:176-327): validates sizes, spacings and the
    Courant number, derives or checks dt against the CFL limit and builds the
    E (half-integer) and H (integer) coordinate vectors."""

    def __init__(self, Nx: int, Ny: int, dx: float, dy: float, *, Nz: int = 1,
                 dz: float | None = None, courant: float = 0.98, dt: float | None = None,
                 device: str | torch.device = "cuda", dtype: torch.dtype = torch.float32) -> None:
        for name, val in (("Nx", Nx), ("Ny", Ny)):
            if not isinstance(val, int) or val < 2:
                raise ValueError(f"{name} must be an integer >= 2, got {val!r}")
        if not isinstance(Nz, int) or Nz < 1:
            raise ValueError(f"Nz must be an integer >= 1 (use Nz=1 for 2-D mode), got {Nz!r}")
        if dx <= 0.0:
            raise ValueError(f"dx must be > 0, got {dx!r}")
        if dy <= 0.0:
            raise ValueError(f"dy must be > 0, got {dy!r}")
        is_3d = Nz > 1
        if is_3d:
            if dz is None:
                raise ValueError("dz is required when Nz > 1 (3-D mode)")
            if dz <= 0.0:
                raise ValueError(f"dz must be > 0, got {dz!r}")
        elif dz is None:
            dz = dx
        if not (0.0 < courant < 1.0):
            raise ValueError(f"courant must satisfy 0 < courant < 1, got {courant!r}")
        dev = self._resolve_device(device)
        stable = compute_stable_dt(dx, dy, dz if is_3d else None, courant)
        if dt is None:
            dt = stable
        else:
            if dt > stable:
                raise ValueError(f"Provided dt={dt:.6e} exceeds CFL-stable limit {stable:.6e}. "
                                 "Simulation will be unstable.")
            if dt < 0.10 * stable:
                warnings.warn(f"Provided dt={dt:.6e} is less than 10 % of the CFL-stable "
                              f"dt={stable:.6e}. This is suspiciously small and may indicate a "
                              "unit error.", UserWarning, stacklevel=2)
        self.meta = GridMetadata(Nx=Nx, Ny=Ny, Nz=Nz, dx=dx, dy=dy, dz=dz, dt=dt, courant=courant,
                                 device=dev, dtype=dtype, is_3d=is_3d)
        self.xs = (torch.arange(Nx, device=dev, dtype=dtype) + 0.5) * dx
        self.ys = (torch.arange(Ny, device=dev, dtype=dtype) + 0.5) * dy
        self.zs = (torch.arange(Nz, device=dev, dtype=dtype) + 0.5) * dz
        self.xs_h = torch.arange(Nx, device=dev, dtype=dtype) * dx
        self.ys_h = torch.arange(Ny, device=dev, dtype=dtype) * dy
        self.zs_h = torch.arange(Nz, device=dev, dtype=dtype) * dz

    @staticmethod
    def _resolve_device(device: str | torch.device) -> torch.device:
        dev = torch.device(device) if isinstance(device, str) else device
        if dev.type == "cuda" and not torch.cuda.is_available():
            raise RuntimeError("CUDA requested but not available: waveforge_b200 runs on the GPU "
                               "only (no silent CPU fallback)")
        if dev.type == "cuda" and dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        return dev

    # -- read-only properties ------------------------------------------------
    Nx = property(lambda self: self.meta.Nx)
    Ny = property(lambda self: self.meta.Ny)
    Nz = property(lambda self: self.meta.Nz)
    dx = property(lambda self: self.meta.dx)
    dy = property(lambda self: self.meta.dy)
    dz = property(lambda self: self.meta.dz)
    dt = property(lambda self: self.meta.dt)
    courant = property(lambda self: self.meta.courant)
    device = property(lambda self: self.meta.device)
    dtype = property(lambda self: self.meta.dtype)

    @property
    def shape(self) -> tuple[int, int, int]:
        return (self.meta.Nx, self.meta.Ny, self.meta.Nz)

    @property
    def cell_volume(self) -> float:
        return self.meta.dx * self.meta.dy * self.meta.dz

    def allocate_field(self, fill: float = 0.0) -> torch.Tensor:
        return torch.full(self.shape, fill, device=self.meta.device, dtype=self.meta.dtype)

    def allocate_material_coeff(self, fill: float = 1.0) -> torch.Tensor:
        return torch.full(self.shape, fill, device=self.meta.device, dtype=self.meta.dtype)

    def cell_index(self, i: int, j: int, k: int = 0) -> int:
        return i * self.meta.Ny * self.meta.Nz + j * self.meta.Nz + k

    def physical_size(self) -> tuple[float, float, float]:
        m = self.meta
        return (m.Nx * m.dx, m.Ny * m.dy, m.Nz * m.dz)

    def wavelength_resolution(self, freq_hz: float) -> float:
        return (C0 / freq_hz) / min(self.meta.dx, self.meta.dy, self.meta.dz)

    def validate_resolution(self, freq_hz: float, min_cells_per_wavelength: float = 10) -> None:
        cpw = self.wavelength_resolution(freq_hz)
        if cpw < min_cells_per_wavelength:
            raise ValueError(f"Grid resolution at {freq_hz:.3e} Hz is {cpw:.2f} cells per "
                             f"wavelength, below the required minimum of "
                             f"{min_cells_per_wavelength}. Reduce cell spacing or lower the "
                             "target frequency.")

    def to(self, device: str | torch.device) -> "YeeGrid":
        dev = self._resolve_device(device)
        g = YeeGrid.__new__(YeeGrid)
        m = self.meta
        g.meta = GridMetadata(Nx=m.Nx, Ny=m.Ny, Nz=m.Nz, dx=m.dx, dy=m.dy, dz=m.dz, dt=m.dt,
                              courant=m.courant, device=dev, dtype=m.dtype, is_3d=m.is_3d)
        for name in ("xs", "ys", "zs", "xs_h", "ys_h", "zs_h"):
            setattr(g, name, getattr(self, name).to(dev))
        return g

    def __repr__(self) -> str:
        m = self.meta
        Lx, Ly, Lz = self.physical_size()
        return (f"YeeGrid(mode={'3D' if m.is_3d else '2D'}, shape={self.shape}, "
                f"physical=({Lx:.3g} m, {Ly:.3g} m, {Lz:.3g} m), spacing=(dx={m.dx:.3g}, "
                f"dy={m.dy:.3g}, dz={m.dz:.3g}) m, dt={m.dt:.6e} s, courant={m.courant}, "
                f"device={m.device}, dtype={m.dtype})")
