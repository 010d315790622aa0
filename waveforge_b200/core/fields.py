"""Six-component SoA field storage (mirror of src/core/fields.py).

Tensors are ``(Nx, Ny, Nz)`` (2D uses Nz=1) or ``(B, Nx, Ny, Nz)`` when
batched, row-major with the last index unit-stride: exactly the layout the
CUDA kernels read and write in place (src/core/fields.py:156-168).
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Tuple

import torch

from .grid import YeeGrid

FIELD_COMPONENTS: Tuple[str, ...] = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


@dataclass
class StaggerOffset:
    component: str
    ox: float
    oy: float
    oz: float


YEE_OFFSETS: dict[str, StaggerOffset] = {
    "Ex": StaggerOffset("Ex", 0.5, 0.0, 0.0),
    "Ey": StaggerOffset("Ey", 0.0, 0.5, 0.0),
    "Ez": StaggerOffset("Ez", 0.0, 0.0, 0.5),
    "Hx": StaggerOffset("Hx", 0.0, 0.5, 0.5),
    "Hy": StaggerOffset("Hy", 0.5, 0.0, 0.5),
    "Hz": StaggerOffset("Hz", 0.5, 0.5, 0.0),
}

# Energy constants of the reference FieldSet (src/core/fields.py:77-78).
_EPS0: float = 8.854e-12
_MU0: float = 1.2566e-6


class FieldSet:
    """Owns six zero tensors on ``grid.device`` (src/core/fields.py:85-150)."""

    def __init__(self, grid: YeeGrid, *, batch_size: int = 1, dtype: torch.dtype | None = None) -> None:
        if batch_size < 1:
            raise ValueError(f"batch_size must be >= 1, got {batch_size!r}")
        self.grid = grid
        self.batch_size = batch_size
        self.dtype = grid.dtype if dtype is None else dtype
        self.offsets = YEE_OFFSETS
        shp = self._tensor_shape()
        self._fields: dict[str, torch.Tensor] = {
            c: torch.zeros(shp, device=grid.device, dtype=self.dtype) for c in FIELD_COMPONENTS}

    def _tensor_shape(self) -> tuple[int, ...]:
        g = self.grid
        return (g.Nx, g.Ny, g.Nz) if self.batch_size == 1 else (self.batch_size, g.Nx, g.Ny, g.Nz)

    def _validate_tensor(self, name: str, t: torch.Tensor) -> None:
        exp = self._tensor_shape()
        if tuple(t.shape) != exp:
            raise ValueError(f"Component '{name}' expected shape {exp}, got {tuple(t.shape)}")
        if t.dtype != self.dtype:
            raise ValueError(f"Component '{name}' expected dtype {self.dtype}, got {t.dtype}")

    def _get(self, name: str) -> torch.Tensor:
        return self._fields[name]

    def _set(self, name: str, t: torch.Tensor) -> None:
        self._validate_tensor(name, t)
        self._fields[name] = t

    Ex = property(lambda s: s._get("Ex"), lambda s, t: s._set("Ex", t))
    Ey = property(lambda s: s._get("Ey"), lambda s, t: s._set("Ey", t))
    Ez = property(lambda s: s._get("Ez"), lambda s, t: s._set("Ez", t))
    Hx = property(lambda s: s._get("Hx"), lambda s, t: s._set("Hx", t))
    Hy = property(lambda s: s._get("Hy"), lambda s, t: s._set("Hy", t))
    Hz = property(lambda s: s._get("Hz"), lambda s, t: s._set("Hz", t))

    @property
    def shape(self) -> tuple[int, ...]:
        return self._tensor_shape()

    @property
    def is_batched(self) -> bool:
        return self.batch_size > 1

    @property
    def device(self) -> torch.device:
        return self.grid.device

    def zero_(self) -> "FieldSet":
        for c in FIELD_COMPONENTS:
            self._fields[c].zero_()
        return self

    def clone(self) -> "FieldSet":
        fs = FieldSet(self.grid, batch_size=self.batch_size, dtype=self.dtype)
        for c in FIELD_COMPONENTS:
            fs._fields[c] = self._fields[c].clone()
        return fs

    def to(self, device: str | torch.device) -> "FieldSet":
        g = self.grid.to(device)
        fs = FieldSet(g, batch_size=self.batch_size, dtype=self.dtype)
        for c in FIELD_COMPONENTS:
            fs._fields[c] = self._fields[c].to(g.device)
        return fs

    def copy_from_(self, other: "FieldSet") -> None:
        if other.shape != self.shape:
            raise ValueError(f"Cannot copy_from_: shape mismatch — self.shape={self.shape}, "
                             f"other.shape={other.shape}")
        for c in FIELD_COMPONENTS:
            self._fields[c].copy_(other._fields[c])

    def as_dict(self) -> dict[str, torch.Tensor]:
        return dict(self._fields)

    def as_tensor(self) -> torch.Tensor:
        return torch.stack([self._fields[c] for c in FIELD_COMPONENTS], dim=1 if self.is_batched else 0)

    def from_tensor(self, t: torch.Tensor) -> None:
        g = self.grid
        unb, bat = (6, g.Nx, g.Ny, g.Nz), (self.batch_size, 6, g.Nx, g.Ny, g.Nz)
        if tuple(t.shape) == unb:
            for i, c in enumerate(FIELD_COMPONENTS):
                self._fields[c] = t[i]
        elif tuple(t.shape) == bat:
            for i, c in enumerate(FIELD_COMPONENTS):
                self._fields[c] = t[:, i]
        else:
            raise ValueError(f"from_tensor: unexpected shape {tuple(t.shape)}. Expected {unb} "
                             f"(unbatched) or {bat} (batched).")

    def electric(self):
        return self._fields["Ex"], self._fields["Ey"], self._fields["Ez"]

    def magnetic(self):
        return self._fields["Hx"], self._fields["Hy"], self._fields["Hz"]

    def energy_density(self) -> torch.Tensor:
        e = sum(self._fields[c] ** 2 for c in ("Ex", "Ey", "Ez")) * (_EPS0 * 0.5)
        m = sum(self._fields[c] ** 2 for c in ("Hx", "Hy", "Hz")) * (_MU0 * 0.5)
        return e + m

    def total_energy(self) -> float:
        return float(self.energy_density().sum().item()) * self.grid.cell_volume

    def max_field(self) -> float:
        return max(float(self._fields[c].abs().max().item()) for c in FIELD_COMPONENTS)

    def norm(self, component: str) -> float:
        if component not in self._fields:
            raise KeyError(f"Unknown field component {component!r}. Valid names: {FIELD_COMPONENTS}")
        return float(torch.linalg.norm(self._fields[component].float()).item())

    def __repr__(self) -> str:
        return (f"FieldSet(shape={self.shape}, batch_size={self.batch_size}, dtype={self.dtype}, "
                f"device={self.device})")
