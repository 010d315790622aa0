"""First-order Mur absorbing boundaries (mirror of src/core/boundaries.py).

The engines do not call ``snapshot``/``apply``: the fused CUDA kernels apply
the Mur update inside every step from the pre-step H they already hold
(double-buffered in shared memory), which removes the reference's full-grid
snapshot copy (src/core/boundaries.py:230-237, 488-497).  These objects keep
the reference surface: coefficient validation, the ``Hz_prev`` buffer, and
``snapshot``/``apply`` as explicit device-tensor operations for callers that
step boundaries by hand.
"""

from __future__ import annotations

import math
from typing import Tuple

import torch

from .grid import YeeGrid

C0: float = 299_792_458.0
EPS0: float = 8.8541878128e-12
ETA0: float = 376.730313


def _pml_bsigma_at_rho(rho, sigma_max, kappa_max, alpha_max, m, dt) -> Tuple[float, float, float]:
    """CPML (sigma, b, c) at normalised depth rho (src/core/boundaries.py:32-48)."""
    rho_m = rho ** m
    sigma_k = sigma_max * rho_m
    kappa_k = 1.0 + (kappa_max - 1.0) * rho_m
    alpha_k = alpha_max * (1.0 - rho)
    b_k = math.exp(-(sigma_k / kappa_k + alpha_k) * dt / EPS0)
    denom = sigma_k * kappa_k + kappa_k ** 2 * alpha_k
    c_k = 0.0 if (sigma_k == 0.0 and alpha_k == 0.0) else sigma_k / denom * (b_k - 1.0)
    return sigma_k, b_k, c_k


def _compute_pml_coeffs(D, dx, dt, device, dtype):
    """Dual-staggered CPML coefficient profiles (src/core/boundaries.py:51-112).
    Stored only; neither engine uses them (the reference engines don't either)."""
    m, R, kmax, amax = 3, 1e-8, 5.0, 0.05
    smax = (m + 1) * math.log(1.0 / R) / (2.0 * ETA0 * D * dx)
    cols = [[], [], [], [], [], []]
    for k in range(D):
        se, be, ce = _pml_bsigma_at_rho(k / D, smax, kmax, amax, m, dt)
        sh, bh, ch = _pml_bsigma_at_rho((k + 0.5) / D, smax, kmax, amax, m, dt)
        for col, v in zip(cols, (be, ce, bh, ch, se, sh)):
            col.append(v)
    return tuple(torch.tensor(c, device=device, dtype=dtype) for c in cols)


def _mur_coeff(dt: float, d: float) -> float:
    return (C0 * dt - d) / (C0 * dt + d)


class MurABC:
    """2D Mur ABC on the four Hz edges (src/core/boundaries.py:119-384)."""

    def __init__(self, grid: YeeGrid, Hz_field: torch.Tensor, *, pml_depth: int = 0) -> None:
        dt = grid.dt
        self.C_mur_x = _mur_coeff(dt, grid.dx)
        self.C_mur_y = _mur_coeff(dt, grid.dy)
        for ax, c in (("x", self.C_mur_x), ("y", self.C_mur_y)):
            if not (-1.0 < c < 0.0):
                raise ValueError(f"C_mur_{ax}={c!r} is not in the open interval (-1, 0). This "
                                 f"indicates a CFL violation — reduce dt or increase d{ax}.")
        self.Hz_prev = torch.zeros_like(Hz_field)
        self.Hz_curr = Hz_field
        self._Nx, self._Ny = grid.Nx, grid.Ny
        self._pml_depth, self._has_pml = pml_depth, pml_depth > 0
        if pml_depth > 0:
            (self.b_x_E, self.c_x_E, self.b_x_H, self.c_x_H, self.sigma_x_E,
             self.sigma_x_H) = _compute_pml_coeffs(pml_depth, grid.dx, dt, grid.device, grid.dtype)
            (self.b_y_E, self.c_y_E, self.b_y_H, self.c_y_H, self.sigma_y_E,
             self.sigma_y_H) = _compute_pml_coeffs(pml_depth, grid.dy, dt, grid.device, grid.dtype)
        else:
            e = torch.empty(0, device=grid.device, dtype=grid.dtype)
            (self.b_x_E, self.c_x_E, self.b_x_H, self.c_x_H, self.sigma_x_E, self.sigma_x_H) = (e,) * 6
            (self.b_y_E, self.c_y_E, self.b_y_H, self.c_y_H, self.sigma_y_E, self.sigma_y_H) = (e,) * 6

    def snapshot(self) -> None:
        self.Hz_prev.copy_(self.Hz_curr)

    def apply(self, Hz: torch.Tensor) -> None:
        """x edges then y edges, from ``Hz_prev`` (boundaries.py:239-274)."""
        nx, ny, cx, cy, hp = self._Nx, self._Ny, self.C_mur_x, self.C_mur_y, self.Hz_prev
        Hz[..., 0, :, 0] = hp[..., 1, :, 0] + cx * (Hz[..., 1, :, 0] - hp[..., 0, :, 0])
        Hz[..., nx - 1, :, 0] = hp[..., nx - 2, :, 0] + cx * (Hz[..., nx - 2, :, 0] - hp[..., nx - 1, :, 0])
        Hz[..., :, 0, 0] = hp[..., :, 1, 0] + cy * (Hz[..., :, 1, 0] - hp[..., :, 0, 0])
        Hz[..., :, ny - 1, 0] = hp[..., :, ny - 2, 0] + cy * (Hz[..., :, ny - 2, 0] - hp[..., :, ny - 1, 0])

    n_boundary_cells = property(lambda s: 2 * (s._Nx + s._Ny))
    mur_coefficient_x = property(lambda s: s.C_mur_x)
    mur_coefficient_y = property(lambda s: s.C_mur_y)
    has_pml = property(lambda s: s._has_pml)
    pml_depth = property(lambda s: s._pml_depth)

    @property
    def pml_coeffs_x(self) -> dict[str, torch.Tensor]:
        return {"b_E": self.b_x_E, "c_E": self.c_x_E, "b_H": self.b_x_H, "c_H": self.c_x_H,
                "sigma_E": self.sigma_x_E, "sigma_H": self.sigma_x_H}

    @property
    def pml_coeffs_y(self) -> dict[str, torch.Tensor]:
        return {"b_E": self.b_y_E, "c_E": self.c_y_E, "b_H": self.b_y_H, "c_H": self.c_y_H,
                "sigma_E": self.sigma_y_E, "sigma_H": self.sigma_y_H}

    def __repr__(self) -> str:
        return (f"MurABC(shape=({self._Nx}, {self._Ny}, 1), C_mur_x={self.C_mur_x:.6f}, "
                f"C_mur_y={self.C_mur_y:.6f}, has_pml={self._has_pml}, "
                f"pml_depth={self._pml_depth}, n_boundary_cells={self.n_boundary_cells})")


class MurABC3D:
    """3D Mur ABC on the tangential H of six faces (src/core/boundaries.py:391-654)."""

    def __init__(self, grid: YeeGrid, Hx_field: torch.Tensor, Hy_field: torch.Tensor,
                 Hz_field: torch.Tensor) -> None:
        dt = grid.dt
        self.C_mur_x = _mur_coeff(dt, grid.dx)
        self.C_mur_y = _mur_coeff(dt, grid.dy)
        self.C_mur_z = _mur_coeff(dt, grid.dz)
        for name, c in (("C_mur_x", self.C_mur_x), ("C_mur_y", self.C_mur_y), ("C_mur_z", self.C_mur_z)):
            if not (-1.0 < c < 0.0):
                raise ValueError(f"{name}={c!r} is not in the open interval (-1, 0). This indicates "
                                 "a CFL violation — reduce dt or increase the corresponding cell "
                                 "spacing.")
        self.Hx_prev = torch.zeros_like(Hx_field)
        self.Hy_prev = torch.zeros_like(Hy_field)
        self.Hz_prev = torch.zeros_like(Hz_field)
        self._Hx, self._Hy, self._Hz = Hx_field, Hy_field, Hz_field
        self._Nx, self._Ny, self._Nz = grid.Nx, grid.Ny, grid.Nz

    def snapshot(self) -> None:
        self.Hx_prev.copy_(self._Hx)
        self.Hy_prev.copy_(self._Hy)
        self.Hz_prev.copy_(self._Hz)

    def apply(self, Hx: torch.Tensor, Hy: torch.Tensor, Hz: torch.Tensor) -> None:
        """Faces x (Hy,Hz) -> y (Hx,Hz) -> z (Hx,Hy) (boundaries.py:499-583)."""
        nx, ny, nz = self._Nx, self._Ny, self._Nz
        cx, cy, cz = self.C_mur_x, self.C_mur_y, self.C_mur_z

        def face(f, p, dim, at, inner, c):
            # dim 0/1/2 = x/y/z, counted among the last three axes
            sl = lambda idx: (Ellipsis,) + (slice(None),) * dim + (idx,) + (slice(None),) * (2 - dim)
            f[sl(at)] = p[sl(inner)] + c * (f[sl(inner)] - p[sl(at)])

        for f, p in ((Hy, self.Hy_prev), (Hz, self.Hz_prev)):
            face(f, p, 0, 0, 1, cx)
        for f, p in ((Hy, self.Hy_prev), (Hz, self.Hz_prev)):
            face(f, p, 0, nx - 1, nx - 2, cx)
        for f, p in ((Hx, self.Hx_prev), (Hz, self.Hz_prev)):
            face(f, p, 1, 0, 1, cy)
        for f, p in ((Hx, self.Hx_prev), (Hz, self.Hz_prev)):
            face(f, p, 1, ny - 1, ny - 2, cy)
        if nz > 1:
            for f, p in ((Hx, self.Hx_prev), (Hy, self.Hy_prev)):
                face(f, p, 2, 0, 1, cz)
            for f, p in ((Hx, self.Hx_prev), (Hy, self.Hy_prev)):
                face(f, p, 2, nz - 1, nz - 2, cz)

    n_boundary_cells = property(lambda s: 2 * (s._Nx * s._Ny + s._Ny * s._Nz + s._Nx * s._Nz))
    mur_coefficient_x = property(lambda s: s.C_mur_x)
    mur_coefficient_y = property(lambda s: s.C_mur_y)
    mur_coefficient_z = property(lambda s: s.C_mur_z)

    def __repr__(self) -> str:
        return (f"MurABC3D(shape=({self._Nx}, {self._Ny}, {self._Nz}), C_mur_x={self.C_mur_x:.6f}, "
                f"C_mur_y={self.C_mur_y:.6f}, C_mur_z={self.C_mur_z:.6f}, "
                f"n_boundary_cells={self.n_boundary_cells})")


class CPML:
    """Convolutional PML of ``depth`` cells on every side of a 2D TM grid, for
    ``FDTD2D(grid, fields, CPML(grid, depth), ...)`` in place of ``MurABC``.

    New: the reference computes these graded profiles (``_compute_pml_coeffs``,
    src/core/boundaries.py:32-112, stored by ``MurABC(pml_depth=...)``) but no
    engine applies them, so ``MurABC(pml_depth=...)`` keeps the reference's
    Mur behaviour and this separate class runs the layer.  Same profile
    (cubic grading, R = 1e-8, kappa_max = 5, alpha_max = 0.05 by default);
    the coefficients (b, c, 1/kappa) are sampled at every position of each
    axis -- integer cells for the E updates, half cells for Hz -- at depth
    rho = (D - x) / D on the low side and (x - (n - 1 - D)) / D on the high
    side.  ``psi`` holds the layers' convolution memories (4 D (Nx + Ny)
    floats) and is zeroed by ``reset``."""

    is_cpml = True

    def __init__(self, grid: YeeGrid, depth: int = 10, *, R: float = 1e-8, m: int = 3,
                 kappa_max: float = 5.0, alpha_max: float = 0.05) -> None:
        if grid.Nz != 1:
            raise ValueError("CPML is implemented for 2D grids (Nz = 1)")
        if depth < 1 or 2 * depth + 2 > min(grid.Nx, grid.Ny):
            raise ValueError(f"a {depth}-cell layer per side does not fit a "
                             f"{grid.Nx}x{grid.Ny} grid")
        self._Nx, self._Ny = grid.Nx, grid.Ny
        self.depth = depth
        self._params = (R, m, kappa_max, alpha_max)
        dt = grid.dt
        tx = self.profile(grid.Nx, grid.dx, dt)
        ty = self.profile(grid.Ny, grid.dy, dt)
        self.tables = torch.tensor(tx + ty, dtype=torch.float32).to(grid.device)
        self.psi = torch.zeros(4 * depth * (grid.Nx + grid.Ny), dtype=torch.float32,
                               device=grid.device)

    def profile(self, n: int, d: float, dt: float) -> list:
        """[b_E, c_E, 1/kappa_E, b_H, c_H, 1/kappa_H] over the n positions of
        one axis (float64, rounded to float32 by the caller); positions
        outside the layer read as (1, 0, 1)."""
        R, m, kmax, amax = self._params
        D = self.depth
        smax = (m + 1) * math.log(1.0 / R) / (2.0 * ETA0 * D * d)
        out = [[], [], [], [], [], []]
        for half, base in ((0.0, 0), (0.5, 3)):
            for i in range(n):
                x = i + half
                rho = max((D - x) / D, (x - (n - 1 - D)) / D, 0.0)
                if rho <= 0.0 or (half and i > n - 2):
                    b, c, ik = 1.0, 0.0, 1.0
                else:
                    rho = min(rho, 1.0)
                    _, b, c = _pml_bsigma_at_rho(rho, smax, kmax, amax, m, dt)
                    ik = 1.0 / (1.0 + (kmax - 1.0) * rho ** m)
                out[base].append(b)
                out[base + 1].append(c)
                out[base + 2].append(ik)
        return [v for col in out for v in col]

    def reset(self) -> None:
        self.psi.zero_()

    def __repr__(self) -> str:
        return f"CPML(grid=({self._Nx}, {self._Ny}), depth={self.depth})"
