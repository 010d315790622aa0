"""CPU restatement of the reference Yee-FDTD time loop (test infrastructure only).

Follows, operation for operation and in the same order, the reference
project's PyTorch-eager update so that float32 results are bit-identical to
the reference run on CPU:

* CFL time step ............ src/core/grid.py:120-169
* Ca/Cb material coefficients src/core/materials.py:61-82
* waveform tables .......... src/core/sources.py:112-138 (t = arange(N)*dt),
                             GaussianPulse :245-248, RickerWavelet :398-402
* soft point/line injection  src/core/sources.py:863-887, :1015-1035
* plane injection .......... src/core/sources.py:730-749
* 2D step .................. src/core/fdtd2d.py:187-266
* 2D Mur ABC ............... src/core/boundaries.py:230-274
* 3D step .................. src/core/fdtd3d.py:261-402
* 3D Mur ABC ............... src/core/boundaries.py:488-583
* stability check .......... src/core/fdtd2d.py:268-295, fdtd3d.py:421-451
* detector gather after each full step: examples/brain_mimo_imaging.py:193-201

The oracle works on plain 2D ``(Nx, Ny)`` / 3D ``(Nx, Ny, Nz)`` CPU tensors and
does not import the ``waveforge_b200`` package.
"""

from __future__ import annotations

import math
from typing import Optional, Sequence

import torch

EPS0 = 8.8541878128e-12   # src/core/fdtd2d.py:40
MU0 = 1.2566370614e-6     # src/core/fdtd2d.py:41
C0 = 299_792_458.0        # src/core/grid.py:23 / boundaries.py:22

COMPONENTS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def stable_dt(dx: float, dy: float, dz: Optional[float] = None, courant: float = 0.98) -> float:
    """CFL time step, src/core/grid.py:120-169 (Python float64)."""
    s = (1.0 / dx) ** 2 + (1.0 / dy) ** 2
    if dz is not None:
        s += (1.0 / dz) ** 2
    return courant / (C0 * math.sqrt(s))


def material_ca_cb(eps_r: float, sigma: float, dt: float) -> tuple[float, float]:
    """Semi-implicit lossy coefficients, src/core/materials.py:61-82."""
    a = sigma * dt / (2.0 * EPS0 * eps_r)
    return (1.0 - a) / (1.0 + a), (dt / (EPS0 * eps_r)) / (1.0 + a)


def _time_axis(n: int, dt: float, dtype) -> torch.Tensor:
    # src/core/sources.py:136-137
    return torch.arange(n, dtype=dtype) * dt


def gaussian_wave(n: int, dt: float, amplitude: float, sigma: float, t0: float,
                  dtype=torch.float32) -> torch.Tensor:
    """GaussianPulse table, src/core/sources.py:245-248."""
    t = _time_axis(n, dt, dtype)
    e = -((t - t0) ** 2) / (2.0 * sigma ** 2)
    return amplitude * torch.exp(e)


def ricker_wave(n: int, dt: float, amplitude: float, fp: float, t0: float,
                dtype=torch.float32) -> torch.Tensor:
    """RickerWavelet table, src/core/sources.py:398-402."""
    t = _time_axis(n, dt, dtype)
    k = (math.pi * fp) ** 2
    u = k * (t - t0) ** 2
    return amplitude * (1.0 - 2.0 * u) * torch.exp(-u)


def gauss_deriv_wave(n: int, dt: float, fc: float = 1e9, amplitude: float = 1.0,
                     dtype=torch.float32) -> torch.Tensor:
    """Gaussian-derivative pulse of the benchmark configurations.

    f(t) = -A*((t-t0)/tau)*exp(-((t-t0)/tau)^2/2), tau = 1/(2*pi*fc), t0 = 3*tau.
    The reference has no class for exactly this pulse; the product's
    ``GaussianDerivativePulse`` evaluates the same expression in the same order.
    """
    tau = 1.0 / (2.0 * math.pi * fc)
    t0 = 3.0 * tau
    t = _time_axis(n, dt, dtype)
    u = (t - t0) / tau
    return amplitude * (-u) * torch.exp(-0.5 * (u * u))


class _Src:
    """One soft source: ``field[cells] += wave[n] * amp`` (sources.py:863-887)."""

    def __init__(self, comp, idx, wave, amp=None, plane=None):
        self.comp = comp
        self.idx = idx          # tuple of index tensors / ints
        self.wave = wave
        self.amp = amp          # tensor of per-cell weights or None (point: 1.0)
        self.plane = plane      # (axis, position) for plane sources


class _OracleBase:
    dims = 2

    def __init__(self, dtype):
        self.dtype = dtype
        self.sources: list[_Src] = []
        self.n = 0
        self.threshold = 1e10
        self.n_check = 10 ** 9
        self.last_field_max = -1.0

    # -- sources --------------------------------------------------------
    def add_point_source(self, comp: str, i: int, j: int, wave: torch.Tensor, k: int = 0):
        """PointSource: amplitude tensor 1.0, values = w[n:n+1]*amp (sources.py:882-887)."""
        cell = (i, j) if self.dims == 2 else (i, j, k)
        idx = tuple(torch.tensor([v]) for v in cell)   # index tensors, as sources.py:882-884
        self.sources.append(_Src(comp, idx, wave.to(self.dtype),
                                 torch.ones(1, dtype=self.dtype)))

    def add_line_source(self, comp: str, axis: str, position: int, start: int, stop: int,
                        wave: torch.Tensor, amp: Optional[torch.Tensor] = None):
        """LineSource along x (vary i) or y (vary j) at k=0, sources.py:960-1035."""
        n = stop - start
        rng = torch.arange(start, stop)
        fixed = torch.full((n,), position, dtype=torch.long)
        ii, jj = (rng, fixed) if axis == "x" else (fixed, rng)
        idx = (ii, jj) if self.dims == 2 else (ii, jj, torch.zeros(n, dtype=torch.long))
        a = torch.ones(n, dtype=self.dtype) if amp is None else amp.to(self.dtype)
        self.sources.append(_Src(comp, idx, wave.to(self.dtype), a))

    def add_box_source(self, comp: str, box: tuple, wave: torch.Tensor,
                       amp: Optional[torch.Tensor] = None):
        """Every cell of the half-open box gets ``w[n]`` (amp None, the point /
        plane case: ``w*1.0 == w``) or ``w[n]*amp[c]`` with c the row-major
        offset inside the box (the line case)."""
        rngs = [torch.arange(box[2 * a], box[2 * a + 1]) for a in range(self.dims)]
        mesh = torch.meshgrid(*rngs, indexing="ij")
        idx = tuple(m.reshape(-1) for m in mesh)
        n = idx[0].numel()
        a = torch.ones(n, dtype=self.dtype) if amp is None else amp.to(self.dtype).reshape(-1)
        self.sources.append(_Src(comp, idx, wave.to(self.dtype), a))

    def add_plane_source(self, comp: str, plane: str, position: int, wave: torch.Tensor):
        """PlaneSource, scalar w[n] broadcast over the plane, sources.py:730-749."""
        self.sources.append(_Src(comp, None, wave.to(self.dtype), None, (plane, position)))

    def _inject(self):
        n = self.n
        for s in self.sources:
            f = getattr(self, s.comp)
            if s.plane is not None:
                plane, pos = s.plane
                w = s.wave[n]
                if plane == "xy":
                    f[..., :, :, pos] += w
                elif plane == "xz":
                    f[..., :, pos, :] += w
                else:
                    f[..., pos, :, :] += w
                continue
            vals = s.wave[n:n + 1] * s.amp
            f[s.idx] += vals

    def _stability(self, names):
        self.n_check_count = getattr(self, "n_check_count", 0) + 1
        for name in names:
            v = float(getattr(self, name).abs().max().item())
            if v > self.last_field_max:
                self.last_field_max = v
            if v > self.threshold:
                raise RuntimeError(f"diverged at step {self.n}: {name} max = {v:.3e}")

    def run(self, nsteps: int, probes: Sequence[tuple] = ()) -> torch.Tensor:
        """Advance ``nsteps`` and gather ``(comp, i, j[, k])`` after each full step."""
        tr = torch.zeros(len(probes), nsteps, dtype=self.dtype)
        for s in range(nsteps):
            self.step()
            for r, p in enumerate(probes):
                tr[r, s] = getattr(self, p[0])[tuple(p[1:])]
        return tr


class Oracle2D(_OracleBase):
    """2D TM {Ex, Ey, Hz} leapfrog, src/core/fdtd2d.py:187-266."""

    dims = 2

    def __init__(self, nx: int, ny: int, dx: float, dy: float, dt: float,
                 ca: Optional[torch.Tensor] = None, cb: Optional[torch.Tensor] = None,
                 dtype=torch.float32):
        super().__init__(dtype)
        self.nx, self.ny = nx, ny
        self.dx, self.dy, self.dt = dx, dy, dt
        self.Ex = torch.zeros(nx, ny, dtype=dtype)
        self.Ey = torch.zeros(nx, ny, dtype=dtype)
        self.Hz = torch.zeros(nx, ny, dtype=dtype)
        self.dh = dt / MU0                                   # fdtd2d.py:158
        self.de = dt / EPS0                                  # fdtd2d.py:159
        self.cmx = (C0 * dt - dx) / (C0 * dt + dx)          # boundaries.py:177
        self.cmy = (C0 * dt - dy) / (C0 * dt + dy)          # boundaries.py:178
        self.ca = None if ca is None else ca.reshape(nx, ny).to(dtype)
        self.cb = None if cb is None else cb.reshape(nx, ny).to(dtype)

    def step(self):
        Ex, Ey, Hz = self.Ex, self.Ey, self.Hz
        dx, dy = self.dx, self.dy
        hp = Hz.clone()                                      # boundaries.py:237 (before injection)
        self._inject()                                       # fdtd2d.py:226-228
        # Faraday, fdtd2d.py:232-235
        Hz[:-1, :-1] += self.dh * ((Ex[:-1, 1:] - Ex[:-1, :-1]) / dy
                                   - (Ey[1:, :-1] - Ey[:-1, :-1]) / dx)
        # Mur, x edges then y edges, boundaries.py:259-274
        nx, ny = self.nx, self.ny
        cx, cy = self.cmx, self.cmy
        Hz[0, :] = hp[1, :] + cx * (Hz[1, :] - hp[0, :])
        Hz[nx - 1, :] = hp[nx - 2, :] + cx * (Hz[nx - 2, :] - hp[nx - 1, :])
        Hz[:, 0] = hp[:, 1] + cy * (Hz[:, 1] - hp[:, 0])
        Hz[:, ny - 1] = hp[:, ny - 2] + cy * (Hz[:, ny - 2] - hp[:, ny - 1])
        # Ampere, fdtd2d.py:244-257
        dhz_dy = (Hz[:, 1:] - Hz[:, :-1]) / dy
        dhz_dx = (Hz[1:, :] - Hz[:-1, :]) / dx
        if self.ca is None:
            Ex[:, 1:] += self.de * dhz_dy
            Ey[1:, :] -= self.de * dhz_dx
        else:
            Ex[:, 1:] = self.ca[:, 1:] * Ex[:, 1:] + self.cb[:, 1:] * dhz_dy
            Ey[1:, :] = self.ca[1:, :] * Ey[1:, :] - self.cb[1:, :] * dhz_dx
        self.n += 1
        if self.n % self.n_check == 0:
            self._stability(("Ex", "Ey", "Hz"))


class Oracle3D(_OracleBase):
    """3D six-component leapfrog, src/core/fdtd3d.py:261-402."""

    dims = 3

    def __init__(self, nx: int, ny: int, nz: int, dx: float, dy: float, dz: float, dt: float,
                 ca: Optional[torch.Tensor] = None, cb: Optional[torch.Tensor] = None,
                 dtype=torch.float32):
        super().__init__(dtype)
        self.nx, self.ny, self.nz = nx, ny, nz
        self.dx, self.dy, self.dz, self.dt = dx, dy, dz, dt
        for c in COMPONENTS:
            setattr(self, c, torch.zeros(nx, ny, nz, dtype=dtype))
        self.dh = dt / MU0
        self.de = dt / EPS0
        self.cmx = (C0 * dt - dx) / (C0 * dt + dx)
        self.cmy = (C0 * dt - dy) / (C0 * dt + dy)
        self.cmz = (C0 * dt - dz) / (C0 * dt + dz)
        self.ca = None if ca is None else ca.reshape(nx, ny, nz).to(dtype)
        self.cb = None if cb is None else cb.reshape(nx, ny, nz).to(dtype)

    def step(self):
        Ex, Ey, Ez, Hx, Hy, Hz = (self.Ex, self.Ey, self.Ez, self.Hx, self.Hy, self.Hz)
        dx, dy, dz, dh, de = self.dx, self.dy, self.dz, self.dh, self.de
        hxp, hyp, hzp = Hx.clone(), Hy.clone(), Hz.clone()  # boundaries.py:495-497
        self._inject()
        # Faraday, fdtd3d.py:312-331
        Hx[:, :-1, :-1] += dh * ((Ey[:, :-1, 1:] - Ey[:, :-1, :-1]) / dz
                                 - (Ez[:, 1:, :-1] - Ez[:, :-1, :-1]) / dy)
        Hy[:-1, :, :-1] += dh * ((Ez[1:, :, :-1] - Ez[:-1, :, :-1]) / dx
                                 - (Ex[:-1, :, 1:] - Ex[:-1, :, :-1]) / dz)
        Hz[:-1, :-1, :] += dh * ((Ex[:-1, 1:, :] - Ex[:-1, :-1, :]) / dy
                                 - (Ey[1:, :-1, :] - Ey[:-1, :-1, :]) / dx)
        # Mur faces x -> y -> z, boundaries.py:523-583
        nx, ny, nz = self.nx, self.ny, self.nz
        cx, cy, cz = self.cmx, self.cmy, self.cmz
        Hy[0] = hyp[1] + cx * (Hy[1] - hyp[0])
        Hz[0] = hzp[1] + cx * (Hz[1] - hzp[0])
        Hy[nx - 1] = hyp[nx - 2] + cx * (Hy[nx - 2] - hyp[nx - 1])
        Hz[nx - 1] = hzp[nx - 2] + cx * (Hz[nx - 2] - hzp[nx - 1])
        Hx[:, 0] = hxp[:, 1] + cy * (Hx[:, 1] - hxp[:, 0])
        Hz[:, 0] = hzp[:, 1] + cy * (Hz[:, 1] - hzp[:, 0])
        Hx[:, ny - 1] = hxp[:, ny - 2] + cy * (Hx[:, ny - 2] - hxp[:, ny - 1])
        Hz[:, ny - 1] = hzp[:, ny - 2] + cy * (Hz[:, ny - 2] - hzp[:, ny - 1])
        if nz > 1:
            Hx[:, :, 0] = hxp[:, :, 1] + cz * (Hx[:, :, 1] - hxp[:, :, 0])
            Hy[:, :, 0] = hyp[:, :, 1] + cz * (Hy[:, :, 1] - hyp[:, :, 0])
            Hx[:, :, nz - 1] = hxp[:, :, nz - 2] + cz * (Hx[:, :, nz - 2] - hxp[:, :, nz - 1])
            Hy[:, :, nz - 1] = hyp[:, :, nz - 2] + cz * (Hy[:, :, nz - 2] - hyp[:, :, nz - 1])
        # Ampere, fdtd3d.py:356-393
        cex = (Hz[:, 1:, 1:] - Hz[:, :-1, 1:]) / dy - (Hy[:, 1:, 1:] - Hy[:, 1:, :-1]) / dz
        cey = (Hx[1:, :, 1:] - Hx[1:, :, :-1]) / dz - (Hz[1:, :, 1:] - Hz[:-1, :, 1:]) / dx
        cez = (Hy[1:, 1:, :] - Hy[:-1, 1:, :]) / dx - (Hx[1:, 1:, :] - Hx[1:, :-1, :]) / dy
        if self.ca is None:
            Ex[:, 1:, 1:] += de * cex
            Ey[1:, :, 1:] += de * cey
            Ez[1:, 1:, :] += de * cez
        else:
            ca, cb = self.ca, self.cb
            Ex[:, 1:, 1:] = ca[:, 1:, 1:] * Ex[:, 1:, 1:] + cb[:, 1:, 1:] * cex
            Ey[1:, :, 1:] = ca[1:, :, 1:] * Ey[1:, :, 1:] + cb[1:, :, 1:] * cey
            Ez[1:, 1:, :] = ca[1:, 1:, :] * Ez[1:, 1:, :] + cb[1:, 1:, :] * cez
        self.n += 1
        if self.n % self.n_check == 0:
            self._stability(COMPONENTS)
