"""Waveforms and soft-source injectors (mirror of src/core/sources.py).

Waveform tables are evaluated once on the host in the grid dtype with the same
tensor expressions as the reference (src/core/sources.py:112-138 and each
``_compute``), then moved to the device.  Injectors keep the reference API
(``step(fields_dict, n)`` for manual stepping) and additionally describe
themselves to the CUDA engine as ``wf_source`` boxes (``native_boxes``), which
the fused kernels apply at the start of every step, before the H update.
"""

from __future__ import annotations

import math
import warnings
from abc import ABC, abstractmethod
from typing import Union

import torch

from .grid import YeeGrid

VALID_COMPONENTS: tuple[str, ...] = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


class Waveform(ABC):
    """Pre-computed source waveform (src/core/sources.py:64-155)."""

    @abstractmethod
    def _compute(self, t: torch.Tensor) -> torch.Tensor: ...

    @property
    @abstractmethod
    def peak_time(self) -> float | None: ...

    @property
    @abstractmethod
    def bandwidth(self) -> float: ...

    @property
    @abstractmethod
    def amplitude(self) -> float: ...

    def build(self, N_steps: int, dt: float, device: torch.device,
              dtype: torch.dtype = torch.float32) -> torch.Tensor:
        """``f(arange(N)*dt)`` of length N_steps.  Evaluated on the host CPU
        (the reference CPU arithmetic) and then placed on ``device``."""
        t = torch.arange(N_steps, dtype=dtype) * dt
        return self._compute(t).to(device)

    def is_causal(self, dt: float) -> bool:
        f0 = float(self._compute(torch.tensor([0.0], dtype=torch.float32)).item())
        return abs(f0) / abs(self.amplitude) < 1e-4


class GaussianPulse(Waveform):
    """A*exp(-(t-t0)^2/(2 sigma^2)) (src/core/sources.py:163-256)."""

    def __init__(self, amplitude: float = 1.0, t0: float | None = None, sigma: float | None = None,
                 *, freq: float | None = None) -> None:
        if amplitude == 0:
            raise ValueError("amplitude must be non-zero.")
        if freq is not None and sigma is not None:
            raise ValueError("Provide either freq or sigma, not both.")
        if freq is not None:
            if freq <= 0:
                raise ValueError(f"freq must be > 0, got {freq!r}")
            sigma = 1.0 / (2.0 * math.pi * freq / 3.0)
        if sigma is None:
            raise ValueError("Either sigma or freq must be supplied.")
        if sigma <= 0:
            raise ValueError(f"sigma must be > 0, got {sigma!r}")
        if t0 is None:
            t0 = 5.0 * sigma
        if t0 <= 0:
            raise ValueError(f"t0 must be > 0, got {t0!r}")
        self._amplitude, self._sigma, self._t0 = float(amplitude), float(sigma), float(t0)
        if not self.is_causal(0.0):
            warnings.warn(f"GaussianPulse: |f(0)|/|A| >= 1e-4 — waveform is not causal. Consider "
                          f"increasing t0 (currently {self._t0:.4g} s) relative to sigma "
                          f"({self._sigma:.4g} s).", UserWarning, stacklevel=2)

    def _compute(self, t):
        e = -((t - self._t0) ** 2) / (2.0 * self._sigma ** 2)
        return self._amplitude * torch.exp(e)

    peak_time = property(lambda s: s._t0)
    bandwidth = property(lambda s: 1.0 / (2.0 * math.pi * s._sigma))
    amplitude = property(lambda s: s._amplitude)


class SinusoidalSource(Waveform):
    """A*sin(2 pi f0 t + phi)*(1-exp(-t/tau)) (src/core/sources.py:264-336)."""

    def __init__(self, amplitude: float = 1.0, frequency: float = 1e9, phase: float = 0.0) -> None:
        if amplitude == 0:
            raise ValueError("amplitude must be non-zero.")
        if frequency <= 0:
            raise ValueError(f"frequency must be > 0, got {frequency!r}")
        self._amplitude, self._frequency, self._phase = float(amplitude), float(frequency), float(phase)
        self._tau_ramp = 3.0 / (2.0 * math.pi * self._frequency)
        if phase != 0.0 and abs(math.sin(phase)) >= 1e-4:
            warnings.warn(f"SinusoidalSource: phase={phase:.4g} rad gives "
                          f"|sin(phi)|={abs(math.sin(phase)):.4g} >= 1e-4 — source is not causal "
                          "at t=0.", UserWarning, stacklevel=2)

    def _compute(self, t):
        omega = 2.0 * math.pi * self._frequency
        return self._amplitude * torch.sin(omega * t + self._phase) * (1.0 - torch.exp(-t / self._tau_ramp))

    peak_time = property(lambda s: -1.0)
    bandwidth = property(lambda s: 0.0)
    amplitude = property(lambda s: s._amplitude)


class RickerWavelet(Waveform):
    """A*(1-2u)*exp(-u), u = (pi fp (t-t0))^2 (src/core/sources.py:344-418)."""

    def __init__(self, amplitude: float = 1.0, peak_freq: float = 1e9, t0: float | None = None) -> None:
        if amplitude == 0:
            raise ValueError("amplitude must be non-zero.")
        if peak_freq <= 0:
            raise ValueError(f"peak_freq must be > 0, got {peak_freq!r}")
        if t0 is None:
            t0 = 1.5 / peak_freq
        if t0 <= 0:
            raise ValueError(f"t0 must be > 0, got {t0!r}")
        self._amplitude, self._peak_freq, self._t0 = float(amplitude), float(peak_freq), float(t0)
        if not self.is_causal(0.0):
            warnings.warn(f"RickerWavelet: |f(0)|/|A| >= 1e-4 — waveform is not causal. Consider "
                          f"increasing t0 (currently {self._t0:.4g} s) relative to 1/peak_freq "
                          f"({1.0 / self._peak_freq:.4g} s).", UserWarning, stacklevel=2)

    def _compute(self, t):
        k = (math.pi * self._peak_freq) ** 2
        u = k * (t - self._t0) ** 2
        return self._amplitude * (1.0 - 2.0 * u) * torch.exp(-u)

    peak_time = property(lambda s: s._t0)
    bandwidth = property(lambda s: s._peak_freq)
    amplitude = property(lambda s: s._amplitude)


class ModulatedGaussian(Waveform):
    """A*sin(2 pi fc t + phi)*exp(-(t-t0)^2/(2 sigma^2)) (src/core/sources.py:426-483)."""

    def __init__(self, amplitude: float = 1.0, fc: float = 1e9, sigma: float | None = None,
                 t0: float | None = None, phi: float = 0.0) -> None:
        if amplitude == 0:
            raise ValueError("amplitude must be non-zero.")
        if fc <= 0:
            raise ValueError(f"fc must be > 0, got {fc!r}")
        if sigma is None:
            raise ValueError("sigma must be supplied.")
        if sigma <= 0:
            raise ValueError(f"sigma must be > 0, got {sigma!r}")
        if t0 is None:
            t0 = 5.0 * sigma
        if t0 <= 0:
            raise ValueError(f"t0 must be > 0, got {t0!r}")
        self._amplitude, self._fc, self._sigma = float(amplitude), float(fc), float(sigma)
        self._t0, self._phi = float(t0), float(phi)
        if not self.is_causal(0.0):
            warnings.warn(f"ModulatedGaussian: |f(0)|/|A| >= 1e-4 — waveform is not causal. With "
                          f"phi={self._phi:.4g} rad, consider increasing t0 (currently "
                          f"{self._t0:.4g} s) to >= 5*sigma ({5.0 * self._sigma:.4g} s).",
                          UserWarning, stacklevel=2)

    def _compute(self, t):
        carrier = torch.sin(2.0 * math.pi * self._fc * t + self._phi)
        envelope = torch.exp(-((t - self._t0) ** 2) / (2.0 * self._sigma ** 2))
        return self._amplitude * carrier * envelope

    peak_time = property(lambda s: s._t0)
    bandwidth = property(lambda s: 1.0 / (2.0 * math.pi * s._sigma))
    amplitude = property(lambda s: s._amplitude)


class Chirp(Waveform):
    """Hann-windowed linear sweep (src/core/sources.py:491-546)."""

    def __init__(self, amplitude: float = 1.0, f_start: float = 1e8, f_end: float = 1e9,
                 t_start: float = 0.0, t_end: float | None = None, phi: float = 0.0) -> None:
        if amplitude == 0:
            raise ValueError("amplitude must be non-zero.")
        if f_start <= 0:
            raise ValueError(f"f_start must be > 0, got {f_start!r}")
        if f_end <= 0:
            raise ValueError(f"f_end must be > 0, got {f_end!r}")
        if t_start < 0:
            raise ValueError(f"t_start must be >= 0, got {t_start!r}")
        if t_end is None:
            t_end = t_start + 10.0 / f_start
        if t_end <= t_start:
            raise ValueError(f"t_end ({t_end!r}) must be > t_start ({t_start!r})")
        self._amplitude, self._f_start, self._f_end = float(amplitude), float(f_start), float(f_end)
        self._t_start, self._t_end, self._phi = float(t_start), float(t_end), float(phi)
        self._duration = self._t_end - self._t_start

    def _compute(self, t):
        inside = (t >= self._t_start) & (t <= self._t_end)
        tau = t - self._t_start
        k = (self._f_end - self._f_start) / (2.0 * self._duration)
        phase = 2.0 * math.pi * (self._f_start * tau + k * tau ** 2) + self._phi
        hann = 0.5 * (1.0 - torch.cos(2.0 * math.pi * tau / self._duration))
        out = self._amplitude * torch.sin(phase) * hann
        return torch.where(inside, out, torch.zeros_like(out))

    peak_time = property(lambda s: (s._t_start + s._t_end) / 2.0)
    bandwidth = property(lambda s: abs(s._f_end - s._f_start))
    amplitude = property(lambda s: s._amplitude)


class UWBPulse(Waveform):
    """Peak-normalised Gaussian monocycle (src/core/sources.py:554-663)."""

    def __init__(self, amplitude: float = 1.0, f_low: float = 1e9, f_high: float = 3e9,
                 t0: float | None = None) -> None:
        if amplitude == 0:
            raise ValueError("amplitude must be non-zero.")
        if f_low <= 0:
            raise ValueError(f"f_low must be > 0, got {f_low!r}")
        if f_high <= f_low:
            raise ValueError(f"f_high must be > f_low, got f_low={f_low!r}, f_high={f_high!r}")
        self._amplitude, self._f_low, self._f_high = float(amplitude), float(f_low), float(f_high)
        self._fc = (f_low + f_high) / 2.0
        self._sigma = 1.0 / (math.sqrt(2.0) * math.pi * self._fc)
        self._norm = self._sigma * math.sqrt(math.e)
        self._t0 = float(t0) if t0 is not None else 6.0 * self._sigma
        if not self.is_causal(0.0):
            warnings.warn(f"UWBPulse: |f(0)|/|A| >= 1e-4 — waveform may not be causal. Consider "
                          f"increasing t0 (currently {self._t0:.4g} s) to >= 5*sigma "
                          f"({5.0 * self._sigma:.4g} s).", UserWarning, stacklevel=2)

    def _compute(self, t):
        tau = t - self._t0
        g = torch.exp(-(tau ** 2) / (2.0 * self._sigma ** 2))
        return self._amplitude * self._norm * (-(tau / self._sigma ** 2) * g)

    fc = property(lambda s: s._fc)
    f_low = property(lambda s: s._f_low)
    f_high = property(lambda s: s._f_high)
    peak_time = property(lambda s: s._t0)
    bandwidth = property(lambda s: s._f_high - s._f_low)
    amplitude = property(lambda s: s._amplitude)


class GaussianDerivativePulse(Waveform):
    """Gaussian-derivative pulse f(t) = -A*u*exp(-u^2/2), u = (t-t0)/tau,
    tau = 1/(2 pi fc), t0 = 3 tau: the excitation of the benchmark workloads.
    The reference has no class for exactly this pulse (its ``UWBPulse`` uses a
    different sigma, t0 and normalisation); with t0 = 3 tau it is intentionally
    not causal by the 1e-4 rule, so no causality warning is raised."""

    def __init__(self, fc: float = 1e9, amplitude: float = 1.0, t0: float | None = None) -> None:
        if amplitude == 0:
            raise ValueError("amplitude must be non-zero.")
        if fc <= 0:
            raise ValueError(f"fc must be > 0, got {fc!r}")
        self._fc, self._amplitude = float(fc), float(amplitude)
        self._tau = 1.0 / (2.0 * math.pi * self._fc)
        self._t0 = 3.0 * self._tau if t0 is None else float(t0)

    def _compute(self, t):
        u = (t - self._t0) / self._tau
        return self._amplitude * (-u) * torch.exp(-0.5 * (u * u))

    peak_time = property(lambda s: s._t0 - s._tau)
    bandwidth = property(lambda s: s._fc)
    amplitude = property(lambda s: s._amplitude)


class TabulatedWaveform(Waveform):
    """A waveform given as an explicit table (values for steps 0..N-1)."""

    def __init__(self, values: torch.Tensor) -> None:
        self._values = torch.as_tensor(values).detach().cpu()
        if self._values.ndim != 1 or self._values.numel() == 0:
            raise ValueError("values must be a non-empty 1-D tensor")
        self._amp = float(self._values.abs().max().item()) or 1.0

    def build(self, N_steps, dt, device, dtype=torch.float32):
        if N_steps > self._values.numel():
            raise ValueError(f"table has {self._values.numel()} entries, {N_steps} requested")
        return self._values[:N_steps].to(dtype).to(device)

    def _compute(self, t):
        raise NotImplementedError("TabulatedWaveform is defined by its table")

    def is_causal(self, dt):
        return abs(float(self._values[0])) / self._amp < 1e-4

    peak_time = property(lambda s: -1.0)
    bandwidth = property(lambda s: 0.0)
    amplitude = property(lambda s: s._amp)


# ---------------------------------------------------------------------------
# Injectors
# ---------------------------------------------------------------------------

class _Injector:
    """Common bits: component, waveform table, native box description."""

    _component: str
    _waveform_tensor: torch.Tensor
    _N_steps: int

    @property
    def waveform_memory_bytes(self) -> int:
        return self._N_steps * self._waveform_tensor.element_size()

    @property
    def is_precomputed(self) -> bool:
        return True

    @property
    def component(self) -> str:
        return self._component

    @property
    def n_steps(self) -> int:
        return self._N_steps

    def native_boxes(self) -> list[tuple]:
        """``(comp, i0, i1, j0, j1, k0, k1, wave, amp_or_None)`` boxes."""
        raise NotImplementedError


class PlaneSource(_Injector):
    """Soft source over a whole xy/xz/yz plane (src/core/sources.py:671-766)."""

    def __init__(self, waveform: Waveform, plane: str, position: int, component: str = "Hz", *,
                 grid: YeeGrid, N_steps: int) -> None:
        if component not in VALID_COMPONENTS:
            raise ValueError(f"component must be one of {VALID_COMPONENTS}, got {component!r}")
        if plane not in ("xy", "xz", "yz"):
            raise ValueError(f"plane must be 'xy', 'xz', or 'yz', got {plane!r}")
        limit, n_cells = {"xy": (grid.Nz, grid.Nx * grid.Ny), "xz": (grid.Ny, grid.Nx * grid.Nz),
                          "yz": (grid.Nx, grid.Ny * grid.Nz)}[plane]
        if not (0 <= position < limit):
            raise ValueError(f"position={position} out of range [0, {limit}) for plane={plane!r}")
        self._component, self._plane, self._position = component, plane, position
        self._N_steps, self._n_cells = N_steps, n_cells
        self._grid_shape = (grid.Nx, grid.Ny, grid.Nz)
        self._waveform_tensor = waveform.build(N_steps, grid.dt, grid.device, grid.dtype)

    def step(self, fields_dict: dict[str, torch.Tensor], n: int) -> None:
        w = self._waveform_tensor[n]
        f = fields_dict[self._component]
        if self._plane == "xy":
            f[..., :, :, self._position] += w
        elif self._plane == "xz":
            f[..., :, self._position, :] += w
        else:
            f[..., self._position, :, :] += w

    def native_boxes(self):
        nx, ny, nz = self._grid_shape
        p = self._position
        box = {"xy": (0, nx, 0, ny, p, p + 1), "xz": (0, nx, p, p + 1, 0, nz),
               "yz": (p, p + 1, 0, ny, 0, nz)}[self._plane]
        return [(self._component, *box, self._waveform_tensor, None)]

    n_cells = property(lambda s: s._n_cells)
    plane = property(lambda s: s._plane)
    position = property(lambda s: s._position)


class PointSource(_Injector):
    """Single-cell soft source, field[i,j,k] += w[n] (src/core/sources.py:774-887)."""

    def __init__(self, waveform: Waveform, i: int, j: int, component: str = "Hz", *, k: int = 0,
                 grid: YeeGrid, N_steps: int) -> None:
        if component not in VALID_COMPONENTS:
            raise ValueError(f"component must be one of {VALID_COMPONENTS}, got {component!r}")
        if not (0 <= i < grid.Nx):
            raise ValueError(f"i={i} out of range [0, {grid.Nx})")
        if not (0 <= j < grid.Ny):
            raise ValueError(f"j={j} out of range [0, {grid.Ny})")
        if not (0 <= k < grid.Nz):
            raise ValueError(f"k={k} out of range [0, {grid.Nz})")
        self._component, self._N_steps = component, N_steps
        self._i, self._j, self._k = i, j, k
        self._waveform_tensor = waveform.build(N_steps, grid.dt, grid.device, grid.dtype)
        dev = grid.device
        self._i_idx = torch.tensor([i], dtype=torch.long, device=dev)
        self._j_idx = torch.tensor([j], dtype=torch.long, device=dev)
        self._k_idx = torch.tensor([k], dtype=torch.long, device=dev)
        self._amp = torch.tensor([1.0], dtype=grid.dtype, device=dev)

    n_cells = property(lambda s: 1)
    position = property(lambda s: (s._i, s._j, s._k))

    def step(self, fields_dict: dict[str, torch.Tensor], n: int) -> None:
        vals = self._waveform_tensor[n:n + 1] * self._amp
        fields_dict[self._component][..., self._i_idx, self._j_idx, self._k_idx] += vals

    def native_boxes(self):
        # w*1.0 == w exactly, so the point source needs no amplitude table.
        i, j, k = self._i, self._j, self._k
        return [(self._component, i, i + 1, j, j + 1, k, k + 1, self._waveform_tensor, None)]


def _validate_range(name: str, start: int, stop: int, limit: int) -> None:
    if start < 0 or stop > limit:
        raise ValueError(f"{name} range [{start}, {stop}) is out of grid bounds [0, {limit})")


def _validate_scalar_index(name: str, index: int, limit: int) -> None:
    if not (0 <= index < limit):
        raise ValueError(f"{name}={index} is out of grid bounds [0, {limit})")


class LineSource(_Injector):
    """Soft source along x or y at k=0 with optional per-cell weights
    (src/core/sources.py:895-1035)."""

    def __init__(self, waveform: Waveform, axis: str, position: int, start: int, stop: int,
                 component: str = "Hz", *, grid: YeeGrid, N_steps: int,
                 amplitude_profile: Union[torch.Tensor, list, None] = None) -> None:
        if axis not in ("x", "y"):
            raise ValueError(f"axis must be 'x' or 'y', got {axis!r}")
        if component not in VALID_COMPONENTS:
            raise ValueError(f"component must be one of {VALID_COMPONENTS}, got {component!r}")
        if start >= stop:
            raise ValueError(f"start ({start}) must be less than stop ({stop})")
        n = stop - start
        dev = grid.device
        if axis == "x":
            _validate_range("i", start, stop, grid.Nx)
            _validate_scalar_index("j (position)", position, grid.Ny)
            self._box = (start, stop, position, position + 1, 0, 1)
        else:
            _validate_range("j", start, stop, grid.Ny)
            _validate_scalar_index("i (position)", position, grid.Nx)
            self._box = (position, position + 1, start, stop, 0, 1)
        i0, i1, j0, j1, _, _ = self._box
        self._i_idx = torch.arange(i0, i1, device=dev).repeat_interleave(j1 - j0)
        self._j_idx = torch.arange(j0, j1, device=dev).repeat(i1 - i0)
        self._k_idx = torch.zeros(n, dtype=torch.long, device=dev)
        self._component, self._N_steps, self._n_cells = component, N_steps, n
        self._waveform_tensor = waveform.build(N_steps, grid.dt, grid.device, grid.dtype)
        if amplitude_profile is None:
            self._amp = torch.ones(n, dtype=grid.dtype, device=dev)
        else:
            a = torch.as_tensor(amplitude_profile, dtype=grid.dtype, device=dev)
            if a.shape != (n,):
                raise ValueError(f"amplitude_profile must have length {n}, got shape {tuple(a.shape)}")
            self._amp = a

    n_cells = property(lambda s: s._n_cells)

    def step(self, fields_dict: dict[str, torch.Tensor], n: int) -> None:
        vals = self._waveform_tensor[n:n + 1] * self._amp
        fields_dict[self._component][..., self._i_idx, self._j_idx, self._k_idx] += vals

    def native_boxes(self):
        return [(self._component, *self._box, self._waveform_tensor, self._amp)]


class SourceCollection:
    """Ordered sources stepped together (src/core/sources.py:1043-1090)."""

    def __init__(self, sources: list) -> None:
        self._sources = list(sources)

    def step(self, fields_dict: dict[str, torch.Tensor], n: int) -> None:
        for s in self._sources:
            s.step(fields_dict, n)

    @property
    def sources(self) -> list:
        return list(self._sources)

    @property
    def total_vram_bytes(self) -> int:
        return sum(s.waveform_memory_bytes for s in self._sources)

    @property
    def sources_graph_compatible(self) -> bool:
        return all(s.is_precomputed for s in self._sources)

    @property
    def n_injection_cells_total(self) -> int:
        return sum(s.n_cells for s in self._sources)
