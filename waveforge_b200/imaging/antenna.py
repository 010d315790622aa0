"""Antenna ring array: ring geometry, transmitter sources, device recording and
the layered-medium DAS image (drop-in for src/datasets/brain/antenna.py).

The reference records every receiver with one ``.item()`` host sync per
receiver per step (antenna.py:173-198) and builds its DAS image with Python
loops over antennas and pixels (:262-341).  Here ``record`` gathers on the
device without a sync, ``detectors()`` lets the fused step kernels record
all receivers (``sim.run(n, record=ring.detectors())`` then ``store``), and
``compute_das_image`` runs the travel-time table and the delay-and-sum on the
device (``wf_das_travel_times``, ``wf_das_envelope_image``): given the same
envelope both are bit-identical to the reference.  The Hilbert envelope is
the analytic-signal magnitude computed with a float64 FFT on the device (the
reference uses scipy's FFT; the envelopes agree to ~1e-7 relative).
"""

from __future__ import annotations

import ctypes
import math
from typing import Optional

import numpy as np
import torch

from .. import _native as nat
from ..core.sources import PointSource, SourceCollection
from ..detectors import Detectors


class AntennaRing:
    """Uniform circular array of N elements in the z = const plane
    (src/datasets/brain/antenna.py:37-101): each element transmits in turn
    and all receive."""

    def __init__(self, n_elements: int, ring_radius_cells: int, z_plane: int, grid,
                 centre: Optional[tuple[int, int]] = None, component: str = "Ez") -> None:
        if n_elements < 2:
            raise ValueError(f"n_elements must be >= 2, got {n_elements}")
        if not (0 < ring_radius_cells < min(grid.Nx, grid.Ny) // 2):
            raise ValueError(f"ring_radius_cells={ring_radius_cells} out of range for grid "
                             f"({grid.Nx}x{grid.Ny})")
        if not (0 <= z_plane < grid.Nz):
            raise ValueError(f"z_plane={z_plane} out of range [0, {grid.Nz})")
        self._n, self._r, self._z = n_elements, ring_radius_cells, z_plane
        self._grid = grid
        self._component = component
        cx = centre[0] if centre else grid.Nx // 2
        cy = centre[1] if centre else grid.Ny // 2
        self._cx, self._cy = cx, cy
        self._positions: list[tuple[int, int, int]] = []
        for k in range(n_elements):
            angle = 2.0 * math.pi * k / n_elements
            i = int(round(cx + ring_radius_cells * math.cos(angle)))
            j = int(round(cy + ring_radius_cells * math.sin(angle)))
            i = max(1, min(grid.Nx - 2, i))
            j = max(1, min(grid.Ny - 2, j))
            self._positions.append((i, j, z_plane))
        self._N_steps = 0
        self._signals: Optional[torch.Tensor] = None
        self._idx = None

    n_elements = property(lambda s: s._n)

    @property
    def positions(self) -> list[tuple[int, int, int]]:
        return list(self._positions)

    @property
    def positions_mm(self) -> list[tuple[float, float, float]]:
        dx = self._grid.dx * 1e3
        return [(i * dx, j * dx, k * dx) for i, j, k in self._positions]

    def _device(self) -> torch.device:
        dev = torch.device(self._grid.device)
        if dev.type != "cuda":
            raise RuntimeError("AntennaRing records and images on a CUDA device only")
        return dev

    # ------------------------------------------------------------------
    def build_sources(self, waveform, tx_idx: int, N_steps: int) -> SourceCollection:
        """One soft point source at element ``tx_idx`` (antenna.py:126-162)."""
        if not (0 <= tx_idx < self._n):
            raise ValueError(f"tx_idx={tx_idx} out of range [0, {self._n})")
        self._N_steps = N_steps
        if self._signals is None:
            self._signals = torch.zeros((self._n, self._n, N_steps), dtype=torch.float32,
                                        device=self._device())
        i, j, k = self._positions[tx_idx]
        return SourceCollection([PointSource(waveform, i, j, self._component, k=k,
                                             grid=self._grid, N_steps=N_steps)])

    def reset(self) -> None:
        if self._signals is not None:
            self._signals.zero_()

    def record(self, field: torch.Tensor, step: int, tx_idx: int) -> None:
        """Field at every receiver for this step (antenna.py:173-198), gathered
        on the device: no host sync per receiver."""
        if self._signals is None:
            raise RuntimeError("Call build_sources() before record().")
        if step >= self._N_steps:
            return
        if self._idx is None or self._idx[0].device != field.device:
            ii, jj, kk = (torch.tensor([p[c] for p in self._positions], device=field.device)
                          for c in range(3))
            self._idx = (ii, jj, kk)
        ii, jj, kk = self._idx
        vals = field[ii, jj, kk] if field.dim() == 3 else field[ii, jj]
        self._signals[tx_idx, :, step] = vals.to(torch.float32)

    def detectors(self) -> Detectors:
        """The receivers as a Detectors set for ``sim.run(n, record=...)``."""
        g = self._grid
        pts = [(self._component, i, j, k) if g.Nz > 1 else (self._component, i, j)
               for i, j, k in self._positions]
        return Detectors(pts)

    def store(self, tx_idx: int, traces: torch.Tensor, step0: int = 0) -> None:
        """Put ``(N_rx, n)`` traces recorded by the step kernels into the
        signal matrix of transmitter ``tx_idx`` from step ``step0``."""
        if self._signals is None:
            raise RuntimeError("Call build_sources() before store().")
        n = min(traces.shape[-1], self._N_steps - step0)
        self._signals[tx_idx, :, step0:step0 + n] = traces[..., :n].to(self._signals.device)

    def get_signals(self) -> np.ndarray:
        """(N_tx, N_rx, N_steps) float32 on the host (antenna.py:204-214)."""
        if self._signals is None:
            raise RuntimeError("No signals recorded yet.")
        return self._signals.cpu().numpy().copy()

    # ------------------------------------------------------------------
    def envelope(self, signals) -> torch.Tensor:
        """|analytic signal| along the last axis (the reference's
        ``np.abs(hilbert(signals, axis=-1))``), float64 FFT on the device."""
        x = torch.as_tensor(signals).to(self._device(), torch.float64)
        N = x.shape[-1]
        h = torch.zeros(N, dtype=torch.float64, device=x.device)
        if N % 2 == 0:
            h[0] = h[N // 2] = 1.0
            h[1:N // 2] = 2.0
        else:
            h[0] = 1.0
            h[1:(N + 1) // 2] = 2.0
        z = torch.fft.ifft(torch.fft.fft(x, dim=-1) * h, dim=-1)
        return z.abs().to(torch.float32).contiguous()

    def compute_das_image(self, signals, image_size: int = 40,
                          head_geometry: Optional[dict] = None) -> np.ndarray:
        """DAS power image (image_size, image_size) float32 on the host
        (antenna.py:262-341): Hilbert envelope, layered ray-circle travel
        times when ``head_geometry`` = {'cx_cells', 'cy_cells', 'layers':
        [(r_cells, eps_r), ...] outermost first} is given, else free space."""
        img = self.compute_das_image_from_envelope(self.envelope(signals), image_size,
                                                   head_geometry)
        return img.cpu().numpy()

    def compute_das_image_from_envelope(self, env: torch.Tensor, image_size: int = 40,
                                        head_geometry: Optional[dict] = None) -> torch.Tensor:
        """The travel-time table and delay-and-sum of ``compute_das_image`` for
        a given (N_tx, N_rx, n) float32 envelope; device tensor result."""
        dev = self._device()
        g = self._grid
        dt, dx = g.dt, g.dx
        env = torch.as_tensor(env).to(dev, torch.float32).contiguous()
        n = self._n
        if tuple(env.shape[:2]) != (n, n):
            raise ValueError(f"envelope must be (N_tx, N_rx, n) with N = {n}")
        n_steps = self._N_steps if self._N_steps else env.shape[-1]
        if env.shape[-1] < n_steps:
            raise ValueError(f"signals hold {env.shape[-1]} samples, the ring {n_steps}")
        x_px = np.linspace(0, (g.Nx - 1) * dx * 1e3, image_size)
        y_px = np.linspace(0, (g.Ny - 1) * dx * 1e3, image_size)
        ant = np.array([(i * dx * 1e3, j * dx * 1e3) for i, j, _ in self._positions])
        host = np.concatenate([ant[:, 0], ant[:, 1], x_px, y_px])
        buf = torch.from_numpy(host).to(dev)
        ax, ay = buf[:n], buf[n:2 * n]
        px, py = buf[2 * n:2 * n + image_size], buf[2 * n + image_size:]
        if head_geometry is not None:
            cx = head_geometry["cx_cells"] * dx * 1e3
            cy = head_geometry["cy_cells"] * dx * 1e3
            layers = [(r * dx * 1e3, e) for r, e in head_geometry["layers"]]
        else:
            cx = cy = 0.0
            layers = []
        lr = (ctypes.c_double * max(1, len(layers)))(*[r for r, _ in layers])
        le = (ctypes.c_double * max(1, len(layers)))(*[float(e) for _, e in layers])
        tt = torch.empty((n, image_size, image_size), dtype=torch.float32, device=dev)
        img = torch.empty((image_size, image_size), dtype=torch.float32, device=dev)
        lib = nat.load()
        st = nat.stream_handle(dev)
        nat.check(lib.wf_das_travel_times(n, ax.data_ptr(), ay.data_ptr(), px.data_ptr(),
                                          image_size, py.data_ptr(), image_size, cx, cy, lr, le,
                                          len(layers), dt, tt.data_ptr(), st))
        if env.shape[-1] != n_steps:
            env = env[..., :n_steps].contiguous()
        nat.check(lib.wf_das_envelope_image(env.data_ptr(), n, n_steps, tt.data_ptr(),
                                            image_size * image_size, img.data_ptr(), st))
        self._keep = (buf, env)
        return img

    def __repr__(self) -> str:
        return (f"AntennaRing(n={self._n}, r={self._r} cells, z={self._z}, "
                f"component='{self._component}')")
