"""Device-side detector recording.

The reference has no detector class: its MIMO drivers gather
``fields.Hz[rx_i, rx_j, 0]`` after every ``sim.step()``
(examples/brain_mimo_imaging.py:193-201) and ``AntennaRing.record`` does one
``.item()`` host sync per receiver per step (src/datasets/brain/antenna.py:
173-214).  ``Detectors`` describes the same sample points once; the fused
kernels write every step's sample straight into a ``(N_rx, n_steps)`` device
trace buffer, recording the value after the full step (H^{n+1/2}, E^{n+1}).
"""

from __future__ import annotations

from typing import Optional, Sequence

import torch

from .core._engine import ProbeTable


class Detectors:
    """Sample points ``(i, j[, k])`` of one component, or explicit
    ``(component, i, j[, k])`` tuples."""

    def __init__(self, positions: Sequence[tuple], component: str = "Hz") -> None:
        pts = []
        for p in positions:
            if isinstance(p[0], str):
                comp, idx = p[0], tuple(int(v) for v in p[1:])
            else:
                comp, idx = component, tuple(int(v) for v in p)
            if len(idx) == 2:
                idx = idx + (0,)
            if len(idx) != 3:
                raise ValueError(f"detector position {p!r} must have 2 or 3 indices")
            pts.append((comp, *idx))
        if not pts:
            raise ValueError("Detectors needs at least one position")
        self._points = pts
        self._cache: dict = {}
        self.traces: Optional[torch.Tensor] = None

    @property
    def points(self) -> list[tuple]:
        return list(self._points)

    def __len__(self) -> int:
        return len(self._points)

    def table(self, device: torch.device, allowed, shape) -> ProbeTable:
        key = (str(device), tuple(allowed), tuple(shape))
        if key not in self._cache:
            self._cache[key] = ProbeTable(self._points, device, allowed, shape)
        return self._cache[key]

    def _store(self, traces: torch.Tensor) -> None:
        self.traces = traces
