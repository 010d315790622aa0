"""CPU restatement of the reference delay-and-sum backprojection (test infrastructure only).

Canonical form: examples/brain_mimo_imaging.py:211-266 (``image_shape`` pixel
pitch ``N*dx/N_img``, float64 distances, ``np.round`` half-to-even delays
clipped to ``[0, n_steps-1]``, float64 accumulation in tx-major/rx-minor
order, squared power image).  Variants covered by keyword arguments:

* ``pitch=dx`` pixel grid ``arange(N)*dx`` of examples/10_breast_tumor_mimo.py:148-165,
* ``gate_start`` time gate of examples/09_brain_clot_dataset_sample.py:176-178,
* ``skip_self`` tx==rx skip of examples/3d/3d_10_breast_tumor_mimo.py:227-228.
"""

from __future__ import annotations

import numpy as np


def das_backprojection_ref(delta_S: np.ndarray, antenna_positions, nx: int, ny: int,
                           dx: float, dt: float, n_steps: int, v_medium: float,
                           image_shape=None, pitch=None, gate_start: int = 0,
                           skip_self: bool = False) -> np.ndarray:
    if image_shape is None:
        nxi, nyi = nx, ny
    else:
        nxi, nyi = image_shape
    data = delta_S
    if gate_start > 0:
        data = delta_S.copy()
        data[:, :, :gate_start] = 0.0
    ax = np.array([p[0] * dx for p in antenna_positions])
    ay = np.array([p[1] * dx for p in antenna_positions])
    if pitch is None:
        px = np.arange(nxi) * (nx * dx / nxi)
        py = np.arange(nyi) * (ny * dx / nyi)
    else:
        px = np.arange(nxi) * pitch
        py = np.arange(nyi) * pitch
    PX, PY = np.meshgrid(px, py, indexing="ij")
    img = np.zeros((nxi, nyi), dtype=np.float64)
    n = len(antenna_positions)
    for tx in range(n):
        for rx in range(n):
            if skip_self and tx == rx:
                continue
            d_tx = np.sqrt((PX - ax[tx]) ** 2 + (PY - ay[tx]) ** 2)
            d_rx = np.sqrt((PX - ax[rx]) ** 2 + (PY - ay[rx]) ** 2)
            tau = (d_tx + d_rx) / v_medium
            k = np.clip(np.round(tau / dt).astype(np.int32), 0, n_steps - 1)
            img += data[tx, rx, k]
    return img ** 2
