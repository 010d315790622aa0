"""CPU restatement of the reference delay-and-sum backprojection (test infrastructure only).

Also: AntennaRing.compute_das_image (src/datasets/brain/antenna.py:216-341),
restated in ``antenna_das_image_ref``.

Canonical form: examples/brain_mimo_imaging.py:211-266 (``image_shape`` pixel
pitch ``N*dx/N_img``, float64 distances, ``np.round`` half-to-even delays
clipped to ``[0, n_steps-1]``, float64 accumulation in tx-major/rx-minor
order, squared power image).  Variants covered by keyword arguments:

* ``pitch=dx`` pixel grid ``arange(N)*dx`` of examples/10_breast_tumor_mimo.py:148-165,
* ``gate_start`` time gate of examples/09_brain_clot_dataset_sample.py:176-178,
* ``skip_self`` tx==rx skip of examples/3d/3d_10_breast_tumor_mimo.py:227-228.
"""

from __future__ import annotations

import math

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


def _chord(ax, ay, bx, by, cx, cy, r):
    """Ray-circle chord length, src/datasets/brain/antenna.py:216-232."""
    dx_ = bx - ax
    dy_ = by - ay
    seg_len = math.sqrt(dx_ ** 2 + dy_ ** 2) + 1e-30
    ux, uy = dx_ / seg_len, dy_ / seg_len
    ox, oy = ax - cx, ay - cy
    b_c = ox * ux + oy * uy
    c_c = ox ** 2 + oy ** 2 - r ** 2
    disc = b_c ** 2 - c_c
    if disc <= 0:
        return 0.0
    sq = math.sqrt(disc)
    t0 = max(0.0, min(seg_len, -b_c - sq))
    t1 = max(0.0, min(seg_len, -b_c + sq))
    return max(0.0, t1 - t0)


def _travel(ax, ay, bx, by, cx, cy, layers, dt):
    """Layered one-way travel time in samples, antenna.py:234-260."""
    C0 = 3e8
    total_d = math.sqrt((bx - ax) ** 2 + (by - ay) ** 2) + 1e-30
    prev = 0.0
    t = 0.0
    for idx, (r_mm, eps) in enumerate(layers):
        co = _chord(ax, ay, bx, by, cx, cy, r_mm)
        ci = _chord(ax, ay, bx, by, cx, cy, layers[idx + 1][0]) if idx + 1 < len(layers) else 0.0
        sc = max(0.0, co - ci)
        t += (sc * 1e-3) / (C0 / math.sqrt(eps))
        prev += sc
    t += (max(0.0, total_d - prev) * 1e-3) / C0
    return t / dt


def antenna_das_image_ref(signals, positions, nx, ny, dx, dt, n_steps, image_size=40,
                          head_geometry=None, env=None):
    """AntennaRing.compute_das_image, src/datasets/brain/antenna.py:262-341:
    Hilbert envelope (scipy, the reference's dependency), float32 travel-time
    table (layered ray-circle chords or free space), nearest-sample DAS in
    float64, squared, float32.  ``env``: an envelope to use instead."""
    from scipy.signal import hilbert
    x_px = np.linspace(0, (nx - 1) * dx * 1e3, image_size)
    y_px = np.linspace(0, (ny - 1) * dx * 1e3, image_size)
    ant = [(i * dx * 1e3, j * dx * 1e3) for i, j, *_ in positions]
    if env is None:
        env = np.abs(hilbert(signals, axis=-1)).astype(np.float32)
    n = len(ant)
    tt = np.zeros((n, image_size, image_size), dtype=np.float32)
    if head_geometry is not None:
        cx = head_geometry["cx_cells"] * dx * 1e3
        cy = head_geometry["cy_cells"] * dx * 1e3
        layers = [(r * dx * 1e3, e) for r, e in head_geometry["layers"]]
        for a in range(n):
            for iy, py in enumerate(y_px):
                for ix, px in enumerate(x_px):
                    tt[a, iy, ix] = _travel(ant[a][0], ant[a][1], px, py, cx, cy, layers, dt)
    else:
        for a in range(n):
            for iy, py in enumerate(y_px):
                for ix, px in enumerate(x_px):
                    d = math.sqrt((px - ant[a][0]) ** 2 + (py - ant[a][1]) ** 2)
                    tt[a, iy, ix] = (d * 1e-3) / 3e8 / dt
    img = np.zeros((image_size, image_size), dtype=np.float64)
    for tx in range(n):
        for rx in range(n):
            delay = np.rint(tt[tx] + tt[rx]).astype(np.int32)
            valid = (delay >= 0) & (delay < n_steps)
            delay = np.clip(delay, 0, n_steps - 1)
            img += np.where(valid, env[tx, rx][delay], 0.0)
    return (img ** 2).astype(np.float32)
