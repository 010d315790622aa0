"""Delay-and-sum backprojection on the GPU (drop-in for the reference DAS).

``das_backprojection`` keeps the signature of the canonical reference
function (examples/brain_mimo_imaging.py:211-266) and reproduces its float64
result bit for bit through ``wf_das2d``: same pixel grid, same float64
distance/delay arithmetic, ``np.round`` half-to-even, clipping, and the same
tx-major accumulation order.  Keyword extensions select the variants found in
the other reference examples: ``v_medium`` / ``eps_eff`` (10_breast_tumor_mimo
.py:153), ``pitch`` (pixel grid ``arange(N)*dx``, 10_breast_tumor_mimo.py:157),
``gate_start`` (09_brain_clot_dataset_sample.py:176-178) and ``skip_self``
(3d/3d_10_breast_tumor_mimo.py:227-228).
"""

from __future__ import annotations

import math
from typing import Optional

import numpy as np
import torch

from .. import _native as nat

C0 = 299_792_458.0


def das_image_device(traces: torch.Tensor, ant_x: torch.Tensor, ant_y: torch.Tensor,
                     px: torch.Tensor, py: torch.Tensor, v_medium: float, dt: float,
                     gate_start: int = 0, skip_self: bool = False,
                     out: Optional[torch.Tensor] = None,
                     traces_ref: Optional[torch.Tensor] = None) -> torch.Tensor:
    """Device-tensor DAS: traces ``(N, N, n_steps)`` float32 on the GPU,
    coordinates float64; returns the ``(len(px), len(py))`` float64 power image.
    With ``traces_ref`` the kernel images ``traces - traces_ref`` (float32
    difference, as the reference forms delta_S)."""
    nat.require_cuda(traces, "traces")
    n, n2, ns = traces.shape
    if n != n2:
        raise ValueError(f"traces must be (N_tx, N_rx, n_steps) with N_tx == N_rx, got {tuple(traces.shape)}")
    dev = traces.device
    tr = traces.to(torch.float32).contiguous()
    tref = None
    if traces_ref is not None:
        if traces_ref.shape != traces.shape:
            raise ValueError("traces_ref must match traces in shape")
        tref = traces_ref.to(device=dev, dtype=torch.float32).contiguous()
    ax = ant_x.to(device=dev, dtype=torch.float64).contiguous()
    ay = ant_y.to(device=dev, dtype=torch.float64).contiguous()
    pxd = px.to(device=dev, dtype=torch.float64).contiguous()
    pyd = py.to(device=dev, dtype=torch.float64).contiguous()
    img = out if out is not None else torch.empty((pxd.numel(), pyd.numel()), dtype=torch.float64, device=dev)
    lib = nat.load()
    nat.check(lib.wf_das2d(tr.data_ptr(), nat.ptr(tref), n, ns, ax.data_ptr(), ay.data_ptr(), pxd.data_ptr(),
                           pxd.numel(), pyd.data_ptr(), pyd.numel(), float(v_medium), float(dt),
                           int(gate_start), 1 if skip_self else 0, img.data_ptr(),
                           nat.stream_handle(dev)))
    return img


def pixel_axes(nx: int, ny: int, dx: float, image_shape=None, pitch: Optional[float] = None):
    """Pixel coordinates (metres) exactly as the reference builds them."""
    nxi, nyi = (nx, ny) if image_shape is None else image_shape
    if pitch is None:
        px = np.arange(nxi) * (nx * dx / nxi)
        py = np.arange(nyi) * (ny * dx / nyi)
    else:
        px = np.arange(nxi) * pitch
        py = np.arange(nyi) * pitch
    return px, py


def das_backprojection(delta_S, antenna_positions, grid, n_steps: int, image_shape=None, *,
                       v_medium: Optional[float] = None, eps_eff: float = 40.0,
                       pitch: Optional[float] = None, gate_start: int = 0,
                       skip_self: bool = False, device=None) -> np.ndarray:
    """Reference-signature DAS (examples/brain_mimo_imaging.py:211-217).

    ``delta_S``: ``(N_tx, N_rx, n_steps)`` NumPy or torch array.  The default
    medium speed is ``c0/sqrt(40)`` as in the reference.  Returns a NumPy
    float64 ``(Nx_img, Ny_img)`` power image computed on the GPU.
    """
    dx, dt = grid.dx, grid.dt
    v = v_medium if v_medium is not None else C0 / math.sqrt(eps_eff)
    dev = torch.device(device) if device is not None else (
        grid.device if getattr(grid.device, "type", "cpu") == "cuda" else torch.device("cuda"))
    tr = torch.as_tensor(np.asarray(delta_S, dtype=np.float32) if not torch.is_tensor(delta_S)
                         else delta_S.detach())
    if tr.shape[-1] < n_steps:
        raise ValueError(f"delta_S holds {tr.shape[-1]} steps, n_steps={n_steps}")
    tr = tr[..., :n_steps].to(dev)
    ant_x = torch.tensor([p[0] * dx for p in antenna_positions], dtype=torch.float64)
    ant_y = torch.tensor([p[1] * dx for p in antenna_positions], dtype=torch.float64)
    px, py = pixel_axes(grid.Nx, grid.Ny, dx, image_shape, pitch)
    img = das_image_device(tr, ant_x, ant_y, torch.from_numpy(px), torch.from_numpy(py), v, dt,
                           gate_start, skip_self)
    return img.cpu().numpy()
