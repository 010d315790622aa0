"""CPU restatement of the 2D TM step with a convolutional PML (test
infrastructure only).

The reference has no CPML update: it only computes the graded profiles
(src/core/boundaries.py:32-112) and keeps applying Mur.  This file restates
the CPML step of waveforge_b200/csrc/cpml2d.cu operation for operation on
float32 CPU tensors, so the device path can be checked bit for bit; physics
(absorption) is checked separately against a larger domain.  Outside the
layers the step is the reference's (src/core/fdtd2d.py:187-266) without the
Mur edges.  Per derivative d inside a layer, with (b, c, ik) of its position:
    psi <- b * psi + c * d ;  d <- d * ik + psi
"""

from __future__ import annotations

import torch

from .fdtd_ref import Oracle2D


class OracleCPML2D(Oracle2D):
    """``tables``: 6 (nx + ny) float32 values -- b_E, c_E, ik_E, b_H, c_H,
    ik_H over the x positions, then the same over y (the CPML class's
    layout); ``depth`` = layer cells per side."""

    def __init__(self, nx, ny, dx, dy, dt, depth, tables, ca=None, cb=None):
        super().__init__(nx, ny, dx, dy, dt, ca, cb)
        t = tables.to(torch.float32).cpu()
        self.tx = t[:6 * nx].view(6, nx)
        self.ty = t[6 * nx:].view(6, ny)
        self.D = depth
        D = depth
        self.phzx = torch.zeros(2 * D, ny)
        self.peyx = torch.zeros(2 * D, ny)
        self.phzy = torch.zeros(nx, 2 * D)
        self.pexy = torch.zeros(nx, 2 * D)

    @staticmethod
    def _layer(n: int, D: int, half: bool):
        """(positions, slab indices) of one axis' layer cells: E at integer i
        in [0, n), H at i + 1/2 for i in [0, n - 1)."""
        if half:
            lo = list(range(D))
            hi = list(range(n - 1 - D, n - 1))
        else:
            lo = list(range(D))
            hi = list(range(n - D, n))
        pos = lo + hi
        return torch.tensor(pos), torch.tensor(list(range(2 * D)))

    def step(self):
        Ex, Ey, Hz = self.Ex, self.Ey, self.Hz
        nx, ny, D = self.nx, self.ny, self.D
        self._inject()
        t2 = (Ex[:-1, 1:] - Ex[:-1, :-1]) / self.dy          # dEx/dy at Hz cells
        t4 = (Ey[1:, :-1] - Ey[:-1, :-1]) / self.dx          # dEy/dx at Hz cells
        # x layer, Hz positions (rows of t4)
        pos, sl = self._layer(nx, D, True)
        b, c, ik = self.tx[3, pos][:, None], self.tx[4, pos][:, None], self.tx[5, pos][:, None]
        p = b * self.phzx[sl, :ny - 1] + c * t4[pos, :]
        self.phzx[sl, :ny - 1] = p
        t4[pos, :] = t4[pos, :] * ik + p
        # y layer, Hz positions (columns of t2)
        pos, sl = self._layer(ny, D, True)
        b, c, ik = self.ty[3, pos][None, :], self.ty[4, pos][None, :], self.ty[5, pos][None, :]
        p = b * self.phzy[:nx - 1, sl] + c * t2[:, pos]
        self.phzy[:nx - 1, sl] = p
        t2[:, pos] = t2[:, pos] * ik + p
        Hz[:-1, :-1] += self.dh * (t2 - t4)
        # Ampere with the E-position layers
        dhz_dy = (Hz[:, 1:] - Hz[:, :-1]) / self.dy          # column c <-> j = c + 1
        dhz_dx = (Hz[1:, :] - Hz[:-1, :]) / self.dx          # row r <-> i = r + 1
        pos, sl = self._layer(ny, D, False)
        keep = pos >= 1
        pos, sl = pos[keep], sl[keep]
        b, c, ik = self.ty[0, pos][None, :], self.ty[1, pos][None, :], self.ty[2, pos][None, :]
        p = b * self.pexy[:, sl] + c * dhz_dy[:, pos - 1]
        self.pexy[:, sl] = p
        dhz_dy[:, pos - 1] = dhz_dy[:, pos - 1] * ik + p
        pos, sl = self._layer(nx, D, False)
        keep = pos >= 1
        pos, sl = pos[keep], sl[keep]
        b, c, ik = self.tx[0, pos][:, None], self.tx[1, pos][:, None], self.tx[2, pos][:, None]
        p = b * self.peyx[sl, :] + c * dhz_dx[pos - 1, :]
        self.peyx[sl, :] = p
        dhz_dx[pos - 1, :] = dhz_dx[pos - 1, :] * ik + p
        if self.ca is None:
            Ex[:, 1:] += self.de * dhz_dy
            Ey[1:, :] -= self.de * dhz_dx
        else:
            Ex[:, 1:] = self.ca[:, 1:] * Ex[:, 1:] + self.cb[:, 1:] * dhz_dy
            Ey[1:, :] = self.ca[1:, :] * Ey[1:, :] - self.cb[1:, :] * dhz_dx
        self.n += 1
        if self.n % self.n_check == 0:
            self._stability(("Ex", "Ey", "Hz"))
