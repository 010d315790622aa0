"""CPU oracle for the WaveForge Yee-FDTD + DAS hot path.

TEST INFRASTRUCTURE ONLY.  Nothing in the ``waveforge_b200`` package imports
this directory; only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may use it, and
only as the checker or the timed CPU baseline, never as the thing measured.

The oracle restates, in plain PyTorch-CPU tensor arithmetic (FDTD) and NumPy
float64 (DAS), the algorithm of the reference project
(shahzaibshazoo/waveforge, pure Python + PyTorch eager).  Every function cites
the reference file:line it follows.  It is pinned against golden vectors that
``tests/golden/make_golden.py`` produced by running the reference itself
(``tests/test_oracle_golden.py`` checks the oracle reproduces them bit for
bit in float32).
"""

from .fdtd_ref import (  # noqa: F401
    EPS0, MU0, C0, stable_dt, material_ca_cb, gauss_deriv_wave, gaussian_wave,
    ricker_wave, Oracle2D, Oracle3D,
)
from .das_ref import antenna_das_image_ref, das_backprojection_ref  # noqa: F401
from . import adjoint_ref  # noqa: F401
