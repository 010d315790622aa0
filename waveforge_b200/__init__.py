"""waveforge_b200 — B200-native (sm_100a) Yee-FDTD time loop and DAS backprojection.

Drop-in for the hot path of shahzaibshazoo/waveforge: the reference's Python
API (``core`` package: YeeGrid, FieldSet, MaterialMap, sources, MurABC,
FDTD2D/FDTD3D; the DAS imager) is mirrored here, and every compute path runs
as hand-written CUDA through the C-ABI library ``lib/libwfb200.so``
(``include/waveforge_b200.h``).  There is no CPU fallback.
"""

from .core import *  # noqa: F401,F403
from .core import __all__ as _core_all
from .detectors import Detectors
from .imaging.das import das_backprojection, das_image_device
from .imaging.antenna import AntennaRing
from .batch import Batch2D, BatchSolve
from .adjoint import FDTDMisfit, MisfitProblem2D, fdtd_misfit

__all__ = list(_core_all) + ["AntennaRing", "Detectors", "das_backprojection", "das_image_device", "Batch2D",
                             "BatchSolve", "FDTDMisfit", "MisfitProblem2D", "fdtd_misfit"]
__version__ = "0.1.0"
