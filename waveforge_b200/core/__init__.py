"""Drop-in mirror of the reference ``core`` package (src/core/__init__.py).

``from waveforge_b200.core import FDTD2D, YeeGrid, ...`` replaces
``from core import FDTD2D, YeeGrid, ...``; submodules keep the reference
names (grid, fields, materials, sources, boundaries, fdtd2d, fdtd3d).
"""

from .grid import C0, GridMetadata, YeeGrid, compute_stable_dt
from .fields import FIELD_COMPONENTS, YEE_OFFSETS, FieldSet, StaggerOffset
from .materials import Material, MaterialMap, MaterialMap3D, TISSUE_LIBRARY
from .sources import (
    Chirp, GaussianDerivativePulse, GaussianPulse, LineSource, ModulatedGaussian, PlaneSource,
    PointSource, RickerWavelet, SinusoidalSource, SourceCollection, TabulatedWaveform, UWBPulse,
    Waveform,
)
from .boundaries import CPML, MurABC, MurABC3D
from .fdtd2d import FDTD2D, SimulationDivergedError
from .fdtd3d import FDTD3D

__all__ = [
    "C0", "Chirp", "FDTD2D", "FDTD3D", "FIELD_COMPONENTS", "FieldSet", "GaussianDerivativePulse",
    "GaussianPulse", "GridMetadata", "LineSource", "Material", "MaterialMap", "MaterialMap3D",
    "ModulatedGaussian", "MurABC", "MurABC3D", "CPML", "PlaneSource", "PointSource", "RickerWavelet",
    "SimulationDivergedError", "SinusoidalSource", "SourceCollection", "StaggerOffset",
    "TISSUE_LIBRARY", "TabulatedWaveform", "UWBPulse", "Waveform", "YEE_OFFSETS", "YeeGrid",
    "compute_stable_dt",
]
