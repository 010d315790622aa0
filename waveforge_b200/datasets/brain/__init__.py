"""Brain phantom, tissue library and antenna ring (drop-in for
src/datasets/brain/__init__.py)."""

from .antenna import AntennaRing
from .phantom import (BLEED_SIZES, PHANTOM_A, PHANTOM_B, BleedConfig, BrainPhantom3D,
                      PhantomGeometry, sample_random_geometry)
from .tissue_library import (BLOOD_AGING, TISSUES, ColeColeParams, all_tissues_at_freq,
                             cole_cole_eps, cole_cole_spectrum, cole_cole_to_fdtd, tissue_at_freq)

__all__ = ["AntennaRing", "BrainPhantom3D", "BleedConfig", "PhantomGeometry", "PHANTOM_A",
           "PHANTOM_B", "BLEED_SIZES", "sample_random_geometry", "ColeColeParams", "TISSUES",
           "BLOOD_AGING", "tissue_at_freq", "all_tissues_at_freq", "cole_cole_eps",
           "cole_cole_to_fdtd", "cole_cole_spectrum"]
