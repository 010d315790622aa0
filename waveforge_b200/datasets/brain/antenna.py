"""The antenna ring under its reference import path
(src/datasets/brain/antenna.py); implemented in waveforge_b200.imaging.antenna."""

from ...imaging.antenna import AntennaRing

__all__ = ["AntennaRing"]
