"""Dataset generation on the batched engine (drop-in for src/datasets)."""

from .generator import BrainDatasetGenerator

__all__ = ["BrainDatasetGenerator"]
