"""Brain-haemorrhage dataset generator on the batched 3D engine (drop-in for
src/datasets/generator.py).

A sample is two MIMO acquisitions of the same head -- with the bleed
(target) and without it (reference) -- each one transmitter at a time with
every ring element receiving, then the scattered signals (target minus
reference) and their layered-medium DAS image.  The reference runs the
2 x n_tx solves one after another, stepping each from Python and reading
every receiver back with one host sync per element per step
(generator.py:162-248).  Here all 2 x n_tx solves of a sample are members of
one batched FieldSet: one ``wf_fdtd3d_batch_run`` launch per step advances
every member, each with its own transmitter, and the step kernel records
all receivers.  Each member's signals are bit-identical to the reference's
single solve; each phantom is painted once per sample on the GPU
(``wf_paint3d``) instead of on the host once per transmitter.  Sample dicts, ``.npz`` files and ``manifest.json`` keep the
reference's keys and layout (generator.py:386-428, :473-532).
"""

from __future__ import annotations

import json
import math
import random
import time
from concurrent.futures import Future, ThreadPoolExecutor
from pathlib import Path
from typing import Optional

import numpy as np
import torch

from ..core.boundaries import MurABC3D
from ..core.fdtd3d import FDTD3D
from ..core.fields import FieldSet
from ..core.grid import YeeGrid
from ..core.sources import ModulatedGaussian, UWBPulse
from ..imaging.antenna import AntennaRing
from .brain.phantom import BrainPhantom3D, sample_random_geometry

# Class balance of bleed ages and sizes (generator.py:52-58)
_BLEED_TYPES = ["epidural", "subdural", "intracerebral"]
_BLEED_AGES = ["acute", "subacute", "chronic"]
_AGE_WEIGHTS = [0.40, 0.35, 0.25]
_SIZE_CATS = ["small", "medium", "large"]
_SIZE_WEIGHTS = [0.30, 0.50, 0.20]
# A requested size falls back to smaller ones when the head has no room
_SIZE_FALLBACK = {"large": ["large", "medium", "small"], "medium": ["medium", "small"],
                  "small": ["small"]}
# Relative permittivity per shell for the DAS travel times (generator.py:368-377)
_DAS_LAYER_EPS = (("scalp_outer_r", 40.0), ("skull_outer_r", 13.1), ("skull_inner_r", 44.0),
                  ("csf_inner_r", 68.0), ("gray_matter_r", 52.7), ("white_matter_r", 38.1))


class BrainDatasetGenerator:
    """Class-balanced haemorrhage dataset of ``grid_size``^3 heads with an
    ``n_tx``-element ring in the mid-axial plane (generator.py:63-160).
    ``freq_low_hz``/``freq_high_hz`` select the UWB monocycle, else a
    modulated Gaussian at ``freq_hz``.  ``device`` must be a CUDA device:
    there is no CPU fallback."""

    def __init__(self, output_dir: str, freq_hz: float = 1e9, freq_low_hz: Optional[float] = None,
                 freq_high_hz: Optional[float] = None, grid_size: int = 64, dx_mm: float = 3.0,
                 n_tx: int = 8, ring_radius_cells: int = 30, n_steps: int = 300,
                 device: str = "cuda", seed: Optional[int] = None, verbose: bool = True) -> None:
        self._output_dir = Path(output_dir)
        self._output_dir.mkdir(parents=True, exist_ok=True)
        if freq_low_hz is not None and freq_high_hz is not None:
            if freq_high_hz <= freq_low_hz:
                raise ValueError("freq_high_hz must be > freq_low_hz")
            self._freq_low, self._freq_high = float(freq_low_hz), float(freq_high_hz)
            self._freq_hz = (freq_low_hz + freq_high_hz) / 2.0
            self._uwb_mode = True
        else:
            self._freq_low = self._freq_high = None
            self._freq_hz = float(freq_hz)
            self._uwb_mode = False
        dev = torch.device(device)
        if dev.type != "cuda":
            raise RuntimeError("BrainDatasetGenerator runs its solves on a CUDA device only")
        self._N = grid_size
        self._dx = dx_mm * 1e-3
        self._n_tx = n_tx
        self._ring_r = ring_radius_cells
        self._n_steps = n_steps
        self._device = str(dev)
        self._seed = seed
        self._rng = random.Random(seed)
        self._grid = YeeGrid(grid_size, grid_size, dx=self._dx, dy=self._dx, Nz=grid_size,
                             dz=self._dx, device=self._device)
        self._ring = AntennaRing(n_elements=n_tx, ring_radius_cells=ring_radius_cells,
                                 z_plane=grid_size // 2, grid=self._grid)
        if verbose:
            band = (f"UWB {self._freq_low / 1e9:.2f}-{self._freq_high / 1e9:.2f} GHz"
                    if self._uwb_mode else f"{self._freq_hz / 1e9:.2f} GHz")
            print(f"BrainDatasetGenerator: {band}, grid {grid_size}^3 dx={dx_mm} mm, "
                  f"{n_tx} antennas r={ring_radius_cells} cells, {n_steps} steps, "
                  f"{self._device}, output {self._output_dir}")

    grid = property(lambda s: s._grid)
    ring = property(lambda s: s._ring)

    # ------------------------------------------------------------------
    def _waveform(self):
        """UWB Gaussian monocycle over the band, or a Gaussian-modulated
        carrier at fc with sigma = 1 / (2 pi fc / 2) (generator.py:181-195)."""
        if self._uwb_mode:
            return UWBPulse(amplitude=1.0, f_low=self._freq_low, f_high=self._freq_high)
        sigma_t = 1.0 / (2.0 * math.pi * (self._freq_hz * 0.5))
        return ModulatedGaussian(amplitude=1.0, fc=self._freq_hz, sigma=sigma_t)

    def _run_members(self, coeffs: list, tx: list) -> tuple[torch.Tensor, float]:
        """One batched solve: member m paints coefficients ``coeffs[m]`` and
        transmits from element ``tx[m]``; returns the (B, n_rx, n_steps)
        receiver signals on the device and the aggregate Mcell-upd/s."""
        B = len(tx)
        g = self._grid
        wave = self._waveform()
        srcs = [self._ring.build_sources(wave, t, self._n_steps) for t in tx]
        if all(c is coeffs[0] for c in coeffs):
            ca, cb = coeffs[0]
        else:
            ca = torch.stack([c[0] for c in coeffs])
            cb = torch.stack([c[1] for c in coeffs])
        fields = FieldSet(g, batch_size=B)
        per_member = dict(member_sources=srcs) if B > 1 else dict(sources=srcs[0])
        sim = FDTD3D(g, fields, MurABC3D(g, fields.Hx, fields.Hy, fields.Hz), Ca=ca, Cb=cb,
                     n_check=99999, **per_member)
        torch.cuda.synchronize(g.device)
        t0 = time.perf_counter()
        traces = sim.run(self._n_steps, record=self._ring.detectors())
        if B == 1:
            traces = traces.unsqueeze(0)
        torch.cuda.synchronize(g.device)
        el = time.perf_counter() - t0
        return traces, B * self._n_steps * self._N ** 3 / max(el, 1e-12) / 1e6

    def _run_simulation(self, phantom: BrainPhantom3D, tx_idx: int) -> tuple[np.ndarray, float]:
        """One transmitter: ((n_rx, n_steps) signals, Mcell-upd/s)
        (generator.py:162-224)."""
        traces, mc = self._run_members([phantom.build_device(self._device)], [tx_idx])
        self._ring.store(tx_idx, traces[0])
        return traces[0].cpu().numpy(), mc

    def _run_full_mimo(self, phantom: BrainPhantom3D) -> tuple[np.ndarray, float]:
        """Every transmitter of one phantom in one batched solve:
        ((n_tx, n_rx, n_steps) signals, Mcell-upd/s) (generator.py:226-248)."""
        self._ring.reset()
        c = phantom.build_device(self._device)
        traces, mc = self._run_members([c] * self._n_tx, list(range(self._n_tx)))
        for t in range(self._n_tx):
            self._ring.store(t, traces[t])
        return traces.cpu().numpy(), mc

    def _run_pair(self, target: BrainPhantom3D, reference: BrainPhantom3D):
        """Both acquisitions of a sample (2 x n_tx solves) in one batched
        solve: (target signals, reference signals, Mcell-upd/s)."""
        ct, cr = target.build_device(self._device), reference.build_device(self._device)
        n = self._n_tx
        traces, mc = self._run_members([ct] * n + [cr] * n, list(range(n)) * 2)
        sig = traces.cpu().numpy()
        return sig[:n].copy(), sig[n:].copy(), mc

    # ------------------------------------------------------------------
    def _prepare(self, label: int, seed: int, phantom_id: str, bleed_age: Optional[str],
                 bleed_size: Optional[str]):
        """Head geometry, bleed and the two phantoms of one sample
        (generator.py:254-336), or None when no bleed placement fits."""
        rng = random.Random(seed)
        geom_seed = seed if phantom_id == "train" else seed + 10_000_000
        geom = sample_random_geometry(seed=geom_seed, grid_size=self._N, dx_mm=self._dx * 1e3)
        target = BrainPhantom3D(self._grid, self._freq_hz, geometry=geom, seed=seed)
        bleed = None
        if label > 0:
            btype = {1: "epidural", 2: "subdural", 3: "intracerebral"}[label]
            age = bleed_age or rng.choices(_BLEED_AGES, weights=_AGE_WEIGHTS)[0]
            size = bleed_size or rng.choices(_SIZE_CATS, weights=_SIZE_WEIGHTS)[0]
            for attempt in range(50):
                trial_geom = sample_random_geometry(geom_seed + attempt, self._N, self._dx * 1e3)
                target = BrainPhantom3D(self._grid, self._freq_hz, geometry=trial_geom,
                                        seed=seed + attempt)
                for trial_size in _SIZE_FALLBACK.get(size, [size]):
                    bleed = target.add_random_bleed(btype, age, trial_size)
                    if bleed is not None:
                        geom = trial_geom
                        break
                if bleed is not None:
                    break
            if bleed is None:
                return None
        reference = BrainPhantom3D(self._grid, self._freq_hz, geometry=geom, seed=seed + 100000)
        return geom, bleed, target, reference

    def _finish(self, label, seed, phantom_id, geom, bleed, signals_total, signals_ref, mc):
        """Scattered signals, layered DAS image and the sample dict
        (generator.py:340-416)."""
        signals_scattered = signals_total - signals_ref
        head_geom = {"cx_cells": geom.center[0], "cy_cells": geom.center[1],
                     "layers": [(getattr(geom, f), e) for f, e in _DAS_LAYER_EPS]}
        das_image = self._ring.compute_das_image(signals_scattered, head_geometry=head_geom)
        center = bleed.center if bleed else (0, 0, 0)
        r = bleed.radius if bleed else 0
        r_mm = r * self._dx * 1e3
        volume_ml = (4 / 3) * math.pi * r_mm ** 3 / 1e3 if r > 0 else 0.0
        return {
            "signals_total": signals_total,
            "signals_reference": signals_ref,
            "signals_scattered": signals_scattered,
            "das_image": das_image,
            "label": np.int32(label),
            "bleed_type": bleed.bleed_type if bleed else "none",
            "bleed_age": bleed.age if bleed else "none",
            "bleed_center_cells": np.array(center, dtype=np.int32),
            "bleed_center_mm": np.array(center, dtype=np.float32) * float(self._dx * 1e3),
            "bleed_radius_cells": np.int32(r),
            "bleed_radius_mm": np.float32(r_mm),
            "bleed_volume_ml": np.float32(volume_ml),
            "freq_hz": np.float32(self._freq_hz),
            "freq_low_hz": np.float32(self._freq_low or self._freq_hz),
            "freq_high_hz": np.float32(self._freq_high or self._freq_hz),
            "uwb_mode": np.bool_(self._uwb_mode),
            "dx_mm": np.float32(self._dx * 1e3),
            "grid_shape": np.array([self._N, self._N, self._N], dtype=np.int32),
            "n_tx": np.int32(self._n_tx),
            "n_rx": np.int32(self._n_tx),
            "n_steps": np.int32(self._n_steps),
            "dt_s": np.float64(self._grid.dt),
            "phantom_id": phantom_id,
            "phantom_seed": np.int32(seed),
            "phantom_skull_inner_r": np.int32(geom.skull_inner_r),
            "phantom_gray_r": np.int32(geom.gray_matter_r),
            "phantom_scalp_outer_r": np.int32(geom.scalp_outer_r),
            "_mcells_per_second": np.float32(mc),
        }

    def generate_sample(self, label: int, seed: int, phantom_id: str = "train",
                        bleed_age: Optional[str] = None,
                        bleed_size: Optional[str] = None) -> Optional[dict]:
        """One sample with its own head geometry (generator.py:254-416).
        ``label`` 0 healthy, 1 epidural, 2 subdural, 3 intracerebral; test
        samples draw geometry from seed + 10^7.  For a bleed, up to 50
        (geometry seed, size) combinations are tried, sizes falling back to
        smaller ones; None when none fits."""
        return self.generate_samples([(label, seed)], phantom_id, bleed_age, bleed_size)[0]

    def generate_samples(self, specs, phantom_id: str = "train", bleed_age: Optional[str] = None,
                         bleed_size: Optional[str] = None) -> list:
        """Several samples, ``specs`` = [(label, seed), ...], with every
        acquisition of all of them (2 x n_tx solves per sample) advanced in
        one batched solve; each sample equals ``generate_sample`` of its spec
        (None where the bleed does not fit)."""
        prep = [self._prepare(label, seed, phantom_id, bleed_age, bleed_size)
                for label, seed in specs]
        live = [p for p in prep if p is not None]
        out = [None] * len(specs)
        if not live:
            return out
        n = self._n_tx
        coeffs, tx = [], []
        for _, _, target, reference in live:
            ct, cr = target.build_device(self._device), reference.build_device(self._device)
            coeffs += [ct] * n + [cr] * n
            tx += list(range(n)) * 2
        traces, mc = self._run_members(coeffs, tx)
        sig = traces.cpu().numpy()
        q = 0
        for k, p in enumerate(prep):
            if p is None:
                continue
            geom, bleed, _, _ = p
            total = sig[2 * n * q:2 * n * q + n].copy()
            ref = sig[2 * n * q + n:2 * n * (q + 1)].copy()
            out[k] = self._finish(specs[k][0], specs[k][1], phantom_id, geom, bleed, total, ref, mc)
            q += 1
        return out

    def save_sample_async(self, sample: dict, sample_idx: int) -> Future:
        """``save_sample`` on a background writer thread (zlib compression
        releases the GIL, so the next sample's solve overlaps the write);
        ``flush()`` waits for every pending write."""
        if getattr(self, "_writer", None) is None:
            self._writer = ThreadPoolExecutor(max_workers=1)
            self._pending: list = []
        fut = self._writer.submit(self.save_sample, sample, sample_idx)
        self._pending.append(fut)
        return fut

    def flush(self) -> list:
        """Wait for the pending background writes; returns their paths."""
        done = [f.result() for f in getattr(self, "_pending", [])]
        self._pending = []
        return done

    def save_sample(self, sample: dict, sample_idx: int) -> Path:
        """``sample_<idx:06d>.npz`` (compressed): every array and numpy
        scalar, plus the string fields as 0-d arrays (generator.py:418-428)."""
        path = self._output_dir / f"sample_{sample_idx:06d}.npz"
        arrays = {k: v for k, v in sample.items() if isinstance(v, (np.ndarray, np.generic))}
        for key in ("bleed_type", "bleed_age", "phantom_id"):
            arrays[key] = np.array(sample[key])
        np.savez_compressed(path, **arrays)
        return path

    def generate_balanced_dataset(self, n_samples: int, phantom_id: str = "train",
                                  base_seed: int = 0, show_progress: bool = True,
                                  batch_samples: int = 4) -> dict:
        """``n_samples`` split evenly over the four classes in a seeded
        shuffled order; sample i of class c uses seed base + 7 i + 1000 c;
        samples whose bleed does not fit are skipped and counted.  Writes
        ``manifest.json`` and returns it (generator.py:434-539).  New:
        ``batch_samples`` consecutive samples share one batched solve (their
        results are the same as one at a time)."""
        per = n_samples // 4
        labels = [0] * per + [1] * per + [2] * per + [3] * per
        labels += [i % 4 for i in range(n_samples - len(labels))]
        random.Random(base_seed).shuffle(labels)
        manifest = {
            "n_requested": n_samples, "n_completed": 0, "n_failed": 0,
            "phantom_id": phantom_id, "class_counts": {0: 0, 1: 0, 2: 0, 3: 0},
            "sample_paths": [], "sample_indices": [], "labels": [], "bleed_types": [],
            "bleed_ages": [], "freq_hz": self._freq_hz,
            "grid_shape": [self._N, self._N, self._N], "dx_mm": self._dx * 1e3,
        }
        t_start = time.time()
        idx = 0
        group = max(1, int(batch_samples))
        for i0 in range(0, len(labels), group):
            part = list(enumerate(labels[i0:i0 + group], start=i0))
            specs = [(label, base_seed + i * 7 + label * 1000) for i, label in part]
            for (i, label), sample in zip(part, self.generate_samples(specs, phantom_id=phantom_id)):
                idx = self._record(manifest, i, label, sample, idx, n_samples, t_start,
                                   show_progress)
        self.flush()
        return self._write_manifest(manifest, n_samples, show_progress)

    def _record(self, manifest: dict, i: int, label: int, sample: Optional[dict], idx: int,
                n_samples: int, t_start: float, show_progress: bool) -> int:
        """Manifest entry and background write of one sample; returns the
        next sample index."""
        if sample is None:
            manifest["n_failed"] += 1
            if show_progress:
                print(f"  [{i + 1}/{n_samples}] SKIP (bleed placement failed, label={label})")
            return idx
        path = self._output_dir / f"sample_{idx:06d}.npz"
        self.save_sample_async(sample, idx)
        manifest["n_completed"] += 1
        manifest["class_counts"][int(label)] += 1
        manifest["sample_paths"].append(str(path))
        manifest["sample_indices"].append(idx)
        manifest["labels"].append(int(label))
        manifest["bleed_types"].append(str(sample["bleed_type"]))
        manifest["bleed_ages"].append(str(sample["bleed_age"]))
        if show_progress:
            el = time.time() - t_start
            eta = el / (i + 1) * (n_samples - i - 1)
            print(f"  [{i + 1:4d}/{n_samples}] label={label} type={sample['bleed_type']:15} "
                  f"age={sample['bleed_age']:9} {float(sample['_mcells_per_second']):.1f}Mc/s "
                  f"ETA:{eta / 60:.0f}min")
        return idx + 1

    def _write_manifest(self, manifest: dict, n_samples: int, show_progress: bool) -> dict:
        path = self._output_dir / "manifest.json"
        with open(path, "w") as fh:
            json.dump(manifest, fh, indent=2)
        if show_progress:
            print(f"\nDone: {manifest['n_completed']}/{n_samples} samples saved")
            print(f"Class counts: {manifest['class_counts']}")
            print(f"Manifest: {path}")
        return manifest
