"""Command line for the brain dataset generator, with the arguments of the
reference's datasets/generate_brain_dataset.py:60-108:

    python -m waveforge_b200.datasets.generate_brain_dataset \\
        --n_samples 2000 --output_dir ./brain_dataset [--phantom A|B] [--base_seed 0]
        [--freq_ghz 1.0 | --freq_low_ghz 1 --freq_high_ghz 3] [--grid_size 64]
        [--dx_mm 3.0] [--n_tx 8] [--ring_radius 30] [--n_steps 300] [--device cuda]
        [--quiet] [--dry_run]

The solves run on a CUDA device (there is no CPU mode).
"""

from __future__ import annotations

import argparse
import sys
import time


def parse_args(argv=None):
    p = argparse.ArgumentParser(description="WaveForge brain haemorrhage FDTD dataset generator "
                                            "(batched B200 engine)",
                                formatter_class=argparse.ArgumentDefaultsHelpFormatter)
    p.add_argument("--n_samples", type=int, required=True, help="total number of samples")
    p.add_argument("--output_dir", type=str, required=True, help="directory for the .npz samples")
    p.add_argument("--phantom", choices=["A", "B"], default="A",
                   help="A = training seed space, B = independent test seed space")
    p.add_argument("--base_seed", type=int, default=0)
    p.add_argument("--freq_ghz", type=float, default=1.0, help="centre frequency (narrow band)")
    p.add_argument("--freq_low_ghz", type=float, default=None, help="UWB band start (with --freq_high_ghz)")
    p.add_argument("--freq_high_ghz", type=float, default=None, help="UWB band end")
    p.add_argument("--grid_size", type=int, default=64, help="cubic grid side N")
    p.add_argument("--dx_mm", type=float, default=3.0, help="cell size in mm")
    p.add_argument("--n_tx", type=int, default=8, help="ring elements (each transmits, all receive)")
    p.add_argument("--ring_radius", type=int, default=30, help="ring radius in cells")
    p.add_argument("--n_steps", type=int, default=300, help="time steps per solve")
    p.add_argument("--device", type=str, default="", help="CUDA device (default cuda)")
    p.add_argument("--quiet", action="store_true", help="no per-sample progress lines")
    p.add_argument("--dry_run", action="store_true", help="print the configuration and exit")
    return p.parse_args(argv)


def main(argv=None) -> int:
    a = parse_args(argv)
    device = a.device or "cuda"
    uwb = a.freq_low_ghz is not None and a.freq_high_ghz is not None
    lo = a.freq_low_ghz * 1e9 if uwb else None
    hi = a.freq_high_ghz * 1e9 if uwb else None
    fc = (lo + hi) / 2.0 if uwb else a.freq_ghz * 1e9
    cells = a.n_tx * 2 * a.n_steps * a.grid_size ** 3
    print("=" * 60)
    print("WaveForge brain haemorrhage dataset generator (B200)")
    print(f"  samples {a.n_samples}, phantom {a.phantom}, base seed {a.base_seed}")
    print(f"  {'UWB %.2f-%.2f GHz' % (a.freq_low_ghz, a.freq_high_ghz) if uwb else '%.2f GHz' % a.freq_ghz}"
          f", grid {a.grid_size}^3 dx={a.dx_mm} mm, {a.n_tx} antennas r={a.ring_radius}, "
          f"{a.n_steps} steps, {device}")
    print(f"  {cells:.3g} cell-updates per sample (2 x {a.n_tx} solves, one batched run)")
    print("=" * 60)
    if a.dry_run:
        print("DRY RUN -- exiting without simulation.")
        return 0
    from .generator import BrainDatasetGenerator
    gen = BrainDatasetGenerator(a.output_dir, freq_hz=fc, freq_low_hz=lo, freq_high_hz=hi,
                                grid_size=a.grid_size, dx_mm=a.dx_mm, n_tx=a.n_tx,
                                ring_radius_cells=a.ring_radius, n_steps=a.n_steps, device=device,
                                seed=a.base_seed)
    t0 = time.time()
    man = gen.generate_balanced_dataset(a.n_samples, phantom_id="train" if a.phantom == "A" else "test",
                                        base_seed=a.base_seed, show_progress=not a.quiet)
    el = time.time() - t0
    print(f"\n{man['n_completed']} samples in {el:.1f} s "
          f"({man['n_completed'] / max(el, 1e-9):.2f} samples/s), {man['n_failed']} skipped")
    return 0


if __name__ == "__main__":
    sys.exit(main())
