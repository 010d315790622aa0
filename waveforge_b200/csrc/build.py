"""Build libwfb200.so (the C-ABI CUDA library) in-tree for sm_100a.

Usage: ``python -m waveforge_b200.csrc.build [--force]``.  Each ``.cu`` file is
compiled to an object with ``nvcc -gencode arch=compute_100a,code=sm_100a``
(IEEE division and no FMA contraction are kept: no --use_fast_math), then
linked with the static CUDA runtime into ``waveforge_b200/lib/libwfb200.so``.
Objects are rebuilt only when a source or header is newer.
"""

from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
PKG = HERE.parent
ROOT = PKG.parent
INCLUDE = ROOT / "include"
OBJDIR = PKG / "lib" / "obj"
LIB = PKG / "lib" / "libwfb200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
         f"-I{INCLUDE}", f"-I{HERE}"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the waveforge_b200 CUDA library cannot be built")


def sources() -> list[Path]:
    return sorted(HERE.glob("*.cu"))


def _includes(path: Path, seen: set) -> None:
    """The library headers a source includes, directly or through other headers."""
    for line in path.read_text().splitlines():
        line = line.strip()
        if line.startswith("#include \""):
            name = line.split('"')[1]
            for d in (HERE, INCLUDE):
                h = d / name
                if h.exists() and h not in seen:
                    seen.add(h)
                    _includes(h, seen)


def _deps_mtime(src: Path) -> float:
    """Newest modification time of a source's own headers (and of this script:
    a change of the build recipe rebuilds everything)."""
    seen: set = set()
    _includes(src, seen)
    return max([p.stat().st_mtime for p in seen] + [Path(__file__).stat().st_mtime])


def _compile(src: Path, force: bool, extra: list[str]) -> Path:
    obj = OBJDIR / (src.stem + ".o")
    if not force and obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, _deps_mtime(src)):
        return obj
    cmd = [nvcc(), *ARCH, *FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, verbose_ptxas: bool = False) -> Path:
    OBJDIR.mkdir(parents=True, exist_ok=True)
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, extra), srcs))
    if force or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *map(str, objs)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    force = "--force" in sys.argv
    print(build(force=force, verbose_ptxas="--ptxas-v" in sys.argv))
