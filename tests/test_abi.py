"""C-ABI checks that need no GPU: the library loads, exports every entry
point declared in include/waveforge_b200.h, and the ctypes mirrors of the C
structs have the C layout (gcc compiles the header and prints sizes and
offsets)."""

from __future__ import annotations

import ctypes
import re
import subprocess
from pathlib import Path

import pytest

from conftest import ROOT
from waveforge_b200 import _native as nat

HEADER = ROOT / "include" / "waveforge_b200.h"


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\S.*?\b(wf_[a-z0-9_]+)\s*\(", text, flags=re.M)))


def test_library_loads_and_reports_abi():
    lib = nat.load()
    assert lib.wf_abi_version() == 1
    assert isinstance(lib.wf_last_error(), bytes)


def test_every_declared_entry_point_is_exported():
    names = declared_functions()
    assert set(nat.EXPORTED) <= set(names)
    lib = ctypes.CDLL(str(nat.LIB_PATH))
    for n in names:
        assert hasattr(lib, n), f"{n} declared in the header but not exported"
    out = subprocess.run(["nm", "-D", "--defined-only", str(nat.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r" T (wf_[a-z0-9_]+)", out))
    assert set(names) <= exported


STRUCTS = {
    "wf_grid2d": (nat.WfGrid2D, ["nx", "ny", "dh", "de", "dx", "dy", "mur_x", "mur_y", "flags"]),
    "wf_grid2d_f64": (nat.WfGrid2DF64, ["nx", "ny", "dh", "de", "dx", "dy", "mur_x", "mur_y"]),
    "wf_grid3d": (nat.WfGrid3D, ["nx", "nz", "dh", "dz", "mur_z", "flags"]),
    "wf_source": (nat.WfSource, ["comp", "k1", "n_wave", "wave", "amp"]),
    "wf_probe": (nat.WfProbe, ["comp", "i", "j", "k"]),
    "wf_tune": (nat.WfTune, ["steps_per_pass", "tile_k", "threads"]),
    "wf_solve2d": (nat.WfSolve2D, ["g", "ex", "sz", "cb", "traces", "trace_ld", "nsrc",
                                   "step0", "nsteps", "n_check", "status", "check_max"]),
    "wf_region2d": (nat.WfRegion2D, ["kind", "material", "p"]),
}


def test_ctypes_layout_matches_c(tmp_path: Path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){"]
    for s, (_, fields) in STRUCTS.items():
        lines.append(f'printf("{s} size %zu\\n", sizeof({s}));')
        for f in fields:
            lines.append(f'printf("{s}.{f} %zu\\n", offsetof({s}, {f}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    r = subprocess.run(["gcc", "-std=c99", "-o", str(exe), str(src)], capture_output=True, text=True)
    if r.returncode != 0:
        pytest.fail(r.stderr)
    got = dict(l.rsplit(" ", 1) for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                          check=True).stdout.splitlines())
    for s, (cls, fields) in STRUCTS.items():
        assert int(got[f"{s} size"]) == ctypes.sizeof(cls), s
        for f in fields:
            assert int(got[f"{s}.{f}"]) == getattr(cls, f).offset, f"{s}.{f}"


def test_argument_errors_need_no_gpu():
    """Validation happens on the host before any CUDA call."""
    lib = nat.load()
    g = nat.WfGrid2D(3, 3, 1.0, 1.0, 1.0, 1.0, -0.5, -0.5, 0)
    rc = lib.wf_fdtd2d_run(ctypes.byref(g), 1, 1, 1, 1, 1, 1, None, None, None, 0, None, 0, None,
                           0, 0, 0, 10, 0, None, None, None)
    assert rc == nat.WF_E_ARG
    assert b"4x4" in lib.wf_last_error()
    g64 = nat.WfGrid2DF64(3, 8, 1.0, 1.0, 1.0, 1.0, -0.5, -0.5)
    rc = lib.wf_fdtd2d_run_f64(ctypes.byref(g64), 1, 1, 1, 1, None, None, None, 0, None, 0, None,
                               0, 0, 0, 10, 0, None, None)
    assert rc == nat.WF_E_ARG and b"4x4" in lib.wf_last_error()
    g64.nx = 8
    # a trace window shorter than the run
    rc = lib.wf_fdtd2d_run_f64(ctypes.byref(g64), 1, 1, 1, 1, None, None, None, 0, 1, 1, 1, 5,
                               0, 0, 10, 0, None, None)
    assert rc == nat.WF_E_ARG
    rc = lib.wf_das2d(None, None, 1, 1, None, None, None, 1, None, 1, 1.0, 1.0, 0, 0, None, None)
    assert rc == nat.WF_E_ARG


def test_new_entry_points_validate_on_host():
    lib = nat.load()
    g = nat.WfGrid2D(3, 8, 1.0, 1.0, 1.0, 1.0, -0.5, -0.5, 0)
    assert lib.wf_adjoint2d_run(ctypes.byref(g), 1, 0, 1, 1, None, None, None, 0, None, 0, 0, 0,
                                0, 1, 1, None, None, None) == nat.WF_E_ARG
    g8 = nat.WfGrid2D(8, 8, 1.0, 1.0, 1.0, 1.0, -0.5, -0.5, 0)
    # several runs need a stride that holds a whole run's slots
    assert lib.wf_adjoint2d_run(ctypes.byref(g8), 1, 10, 2, 1, None, None, None, 0, None, 0, 0, 0,
                                0, 1, 1, None, None, None) == nat.WF_E_ARG
    assert lib.wf_fdtd2d_states(ctypes.byref(g), 1, 0, 1, 1, None, None, None, 0, 0,
                                None) == nat.WF_E_ARG
    assert lib.wf_fdtd2d_states(ctypes.byref(g8), 1, 10, 2, 1, None, None, None, 0, 0,
                                None) == nat.WF_E_ARG
    assert lib.wf_material_coeffs(None, None, 4, 1e-12, None, None, None) == nat.WF_E_ARG
    assert lib.wf_material_grad(None, None, 4, 1e-12, None, None, 1, 1.0, None, None,
                                None) == nat.WF_E_ARG
    assert lib.wf_material_grad(1, 1, 4, 1e-12, 1, 1, 0, 1.0, 1, 1, None) == nat.WF_E_ARG
    assert lib.wf_paint2d(0, 4, None, 0, None, None, None, None, 1, None, None, None, None, None,
                          None) == nat.WF_E_ARG
    assert lib.wf_paint2d(4, 4, 1, 2000, 1, 1, None, None, 1, 1, 1, None, None, None,
                          None) == nat.WF_E_LIMIT
    assert lib.wf_paint2d(4, 4, 1, 2, 1, 1, None, None, 1, 1, 1, 1, None, None,
                          None) == nat.WF_E_ARG
