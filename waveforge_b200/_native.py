"""ctypes binding of the C-ABI library ``lib/libwfb200.so`` (declared in
``include/waveforge_b200.h``).

The structures below mirror the C structs field for field; a CPU test
compiles the header with gcc and checks sizes and offsets against them.  The
library is loaded lazily on first use; when it is missing the product fails
loudly (there is no CPU fallback for any compute path).
"""

from __future__ import annotations

import ctypes
from ctypes import c_double, c_float, c_int32, c_int64, c_void_p, POINTER
from pathlib import Path
from typing import Optional

import torch

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libwfb200.so"

WF_OK, WF_E_ARG, WF_E_CUDA, WF_E_LIMIT, WF_E_DIVERGED, WF_E_TIMEOUT = range(6)
COMP_CODE = {"Ex": 0, "Ey": 1, "Ez": 2, "Hx": 3, "Hy": 4, "Hz": 5}

EXPORTED = ("wf_abi_version", "wf_last_error", "wf_check_fastdiv", "wf_fdtd2d_run",
            "wf_fdtd2d_run_noalloc", "wf_fdtd2d_run_f64", "wf_fdtd3d_run", "wf_fdtd3d_batch_run", "wf_batch2d_run", "wf_batch2d_pass", "wf_batch2d_queue", "wf_fdtd2d_states",
            "wf_adjoint2d_run", "wf_material_coeffs", "wf_material_grad", "wf_paint2d", "wf_paint3d", "wf_fdtd3d_take_status", "wf_fdtd3d_set_wait_limit", "wf_cpml2d_run",
            "wf_das2d", "wf_das_travel_times", "wf_das_envelope_image")
NOALLOC_MAX_CELLS = 1 << 20   # WF_NOALLOC_MAX_CELLS of the header
WF_FASTDIV_X, WF_FASTDIV_Y, WF_FASTDIV_Z = 1, 2, 4


class NativeError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"[wf status {code}] {message}")
        self.code = code


class WfGrid2D(ctypes.Structure):
    _fields_ = [("nx", c_int32), ("ny", c_int32), ("dh", c_float), ("de", c_float),
                ("dx", c_float), ("dy", c_float), ("mur_x", c_float), ("mur_y", c_float),
                ("flags", c_int32)]


class WfGrid2DF64(ctypes.Structure):
    _fields_ = [("nx", c_int32), ("ny", c_int32), ("dh", c_double), ("de", c_double),
                ("dx", c_double), ("dy", c_double), ("mur_x", c_double), ("mur_y", c_double)]


class WfGrid3D(ctypes.Structure):
    _fields_ = [("nx", c_int32), ("ny", c_int32), ("nz", c_int32), ("dh", c_float),
                ("de", c_float), ("dx", c_float), ("dy", c_float), ("dz", c_float),
                ("mur_x", c_float), ("mur_y", c_float), ("mur_z", c_float), ("flags", c_int32)]


class WfSource(ctypes.Structure):
    _fields_ = [("comp", c_int32), ("i0", c_int32), ("i1", c_int32), ("j0", c_int32),
                ("j1", c_int32), ("k0", c_int32), ("k1", c_int32), ("n_wave", c_int32),
                ("wave", c_void_p), ("amp", c_void_p)]


class WfProbe(ctypes.Structure):
    _fields_ = [("comp", c_int32), ("i", c_int32), ("j", c_int32), ("k", c_int32)]


class WfRegion2D(ctypes.Structure):
    _fields_ = [("kind", c_int32), ("material", c_int32), ("p", c_float * 8)]


class WfRegion3D(ctypes.Structure):
    _fields_ = [("kind", c_int32), ("material", c_int32), ("p", c_float * 8)]


class WfTune(ctypes.Structure):
    _fields_ = [("steps_per_pass", c_int32), ("tile_i", c_int32), ("tile_j", c_int32),
                ("tile_k", c_int32), ("threads", c_int32)]


class WfSolve2D(ctypes.Structure):
    _fields_ = [("g", WfGrid2D),
                ("ex", c_void_p), ("ey", c_void_p), ("hz", c_void_p),
                ("sx", c_void_p), ("sy", c_void_p), ("sz", c_void_p),
                ("ca", c_void_p), ("cb", c_void_p),
                ("src", c_void_p), ("probes", c_void_p), ("traces", c_void_p),
                ("trace_ld", c_int64),
                ("nsrc", c_int32), ("nprobe", c_int32), ("trace_step0", c_int32),
                ("step0", c_int32), ("nsteps", c_int32), ("n_check", c_int32),
                ("status", c_int32), ("check_max", c_void_p)]


_lib: Optional[ctypes.CDLL] = None


def load() -> ctypes.CDLL:
    """Load and type the library (raises RuntimeError when it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"waveforge_b200 CUDA library missing at {LIB_PATH}; build it with "
            "`python -m waveforge_b200.csrc.build` (there is no CPU fallback)")
    lib = ctypes.CDLL(str(LIB_PATH))
    lib.wf_abi_version.restype = c_int32
    lib.wf_last_error.restype = ctypes.c_char_p
    lib.wf_check_fastdiv.restype = c_int32
    lib.wf_check_fastdiv.argtypes = [c_float, c_void_p, c_void_p]
    lib.wf_fdtd2d_run.restype = c_int32
    lib.wf_fdtd2d_run.argtypes = [
        POINTER(WfGrid2D), c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
        c_void_p, c_void_p, c_void_p, c_int32, c_void_p, c_int32, c_void_p, c_int64, c_int32,
        c_int32, c_int32, c_int32, c_void_p, POINTER(WfTune), c_void_p]
    lib.wf_fdtd2d_run_f64.restype = c_int32
    lib.wf_fdtd2d_run_f64.argtypes = [
        POINTER(WfGrid2DF64), c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
        c_void_p, c_int32, c_void_p, c_int32, c_void_p, c_int64, c_int32, c_int32, c_int32,
        c_int32, c_void_p, c_void_p]
    lib.wf_fdtd2d_run_noalloc.restype = c_int32
    lib.wf_fdtd2d_run_noalloc.argtypes = [
        POINTER(WfGrid2D), c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int32,
        c_void_p, c_int32, c_void_p, c_int64, c_int32, c_int32, c_int32, c_int32, c_void_p,
        POINTER(WfTune), c_void_p]
    lib.wf_fdtd3d_run.restype = c_int32
    lib.wf_fdtd3d_run.argtypes = [
        POINTER(WfGrid3D), POINTER(c_void_p), POINTER(c_void_p), c_void_p, c_void_p,
        c_void_p, c_int32, c_void_p, c_int32, c_void_p, c_int64, c_int32, c_int32, c_int32,
        c_int32, c_void_p, POINTER(WfTune), c_void_p]
    lib.wf_fdtd3d_batch_run.restype = c_int32
    lib.wf_fdtd3d_batch_run.argtypes = [
        POINTER(WfGrid3D), c_int32, c_int64, POINTER(c_void_p), POINTER(c_void_p), c_void_p,
        c_void_p, c_int64, c_void_p, c_int32, c_int32, c_void_p, c_int32, c_void_p, c_int64,
        c_int64, c_int32, c_int32, c_int32, c_int32, c_void_p, POINTER(WfTune), c_void_p]
    lib.wf_batch2d_run.restype = c_int32
    lib.wf_batch2d_run.argtypes = [c_void_p, c_int32, c_void_p, c_void_p, POINTER(WfTune),
                                   c_int32, c_int32, c_void_p]
    lib.wf_batch2d_pass.restype = c_int32
    lib.wf_batch2d_pass.argtypes = [c_void_p, c_void_p, c_int32, c_int32, c_int32, c_int32,
                                    POINTER(WfTune), c_int32, c_void_p]
    lib.wf_fdtd2d_states.restype = c_int32
    lib.wf_fdtd2d_states.argtypes = [POINTER(WfGrid2D), c_void_p, c_int64, c_int32, c_int32,
                                     c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_void_p]
    lib.wf_adjoint2d_run.restype = c_int32
    lib.wf_adjoint2d_run.argtypes = [POINTER(WfGrid2D), c_void_p, c_int64, c_int32, c_int32,
                                     c_void_p, c_void_p, c_void_p, c_int32, c_void_p, c_int64,
                                     c_int64, c_int32, c_int32, c_void_p, c_void_p, c_void_p,
                                     c_void_p, c_void_p]
    lib.wf_material_coeffs.restype = c_int32
    lib.wf_material_coeffs.argtypes = [c_void_p, c_void_p, c_int64, c_double, c_void_p, c_void_p,
                                       c_void_p]
    lib.wf_material_grad.restype = c_int32
    lib.wf_material_grad.argtypes = [c_void_p, c_void_p, c_int64, c_double, c_void_p, c_void_p,
                                     c_int32, c_double, c_void_p, c_void_p, c_void_p]
    lib.wf_cpml2d_run.restype = c_int32
    lib.wf_cpml2d_run.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                  c_int32, c_void_p, c_void_p, c_void_p, c_int32, c_void_p,
                                  c_int32, c_void_p, c_int64, c_int32, c_int32, c_int32,
                                  c_int32, c_void_p, c_void_p]
    lib.wf_batch2d_queue.restype = c_int32
    lib.wf_batch2d_queue.argtypes = [c_void_p, c_void_p, c_int32, c_void_p, c_void_p, c_void_p,
                                     c_int32, c_void_p, c_int32, c_int64, c_void_p]
    lib.wf_fdtd3d_take_status.restype = c_int32
    lib.wf_fdtd3d_take_status.argtypes = [c_void_p]
    lib.wf_fdtd3d_set_wait_limit.restype = c_int32
    lib.wf_fdtd3d_set_wait_limit.argtypes = [c_int64]
    lib.wf_paint3d.restype = c_int32
    lib.wf_paint3d.argtypes = [c_int32, c_int32, c_int32, c_void_p, c_int32, c_void_p, c_void_p,
                               c_int32, c_void_p, c_void_p, c_void_p, c_void_p]
    lib.wf_paint2d.restype = c_int32
    lib.wf_paint2d.argtypes = [c_int32, c_int32, c_void_p, c_int32, c_void_p, c_void_p, c_void_p,
                               c_void_p, c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                               c_void_p]
    lib.wf_das_travel_times.restype = c_int32
    lib.wf_das_travel_times.argtypes = [c_int32, c_void_p, c_void_p, c_void_p, c_int32, c_void_p,
                                        c_int32, c_double, c_double, POINTER(c_double),
                                        POINTER(c_double), c_int32, c_double, c_void_p, c_void_p]
    lib.wf_das_envelope_image.restype = c_int32
    lib.wf_das_envelope_image.argtypes = [c_void_p, c_int32, c_int32, c_void_p, c_int32, c_void_p,
                                          c_void_p]
    lib.wf_das2d.restype = c_int32
    lib.wf_das2d.argtypes = [c_void_p, c_void_p, c_int32, c_int32, c_void_p, c_void_p, c_void_p, c_int32,
                             c_void_p, c_int32, c_double, c_double, c_int32, c_int32, c_void_p,
                             c_void_p]
    if lib.wf_abi_version() != 1:
        raise RuntimeError("waveforge_b200 CUDA library ABI mismatch; rebuild it")
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc != WF_OK:
        msg = load().wf_last_error().decode(errors="replace")
        raise NativeError(rc, msg)


def ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    return None if t is None else t.data_ptr()


def stream_handle(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def require_cuda(t: torch.Tensor, what: str) -> None:
    if not t.is_cuda:
        raise RuntimeError(
            f"{what} must live on a CUDA device: waveforge_b200 runs only on the GPU "
            "(there is no CPU fallback)")


def to_device_bytes(arr: ctypes.Array, device: torch.device) -> torch.Tensor:
    """Copy a ctypes struct array into a device byte tensor (descriptor upload)."""
    raw = bytes(memoryview(arr).cast("B"))
    host = torch.frombuffer(bytearray(raw), dtype=torch.uint8)
    return host.to(device, non_blocking=False)


def f32(x: float) -> float:
    """Round a Python float to float32 (the scalar rounding PyTorch applies)."""
    return float(torch.tensor(x, dtype=torch.float32).item())


_fastdiv_ok: dict = {}


def fastdiv_ok(d: float, device: torch.device) -> bool:
    """True when the fast exact division by float32(d) matches IEEE division
    for every float32 input on this device (checked once per value)."""
    key = (f32(d), str(device))
    if key not in _fastdiv_ok:
        lib = load()
        cnt = torch.zeros(1, dtype=torch.int32, device=device)
        check(lib.wf_check_fastdiv(key[0], cnt.data_ptr(), stream_handle(device)))
        _fastdiv_ok[key] = int(cnt.item()) == 0
    return _fastdiv_ok[key]


def fastdiv_flags(device: torch.device, dx: float, dy: float, dz: Optional[float] = None) -> int:
    flags = 0
    if fastdiv_ok(dx, device):
        flags |= WF_FASTDIV_X
    if fastdiv_ok(dy, device):
        flags |= WF_FASTDIV_Y
    if dz is not None and fastdiv_ok(dz, device):
        flags |= WF_FASTDIV_Z
    return flags
