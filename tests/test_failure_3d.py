"""Failure handling of the 3D TMA pass without any device fault.

k3d_tma waits on an mbarrier for the bulk-tensor loads of each i-plane.
Every such wait is bounded: when it gives up, the CTA writes WF_E_TIMEOUT to a
device status word, waits (with the full bound) for the copies it still has in
flight, and stops; ``FDTD3D.run`` reads the word after the run and raises.
Here the bound is set so low (one non-blocking look, no suspended polls) that
waits give up on loads that do complete, so the timeout path runs with no hung
or faulting load.  A normal run afterwards must be bit-identical to the
reference's golden (the context is intact and the status word was cleared).
"""

from __future__ import annotations

import ctypes

import pytest
import torch

from _cases import head_coeffs, load
from conftest import sha
from waveforge_b200 import Detectors, TabulatedWaveform, _native as nat
from test_parity_3d import COMPS, sim3d

pytestmark = pytest.mark.gpu


def _head_sim(cuda, g, ca, cb):
    n, steps = int(g["n"]), int(g["steps"])
    i, j, k = (int(v) for v in g["src"])
    return sim3d(cuda, (n, n, n), float(g["dx"]), float(g["courant"]),
                 [("Ez", (i, i + 1, j, j + 1, k, k + 1), torch.from_numpy(g["wave"]))],
                 ca, cb, steps=steps)


def test_tma_wait_timeout_raises_then_normal_run_is_exact(cuda):
    lib = nat.load()
    g = load("head3d_32")          # 32^3: Nz % 4 == 0, so the default is the TMA pass
    ca, cb = head_coeffs(g)
    steps = int(g["steps"])
    try:
        nat.check(lib.wf_fdtd3d_set_wait_limit(0))
        sim, _ = _head_sim(cuda, g, ca, cb)
        with pytest.raises(RuntimeError, match="gave up"):
            sim.run(6)
        # the status word was read and cleared by run()
        st = ctypes.c_int32(-1)
        nat.check(lib.wf_fdtd3d_take_status(ctypes.byref(st)))
        assert st.value == 0
    finally:
        nat.check(lib.wf_fdtd3d_set_wait_limit(-1))
    sim, f = _head_sim(cuda, g, ca, cb)
    tr = sim.run(steps, record=Detectors([("Ez", *(int(v) for v in r)) for r in g["rx"]]))
    assert sha(tr) == str(g["sha_traces"])
    for c in COMPS:
        assert sha(getattr(f, c)) == str(g[f"sha_{c.lower()}"]), c
    st = ctypes.c_int32(-1)
    nat.check(lib.wf_fdtd3d_take_status(ctypes.byref(st)))
    assert st.value == 0
