"""The fast spacing division is only ever used where it is exact.

wf_check_fastdiv compares the FMA-corrected quotient with IEEE division on
all 2^32 float32 inputs.  For the spacings of the benchmark workloads the
check is run and, where it passes, a run with the fast path forced ON is
compared bit for bit with the same run forced OFF (IEEE division)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from waveforge_b200 import _native as nat
from test_parity_2d import _random_case, sim2d

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("d", [1e-3, 0.5e-3, 2e-3, 1.5e-3])
def test_fastdiv_check_runs(cuda, d):
    ok = nat.fastdiv_ok(d, cuda)
    assert isinstance(ok, bool)


def test_fastdiv_forced_on_equals_ieee(cuda):
    if not nat.fastdiv_ok(1e-3, cuda):
        pytest.skip("fast division not exact for 1e-3 on this device: IEEE path is used")
    rng = np.random.default_rng(17)
    spec, ca, cb = _random_case(rng, 50, 45, 80, True, 3)
    outs = []
    for flags in (0, nat.WF_FASTDIV_X | nat.WF_FASTDIV_Y):
        sim, f = sim2d(cuda, 50, 45, 1e-3, 0.9, spec, ca, cb, steps=80, tune=(4, 32, 64, 1, 0))
        sim._g.flags = flags
        sim.run(80)
        outs.append(torch.cat([f.Ex.flatten(), f.Ey.flatten(), f.Hz.flatten()]))
    assert torch.equal(outs[0].view(torch.int32), outs[1].view(torch.int32))
