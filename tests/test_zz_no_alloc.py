"""wf_fdtd2d_run_noalloc: the 2D run for callers that cannot allocate.

Some callers cannot allocate device memory (their own pool allocator owns
the GPU memory, or their loop must not call cudaMalloc/cudaFree because those
can synchronise the device), so they cannot supply the scratch fields that
wf_fdtd2d_run needs.  wf_fdtd2d_run_noalloc keeps that scratch in a device
array built into the library.  This test calls it through the C-ABI, twice in
a row (the second call starts from whatever the first left in the shared
array), after a call on a grid of another shape has left non-zero values at
other cells of that array, and demands the same bits as wf_fdtd2d_run with
caller scratch, our parity tolerance.  It also checks the size limit and the
rejection of negative sizes.  The file is named to be collected last.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from waveforge_b200 import _native as nat

pytestmark = pytest.mark.gpu


def _case(dev, nx, ny, steps, seed):
    rng = np.random.default_rng(seed)
    g = nat.WfGrid2D(nx, ny, nat.f32(9.4e-7), nat.f32(0.13), nat.f32(1e-3), nat.f32(1e-3),
                     nat.f32(-0.4), nat.f32(-0.4), 0)
    ca = torch.from_numpy(rng.uniform(0.6, 1.0, (nx, ny)).astype(np.float32)).to(dev)
    cb = torch.from_numpy(rng.uniform(0.001, 0.05, (nx, ny)).astype(np.float32)).to(dev)
    wave = torch.from_numpy(rng.standard_normal(2 * steps).astype(np.float32)).to(dev)
    src = (nat.WfSource * 1)(nat.WfSource(nat.COMP_CODE["Hz"], nx // 3, nx // 3 + 1, ny // 2,
                                          ny // 2 + 1, 0, 1, wave.numel(), wave.data_ptr(), None))
    # probes a few cells from the source (a short run reaches only those)
    # plus one on the Mur edge
    si, sj = nx // 3, ny // 2
    prb = (nat.WfProbe * 3)(nat.WfProbe(5, si + 5, sj + 3, 0), nat.WfProbe(0, si - 4, sj, 0),
                            nat.WfProbe(1, 0, sj, 0))
    return g, ca, cb, wave, nat.to_device_bytes(src, dev), nat.to_device_bytes(prb, dev)


def _run(lib, dev, noalloc, g, fields, ca, cb, src_d, prb_d, traces, step0, nsteps):
    ex, ey, hz = fields
    stream = nat.stream_handle(dev)
    common = (ca.data_ptr(), cb.data_ptr(), src_d.data_ptr(), 1, prb_d.data_ptr(), 3,
              traces.data_ptr(), traces.stride(0), 0, step0, nsteps, 0, None, None, stream)
    if noalloc:
        rc = lib.wf_fdtd2d_run_noalloc(ctypes.byref(g), ex.data_ptr(), ey.data_ptr(),
                                       hz.data_ptr(), *common)
    else:
        scratch = torch.empty((3,) + tuple(ex.shape), dtype=torch.float32, device=dev)
        rc = lib.wf_fdtd2d_run(ctypes.byref(g), ex.data_ptr(), ey.data_ptr(), hz.data_ptr(),
                               scratch[0].data_ptr(), scratch[1].data_ptr(),
                               scratch[2].data_ptr(), *common)
    nat.check(rc)


def _plant_leftovers(lib, dev):
    """Run the no-alloc entry point once on a grid of another shape with
    non-zero fields, so the shared array holds values that sit at other cells
    (a different row length) than the calls that follow will use."""
    nx, ny, steps = 97, 233, 5
    g, ca, cb, wave, src_d, prb_d = _case(dev, nx, ny, steps, 11)
    gen = torch.Generator(device="cpu").manual_seed(3)
    fields = [torch.randn((nx, ny), generator=gen).to(dev) for _ in range(3)]
    traces = torch.zeros((3, 2 * steps), dtype=torch.float32, device=dev)
    _run(lib, dev, True, g, fields, ca, cb, src_d, prb_d, traces, 0, steps)
    torch.cuda.synchronize(dev)


def test_noalloc_matches_caller_scratch_on_two_calls(cuda):
    lib = nat.load()
    _plant_leftovers(lib, cuda)
    nx, ny, steps = 203, 151, 37
    g, ca, cb, wave, src_d, prb_d = _case(cuda, nx, ny, steps, 5)
    out = {}
    for noalloc in (False, True):
        fields = [torch.zeros((nx, ny), dtype=torch.float32, device=cuda) for _ in range(3)]
        traces = torch.zeros((3, 2 * steps), dtype=torch.float32, device=cuda)
        # two calls in a row: an odd-length first call (its last pass lands in
        # the scratch array and is copied back), then a continuation
        _run(lib, cuda, noalloc, g, fields, ca, cb, src_d, prb_d, traces, 0, steps)
        first = [f.clone() for f in fields]
        _run(lib, cuda, noalloc, g, fields, ca, cb, src_d, prb_d, traces, steps, steps)
        torch.cuda.synchronize(cuda)
        out[noalloc] = (first, fields, traces)
    for a, b in zip(out[False][0] + out[False][1] + [out[False][2]],
                    out[True][0] + out[True][1] + [out[True][2]]):
        assert torch.equal(a.view(torch.int32), b.view(torch.int32))
    # not vacuous: the wave reached the probes and the fields
    assert float(out[True][2][0].abs().max()) > 0.0
    assert float(out[True][2][1].abs().max()) > 0.0
    assert all(float(f.abs().max()) > 0.0 for f in out[True][1])


def test_noalloc_rejects_grids_above_its_limit(cuda):
    lib = nat.load()
    nx = 1025
    ny = nat.NOALLOC_MAX_CELLS // 1024 + 1   # nx*ny > limit
    g = nat.WfGrid2D(nx, ny, 1.0, 1.0, 1.0, 1.0, -0.5, -0.5, 0)
    dummy = torch.zeros(1, device=cuda)
    rc = lib.wf_fdtd2d_run_noalloc(ctypes.byref(g), dummy.data_ptr(), dummy.data_ptr(),
                                   dummy.data_ptr(), None, None, None, 0, None, 0, None, 0, 0, 0,
                                   1, 0, None, None, nat.stream_handle(cuda))
    assert rc == nat.WF_E_LIMIT
    assert b"limit" in lib.wf_last_error()


def test_noalloc_rejects_negative_sizes(cuda):
    lib = nat.load()
    dummy = torch.zeros(1, device=cuda)
    for nx, ny in ((-1, 8), (8, -3)):
        g = nat.WfGrid2D(nx, ny, 1.0, 1.0, 1.0, 1.0, -0.5, -0.5, 0)
        rc = lib.wf_fdtd2d_run_noalloc(ctypes.byref(g), dummy.data_ptr(), dummy.data_ptr(),
                                       dummy.data_ptr(), None, None, None, 0, None, 0, None, 0,
                                       0, 0, 1, 0, None, None, nat.stream_handle(cuda))
        assert rc == nat.WF_E_ARG
        assert b"negative" in lib.wf_last_error()
