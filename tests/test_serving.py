"""Continuous-batching server: results are the same alone and in the mix.

A request's traces (and, for a gradient request, its loss and gradients) come
out bit-identical when it runs alone, when it joins a running mix of other
requests between chunks, and when it runs through the one-at-a-time plain
path (each transmitter a separate wf_fdtd2d_run; fdtd_misfit for gradients).
The server never holds more than its HBM budget, and rejects requests under
an explicit wait bound.
"""

from __future__ import annotations

import pytest
import torch

from waveforge_b200 import workloads as W
from waveforge_b200.serving import (ImagingRequest, Server, request_footprint, request_work,
                                    serve_one_at_a_time)


def _req(side, steps, seed, grad=False, n_ant=6):
    return W.serving_request(side, steps, seed, n_ant=n_ant, gradient=grad, dx=1e-3)


def test_footprint_and_work_accounting():
    r = _req(64, 100, 1)
    cells = 64 * 64
    assert request_work(r) == 6 * cells * 100
    assert request_footprint(r, 32) == 6 * 6 * cells * 4 + 2 * cells * 4 + 6 * 6 * 100 * 4
    rg = _req(64, 100, 1, grad=True)
    assert request_work(rg) == 2 * 6 * cells * 100
    assert request_footprint(rg, 32) > request_footprint(r, 32)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["tiled", "persistent"])
def test_forward_request_same_alone_in_mix_and_one_at_a_time(cuda, mode):
    probe = _req(72, 150, 7)
    alone = Server(cuda, chunk_steps=32, mode=mode)
    tk = alone.submit(probe)
    alone.drain()
    assert tk.status == "done"
    ref = tk.traces.clone()
    assert float(ref.abs().max()) > 0

    mix = Server(cuda, chunk_steps=32, mode=mode, max_active_cells=2e5)
    others = [_req(s, n, 100 + s) for s, n in ((96, 200), (48, 90), (130, 260), (64, 40))]
    tks = [mix.submit(r) for r in others[:2]]
    mix.step()
    mix.step()
    tk2 = mix.submit(probe)              # joins mid-flight, between chunks
    mix.step()
    tks += [mix.submit(r) for r in others[2:]]
    mix.drain()
    assert all(t.status == "done" for t in tks + [tk2])
    assert torch.equal(tk2.traces, ref)

    plain = serve_one_at_a_time(cuda, [(0.0, probe)])
    assert torch.equal(plain[0].traces, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["tiled", "persistent"])
def test_gradient_request_same_alone_in_mix_and_one_at_a_time(cuda, mode):
    g = _req(64, 120, 3, grad=True, n_ant=4)
    alone = Server(cuda, chunk_steps=16, mode=mode)
    tk = alone.submit(g)
    alone.drain()
    assert tk.status == "done" and tk.grad_eps is not None
    assert float(tk.grad_eps.abs().max()) > 0 and tk.loss > 0

    mix = Server(cuda, chunk_steps=16, mode=mode)
    first = [mix.submit(_req(80, 150, 21)), mix.submit(_req(50, 60, 22, grad=True, n_ant=4))]
    mix.step()
    tk2 = mix.submit(g)
    mix.step()
    last = mix.submit(_req(90, 100, 23))
    mix.drain()
    assert all(t.status == "done" for t in first + [tk2, last])
    assert torch.equal(tk2.traces, tk.traces)
    assert torch.equal(tk2.grad_eps, tk.grad_eps)
    assert torch.equal(tk2.grad_sigma, tk.grad_sigma)
    assert tk2.loss == tk.loss

    plain = serve_one_at_a_time(cuda, [(0.0, g)])[0]
    assert torch.equal(plain.traces, tk.traces)
    assert torch.equal(plain.grad_eps.reshape(tk.grad_eps.shape), tk.grad_eps)
    assert torch.equal(plain.grad_sigma.reshape(tk.grad_sigma.shape), tk.grad_sigma)


@pytest.mark.gpu
def test_admission_respects_hbm_budget(cuda):
    reqs = [_req(s, 80, 40 + s) for s in (64, 96, 128, 80, 112)]
    budget = max(request_footprint(r, 32) for r in reqs) * 2
    srv = Server(cuda, chunk_steps=32, hbm_budget=budget)
    tks = [srv.submit(r) for r in reqs]
    peak = 0
    while srv.queue or srv.live:
        srv.step()
        peak = max(peak, srv.used)
        assert srv.used <= budget
    srv.drain()
    assert all(t.status == "done" for t in tks)
    assert srv.used == 0
    assert peak > 0


@pytest.mark.gpu
def test_overload_policy_rejects_beyond_wait_bound(cuda):
    srv = Server(cuda, chunk_steps=32, max_wait_s=1e-6)
    srv.rate = 1e9   # a tiny bound: only an empty server admits
    tks = [srv.submit(_req(64, 60, 70 + q)) for q in range(4)]
    srv.drain()
    assert tks[0].status == "done"
    assert all(t.status == "rejected" and "overloaded" in t.reason for t in tks[1:])
