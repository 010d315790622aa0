"""Multi-process path of bench.py on CPU (gloo, world size 2).

On GPUs the bench runs one process per GPU as independent replicas; the only
cross-rank operations are the barrier and the max-over-ranks of the timed
region.  These tests run the same helpers and the `--impl reference` arm
under torch.distributed with the gloo backend on 127.0.0.1.
"""

from __future__ import annotations

import json
import os
import socket
import subprocess
import sys

import pytest
import torch
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2",
                      RANK=str(rank), LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench
    ws, r, _ = bench.dist_setup()
    v = bench.reduce_max(float(10 + 5 * rank), ws, torch.device("cpu"))
    bench.barrier(ws)
    out[rank] = v
    import torch.distributed as dist
    dist.destroy_process_group()


def test_reduce_max_and_barrier_over_two_gloo_ranks():
    port = _free_port()
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_worker, args=(r, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert out[0] == out[1] == 15.0


def test_reference_arm_under_torchrun_two_ranks():
    """`bench.py --impl reference` launched like the multi-GPU driver
    launches it: rank 0 prints one JSON line, rank 1 exits 0."""
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(ROOT / "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3",
           "--ref-budget", "0.05"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
