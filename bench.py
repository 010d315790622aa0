"""Benchmark: batched uneven breast-MIMO 2D FDTD + DAS on B200.

Workload (one bench "step"): 64 seeded breast phantoms (sides drawn from
{150,200,256,384,512}, dx = 0.5 mm, Courant 0.5), each with a 16-antenna
ring; every transmitter is a separate 3000-step solve recording 16 receivers,
for the tumour phantom AND its healthy twin (2 x 1024 solves; each batch's
launch shape is picked by the autotuner and its whole run replayed from a
CUDA graph), followed by one 128x128 DAS image per phantom of
S_tumour - S_healthy.  Metric: aggregate Gcell-updates/s (cells x steps of all
solves / time).  Inputs (fields 2 x 1.3 GB) are far larger than L2, so no L2
flush is needed between steps.

Legs reported on one JSON line:
  value      device-resident, CUDA-event timed, max over ranks (replicas per GPU)
  e2e        same work through the public API from pinned HOST buffers: H2D of
             coefficients/waveforms and D2H of all traces and images inside
             the timed region
  plain_per_solve  the same solves one wf_fdtd2d_run at a time (measured on a
             stratified sample, one phantom per grid size, extrapolated)
  roofline   k_batch2d: 32 algorithmic bytes per cell-update / launch time
  cpu_baseline  the CPU port of the reference loop (oracle) on a bounded sample
`--impl reference` runs only the reference CPU port (rank 0) on the same metric.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "batched Gcell-upd/s (uneven breast MIMO, 2D TM lossy fp32)"
UNIT = "Gcell-upd/s"
BYTES_PER_CELL_UPDATE = 32  # read Ex,Ey,Hz,Ca,Cb + write Ex,Ey,Hz (float32)
DAS_SIZE = 128
EPS_EFF = 0.6 * 5.0 + 0.3 * 40.0 + 0.1 * 36.0  # breast volume-weighted average


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------

def build_workload(dev, n_phantoms, n_tx, steps, seed, mode="persistent", tune=None):
    from waveforge_b200 import (Batch2D, BatchSolve, Detectors, PointSource, SourceCollection,
                                YeeGrid)
    from waveforge_b200.core.materials import Material, MaterialMap
    from waveforge_b200.core.sources import GaussianDerivativePulse
    from waveforge_b200 import workloads as W

    wl = W.BreastMIMO(n_phantoms=n_phantoms, n_tx=n_tx, steps=steps, seed=seed)
    phantoms = wl.phantoms()
    host_coeffs = {}   # (p, twin) -> (ca, cb) pinned host
    dev_coeffs = {}
    waves = {}
    solves = {True: [], False: []}
    for p, ph in enumerate(phantoms):
        gh = YeeGrid(ph.side, ph.side, wl.dx, wl.dx, courant=wl.courant, device="cpu")
        g = YeeGrid(ph.side, ph.side, wl.dx, wl.dx, courant=wl.courant, device=dev)
        if ph.side not in waves:
            waves[ph.side] = GaussianDerivativePulse(1e9).build(steps, g.dt, dev)
        ant = ph.antennas(16)
        for tumor in (True, False):
            mm = MaterialMap(gh, default=ph.background(Material))
            ph.paint(mm, Material, with_tumor=tumor)
            ca, cb = mm.build()
            host_coeffs[(p, tumor)] = (ca.pin_memory(), cb.pin_memory())
            cad, cbd = ca.to(dev), cb.to(dev)
            dev_coeffs[(p, tumor)] = (cad, cbd)
            for tx in range(n_tx):
                i, j = ant[tx]
                src = PointSource(_TableWave(waves[ph.side]), i, j, "Hz", grid=g, N_steps=steps)
                solves[tumor].append(BatchSolve(g, SourceCollection([src]), Detectors(ant), cad, cbd,
                                                tag=(p, tx)))
    batches = {t: Batch2D(solves[t], steps, mode=mode, tune=tune) for t in (True, False)}
    return wl, phantoms, batches, host_coeffs, dev_coeffs, waves


class _TableWave:
    """Waveform already on the device (shared by all solves of one grid size)."""

    def __init__(self, t):
        self.t = t

    def build(self, N_steps, dt, device, dtype=torch.float32):
        return self.t[:N_steps]


def das_all(batches, phantoms, wl, n_tx, dev, out_images):
    from waveforge_b200.imaging.das import das_image_device, pixel_axes
    v = 299_792_458.0 / math.sqrt(EPS_EFF)
    for p, ph in enumerate(phantoms):
        q0 = p * n_tx
        tr_t = batches[True].traces_block(q0, n_tx)
        tr_h = batches[False].traces_block(q0, n_tx)
        ant = ph.antennas(16)
        ax = torch.tensor([a[0] * wl.dx for a in ant], dtype=torch.float64)
        ay = torch.tensor([a[1] * wl.dx for a in ant], dtype=torch.float64)
        px, py = pixel_axes(ph.side, ph.side, wl.dx, (DAS_SIZE, DAS_SIZE))
        dt = batches[True].solves[q0].grid.dt
        das_image_device(tr_t, ax, ay, torch.from_numpy(px), torch.from_numpy(py), v, dt,
                         out=out_images[p], traces_ref=tr_h)


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            # raw samples go to WAVEFORGE_B200_CLOCKS_DIR (default: the temp
            # dir); the JSON line carries their summary
            out_dir = Path(os.environ.get("WAVEFORGE_B200_CLOCKS_DIR", tempfile.gettempdir()))
            out_dir.mkdir(parents=True, exist_ok=True)
            self.path = out_dir / f"clocks_gpu{self.gpu}.csv"
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                stderr=subprocess.DEVNULL)
        except Exception:  # nvidia-smi absent: report no clock record
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU reference port (oracle) timing
# ---------------------------------------------------------------------------

def cpu_reference_sample(budget_s=12.0, threads=None):
    """Time the CPU port of the reference 2D loop on solves of the workload
    until ``budget_s`` of work; returns (Gcell-upd/s, cores, sample text)."""
    import oracle
    from waveforge_b200 import workloads as W
    from waveforge_b200.core.grid import YeeGrid
    from waveforge_b200.core.materials import Material, MaterialMap

    threads = threads or os.cpu_count() or 1
    torch.set_num_threads(threads)
    wl = W.BreastMIMO()
    phantoms = wl.phantoms()
    done_cells = 0
    t_total = 0.0
    solves = 0
    steps_each = 300
    for ph in phantoms:
        g = YeeGrid(ph.side, ph.side, wl.dx, wl.dx, courant=wl.courant, device="cpu")
        mm = MaterialMap(g, default=ph.background(Material))
        ph.paint(mm, Material)
        ca, cb = mm.build()
        ant = ph.antennas(16)
        o = oracle.Oracle2D(ph.side, ph.side, wl.dx, wl.dx, g.dt, ca[..., 0], cb[..., 0])
        o.add_point_source("Hz", *ant[0], oracle.gauss_deriv_wave(steps_each, g.dt))
        t0 = time.perf_counter()
        o.run(steps_each, [("Hz", i, j) for i, j in ant])
        t_total += time.perf_counter() - t0
        done_cells += ph.side * ph.side * steps_each
        solves += 1
        if t_total >= budget_s:
            break
    return (done_cells / t_total / 1e9, threads,
            f"{solves} solves of the workload (first phantoms, TX 0), {steps_each} steps each, "
            f"16 receivers gathered per step; {done_cells:.3e} cell-updates in {t_total:.1f} s")


# ---------------------------------------------------------------------------

def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return ws, rank, local


def reduce_max(x, ws, dev):
    if ws == 1:
        return x
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def run_reference_arm(args, ws, rank):
    if rank != 0:
        return
    t0 = time.perf_counter()
    vals = []
    samples = ""
    for s in range(args.warmup + args.steps):
        v, cores, samples = cpu_reference_sample(budget_s=args.ref_budget)
        if s >= args.warmup:
            vals.append(v)
    value = statistics.median(vals)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "breast_mimo_64ph_16tx_3000steps", "parallelism": "replicas"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": samples},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": time.perf_counter() - t0}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# single-solve workloads: plain 2D (4096^2 lossy ellipses) and 3D head (256^3)
# ---------------------------------------------------------------------------

def default_depth(workload, cells):
    """Temporal block depth the library picks without a tune (fdtd2d.cu
    default_tune2d; fdtd3d.cu uses single-step passes)."""
    if workload == "head3d":
        return 1
    return 6 if cells >= 1024 * 1024 else 4


def pass_launches(nsteps, k):
    """Kernel launches of one run: the pass plan of wf_common.cuh PassPlan
    (the first pass is split when the pass count is odd and it has >= 2
    steps) plus a copy-back when the pass count stays odd."""
    p0 = -(-nsteps // k)
    split = 1 if (p0 % 2 == 1 and min(nsteps, k) >= 2) else 0
    passes = p0 + split
    return passes + (passes % 2)


def _tune_arg(args):
    return None if args.tune is None else tuple(int(v) for v in args.tune.split(","))


def build_single(args, dev):
    """The solve of --workload plain2d / head3d: returns (sim, detectors,
    host (ca, cb), device (ca, cb), wave, cells, bytes per cell-update, oracle factory)."""
    import oracle
    from waveforge_b200 import workloads as W
    from waveforge_b200 import (FDTD2D, FDTD3D, Detectors, FieldSet, MurABC, MurABC3D,
                                PointSource, SourceCollection, YeeGrid)
    from waveforge_b200.core.materials import Material, MaterialMap, MaterialMap3D
    from waveforge_b200.core.sources import GaussianDerivativePulse

    if args.workload == "plain2d":
        wl = W.LossyEllipses(n=args.side or 4096, steps=args.nsteps)
        n = wl.n
        gh = YeeGrid(n, n, wl.dx, wl.dx, courant=wl.courant, device="cpu")
        mm = MaterialMap(gh, default=wl.background(Material))
        wl.paint(mm, Material)
        ca, cb = mm.build()
        g = YeeGrid(n, n, wl.dx, wl.dx, courant=wl.courant, device=dev)
        f = FieldSet(g)
        wave = GaussianDerivativePulse(1e9).build(wl.steps, g.dt, dev)
        i, j = wl.source
        src = PointSource(_TableWave(wave), i, j, "Hz", grid=g, N_steps=wl.steps)
        cad, cbd = ca.to(dev), cb.to(dev)
        sim = FDTD2D(g, f, MurABC(g, f.Hz), SourceCollection([src]), Ca=cad, Cb=cbd,
                     tune=_tune_arg(args))
        det = Detectors(wl.receivers)

        def make_oracle():
            o = oracle.Oracle2D(n, n, wl.dx, wl.dx, gh.dt, ca[..., 0], cb[..., 0])
            o.add_point_source("Hz", i, j, oracle.gauss_deriv_wave(wl.steps, gh.dt))
            return o, [("Hz", a, b) for a, b in wl.receivers]

        name = f"lossy_ellipses_{n}x{n}_{wl.steps}steps_16rx"
        return sim, det, (ca, cb), (cad, cbd), wave, n * n, 32, make_oracle, name, "k2d_pass"

    B = max(1, args.instances)
    wls = [W.Head3D(n=args.side or 256, steps=args.nsteps, seed=4 + q) for q in range(B)]
    wl = wls[0]
    n = wl.n
    gh = YeeGrid(n, n, wl.dx, wl.dx, Nz=n, dz=wl.dx, courant=wl.courant, device="cpu")
    cas, cbs = [], []
    for w in wls:
        mm = MaterialMap3D(gh, default=w.background(Material))
        w.paint(mm, Material)
        a, c = mm.build3d()
        cas.append(a)
        cbs.append(c)
    ca, cb = (cas[0], cbs[0]) if B == 1 else (torch.stack(cas), torch.stack(cbs))
    g = YeeGrid(n, n, wl.dx, wl.dx, Nz=n, dz=wl.dx, courant=wl.courant, device=dev)
    f = FieldSet(g, batch_size=B)
    wave = GaussianDerivativePulse(1e9).build(wl.steps, g.dt, dev)
    i, j, k = wl.source
    src = PointSource(_TableWave(wave), i, j, "Ez", k=k, grid=g, N_steps=wl.steps)
    cad, cbd = ca.to(dev), cb.to(dev)
    sim = FDTD3D(g, f, MurABC3D(g, f.Hx, f.Hy, f.Hz), SourceCollection([src]), Ca=cad, Cb=cbd,
                 tune=_tune_arg(args))
    det = Detectors([("Ez",) + tuple(r) for r in wl.receivers()])

    def make_oracle():
        o = oracle.Oracle3D(n, n, n, wl.dx, wl.dx, wl.dx, gh.dt, cas[0], cbs[0])
        o.add_point_source("Ez", i, j, oracle.gauss_deriv_wave(wl.steps, gh.dt), k=k)
        return o, [("Ez",) + tuple(r) for r in wl.receivers()]

    name = f"head3d_{n}^3_{wl.steps}steps_{wl.n_rx}rx" + (f"_x{B}_instances" if B > 1 else "")
    # the library runs the TMA-ring kernel when Nz % 4 == 0 unless a tune picks
    # the register streaming kernel (variant 1 or 2) or the tile kernel
    t = _tune_arg(args)
    kern = ("k3d_tma" if n % 4 == 0 and (t is None or (t[1] == 0 and t[4] == 0))
            else "k3d_stream" if t is None or t[1] == 0 else "k3d_pass")
    return sim, det, (ca, cb), (cad, cbd), wave, B * n ** 3, 56, make_oracle, name, kern


def cpu_single_sample(make_oracle, cells, max_steps, budget_s=12.0):
    """Time the CPU port of the reference loop on the same solve until
    ``budget_s`` of work (or the solve's last step); returns (Gcell-upd/s,
    cores, sample text)."""
    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    o, probes = make_oracle()
    o.run(1, probes)   # warm-up
    done, t = 0, 0.0
    while t < budget_s and done + 6 <= max_steps:
        t0 = time.perf_counter()
        o.run(5, probes)
        t += time.perf_counter() - t0
        done += 5
    return (cells * done / t / 1e9, threads,
            f"the same solve, first {done + 1} steps with its receivers gathered per step "
            f"({cells * done:.3e} cell-updates in {t:.1f} s)")


def companion_legs(args, dev):
    """The rest of the metric on the same GPU, reported beside the headline:
    the plain kernel at 4096^2 (its HBM-roofline target), the 256^3 head
    solve, and the served stream with p50/p99 latency.  Each runs its whole
    workload once untimed, then is timed with CUDA events (plain2d, head3d:
    two full solves; serve: one full stream and its one-at-a-time baseline)."""
    import copy
    from waveforge_b200 import workloads as W
    from waveforge_b200.serving import Server, serve_one_at_a_time
    peak, peak_kind = measured_peaks()
    stream = torch.cuda.current_stream(dev)
    out = {}
    for wk, nsteps, side in (("plain2d", 2000, 4096), ("head3d", 1500, 256)):
        a = copy.copy(args)
        a.workload, a.nsteps, a.side, a.tune, a.instances = wk, nsteps, side, None, 1
        sim, det, _, _, _, cells, bpc, _, name, kname = build_single(a, dev)
        sim.reset()
        sim.run(nsteps, record=det)
        ms = []
        for _ in range(2):
            sim.reset()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            sim.run(nsteps, record=det)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            ms.append(e0.elapsed_time(e1))
        t = statistics.mean(ms) * 1e-3
        gcu = cells * nsteps / t / 1e9
        dram = None
        tfile = ROOT / "profiles" / f"{kname}_traffic.txt"
        if tfile.exists():
            for tl in tfile.read_text().splitlines():
                if tl.startswith("dram_bytes_per_cell_update="):
                    dram = float(tl.split("=")[1])
        out[f"{wk}_{side}"] = {
            "workload": name, "value": gcu, "unit": UNIT, "ms_per_solve": t * 1e3,
            "kernel": kname, "bytes_per_cell_update": bpc,
            "frac_algorithmic": gcu * bpc / peak, "peak_gbs": peak, "peak_kind": peak_kind,
            "dram_bytes_per_cell_update_ncu": dram,
            "dram_frac_of_peak": None if dram is None else gcu * dram / peak}
        del sim, det
        torch.cuda.empty_cache()
    arrivals = W.ServingStream(rate=200.0, duration=10.0, seed=args.seed,
                               grad_fraction=0.1).arrivals()
    warm = W.ServingStream(rate=20.0, duration=0.3, seed=args.seed + 1, side_max=256,
                           steps_max=1200).arrivals()
    Server(dev, max_wait_s=2.0).serve(warm)
    srv = Server(dev, chunk_steps=128, max_wait_s=2.0, hbm_budget=60e9, max_active_cells=3.2e7)
    tickets = srv.serve(arrivals)
    stats = _stream_stats(tickets, max(t.t_done for t in tickets if t.t_done is not None))
    base = serve_one_at_a_time(dev, arrivals, max_wait_s=2.0)
    bstats = _stream_stats(base, max(t.t_done for t in base if t.t_done is not None))
    out["serve"] = {
        "workload": "serve_poisson200_10s_side128-1024_steps1000-5000_16tx_grad10pct",
        "requests": len(arrivals), "p50_s": stats["p50_s"], "p99_s": stats["p99_s"],
        "served": stats["served"], "rejected": stats["rejected"],
        "gradient_served": stats["gradient_served"],
        "served_gcell_upd_per_s": stats["gcell_upd_per_s"], "solves_per_s": stats["solves_per_s"],
        "one_at_a_time": {"p50_s": bstats["p50_s"], "p99_s": bstats["p99_s"],
                          "served": bstats["served"], "rejected": bstats["rejected"],
                          "served_gcell_upd_per_s": bstats["gcell_upd_per_s"]},
        "policy": "FIFO admission by HBM footprint (60 GB) and in-flight cells; reject at "
                  "arrival when the estimated wait exceeds 2 s; latency = arrival -> traces "
                  "(and gradients) in pinned host memory"}
    return out


def bench_single(args, ws, rank, local):
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    sim, det, host_c, dev_c, wave, cells, bpc, make_oracle, name, kname = build_single(args, dev)
    stream = torch.cuda.current_stream(dev)
    nsteps = args.nsteps
    upd = cells * nsteps

    def one_step():
        sim.reset()
        return sim.run(nsteps, record=det)

    for _ in range(args.warmup):
        tr_shape = tuple(one_step().shape)
    torch.cuda.synchronize(dev)
    barrier(ws)
    clk = ClockSampler(local)
    clk.start()
    times = []
    for _ in range(args.steps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        one_step()
        b.record(stream)
        torch.cuda.synchronize(dev)
        times.append(a.elapsed_time(b))
    barrier(ws)
    clocks = clk.stop()
    ms_step = reduce_max(sum(times) / len(times), ws, dev)
    value = ws * upd / (ms_step * 1e-3) / 1e9

    # e2e: coefficients and waveform from pinned host memory, traces back to the host
    ca_h, cb_h = (c.pin_memory() for c in host_c)
    wave_h = wave.cpu().pin_memory()
    tr_h = torch.empty(tr_shape, dtype=torch.float32, pin_memory=True)

    def e2e_step():
        dev_c[0].copy_(ca_h, non_blocking=True)
        dev_c[1].copy_(cb_h, non_blocking=True)
        wave.copy_(wave_h, non_blocking=True)
        tr = one_step()
        tr_h.copy_(tr, non_blocking=True)

    for _ in range(args.warmup):
        e2e_step()
    torch.cuda.synchronize(dev)
    barrier(ws)
    s2 = torch.cuda.Event(enable_timing=True)
    e2 = torch.cuda.Event(enable_timing=True)
    s2.record(stream)
    for _ in range(args.steps):
        e2e_step()
    e2.record(stream)
    torch.cuda.synchronize(dev)
    ms_e2e = reduce_max(s2.elapsed_time(e2), ws, dev) / args.steps
    h2d = (ca_h.numel() + cb_h.numel() + wave_h.numel()) * 4
    d2h = tr_h.numel() * 4

    peak, peak_kind = measured_peaks()
    achieved = bpc * upd / (ms_step * 1e-3) / 1e9
    k = sim._tune.steps_per_pass if sim._tune is not None else None
    # DRAM bytes of one launch: the ncu figure per cell-update (profiles/) x
    # the cell-updates of one launch (2D: one pass of the default depth 6 on
    # grids >= 2^20 cells; 3D: one step of every member)
    traffic = None
    tfile = ROOT / "profiles" / f"{kname}_traffic.txt"
    per_launch = cells * (6 if kname == "k2d_pass" and cells >= 1 << 20 else 1)
    if tfile.exists() and (kname != "k2d_pass" or args.tune is None):
        for tl in tfile.read_text().splitlines():
            if tl.startswith("dram_bytes_per_cell_update="):
                traffic = float(tl.split("=")[1]) * per_launch
    roof = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
            "bytes_per_cell_update": bpc,
            "note": f"algorithmic bytes = {bpc} B x cell-updates / run time (all passes); "
                    "temporal blocking re-uses tiles on chip, so frac may exceed 1"}
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        per_solve = cells // sim.fields.batch_size
        v, cores, sample = cpu_single_sample(make_oracle, per_solve, nsteps, args.ref_budget)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}
    if rank == 0:
        line = {
            "metric": f"Gcell-upd/s ({args.workload}, fp32)", "value": value, "unit": UNIT,
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": name, "cell_updates_per_step": upd, "tune": k,
                       "l2": "fields + coefficients > L2, no flush", "parallelism": f"replicas x{ws}"},
            "e2e": {"value": ws * upd / (ms_e2e * 1e-3) / 1e9, "unit": UNIT,
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": ms_e2e},
            "roofline": roof, "cpu_baseline": cpu, "clocks": clocks,
            "gpu_launches": args.steps * pass_launches(nsteps, k or default_depth(args.workload, cells)),
        }
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# serving: Poisson stream through the continuous-batching server
# ---------------------------------------------------------------------------

def _stream_stats(tickets, window_s):
    from waveforge_b200.serving import request_work
    done = [t for t in tickets if t.status == "done"]
    lat = sorted(t.latency for t in done)

    def pct(p):
        return lat[min(len(lat) - 1, int(math.ceil(p * len(lat))) - 1)] if lat else None

    upd = sum(request_work(t.request) for t in done)
    solves = sum(len(t.request.transmitters) for t in done)
    return {"served": len(done), "rejected": sum(t.status == "rejected" for t in tickets),
            "gradient_served": sum(t.request.target is not None for t in done),
            "p50_s": pct(0.50), "p99_s": pct(0.99),
            "mean_s": statistics.mean(lat) if lat else None,
            "solves_per_s": solves / window_s, "gcell_upd_per_s": upd / window_s / 1e9,
            "window_s": window_s, "cell_updates": upd}


def bench_serve(args, ws, rank, local):
    from waveforge_b200 import workloads as W
    from waveforge_b200.serving import Server, serve_one_at_a_time
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    t_gen = time.perf_counter()
    arrivals = W.ServingStream(rate=args.rate, duration=args.duration, seed=args.seed,
                               grad_fraction=args.grad_fraction).arrivals()
    log(f"[bench] {len(arrivals)} requests generated in {time.perf_counter() - t_gen:.1f}s")
    warm = W.ServingStream(rate=20.0, duration=0.3, seed=args.seed + 1, side_max=256,
                           steps_max=1200).arrivals()
    for _ in range(args.warmup):
        Server(dev, max_wait_s=args.max_wait).serve(warm)
    serve_one_at_a_time(dev, warm[:2])
    torch.cuda.synchronize(dev)
    barrier(ws)
    clk = ClockSampler(local)
    clk.start()
    stats = srv = None
    for _ in range(args.steps):
        srv = Server(dev, chunk_steps=args.chunk, max_wait_s=args.max_wait,
                     hbm_budget=args.hbm_budget * 1e9, max_active_cells=args.max_cells)
        tickets = srv.serve(arrivals)
        window = max(t.t_done for t in tickets if t.t_done is not None)
        stats = _stream_stats(tickets, window)
    clocks = clk.stop()
    base = serve_one_at_a_time(dev, arrivals, max_wait_s=args.max_wait)
    bwin = max(t.t_done for t in base if t.t_done is not None)
    bstats = _stream_stats(base, bwin)
    value = reduce_max(-stats["gcell_upd_per_s"], ws, dev) * -1.0   # slowest replica
    if rank == 0:
        line = {
            "metric": "served Gcell-upd/s (continuous batching, Poisson stream, fp32)",
            "value": value * ws, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": stats["window_s"] * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": f"serve_poisson{args.rate:g}_{args.duration:g}s_side128-1024_"
                                   "steps1000-5000_16tx_grad10pct",
                       "requests": len(arrivals), "hbm_budget_gb": args.hbm_budget,
                       "chunk_steps": args.chunk, "max_wait_s": args.max_wait,
                       "policy": "FIFO admission by HBM footprint and <= 3 solves/SM in flight; "
                                 "reject at arrival when the estimated wait exceeds max_wait_s",
                       "parallelism": f"replicas x{ws}"},
            "latency_s": {"p50": stats["p50_s"], "p99": stats["p99_s"], "mean": stats["mean_s"]},
            "serving": stats,
            "one_at_a_time": bstats,
            "served_over_one_at_a_time": stats["gcell_upd_per_s"] / bstats["gcell_upd_per_s"],
            "e2e": {"value": value * ws, "unit": UNIT, "h2d_bytes_per_step": srv.h2d_bytes,
                    "d2h_bytes_per_step": srv.d2h_bytes,
                    "note": "requests enter as host objects (phantom region lists) and leave as "
                            "pinned host traces/gradients: the served figure is end to end"},
            "clocks": clocks, "gpu_launches": srv.launches,
        }
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# adjoint: one misfit gradient (forward with checkpoints + reverse pass)
# ---------------------------------------------------------------------------

def bench_adjoint(args, ws, rank, local):
    from waveforge_b200 import MisfitProblem2D, PointSource, SourceCollection, YeeGrid, fdtd_misfit
    from waveforge_b200 import workloads as W
    from waveforge_b200.core.sources import TabulatedWaveform
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    side, steps = args.side or 512, args.nsteps
    req = W.serving_request(side, steps, args.seed, gradient=True)
    gh = req.material._grid
    g = YeeGrid(side, side, gh.dx, gh.dy, courant=gh.courant, device=dev)
    wave = TabulatedWaveform(req.waveform.build(steps, g.dt, "cpu"))
    srcs = [SourceCollection([PointSource(wave, i, j, "Hz", grid=g, N_steps=steps)])
            for i, j in req.transmitters]
    n_tx, n_rx = len(srcs), len(req.receivers)
    eps_t = torch.empty((side, side), dtype=torch.float64, device=dev)
    sig_t = torch.empty_like(eps_t)
    req.target.build_device(dev, eps_sigma=(eps_t, sig_t))
    tp = MisfitProblem2D(g, srcs, list(req.receivers), torch.zeros(n_tx, n_rx, steps), steps)
    with torch.no_grad():
        fdtd_misfit(eps_t, sig_t, tp)
    prob = MisfitProblem2D(g, srcs, list(req.receivers), tp.traces, steps)
    eps = torch.empty_like(eps_t)
    sig = torch.empty_like(eps_t)
    req.material.build_device(dev, eps_sigma=(eps, sig))

    def one():
        e = eps.clone().requires_grad_(True)
        s = sig.clone().requires_grad_(True)
        a = torch.cuda.Event(enable_timing=True)
        m = torch.cuda.Event(enable_timing=True)
        z = torch.cuda.Event(enable_timing=True)
        a.record()
        loss = fdtd_misfit(e, s, prob)
        m.record()
        loss.backward()
        z.record()
        return a, m, z, e.grad

    for _ in range(args.warmup):
        one()
    torch.cuda.synchronize(dev)
    barrier(ws)
    clk = ClockSampler(local)
    clk.start()
    fw, bw, tot = [], [], []
    for _ in range(args.steps):
        a, m, z, gr = one()
        torch.cuda.synchronize(dev)
        fw.append(a.elapsed_time(m))
        bw.append(m.elapsed_time(z))
        tot.append(a.elapsed_time(z))
    clocks = clk.stop()
    ms = reduce_max(statistics.mean(tot), ws, dev)
    upd = n_tx * side * side * steps
    if rank == 0:
        line = {
            "metric": "gradient Gcell-upd/s (misfit forward + adjoint, fp32)",
            "value": ws * upd / (ms * 1e-3) / 1e9, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": f"adjoint_lossy_{side}x{side}_{steps}steps_{n_tx}tx",
                       "checkpoint_every": prob.K, "parallelism": f"replicas x{ws}",
                       "note": "value counts the forward cell-updates of the model phantom; "
                               "one step = forward with sqrt(N) checkpoints + reverse pass "
                               "(segment recompute + time-reversed Yee step per step)"},
            "forward_ms": statistics.mean(fw), "backward_ms": statistics.mean(bw),
            "backward_over_forward": statistics.mean(bw) / statistics.mean(fw),
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)


def bench_dataset(args, ws, rank, local):
    """Brain dataset generation at the reference generator's defaults (64^3,
    3 mm, 8-element ring r = 30 cells, 300 steps, 1 GHz): one step = one
    sample (two phantoms painted, both MIMO acquisitions as one batched
    2 x 8-member solve, scattered signals, DAS image, compressed .npz)."""
    import tempfile
    import oracle
    from waveforge_b200.datasets import BrainDatasetGenerator
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    n, n_tx, steps = args.side or 64, 8, args.nsteps
    tmp = tempfile.TemporaryDirectory()
    gen = BrainDatasetGenerator(tmp.name, grid_size=n, dx_mm=3.0, n_tx=n_tx,
                                ring_radius_cells=min(30, n // 2 - 2), n_steps=steps,
                                device=str(dev), seed=args.seed, verbose=False)
    counter = iter(range(10 ** 9))
    per_step = max(1, args.batch_samples)

    def one():
        """``per_step`` samples, all acquisitions in one batched solve."""
        ids = [next(counter) for _ in range(per_step)]
        out = gen.generate_samples([(i % 4, args.seed * 1000 + i) for i in ids])
        for i, smp in zip(ids, out):
            if smp is not None:
                gen.save_sample_async(smp, i)   # written while the next solve runs
        return sum(smp is not None for smp in out)

    def plain():
        """The same two acquisitions, one solve at a time (the reference's
        per-transmitter loop on this library's kernels)."""
        from waveforge_b200.datasets.brain import BrainPhantom3D, sample_random_geometry
        ph = BrainPhantom3D(gen.grid, 1e9, geometry=sample_random_geometry(args.seed, n, 3.0),
                            seed=args.seed)
        t0 = time.perf_counter()
        for _ in range(2):
            for t in range(n_tx):
                gen._run_simulation(ph, t)
        torch.cuda.synchronize(dev)
        return time.perf_counter() - t0

    for _ in range(args.warmup):
        one()
    gen.flush()
    torch.cuda.synchronize(dev)
    barrier(ws)
    clk = ClockSampler(local)
    clk.start()
    t0 = time.perf_counter()
    done = 0
    for _ in range(args.steps):
        done += one()
    gen.flush()
    torch.cuda.synchronize(dev)
    el = time.perf_counter() - t0
    clocks = clk.stop()
    el = reduce_max(el, ws, dev)
    plain_s = plain() if rank == 0 and not args.no_plain else None
    upd = 2 * n_tx * n ** 3 * steps   # per sample
    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline:
            from waveforge_b200.datasets.brain import BrainPhantom3D, sample_random_geometry
            from waveforge_b200.core.grid import YeeGrid
            gh = YeeGrid(n, n, 3e-3, 3e-3, Nz=n, dz=3e-3, device="cpu")
            ph = BrainPhantom3D(gh, 1e9, geometry=sample_random_geometry(args.seed, n, 3.0),
                                seed=args.seed)
            ca, cb = ph.build()
            pos = gen.ring.positions
            wave = gen._waveform().build(steps, gh.dt, "cpu")

            def make_oracle():
                o = oracle.Oracle3D(n, n, n, gh.dx, gh.dy, gh.dz, gh.dt, ca, cb)
                o.add_point_source("Ez", pos[0][0], pos[0][1], wave, k=pos[0][2])
                return o, [("Ez", i, j, k) for i, j, k in pos]
            v, cores, sample = cpu_single_sample(make_oracle, n ** 3, steps, args.ref_budget)
            cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                   "sample": "one transmitter solve of a sample: " + sample}
        rate = ws * done / el
        # per sample: two phantoms' region lists (<= 7 spheres x 40 B) and
        # material tables (<= 8 x 8 B) cross to the device; Ca/Cb are painted there
        h2d = per_step * 2 * (7 * 40 + 8 * 8)
        d2h = per_step * 2 * n_tx * n_tx * steps * 4
        line = {
            "metric": "dataset samples/s (brain haemorrhage, 2 x 8-TX MIMO per sample)",
            "value": rate, "unit": "samples/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3,
            "samples_per_step": per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": f"brain_dataset_{n}^3_3mm_{n_tx}tx_{steps}steps",
                       "cell_updates_per_sample": upd, "parallelism": f"replicas x{ws}",
                       "samples_per_solve": per_step,
                       "note": "wall clock: seeded geometry and bleed placement on the host, "
                               "phantoms painted on the device, the acquisitions of "
                               "samples_per_solve samples (16 each) in one batched solve, DAS, "
                               "compressed npz write on a background thread"},
            "gcell_upd_per_s": rate * upd / 1e9,
            "plain_per_solve_samples_per_s": None if plain_s is None else 1.0 / plain_s,
            "e2e": {"value": rate, "unit": "samples/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "cpu_baseline": cpu, "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    tmp.cleanup()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="mimo",
                    choices=["mimo", "plain2d", "head3d", "serve", "adjoint", "dataset"],
                    help="mimo: batched uneven breast MIMO (default, the headline metric); "
                         "plain2d: one 4096^2 lossy 2D solve; head3d: one 256^3 head solve; "
                         "serve: Poisson request stream through the continuous-batching server; "
                         "adjoint: one misfit gradient (forward + adjoint) of a 512^2 16-TX phantom; "
                         "dataset: brain dataset samples (two batched 8-TX MIMO acquisitions each)")
    ap.add_argument("--batch-mode", default="auto", choices=["persistent", "tiled", "queue", "auto"],
                    help="mimo: one persistent launch per batch (a CTA per solve), one tile launch "
                         "per pass, one persistent launch over a (pass, tile) queue, or the "
                         "autotuner's pick (default)")
    ap.add_argument("--no-graph", dest="graph", action="store_false",
                    help="mimo: launch each run directly instead of replaying its CUDA graph")
    ap.add_argument("--tune", default=None, help="K,tile_i,tile_j,tile_k,threads of the kernel (mimo: batched; plain2d/head3d: "
                         "the solve's tune)")
    ap.add_argument("--rate", type=float, default=200.0, help="serve: arrivals per second")
    ap.add_argument("--duration", type=float, default=10.0, help="serve: arrival window (s)")
    ap.add_argument("--max-wait", type=float, default=2.0, help="serve: wait bound (s)")
    ap.add_argument("--chunk", type=int, default=128, help="serve: steps per chunk")
    ap.add_argument("--hbm-budget", type=float, default=60.0, help="serve: admission budget (GB)")
    ap.add_argument("--grad-fraction", type=float, default=0.1, help="serve: gradient requests")
    ap.add_argument("--max-cells", type=float, default=3.2e7, help="serve: in-flight cell cap")
    ap.add_argument("--side", type=int, default=None,
                    help="grid side of plain2d (4096) / head3d (256)")
    ap.add_argument("--instances", type=int, default=1,
                    help="head3d: independent instances advanced in one launch per step")
    ap.add_argument("--phantoms", type=int, default=64)
    ap.add_argument("--tx", type=int, default=16)
    ap.add_argument("--nsteps", type=int, default=None,
                    help="time steps per solve (mimo 3000, plain2d 2000, head3d 1500)")
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--ref-budget", type=float, default=12.0)
    ap.add_argument("--batch-samples", type=int, default=4,
                    help="dataset: samples whose acquisitions share one batched solve")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="mimo: skip the plain2d/head3d/serve companion legs")
    args = ap.parse_args()
    if args.warmup < 3:
        raise SystemExit("--warmup must be >= 3")
    if args.nsteps is None:
        args.nsteps = {"mimo": 3000, "plain2d": 2000, "head3d": 1500, "serve": 0,
                       "adjoint": 1000, "dataset": 300}[args.workload]
    ws, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference_arm(args, ws, rank)
        barrier(ws)
        return
    if args.workload == "adjoint":
        bench_adjoint(args, ws, rank, local)
        barrier(ws)
        return
    if args.workload == "dataset":
        bench_dataset(args, ws, rank, local)
        barrier(ws)
        return
    if args.workload == "serve":
        if "--steps" not in sys.argv:
            args.steps = 1   # one timed stream unless asked
        bench_serve(args, ws, rank, local)
        barrier(ws)
        return
    if args.workload != "mimo":
        bench_single(args, ws, rank, local)
        barrier(ws)
        return

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    t_setup = time.perf_counter()
    tune = None if args.tune is None else tuple(int(v) for v in args.tune.split(","))
    wl, phantoms, batches, host_coeffs, dev_coeffs, waves = build_workload(
        dev, args.phantoms, args.tx, args.nsteps, args.seed, args.batch_mode, tune)
    images = torch.zeros((len(phantoms), DAS_SIZE, DAS_SIZE), dtype=torch.float64, device=dev)
    cells_per_step = 2 * batches[True].cells * args.nsteps   # both twins
    log(f"[bench] setup {time.perf_counter() - t_setup:.1f}s, {2 * len(batches[True].solves)} solves, "
        f"{cells_per_step:.3e} cell-updates per step")
    stream = torch.cuda.current_stream(dev)

    kern_ms = []

    if args.graph:
        for b in batches.values():
            b.capture()

    def one_step(record=False):
        if not args.graph:
            for b in batches.values():
                b.reset()
        ev = []
        for t in (True, False):
            b = batches[t]
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            if args.graph:
                e0.record(stream)
                b.replay()
                e1.record(stream)
            else:
                b._upload(0, args.nsteps)
                e0.record(stream)
                b.launch()
                e1.record(stream)
                b.step = args.nsteps
            ev.append((e0, e1))
        das_all(batches, phantoms, wl, args.tx, dev, images)
        return ev

    # ---- device-resident leg -------------------------------------------
    for _ in range(args.warmup):
        one_step()
    torch.cuda.synchronize(dev)
    barrier(ws)
    clk = ClockSampler(local)
    clk.start()
    torch.cuda.synchronize(dev)
    barrier(ws)
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    evs = []
    for _ in range(args.steps):
        evs.append(one_step())
    end.record(stream)
    torch.cuda.synchronize(dev)
    barrier(ws)
    clocks = clk.stop()
    ms_total = start.elapsed_time(end)
    for ev in evs:
        for e0, e1 in ev:
            kern_ms.append(e0.elapsed_time(e1))
    statuses = batches[True].statuses() + batches[False].statuses()
    if any(statuses):
        raise RuntimeError(f"batched solves reported status {set(statuses)}")
    ms_total = reduce_max(ms_total, ws, dev)
    ms_step = ms_total / args.steps
    value = ws * cells_per_step / (ms_step * 1e-3) / 1e9

    # ---- e2e leg: host buffers through the public API ---------------------
    host_traces = {t: torch.empty(batches[t]._traces.shape, dtype=torch.float32, pin_memory=True)
                   for t in batches}
    host_images = torch.empty(images.shape, dtype=torch.float64, pin_memory=True)
    h2d = sum(c.numel() * 4 * 2 for c, _ in host_coeffs.values()) + sum(
        w.numel() * 4 for w in waves.values())
    d2h = sum(h.numel() * 4 for h in host_traces.values()) + host_images.numel() * 8
    host_waves = {k: w.cpu().pin_memory() for k, w in waves.items()}

    def e2e_step():
        for key, (ca_h, cb_h) in host_coeffs.items():
            ca_d, cb_d = dev_coeffs[key]
            ca_d.copy_(ca_h, non_blocking=True)
            cb_d.copy_(cb_h, non_blocking=True)
        for k, w in host_waves.items():
            waves[k].copy_(w, non_blocking=True)
        one_step()
        for t in batches:
            host_traces[t].copy_(batches[t]._traces, non_blocking=True)
        host_images.copy_(images, non_blocking=True)

    # the e2e leg repeats the same multi-second step: a few steps bound it tightly
    e2e_steps = min(args.steps, 5)
    for _ in range(min(args.warmup, 3)):
        e2e_step()
    torch.cuda.synchronize(dev)
    barrier(ws)
    s2 = torch.cuda.Event(enable_timing=True)
    e2 = torch.cuda.Event(enable_timing=True)
    s2.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    e2.record(stream)
    torch.cuda.synchronize(dev)
    barrier(ws)
    ms_e2e = reduce_max(s2.elapsed_time(e2), ws, dev) / e2e_steps
    e2e_value = ws * cells_per_step / (ms_e2e * 1e-3) / 1e9

    # ---- plain per-solve comparison (stratified sample) -------------------
    plain = None
    if not args.no_plain:
        by_side = {}
        for p, ph in enumerate(phantoms):
            by_side.setdefault(ph.side, p)
        counts = {}
        for ph in phantoms:
            counts[ph.side] = counts.get(ph.side, 0) + 1
        sub_solves = []
        for side, p in sorted(by_side.items()):
            sub_solves += [batches[True].solves[p * args.tx + tx] for tx in range(2)]
        from waveforge_b200 import Batch2D
        sub = Batch2D(sub_solves, args.nsteps)
        per_side_ms, per_side_graph_ms = {}, {}
        for q in range(0, len(sub_solves), 2):
            side = sub_solves[q].grid.Nx
            times, gtimes = [], []
            for rep in range(2):
                sub.reset()
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                sub.run_plain_one(q)
                b.record(stream)
                torch.cuda.synchronize(dev)
                times.append(a.elapsed_time(b))
            # the same solve with its pass launches replayed from a CUDA graph
            graph = torch.cuda.CUDAGraph()
            side_stream = torch.cuda.Stream(dev)
            side_stream.wait_stream(stream)
            with torch.cuda.stream(side_stream):
                with torch.cuda.graph(graph, stream=side_stream, capture_error_mode="relaxed"):
                    sub._state.zero_()
                    sub.run_plain_one(q)
            stream.wait_stream(side_stream)
            for rep in range(3):
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                graph.replay()
                b.record(stream)
                torch.cuda.synchronize(dev)
                gtimes.append(a.elapsed_time(b))
            del graph
            per_side_ms[side] = min(times)
            per_side_graph_ms[side] = min(gtimes[1:])
        total_ms = sum(counts[s] * args.tx * per_side_ms[s] for s in counts) * 2  # both twins
        total_gms = sum(counts[s] * args.tx * per_side_graph_ms[s] for s in counts) * 2
        plain_value = cells_per_step / (total_ms * 1e-3) / 1e9
        plain_graph_value = cells_per_step / (total_gms * 1e-3) / 1e9
        best_plain = max(plain_value, plain_graph_value)
        plain = {"value": best_plain, "unit": UNIT,
                 "launched": plain_value, "graph_replayed": plain_graph_value,
                 "ms_per_solve_by_side": {str(k): round(v, 3) for k, v in sorted(per_side_ms.items())},
                 "ms_per_solve_by_side_graph": {str(k): round(v, 3)
                                                for k, v in sorted(per_side_graph_ms.items())},
                 "sample": "one phantom per grid size, 2 TX each, timed one solve at a time with "
                           "wf_fdtd2d_run, launched pass by pass and replayed from a CUDA graph of "
                           "its passes; the faster of the two is the comparison; extrapolated by "
                           "the workload's size histogram",
                 "batched_over_plain": value / ws / best_plain}

    # ---- roofline of the dominant kernel ----------------------------------
    peak, peak_kind = measured_peaks()
    k_ms = statistics.mean(kern_ms)
    achieved = BYTES_PER_CELL_UPDATE * (cells_per_step / 2) / (k_ms * 1e-3) / 1e9
    traffic = None
    kname = {"persistent": "k_batch2d", "tiled": "k_batch_pass",
             "queue": "k_batch_queue"}[batches[True].mode]
    tfile = ROOT / "profiles" / f"{kname}_traffic.txt"
    if tfile.exists():
        for line in tfile.read_text().splitlines():
            if line.startswith("dram_bytes_per_cell_update="):
                traffic = float(line.split("=")[1]) * cells_per_step / 2
    roof = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak,
            "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
            "bytes_per_cell_update": BYTES_PER_CELL_UPDATE,
            "launch_ms": k_ms, "note": "algorithmic bytes = 32 B x cell-updates of one batch run "
                                       "(persistent: one launch; tiled: all its pass launches); "
                                       "temporal blocking re-uses tiles on chip, so frac may exceed 1"}

    extra = {}
    if ws == 1 and not args.no_extras:
        extra = companion_legs(args, dev)

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        v, cores, sample = cpu_reference_sample()
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"breast_mimo_{len(phantoms)}ph_{args.tx}tx_{args.nsteps}steps",
                       "solves_per_step": 2 * len(batches[True].solves),
                       "twins": "tumour + healthy", "das": f"{len(phantoms)} x {DAS_SIZE}x{DAS_SIZE}",
                       "cell_updates_per_step": cells_per_step, "grid_sides": "150-512",
                       "dx_mm": 0.5, "courant": 0.5, "l2": "inputs > L2 (2.6 GB fields), no flush",
                       "batch_mode": batches[True].mode, "graph": args.graph,
                       "tune": args.tune if args.batch_mode != "auto" else
                       [batches[True].depth, *batches[True].region, batches[True].threads],
                       "parallelism": f"replicas x{ws}"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": ms_e2e, "steps": e2e_steps},
            "plain_per_solve": plain, "roofline": roof, "cpu_baseline": cpu, "clocks": clocks,
            "gpu_launches": args.steps * (2 * batches[True].launches_per_run() + len(phantoms)),
        }
        if "serve" in extra:
            line["latency_s"] = {"p50": extra["serve"]["p50_s"], "p99": extra["serve"]["p99_s"],
                                 "of": "the served Poisson stream (key serve)"}
        line.update(extra)
        print(json.dumps(line), flush=True)
    barrier(ws)


if __name__ == "__main__":
    main()
