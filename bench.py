#!/usr/bin/env python
"""bench.py -- throughput of the cpsFDTD time-stepping loop on B200.

Workload (default): the dispersive-scattering deck -- 256^3 cells, dx 5 nm,
CPML 12, TF/SF Gaussian beam (inset 20, 550 nm, theta 30, phi 45, pulse
tau 4 fs), 4x4x4 Drude-Lorentz spheres (r 15, pitch 40), six planar ports with
64-frequency FP64 DFTs; FP32 fields, fused path.  One bench step = one whole
job of --job-steps time steps (default 4000) from a reset state, ports flushed.
Synthetic geometry from the seeded deck generator; no dataset.

Metric: Gcell-upd/s = cells x time steps / time, whole job, all ranks.
  value  : device-timed (CUDA events on the grid's stream), inputs in HBM
  e2e    : through the C ABI from host buffers: grid setup from the deck and
           the host ID grid, the run, and the port spectra read back to host
  roofline: the E sweep (dominant kernel) algorithmic bytes / its mean
           event-timed duration (events around each sweep of one job run
           after the timed region), against the measured HBM copy bandwidth
  cpu_baseline: the reference's own OpenMP code (oracle/_ref/ref_bench; its
           3-D Drude-Lorentz from the oracle restatement) on the same deck
Multi-GPU: one replica job per rank (the path does not shard), weak scaling.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FALLBACK = {"hbm_gbs": 6650.0}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=256, help="grid edge (cells)")
    ap.add_argument("--workload", default="dispersive", choices=["dispersive", "laser"],
                    help="bench deck: dispersive scattering (default) or the photonic-crystal laser")
    ap.add_argument("--job-steps", type=int, default=4000)
    ap.add_argument("--path", default="fused", choices=["fused", "onepass"],
                    help="one-grid stepping path: two TMA sweeps per step (default) or the one-pass step")
    ap.add_argument("--e2e-steps", type=int, default=2, help="end-to-end jobs to time")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--cpu-steps", type=int, default=3, help="time steps in the CPU baseline sample")
    ap.add_argument("--ens-grids", type=int, default=256, help="grids of the batched ensemble leg (0: skip)")
    ap.add_argument("--ens-steps", type=int, default=128, help="timed steps of the batched ensemble")
    ap.add_argument("--ens-loop-steps", type=int, default=8,
                    help="steps per grid of the one-grid-per-launch comparison loops")
    ap.add_argument("--serve-jobs", type=int, default=24, help="jobs of the serving leg (0: skip)")
    ap.add_argument("--serve-step-scale", type=float, default=2.0,
                    help="job step counts are the log-uniform [500, 20000] draws divided by this")
    ap.add_argument("--serve-tile", default="",
                    help="batch tile of the serving loop as rows,planes,mode (empty: the library default)")
    ap.add_argument("--serve-load", type=float, default=2.0,
                    help="offered load: arrival rate x job work / 20 Gcell-upd/s")
    return ap.parse_args()


class Clocks:
    """nvidia-smi sampling of SM clock and throttle reasons during a region."""

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(prefix="cps_clk_", suffix=".csv")
        os.close(fd)
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                smax.append(float(f[1]))
            except ValueError:
                continue
            for nm, v in zip(names, f[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def workload(n, job_steps, kind="dispersive"):
    """The bench deck: the dispersive-scattering deck (default), or the
    disordered photonic-crystal laser deck (four-level gain, 32-frequency
    spherical-port DFT)."""
    from cpsfdtd_b200 import decks
    if kind == "laser":
        return decks.config3(n=n, steps=job_steps, seed=0, nfreq=32)
    return decks.config2(n=n, steps=job_steps, nfreq=64)


def workload_name(dk, kind):
    if kind == "laser":
        return (f"disordered photonic-crystal laser {dk.nx}^3, eps 11.9 spheres in gain-doped eps 2.25, CPML "
                f"{dk.pml['npml'][0]}, Ez seed pulse, spherical port x 32-freq FP64 DFT; 1 bench step = 1 job of "
                f"{dk.nsteps} time steps")
    return (f"dispersive scattering {dk.nx}^3, Drude-Lorentz 4x4x4 spheres, CPML {dk.pml['npml'][0]}, TF/SF "
            f"Gaussian beam, 6 ports x 64-freq FP64 DFT; 1 bench step = 1 job of {dk.nsteps} time steps")


def config_of(dk, kind, world, path="fused"):
    return {"workload": workload_name(dk, kind), "grid": [dk.nx, dk.ny, dk.nz], "time_steps_per_job": dk.nsteps,
            "precision": "fp32 fields, fp64 port accumulators", "path": path,
            "l2": f"inputs larger than L2 (fields {6 * 4 * (dk.nx + 1) * (dk.ny + 1) * (dk.nz + 1) / 1e9:.2f} GB "
                  "per grid)", "parallelism": f"replicas x{world}"}


def aggregate(units_local, ms_local, dist=None, device=None):
    """Whole-job throughput of replicas: units summed over ranks / the slowest
    rank's time (max over ranks); returns (units per second, max ms)."""
    if dist is None:
        return units_local / (ms_local / 1e3), ms_local
    import torch
    t = torch.tensor([ms_local, units_local], dtype=torch.float64, device=device)
    mx = t[:1].clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    tot = t[1:].clone()
    dist.all_reduce(tot, op=dist.ReduceOp.SUM)
    return float(tot.item()) / (float(mx.item()) / 1e3), float(mx.item())


def sweep_bytes(dk, ndl, prec_bytes=4, ngain=0):
    """Algorithmic bytes of one H sweep and one E sweep (FP32): each field word
    read and written once, 1 B material ID, CPML psi (2 words read+write per
    slab cell per sweep), Drude-Lorentz state (3 x (nD + 2 nL + 1) words read
    + write per ID-2 cell), gain state (12 polarisation + 3 population words
    read + write per gain cell).  Neighbour re-reads are not counted."""
    nx, ny, nz, s = dk.nx, dk.ny, dk.nz, prec_bytes
    np_ = dk.pml["npml"][0] if dk.pml else 0
    h_cells = nx * ny * nz
    e_cells = (nx - 1) * (ny - 1) * (nz - 1)
    h_slab = 2 * np_ * (ny * nz + nx * nz + nx * ny)
    e_slab = 2 * np_ * ((ny - 1) * (nz - 1) + (nx - 1) * (nz - 1) + (nx - 1) * (ny - 1))
    psi = 2 * 2 * s
    h = h_cells * (9 * s + 1) + h_slab * psi
    stride = len(dk.dl["fD"]) + 2 * len(dk.dl["fL"]) + 1 if dk.dl else 0
    e = e_cells * (9 * s + 1) + e_slab * psi + ndl * 3 * stride * 2 * s + ngain * 15 * 2 * s
    return h, e


def onepass_bytes(dk, ngain, prec_bytes=4):
    """Algorithmic bytes of one one-pass sweep (FP32): the six fields read and
    written once, 1 B ID, CPML psi of both sides (2 words read + write per slab
    cell and side), gain state; the Drude-Lorentz cells run in their own kernel."""
    h, e = sweep_bytes(dk, 0, prec_bytes, ngain)
    nx, ny, nz, s = dk.nx, dk.ny, dk.nz, prec_bytes
    return h + e - nx * ny * nz * (9 * s + 1) - (nx - 1) * (ny - 1) * (nz - 1) * (9 * s + 1) + nx * ny * nz * (12 * s + 1)


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return world, rank, local, dist


def cpu_baseline(dk, steps, deck_kind="dispersive"):
    """The reference's own code on the same deck, bounded sample on all host cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    threads = os.cpu_count() or 1
    if os.path.exists(oracle.REF_BENCH):
        r = oracle.ref_bench(dk, 1, steps, threads=threads)
        kind = "reference"
        extra = "3-D Drude-Lorentz" if deck_kind == "dispersive" else "3-D four-level gain"
        sample = (f"{dk.nx}^3 deck, {steps} time steps after 1 warm-up, reference BasicFDTD/CPML/TF_SF/Ports "
                  f"(OpenMP) + {extra} from the oracle restatement")
    else:
        o = oracle.Oracle.from_deck(dk, _ids(dk))
        oracle.Oracle.threads(threads)
        o.step(1)
        t0 = time.perf_counter()
        o.step(steps)
        r = {"cells": dk.cells, "steps": steps, "seconds": time.perf_counter() - t0, "threads": threads}
        kind = "port"
        sample = f"{dk.nx}^3 deck, {steps} time steps after 1 warm-up, oracle restatement (OpenMP)"
    gcell = r["cells"] * r["steps"] / r["seconds"] / 1e9
    return {"value": gcell, "unit": "Gcell-upd/s", "cores": r["threads"], "kind": kind, "sample": sample}


_IDS = {}


def _ids(dk):
    import cpsfdtd_b200 as cps
    key = (dk.nx, dk.ny, dk.nz)
    if key not in _IDS:
        _IDS[key] = dk.ids if dk.ids is not None else cps.rasterize(dk.nx, dk.ny, dk.nz, dk.dx, dk.dy, dk.dz, dk.shapes)
    return _IDS[key]


def run_reference(args):
    world, rank, local, dist = dist_setup()
    if rank != 0:
        return
    dk = workload(args.n, args.job_steps, args.workload)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    threads = os.cpu_count() or 1
    if os.path.exists(oracle.REF_BENCH):
        r = oracle.ref_bench(dk, args.warmup, args.steps, threads=threads)
        extra = "3-D Drude-Lorentz" if args.workload == "dispersive" else "3-D four-level gain"
        kind, what = "reference", f"reference BasicFDTD/CPML/TF_SF/Ports (OpenMP) + {extra} from the oracle restatement"
    else:
        o = oracle.Oracle.from_deck(dk, _ids(dk))
        oracle.Oracle.threads(threads)
        o.step(args.warmup)
        t0 = time.perf_counter()
        o.step(args.steps)
        r = {"cells": dk.cells, "steps": args.steps, "seconds": time.perf_counter() - t0, "threads": threads}
        kind, what = "port", "oracle restatement (OpenMP)"
    v = r["cells"] * r["steps"] / r["seconds"] / 1e9
    sample = (f"{dk.nx}^3 {args.workload} deck: each bench step is 1 time step of the job (bounded sample), "
              f"{args.steps} timed after {args.warmup} warm-up, {what}")
    line = {"metric": "Gcell-upd/s", "value": v, "unit": "Gcell-upd/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["seconds"] / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded deck generator)",
            "config": config_of(dk, args.workload, args.gpus, args.path),
            "cpu_baseline": {"value": v, "unit": "Gcell-upd/s", "cores": r["threads"], "kind": kind, "sample": sample},
            "e2e": {"value": v, "unit": "Gcell-upd/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def ensemble(args, local, dist):
    """Batched ensemble: --ens-grids disordered-crystal realizations (edges
    drawn from {64,80,96,112,128} per axis, CPML 8, gain, 32-frequency
    spherical-port DFT) advanced together by the batched engine (autotuned
    tiling, graph-replayed 64-step chunks), against the same grids stepped one
    grid per launch, one after another, on the plain per-routine path and on
    the fused path."""
    import torch
    import cpsfdtd_b200 as cps
    from cpsfdtd_b200 import decks
    t0 = time.perf_counter()
    shapes = decks.config4_shapes(args.ens_grids, seed=0)
    grids = []
    for i, (nx, ny, nz) in enumerate(shapes):
        dk = decks.config4_member(nx, ny, nz, seed=i, steps=5000, nfreq=32)
        grids.append(cps.Grid.from_deck(dk, cps.FP32, device=local))
    setup_s = time.perf_counter() - t0
    cells = sum(nx * ny * nz for nx, ny, nz in shapes)
    b = cps.Batch(cps.FP32)
    for g in grids:
        b.add(g)
    cache = os.path.join(os.path.expanduser("~"), ".cache", "cpsfdtd_b200", "batch_tune.txt")
    os.makedirs(os.path.dirname(cache), exist_ok=True)
    t1 = time.perf_counter()
    tuned_steps = b.autotune(cache, trial_steps=4)
    tune_s = time.perf_counter() - t1
    b.step(128)  # warm-up: a direct 64-step chunk, then its graph capture and replay
    b.sync()
    stream = torch.cuda.ExternalStream(b.stream(), device=local)
    l0 = b.launches()
    if dist:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.step(args.ens_steps)
    e1.record(stream)
    b.sync()
    batched, ms = aggregate(cells * args.ens_steps, e0.elapsed_time(e1), dist, f"cuda:{local}")
    batched /= 1e9
    launches = b.launches() - l0
    tile = list(b.get_tile())
    b.close()

    def loop(path):
        torch.cuda.synchronize()
        ts = time.perf_counter()
        for g in grids:
            g.step(args.ens_loop_steps, path)
            g.sync()
        torch.cuda.synchronize()
        return cells * args.ens_loop_steps / (time.perf_counter() - ts) / 1e9

    loop(cps.FUSED)  # warm-up of the one-grid kernels
    plain = loop(cps.PLAIN)
    fused = loop(cps.FUSED)
    for g in grids:
        g.close()
    return {"workload": f"{args.ens_grids} disordered-crystal realizations, edges U{{64,80,96,112,128}} per axis, "
                        "CPML 8, four-level gain, Ez seed pulse, 32-freq FP64 spherical-port DFT; FP32 fields",
            "grids": args.ens_grids, "cells": int(cells), "metric": "Gcell-upd/s", "value": batched,
            "steps_timed": args.ens_steps, "ms": ms, "tile": tile,
            "plain_one_grid_per_launch": plain, "fused_one_grid_per_launch": fused,
            "speedup_vs_plain_loop": batched / plain if plain else None,
            "speedup_vs_fused_loop": batched / fused if fused else None,
            "gpu_launches": int(launches), "setup_s": setup_s, "autotune_s": tune_s,
            "autotune_steps": tuned_steps, "loop_steps_per_grid": args.ens_loop_steps,
            "timing": "batched: CUDA events on the batch stream; loops: host clock with a device sync per grid"}


def serve_jobs(count, step_scale, seed=0):
    """Seeded job stream: edge log-uniform in [48, 320], steps log-uniform in
    [500, 20000] (divided by step_scale), material mix 40% dielectric (the
    sphere-scatterer deck), 35% Drude-Lorentz spheres + TF/SF + six 64-frequency
    planar-port DFTs (dispersive-scattering parameters), 25% four-level gain
    photonic crystal with a 32-frequency spherical-port DFT (laser parameters)."""
    from cpsfdtd_b200 import decks
    rng = np.random.Generator(np.random.PCG64(seed))
    jobs = []
    for n in range(count):
        edge = int(round(math.exp(rng.uniform(math.log(48), math.log(320)))))
        steps = int(round(math.exp(rng.uniform(math.log(500), math.log(20000))) / step_scale))
        steps = max(1, steps)
        u = rng.uniform()
        kind = "dielectric" if u < 0.40 else ("drude-lorentz" if u < 0.75 else "gain")
        jobs.append((kind, edge, steps, n))
    return jobs


def serve_deck(kind, edge, steps, seed):
    from cpsfdtd_b200 import decks
    if kind == "dielectric":
        return decks.config1(n=edge, steps=steps)
    if kind == "drude-lorentz":
        return decks.config2(n=edge, steps=steps, nfreq=64)
    return decks.config3(n=edge, steps=steps, seed=seed, nfreq=32)


def serving(args, local):
    """Served job stream through the library's serving loop (Poisson arrivals
    offered at --serve-load times a 20 Gcell-upd/s service rate, admission
    against a 180 GB budget, continuous batching), against the same jobs run
    one at a time on the plain per-routine GPU path, queued in arrival order."""
    import torch
    import cpsfdtd_b200 as cps
    jobs = serve_jobs(args.serve_jobs, args.serve_step_scale)
    work = [e ** 3 * st for _, e, st, _ in jobs]
    rng = np.random.Generator(np.random.PCG64(1))
    mean_gap = sum(work) / (args.serve_load * 20e9) / len(jobs)
    arrivals = np.cumsum(rng.exponential(mean_gap, size=len(jobs)))
    arrivals -= arrivals[0]
    budget = 180 * 10 ** 9
    free, total = torch.cuda.mem_get_info(local)
    budget = min(budget, int(free * 0.9))
    tile = tuple(int(v) for v in args.serve_tile.split(",")) if args.serve_tile else None
    srv = cps.Server(cps.FP32, max_jobs=256, budget_bytes=budget, chunk_steps=64, tile=tile)
    done = {}
    t0 = time.perf_counter()
    nxt = 0
    while len(done) < len(jobs):
        now = time.perf_counter() - t0
        while nxt < len(jobs) and arrivals[nxt] <= now:
            kind, edge, steps, seed = jobs[nxt]
            dk = serve_deck(kind, edge, steps, seed)

            def fin(g, status, n=nxt):
                if g is not None and status == 0:
                    for p in range(len(g.ports)):
                        if g.ports[p][2] > 0:
                            g.port_dft(p, raw=True)
                done[n] = (status, time.perf_counter() - t0)

            srv.submit(lambda dk=dk: cps.Grid.from_deck(dk, cps.FP32, device=local), fin, steps,
                       cps.footprint(dk))
            nxt += 1
        live, queued = srv.poll()
        if live == 0 and queued == 0 and nxt < len(jobs):
            time.sleep(max(0.0, min(0.05, arrivals[nxt] - (time.perf_counter() - t0))))
    span = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    lat = sorted(done[n][1] - arrivals[n] for n in range(len(jobs)))
    cells_total = float(sum(work))

    # the same jobs one at a time on the plain path, in arrival order
    service = []
    for kind, edge, steps, seed in jobs:
        dk = serve_deck(kind, edge, steps, seed)
        torch.cuda.synchronize()
        ts = time.perf_counter()
        g = cps.Grid.from_deck(dk, cps.FP32, device=local)
        g.step(steps, cps.PLAIN)
        for p in range(len(g.ports)):
            if g.ports[p][2] > 0:
                g.port_dft(p, raw=True)
        g.sync()
        g.close()
        service.append(time.perf_counter() - ts)
    finish, plain_lat = 0.0, []
    for a, sv in zip(arrivals, service):
        finish = max(finish, a) + sv
        plain_lat.append(finish - a)
    plain_lat.sort()
    pct = lambda v, q: float(np.percentile(v, q))
    return {"workload": f"{len(jobs)} jobs, edge log-uniform [48,320], steps log-uniform [500,20000]/"
                        f"{args.serve_step_scale:g}, mix 40% dielectric / 35% Drude-Lorentz+TF/SF / 25% gain; "
                        f"Poisson arrivals at {args.serve_load:g}x a 20 Gcell-upd/s service rate; FP32 fields, "
                        "FP64 port accumulators",
            "jobs": len(jobs), "jobs_per_s": len(jobs) / span, "gcell_upd_per_s": cells_total / span / 1e9,
            "latency_p50_s": pct(lat, 50), "latency_p99_s": pct(lat, 99),
            "server_latency_p50_ms": st["latency_p50_ms"], "server_latency_p99_ms": st["latency_p99_ms"],
            "wait_p50_ms": st["wait_p50_ms"], "chunks": st["chunks"], "failed": st["jobs_failed"],
            "gpu_busy_s": st["gpu_busy_s"],
            "budget_bytes": budget, "span_s": span, "batch_tile": args.serve_tile or "library default (4,16,2)",
            "plain_one_at_a_time": {"jobs_per_s": len(jobs) / max(finish, 1e-9),
                                    "gcell_upd_per_s": cells_total / sum(service) / 1e9,
                                    "latency_p50_s": pct(plain_lat, 50), "latency_p99_s": pct(plain_lat, 99)},
            "speedup_gcell_vs_plain": (cells_total / span) / (cells_total / sum(service)),
            "timing": "host clock: job latency = completion - arrival, including deck generation and grid "
                      "set-up; plain latencies from measured service times queued in arrival order"}


def run_ours(args):
    import torch
    world, rank, local, dist = dist_setup()
    import cpsfdtd_b200 as cps
    torch.cuda.set_device(local)
    dk = workload(args.n, args.job_steps, args.workload)
    ids = _ids(dk)
    pts = [cps.port_points(dk, p) for p in dk.ports]
    g = cps.Grid.from_deck(dk, cps.FP32, ids=ids, port_points_list=pts, device=local)
    stream = torch.cuda.ExternalStream(g.stream(), device=local)

    path = cps.ONEPASS if args.path == "onepass" else cps.FUSED

    def job(grid):
        grid.reset(dk.n0)
        grid.step(dk.nsteps, path)
        grid.flush_ports()

    for _ in range(args.warmup):
        job(g)
    g.sync()
    launches0 = g.launches()
    clocks = Clocks(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        job(g)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    launches = g.launches() - launches0
    # the sweeps' own durations: per-step CUDA events on one more job, stepped
    # as the direct launch sequence (the timed jobs replay the same kernels in
    # CUDA-graph chunks, where single launches are not timed)
    g.set_timing(1)
    job(g)
    g.sync()
    h_ms, e_ms, nsamp = g.timing()
    g.set_timing(0)
    cells = dk.cells
    value, ms = aggregate(cells * dk.nsteps * args.steps, ms, dist, f"cuda:{local}")
    value /= 1e9

    # roofline of the dominant kernel (E sweep)
    P, src = peaks()
    ndl = 0
    from cpsfdtd_b200 import decks
    ndl = int(((ids[1:-1, 1:-1, 1:-1]) == decks.ID_DISPERSIVE).sum()) if dk.dl else 0
    ngain = int(((ids[1:-1, 1:-1, 1:-1]) == decks.ID_GAIN).sum()) if dk.gain else 0
    hb, eb = sweep_bytes(dk, ndl, ngain=ngain)
    if path == cps.ONEPASS:  # h_ms: the one-pass sweep (with its TF/SF terms); e_ms: the Drude-Lorentz cells
        dom_ms, dom_bytes, dom = h_ms, onepass_bytes(dk, ngain), "one-pass sweep"
    else:
        dom_ms, dom_bytes, dom = (e_ms, eb, "E sweep") if e_ms >= h_ms else (h_ms, hb, "H sweep")
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9 if dom_ms > 0 else 0.0
    roof = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": P["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / P["hbm_gbs"], "peak_source": src, "traffic": None,
            "algorithmic_bytes_per_launch": dom_bytes, "launch_ms": dom_ms, "samples": nsamp,
            "launch_timing": "CUDA events around each sweep on the grid's stream, one job after the timed region",
            "h_sweep_ms": h_ms, "e_sweep_ms": e_ms,
            "step_bytes_per_cell": (hb + eb) / cells,
            "step_frac_at_50B": value / world * 50 / P["hbm_gbs"]}
    tr = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tr) and args.workload == "dispersive" and args.n == 256 and path == cps.FUSED:
        try:
            roof["traffic"] = json.load(open(tr)).get("e_sweep_bytes_per_launch")
        except (ValueError, OSError):
            pass

    # end to end through the C ABI from host buffers
    e2e = None
    if args.e2e_steps > 0:
        pinned_ids = torch.from_numpy(np.ascontiguousarray(ids)).pin_memory()
        # spectra land in pinned host buffers allocated once, like the inputs
        pinned_out = [torch.empty(len(pp) * bin(p.dft_mask).count("1") * len(p.dft_freqs) * 2, dtype=torch.float64)
                      .pin_memory().numpy() if p.dft_freqs is not None else None for p, pp in zip(dk.ports, pts)]
        outs = []
        h2d = d2h = 0
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            gg = cps.Grid.from_deck(dk, cps.FP32, ids=pinned_ids.numpy(), port_points_list=pts, device=local)
            gg.step(dk.nsteps, path)
            outs = [gg.port_dft(n, raw=True, out=pinned_out[n]) for n in range(len(dk.ports))
                    if pinned_out[n] is not None]
            gg.close()
        torch.cuda.synchronize()
        t_e2e = time.perf_counter() - t0
        if dist:
            t = torch.tensor([t_e2e], device=f"cuda:{local}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            t_e2e = float(t.item())
        h2d = ids.nbytes + sum(p.nbytes for p in pts) + sum(len(w) * 8 for *_, w in dk.sources)
        d2h = sum(o.nbytes for o in outs)
        e2e = {"value": cells * dk.nsteps * args.e2e_steps * world / t_e2e / 1e9, "unit": "Gcell-upd/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            cpu = cpu_baseline(workload(args.n, args.job_steps, args.workload), args.cpu_steps, args.workload)
        except Exception as ex:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "Gcell-upd/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"failed: {ex}"}
    srv = None
    if args.serve_jobs > 0 and world == 1:
        try:
            srv = serving(args, local)
        except Exception as ex:
            srv = {"error": str(ex)}
    ens = None
    if args.ens_grids > 0:
        try:
            ens = ensemble(args, local, dist)
        except Exception as ex:
            ens = {"error": str(ex)}
    if rank == 0:
        line = {"metric": "Gcell-upd/s", "value": value, "unit": "Gcell-upd/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
                "data": "synthetic (seeded deck generator)",
                "config": config_of(dk, args.workload, world, args.path),
                "roofline": roof, "clocks": clk, "gpu_launches": int(launches),
                "e2e": e2e, "cpu_baseline": cpu, "ensemble": ens, "serving": srv}
        print(json.dumps(line), flush=True)
    g.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
