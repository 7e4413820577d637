#!/usr/bin/env python
"""bench.py -- throughput of the cpsFDTD time-stepping loop on B200.

Headline workload (default, the largest single-GPU configuration): the
disordered photonic-crystal laser -- 384^3 cells, dx 10 nm, CPML 16, eps 11.9
spheres (r 8, pitch 30, jittered +-4) in an eps 2.25 background doped with
four-level gain, Ez seed pulse, spherical port r 150 with a 32-frequency FP64
DFT; 20000-step jobs.  FP32 fields, FP64 port accumulators, fused path.  One
bench step = --chunk time steps of the job (default 500; the job restarts
from its initial state after its last step).  Synthetic geometry from the
seeded deck generator; no dataset.

Metric: Gcell-upd/s = cells x time steps / time, all ranks.
  value    : device-timed (CUDA events on the grid's stream), inputs in HBM
  e2e      : through the C ABI from host buffers: per e2e step one whole job
             (grid set-up from the host deck, IDs and port points in pinned
             memory, all its time steps, port spectra read back to pinned
             memory)
  fp64     : the same deck in FP64 on the plain path (one kernel per
             reference routine) and on the fused path, value and e2e
  roofline : the E sweep (dominant kernel), algorithmic bytes / its mean
             event-timed duration, against the measured HBM copy bandwidth;
             bytes counted as each field word of the swept side read and
             written once + 1 B ID + CPML psi + gain/Drude-Lorentz state,
             and (printed beside) the two-sweep count that adds the other
             side's field read
  c2       : the dispersive-scattering deck (256^3, Drude-Lorentz spheres,
             TF/SF beam, six 64-frequency ports, 4000-step jobs) beside it
  accuracy : each chosen form against FP64 per config -- field relative L2,
             port-spectrum relative error, resonance-frequency shift
  cpu_baseline: the reference's own OpenMP code (oracle/_ref/ref_bench; the
             3-D gain and Drude-Lorentz from the oracle restatement)
  ensemble : 256 uneven grids (C4) batched vs one grid per launch
  serving  : a Poisson job stream (C5) served vs one job at a time
Multi-GPU: one replica per rank (the path does not shard), weak scaling.

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
    ap.add_argument("--workload", default="laser", choices=["laser", "dispersive"],
                    help="headline deck: the photonic-crystal laser (default) or the dispersive scattering deck")
    ap.add_argument("--n", type=int, default=0, help="grid edge (cells); 0: the workload's own (384 / 256)")
    ap.add_argument("--job-steps", type=int, default=0, help="time steps per job; 0: the workload's own")
    ap.add_argument("--chunk", type=int, default=0,
                    help="time steps per bench step; 0: 500 for the laser deck, a whole job for the dispersive one")
    ap.add_argument("--path", default="fused", choices=["fused", "onepass"],
                    help="one-grid stepping path: two TMA sweeps per step (default) or the one-pass step")
    ap.add_argument("--e2e-jobs", type=int, default=1, help="whole jobs of the end-to-end leg")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 legs")
    ap.add_argument("--fp64-chunks", type=int, default=2, help="timed bench steps of each FP64 leg")
    ap.add_argument("--fp64-e2e-steps", type=int, default=1000,
                    help="time steps of the FP64 end-to-end job (set-up + steps + read-back)")
    ap.add_argument("--no-c2", action="store_true", help="skip the dispersive-scattering deck beside the headline")
    ap.add_argument("--c2-jobs", type=int, default=3, help="timed 4000-step jobs of the C2 leg")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the accuracy legs")
    ap.add_argument("--acc-c3-steps", type=int, default=2000, help="time steps of the C3 accuracy sample")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--cpu-steps", type=int, default=3, help="time steps in the CPU baseline sample")
    ap.add_argument("--ens-grids", type=int, default=256, help="grids of the batched ensemble leg (0: skip)")
    ap.add_argument("--ens-steps", type=int, default=128, help="timed steps of the batched ensemble")
    ap.add_argument("--ens-tile", default="",
                    help="batch tile of the ensemble as rows,planes,mode (empty: autotuned)")
    ap.add_argument("--ens-loop-steps", type=int, default=64,
                    help="steps per grid of the one-grid-per-launch comparison loops (0: skip them)")
    ap.add_argument("--serve-jobs", type=int, default=24, help="jobs of the serving leg (0: skip)")
    ap.add_argument("--serve-step-scale", type=float, default=1.0,
                    help="job step counts are the log-uniform [500, 20000] draws divided by this")
    ap.add_argument("--serve-fp64-steps", type=int, default=500,
                    help="steps of each job timed on the FP64 plain path (scaled to the job's length; 0: skip)")
    ap.add_argument("--serve-tile", default="",
                    help="batch tile of the serving loop as rows,planes,mode (empty: the library default)")
    ap.add_argument("--serve-load", type=float, default=4.0,
                    help="offered load: arrival rate x job work / 20 Gcell-upd/s (4: about twice what the "
                         "server completes, so the GPU stays saturated while jobs arrive)")
    a = ap.parse_args()
    if a.n == 0:
        a.n = 384 if a.workload == "laser" else 256
    if a.job_steps == 0:
        a.job_steps = 20000 if a.workload == "laser" else 4000
    if a.chunk == 0:
        a.chunk = 500 if a.workload == "laser" else a.job_steps
    a.chunk = min(a.chunk, a.job_steps)
    return a


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


# ------------------------------------------------------------------ decks

def workload(kind, n, job_steps):
    """The bench decks: the disordered photonic-crystal laser (four-level
    gain, 32-frequency spherical-port DFT) or the dispersive-scattering deck
    (Drude-Lorentz spheres, TF/SF beam, six 64-frequency planar ports)."""
    from cpsfdtd_b200 import decks
    if kind == "laser":
        return decks.config3(n=n, steps=job_steps, seed=0, nfreq=32)
    return decks.config2(n=n, steps=job_steps, nfreq=64)


def workload_name(dk, kind, chunk):
    step = (f"1 bench step = {chunk} time steps of a {dk.nsteps}-step job" if chunk < dk.nsteps
            else f"1 bench step = 1 job of {dk.nsteps} time steps")
    if kind == "laser":
        return (f"disordered photonic-crystal laser {dk.nx}^3, eps 11.9 spheres in gain-doped eps 2.25, CPML "
                f"{dk.pml['npml'][0]}, Ez seed pulse, spherical port x 32-freq FP64 DFT; {step}")
    return (f"dispersive scattering {dk.nx}^3, Drude-Lorentz 4x4x4 spheres, CPML {dk.pml['npml'][0]}, TF/SF "
            f"Gaussian beam, 6 ports x 64-freq FP64 DFT; {step}")


def config_of(dk, kind, world, chunk, path="fused"):
    return {"workload": workload_name(dk, kind, chunk), "grid": [dk.nx, dk.ny, dk.nz],
            "time_steps_per_job": dk.nsteps, "time_steps_per_bench_step": chunk,
            "precision": "fp32 fields, fp32 gain state (population offsets), fp64 port accumulators"
            if kind == "laser" else "fp32 fields, fp64 port accumulators", "path": path,
            "l2": f"inputs larger than L2 (fields {6 * 4 * (dk.nx + 1) * (dk.ny + 1) * (dk.nz + 1) / 1e9:.2f} GB "
                  "per grid)", "parallelism": f"replicas x{world}"}


class Prepared:
    """A deck with its host inputs (IDs, port points) and aux cell counts."""

    def __init__(self, kind, n, job_steps):
        import cpsfdtd_b200 as cps
        from cpsfdtd_b200 import decks
        self.kind = kind
        self.dk = workload(kind, n, job_steps)
        dk = self.dk
        self.ids = dk.ids if dk.ids is not None else cps.rasterize(dk.nx, dk.ny, dk.nz, dk.dx, dk.dy, dk.dz,
                                                                   dk.shapes)
        self.pts = [cps.port_points(dk, p) for p in dk.ports]
        inner = self.ids[1:-1, 1:-1, 1:-1]
        self.ndl = int((inner == decks.ID_DISPERSIVE).sum()) if dk.dl else 0
        self.ngain = int((inner == decks.ID_GAIN).sum()) if dk.gain else 0

    def grid(self, prec, device, ids=None):
        import cpsfdtd_b200 as cps
        return cps.Grid.from_deck(self.dk, prec, ids=self.ids if ids is None else ids, port_points_list=self.pts,
                                  device=device)

    @property
    def cells(self):
        return self.dk.nx * self.dk.ny * self.dk.nz


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
    """Algorithmic bytes of one H sweep and one E sweep.  Returns two models as
    ((h, e), (h2, e2)):
      model 1: each field word of the swept side read and written once
               (3 x 2 x s), 1 B material ID, CPML psi (2 words read + write
               per slab cell of that side), Drude-Lorentz state (3 x (nD +
               2 nL + 1) words read + write per ID-2 cell, E side), gain state
               (12 polarisation + 3 population words read + write per gain
               cell, E side) -- a step is 50 B per cell at s = 4 plus aux;
      model 2: model 1 plus the read of the other side's three components,
               which a design with separate H and E sweeps makes every sweep.
    Neighbour and halo re-reads are not counted in either."""
    nx, ny, nz, s = dk.nx, dk.ny, dk.nz, prec_bytes
    np_ = dk.pml["npml"][0] if dk.pml else 0
    h_cells = nx * ny * nz
    e_cells = (nx - 1) * (ny - 1) * (nz - 1)
    h_slab = 2 * np_ * (ny * nz + nx * nz + nx * ny)
    e_slab = 2 * np_ * ((ny - 1) * (nz - 1) + (nx - 1) * (nz - 1) + (nx - 1) * (ny - 1))
    psi = 2 * 2 * s
    h = h_cells * (6 * s + 1) + h_slab * psi
    stride = len(dk.dl["fD"]) + 2 * len(dk.dl["fL"]) + 1 if dk.dl else 0
    e = e_cells * (6 * s + 1) + e_slab * psi + ndl * 3 * stride * 2 * s + ngain * 15 * 2 * s
    return (h, e), (h + h_cells * 3 * s, e + e_cells * 3 * s)


def onepass_bytes(dk, ngain, prec_bytes=4):
    """Algorithmic bytes of one one-pass sweep: the six fields read and written
    once, 1 B ID, CPML psi of both sides, gain state (Drude-Lorentz cells run
    in their own kernel)."""
    (h, e), _ = sweep_bytes(dk, 0, prec_bytes, ngain)
    nx, ny, nz, s = dk.nx, dk.ny, dk.nz, prec_bytes
    return h + e - nx * ny * nz * (6 * s + 1) - (nx - 1) * (ny - 1) * (nz - 1) * (6 * s + 1) + nx * ny * nz * (12 * s + 1)


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


# ------------------------------------------------------------ CPU legs

def cpu_run(dk, ids, warm, steps, kind):
    """The reference's own code on the deck (oracle/_ref/ref_bench) on all host
    cores, or the oracle restatement when the reference build is absent."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    threads = os.cpu_count() or 1
    extra = "3-D four-level gain" if kind == "laser" else "3-D Drude-Lorentz"
    if os.path.exists(oracle.REF_BENCH):
        r = oracle.ref_bench(dk, warm, steps, threads=threads)
        what = f"reference BasicFDTD/CPML/TF_SF/Ports (OpenMP) + {extra} from the oracle restatement"
        return r, "reference", what
    o = oracle.Oracle.from_deck(dk, ids)
    oracle.Oracle.threads(threads)
    o.step(warm)
    t0 = time.perf_counter()
    o.step(steps)
    r = {"cells": dk.cells, "steps": steps, "seconds": time.perf_counter() - t0, "threads": threads}
    return r, "port", "oracle restatement (OpenMP)"


def cpu_baseline(prep, steps):
    try:
        r, kind, what = cpu_run(prep.dk, prep.ids, 1, steps, prep.kind)
    except Exception as ex:  # the baseline is reported, never required
        return {"value": None, "unit": "Gcell-upd/s", "cores": os.cpu_count(), "kind": "reference",
                "sample": f"failed: {ex}"}
    return {"value": r["cells"] * r["steps"] / r["seconds"] / 1e9, "unit": "Gcell-upd/s", "cores": r["threads"],
            "kind": kind, "sample": f"{prep.dk.nx}^3 {prep.kind} deck, {steps} time steps after 1 warm-up, {what}"}


def run_reference(args):
    world, rank, local, dist = dist_setup()
    if rank != 0:
        return
    dk = workload(args.workload, args.n, args.job_steps)
    ids = dk.ids
    if ids is None:
        import cpsfdtd_b200 as cps
        ids = cps.rasterize(dk.nx, dk.ny, dk.nz, dk.dx, dk.dy, dk.dz, dk.shapes)
    r, kind, what = cpu_run(dk, ids, args.warmup, args.steps, args.workload)
    v = r["cells"] * r["steps"] / r["seconds"] / 1e9
    sample = (f"{dk.nx}^3 {args.workload} deck: each bench step is 1 time step of the job (bounded sample), "
              f"{args.steps} timed after {args.warmup} warm-up, {what}")
    line = {"metric": "Gcell-upd/s", "value": v, "unit": "Gcell-upd/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["seconds"] / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded deck generator)",
            "config": config_of(dk, args.workload, args.gpus, args.chunk, args.path),
            "cpu_baseline": {"value": v, "unit": "Gcell-upd/s", "cores": r["threads"], "kind": kind, "sample": sample},
            "e2e": {"value": v, "unit": "Gcell-upd/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------ GPU legs

class Stepper:
    """Bench steps of `chunk` time steps over consecutive jobs of one grid: a
    job that has run all its steps has its spectra flushed and restarts from
    the initial state."""

    def __init__(self, g, dk, chunk, path):
        self.g, self.dk, self.chunk, self.path = g, dk, chunk, path
        self.left = dk.nsteps

    def step(self):
        if self.left == 0:
            self.g.flush_ports()
            self.g.reset(self.dk.n0)
            self.left = self.dk.nsteps
        n = min(self.chunk, self.left)
        self.g.step(n, self.path)
        self.left -= n
        return n


def timed_chunks(g, st, warm, steps, dist=None, clocks=None):
    """warm untimed bench steps, then `steps` timed with CUDA events on the
    grid's stream (barrier + synchronize on both sides); returns (ms, time
    steps, launches, clocks)."""
    import torch
    stream = torch.cuda.ExternalStream(g.stream(), device=torch.cuda.current_device())
    for _ in range(warm):
        st.step()
    g.sync()
    l0 = g.launches()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    if clocks:
        clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    nts = 0
    for _ in range(steps):
        nts += st.step()
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop() if clocks else None
    return e0.elapsed_time(e1), nts, g.launches() - l0, clk


def sweep_roofline(prep, g, path, value_per_gpu):
    """Mean event-timed H and E sweep durations over 200 more time steps of
    the job the timed region left off (fields and gain state as the timed
    steps had them: the sweeps run slower on a developed field than on the
    near-zero one of a job's first steps), run as the direct launch sequence
    (the timed steps replay the same kernels in CUDA-graph chunks, where
    single launches are not timed)."""
    import cpsfdtd_b200 as cps
    dk = prep.dk
    g.set_timing(1)
    g.step(200, path)
    g.sync()
    h_ms, e_ms, nsamp = g.timing()
    g.set_timing(0)
    P, src = peaks()
    (hb, eb), (hb2, eb2) = sweep_bytes(dk, prep.ndl, ngain=prep.ngain)
    if path == cps.ONEPASS:  # h_ms: the one-pass sweep (with its TF/SF terms); e_ms: the Drude-Lorentz cells
        dom_ms, dom_b, dom_b2, dom = h_ms, onepass_bytes(dk, prep.ngain), onepass_bytes(dk, prep.ngain), "one-pass sweep"
    elif e_ms >= h_ms:
        dom_ms, dom_b, dom_b2, dom = e_ms, eb, eb2, "E sweep"
    else:
        dom_ms, dom_b, dom_b2, dom = h_ms, hb, hb2, "H sweep"
    ach = dom_b / (dom_ms / 1e3) / 1e9 if dom_ms > 0 else 0.0
    ach2 = dom_b2 / (dom_ms / 1e3) / 1e9 if dom_ms > 0 else 0.0
    step_b = (hb + eb) / prep.cells
    roof = {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": P["hbm_gbs"], "unit": "GB/s",
            "frac": ach / P["hbm_gbs"], "peak_source": src, "traffic": None,
            "algorithmic_bytes_per_launch": dom_b,
            "byte_model": "swept side's fields read+written once + 1 B ID + psi + aux state (other side not counted)",
            "two_sweep_bytes_per_launch": dom_b2, "achieved_two_sweep": ach2, "frac_two_sweep": ach2 / P["hbm_gbs"],
            "launch_ms": dom_ms, "samples": nsamp,
            "launch_timing": "CUDA events around each sweep on the grid's stream, the 200 time steps that follow "
                             "the timed region in the same job",
            "h_sweep_ms": h_ms, "e_sweep_ms": e_ms,
            "h_sweep_frac": hb / (h_ms / 1e3) / 1e9 / P["hbm_gbs"] if h_ms else 0,
            "step_bytes_per_cell": step_b,
            "step_frac": value_per_gpu * step_b / P["hbm_gbs"]}
    tr = os.path.join(ROOT, "profiles", "traffic.json")
    key = f"{prep.kind}_{dk.nx}_{'onepass' if path == cps.ONEPASS else 'fused'}"
    if os.path.exists(tr):
        try:
            t = json.load(open(tr)).get(key)
            if t:
                roof["traffic"] = t["e_sweep_bytes_per_launch"] if dom == "E sweep" else t.get("h_sweep_bytes_per_launch")
                roof["traffic_source"] = t["source"]
        except (ValueError, OSError, KeyError):
            pass
    return roof


def e2e_jobs(prep, prec, path, jobs, local, dist, steps=None):
    """Whole jobs through the C ABI from host buffers: grid set-up from the
    deck with the IDs and port points in pinned host memory, `steps` time
    steps (the job's own count by default), the port spectra read back into
    pinned host buffers allocated once, teardown."""
    import torch
    dk = prep.dk
    steps = steps or dk.nsteps
    pinned_ids = torch.from_numpy(np.ascontiguousarray(prep.ids)).pin_memory()
    pinned_out = [torch.empty(len(pp) * bin(p.dft_mask).count("1") * len(p.dft_freqs) * 2, dtype=torch.float64)
                  .pin_memory().numpy() if p.dft_freqs is not None else None for p, pp in zip(dk.ports, prep.pts)]
    outs = []
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(jobs):
        gg = prep.grid(prec, local, ids=pinned_ids.numpy())
        gg.step(steps, path)
        outs = [gg.port_dft(n, raw=True, out=pinned_out[n]) for n in range(len(dk.ports))
                if pinned_out[n] is not None]
        gg.close()
    torch.cuda.synchronize()
    t = time.perf_counter() - t0
    if dist:
        tt = torch.tensor([t], device=f"cuda:{local}")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t = float(tt.item())
    world = dist.get_world_size() if dist else 1
    h2d = prep.ids.nbytes + sum(p.nbytes for p in prep.pts) + sum(len(w) * 8 for *_, w in dk.sources)
    d2h = sum(o.nbytes for o in outs)
    return {"value": prep.cells * steps * jobs * world / t / 1e9, "unit": "Gcell-upd/s",
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "job_time_steps": steps, "seconds": t}


def fp64_legs(prep, args, local, dist):
    """The deck in FP64: the plain path (one kernel per reference routine, the
    form the oracle pins) and the fused path, each over args.fp64_chunks
    bench steps after one warm-up; e2e on the plain path over a job of
    args.fp64_e2e_steps time steps."""
    import cpsfdtd_b200 as cps
    out = {}
    for name, path in (("plain", cps.PLAIN), ("fused", cps.FUSED)):
        g = prep.grid(cps.FP64, local)
        st = Stepper(g, prep.dk, args.chunk, path)
        ms, nts, launches, _ = timed_chunks(g, st, 1, args.fp64_chunks, dist)
        v, ms = aggregate(prep.cells * nts, ms, dist, f"cuda:{local}")
        out[name] = {"value": v / 1e9, "unit": "Gcell-upd/s", "ms_per_step": ms / args.fp64_chunks,
                     "steps": args.fp64_chunks, "time_steps_per_step": args.chunk, "gpu_launches": int(launches)}
        g.close()
    out["e2e_plain"] = e2e_jobs(prep, cps.FP64, cps.PLAIN, 1, local, dist,
                                steps=min(args.fp64_e2e_steps, prep.dk.nsteps))
    out["dtype"] = "f64"
    return out


def fp64_with_peak(dk, steps, local, checkpoints=20):
    """The deck alone in FP64 on the fused path, stepped in chunks; returns the
    grid and, per field component, the largest L2 norm seen at the
    checkpoints (the scale against which a decayed final field's error is
    read)."""
    import cpsfdtd_b200 as cps
    g = cps.Grid.from_deck(dk, cps.FP64, device=local)
    peak = np.zeros(6)
    chunk = max(1, -(-steps // checkpoints))
    done = 0
    while done < steps:
        n = min(chunk, steps - done)
        g.step(n, cps.FUSED)
        done += n
        peak = np.maximum(peak, [float(np.linalg.norm(g.field(c))) for c in range(6)])
    g.sync()
    return g, peak


def err_vs_peak(a_fields, b_fields, peak):
    """max over components of |a - b|_2 / (the component's peak norm)"""
    return max(float(np.linalg.norm(np.asarray(x, np.float64) - np.asarray(y, np.float64))) / p
               for x, y, p in zip(a_fields, b_fields, peak) if p > 0)


def grid_report(a, b, dk):
    """accuracy of grid a against grid b: fields and every DFT port"""
    from cpsfdtd_b200 import accuracy
    ports = [accuracy.port_errors(p.dft_freqs, a.port_dft(n, raw=True), b.port_dft(n, raw=True))
             for n, p in enumerate(dk.ports) if p.dft_freqs is not None]
    return accuracy.summarize(accuracy.field_errors([a.field(c) for c in range(6)], [b.field(c) for c in range(6)]),
                              ports)


def accuracy_legs(args, local, c3_prep, c2_prep):
    """Per config, the chosen FP32 forms against FP64 runs of the same decks:
    C1 (96^3, 1000 steps), C2 (256^3, 4000 steps) and C3 (384^3, the first
    args.acc_c3_steps steps) fused FP32 against FP64; C4, one 128^3 member
    batched with two others for its 5000 steps against it alone in FP64.  The
    FP64 side is the fused FP64 path, checked here against the plain FP64
    path (which equals the oracle bit for bit on C1)."""
    import cpsfdtd_b200 as cps
    from cpsfdtd_b200 import decks
    rep = {"reference": "FP64 fused path on the GPU (agreement with the FP64 plain path reported as "
                        "fp64_fused_vs_plain; the plain path equals the oracle bit for bit on C1 at 96^3 x 1000)"}
    c1 = decks.config1(n=96, steps=1000)
    cases = [("c1", c1, cps.rasterize(c1.nx, c1.ny, c1.nz, c1.dx, c1.dy, c1.dz, c1.shapes),
              [cps.port_points(c1, p) for p in c1.ports], c1.nsteps)]
    if c2_prep is not None:
        cases.append(("c2", c2_prep.dk, c2_prep.ids, c2_prep.pts, c2_prep.dk.nsteps))
    if c3_prep is not None:
        cases.append(("c3", c3_prep.dk, c3_prep.ids, c3_prep.pts, min(args.acc_c3_steps, c3_prep.dk.nsteps)))
    for name, dk, ids, pts, steps in cases:

        def run(prec, path):
            g = cps.Grid.from_deck(dk, prec, ids=ids, port_points_list=pts, device=local)
            g.step(steps, path)
            g.sync()
            return g

        f64 = run(cps.FP64, cps.FUSED)
        p64 = run(cps.FP64, cps.PLAIN)
        r64 = grid_report(f64, p64, dk)
        p64.close()
        f32 = run(cps.FP32, cps.FUSED)
        r = grid_report(f32, f64, dk)
        r["time_steps"] = steps
        r["grid"] = [dk.nx, dk.ny, dk.nz]
        r["form"] = "fp32 fused, one grid"
        r["fp64_fused_vs_plain_field_rel_l2"] = r64["field_rel_l2"]
        if dk.gain:
            r["population_max_abs_err"] = float(np.abs(f32.populations() - f64.populations()).max())
        f32.close()
        f64.close()
        rep[name] = r
    # C4: a member inside a batch
    dks = [decks.config4_member(128, 128, 128, seed=7, steps=5000, nfreq=32),
           decks.config4_member(64, 96, 80, seed=8, steps=5000, nfreq=32),
           decks.config4_member(112, 64, 128, seed=9, steps=5000, nfreq=32)]
    b = cps.Batch(cps.FP32)
    gs = [cps.Grid.from_deck(d, cps.FP32, device=local) for d in dks]
    for g in gs:
        b.add(g)
    b.step(5000)
    b.sync()
    ref, peak = fp64_with_peak(dks[0], 5000, local)
    r = grid_report(gs[0], ref, dks[0])
    r["field_err_vs_peak"] = err_vs_peak([gs[0].field(c) for c in range(6)], [ref.field(c) for c in range(6)], peak)
    r.update({"time_steps": 5000, "grid": [128, 128, 128], "form": "fp32 batched (3 members) vs fp64 alone"})
    rep["c4"] = r
    b.close()
    for g in gs + [ref]:
        g.close()
    return rep


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
    if args.ens_tile:
        b.set_tile(*(int(v) for v in args.ens_tile.split(",")))
        tuned_steps = 0
    else:
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

    def loop(path, steps, grids=grids):
        # one grid after another on the device: each grid's stream waits for
        # the previous grid's last launch; events on the current stream bracket
        # the chain
        cur = torch.cuda.current_stream(local)
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        s0.record(cur)
        prev = s0
        for g in grids:
            gs = torch.cuda.ExternalStream(g.stream(), device=local)
            gs.wait_event(prev)
            g.step(steps, path)
            prev = torch.cuda.Event()
            prev.record(gs)
        cur.wait_event(prev)
        s1.record(cur)
        s1.synchronize()
        return cells * steps / (s0.elapsed_time(s1) / 1e3) / 1e9

    plain = fused = None
    if args.ens_loop_steps > 0:
        loop(cps.FUSED, 2)  # warm-up of the one-grid kernels
        plain = loop(cps.PLAIN, args.ens_loop_steps)
        fused = loop(cps.FUSED, args.ens_loop_steps)
    for g in grids:
        g.close()
    # the plain form proper: FP64, one grid per launch (the parity form)
    plain64 = None
    if not args.no_fp64 and args.ens_loop_steps > 0:
        g64 = [cps.Grid.from_deck(decks.config4_member(nx, ny, nz, seed=i, steps=5000, nfreq=32), cps.FP64,
                                  device=local) for i, (nx, ny, nz) in enumerate(shapes)]
        loop(cps.PLAIN, 2, g64)
        plain64 = loop(cps.PLAIN, args.ens_loop_steps, g64)
        for g in g64:
            g.close()
    return {"workload": f"{args.ens_grids} disordered-crystal realizations, edges U{{64,80,96,112,128}} per axis, "
                        "CPML 8, four-level gain, Ez seed pulse, 32-freq FP64 spherical-port DFT; FP32 fields",
            "grids": args.ens_grids, "cells": int(cells), "metric": "Gcell-upd/s", "value": batched,
            "steps_timed": args.ens_steps, "ms": ms, "tile": tile,
            "plain_one_grid_per_launch": plain, "fused_one_grid_per_launch": fused,
            "plain_fp64_one_grid_per_launch": plain64,
            "speedup_vs_plain_loop": batched / plain if plain else None,
            "speedup_vs_fused_loop": batched / fused if fused else None,
            "speedup_vs_plain_fp64_loop": batched / plain64 if plain64 else None,
            "arms": "batched: FP32 fields (the chosen form, within 1e-4 of FP64); plain and fused loops: the same "
                    "FP32 grids one grid per launch; plain FP64 loop: the parity form (FP64, one kernel per "
                    "reference routine, one grid per launch) on the same decks",
            "gpu_launches": int(launches), "setup_s": setup_s, "autotune_s": tune_s,
            "autotune_steps": tuned_steps, "loop_steps_per_grid": args.ens_loop_steps,
            "timing": "all arms: CUDA events around the whole loop on the device (the loops' grids stepped one "
                      "after another, each grid's stream waiting for the previous grid's last launch)"}


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


def trim_device_pool(local):
    """Hand the memory that the library's grids returned to the device's
    default pool (it keeps freed blocks for the next grid) back to the driver,
    so that the free-memory figure counts it."""
    import torch
    torch.cuda.synchronize(local)
    try:
        from cuda.bindings import runtime as rt
        err, pool = rt.cudaDeviceGetDefaultMemPool(local)
        if err == rt.cudaError_t.cudaSuccess:
            rt.cudaMemPoolTrimTo(pool, 0)
    except ImportError:
        pass


def serving(args, local):
    """Served job stream through the library's serving loop (Poisson arrivals
    offered at --serve-load times a 20 Gcell-upd/s service rate, admission
    against a 180 GB budget, continuous batching), against the same jobs run
    one at a time on the plain per-routine GPU path, queued in arrival order.
    Accuracy: the smallest job of each material kind, served in FP32, against
    the same deck run alone in FP64."""
    import torch
    import cpsfdtd_b200 as cps
    from cpsfdtd_b200 import accuracy
    jobs = serve_jobs(args.serve_jobs, args.serve_step_scale)
    work = [e ** 3 * st for _, e, st, _ in jobs]
    rng = np.random.Generator(np.random.PCG64(1))
    mean_gap = sum(work) / (args.serve_load * 20e9) / len(jobs)
    arrivals = np.cumsum(rng.exponential(mean_gap, size=len(jobs)))
    arrivals -= arrivals[0]
    budget = 180 * 10 ** 9
    trim_device_pool(local)
    free, total = torch.cuda.mem_get_info(local)
    budget = min(budget, int(free * 0.9))
    tile = tuple(int(v) for v in args.serve_tile.split(",")) if args.serve_tile else None
    srv = cps.Server(cps.FP32, max_jobs=256, budget_bytes=budget, chunk_steps=64, tile=tile)
    # the smallest job of each material kind is checked against an FP64 run alone
    checked = {}
    for n, (kind, edge, steps, seed) in enumerate(jobs):
        if kind not in checked or edge ** 3 * steps < jobs[checked[kind]][1] ** 3 * jobs[checked[kind]][2]:
            checked[kind] = n
    check_ids = set(checked.values())
    kept = {}
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
                    dfts = [g.port_dft(p, raw=True) for p in range(len(g.ports)) if g.ports[p][2] > 0]
                    if n in check_ids:
                        kept[n] = ([g.field(c) for c in range(6)], dfts)
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
    def queued(service):
        finish, out = 0.0, []
        for a, sv in zip(arrivals, service):
            finish = max(finish, a) + sv
            out.append(finish - a)
        return finish, sorted(out)

    finish, plain_lat = queued(service)

    # the plain form proper (FP64, one grid per launch): set-up and spectrum
    # read-out measured per job, stepping timed over the job's first
    # --serve-fp64-steps steps and scaled to its step count
    plain64 = None
    if not args.no_fp64 and args.serve_fp64_steps > 0:
        service64 = []
        for kind, edge, steps, seed in jobs:
            dk = serve_deck(kind, edge, steps, seed)
            torch.cuda.synchronize()
            ts = time.perf_counter()
            g = cps.Grid.from_deck(dk, cps.FP64, device=local)
            g.sync()
            t1 = time.perf_counter()
            n = min(steps, args.serve_fp64_steps)
            g.step(n, cps.PLAIN)
            g.sync()
            t2 = time.perf_counter()
            for p in range(len(g.ports)):
                if g.ports[p][2] > 0:
                    g.port_dft(p, raw=True)
            g.sync()
            t3 = time.perf_counter()
            g.close()
            service64.append((t1 - ts) + (t2 - t1) * steps / n + (t3 - t2))
        finish64, lat64 = queued(service64)
        plain64 = {"jobs_per_s": len(jobs) / max(finish64, 1e-9),
                   "gcell_upd_per_s": float(sum(work)) / sum(service64) / 1e9,
                   "latency_p50_s": float(np.percentile(lat64, 50)),
                   "latency_p99_s": float(np.percentile(lat64, 99)),
                   "timing": f"host clock; set-up and read-out measured, stepping timed over each job's first "
                             f"{args.serve_fp64_steps} steps and scaled to its step count"}

    # accuracy of the served results against FP64 runs alone
    acc = {}
    for kind, n in sorted(checked.items()):
        if n not in kept:
            continue
        _, edge, steps, seed = jobs[n]
        dk = serve_deck(kind, edge, steps, seed)
        g, peak = fp64_with_peak(dk, steps, local)
        fields, dfts = kept[n]
        ports = []
        k = 0
        for p_i, p in enumerate(dk.ports):
            if p.dft_freqs is not None:
                ports.append(accuracy.port_errors(p.dft_freqs, dfts[k], g.port_dft(p_i, raw=True)))
                k += 1
        ref = [g.field(c) for c in range(6)]
        r = accuracy.summarize(accuracy.field_errors(fields, ref), ports)
        r["field_err_vs_peak"] = err_vs_peak(fields, ref, peak)
        r["final_field_over_peak"] = max(float(np.linalg.norm(x)) for x in ref) / float(peak.max())
        r.update({"job": n, "grid": [edge] * 3, "time_steps": steps, "form": "fp32 served vs fp64 alone"})
        acc[kind] = r
        g.close()

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
            "plain_fp64_one_at_a_time": plain64,
            "speedup_gcell_vs_plain_fp64": (cells_total / span) / (plain64["gcell_upd_per_s"] * 1e9)
            if plain64 else None,
            "accuracy": acc,
            "timing": "host clock: job latency = completion - arrival, including deck generation and grid "
                      "set-up; plain latencies from measured service times queued in arrival order"}


def headline(prep, args, local, dist, clocks_on=True):
    """FP32 value, roofline and e2e of one deck."""
    import cpsfdtd_b200 as cps
    import torch
    path = cps.ONEPASS if args.path == "onepass" else cps.FUSED
    g = prep.grid(cps.FP32, local)
    st = Stepper(g, prep.dk, args.chunk, path)
    clocks = Clocks(local) if clocks_on else None
    ms, nts, launches, clk = timed_chunks(g, st, args.warmup, args.steps, dist, clocks)
    value, ms = aggregate(prep.cells * nts, ms, dist, f"cuda:{local}")
    value /= 1e9
    world = dist.get_world_size() if dist else 1
    roof = sweep_roofline(prep, g, path, value / world)
    g.close()
    torch.cuda.synchronize()
    e2e = e2e_jobs(prep, cps.FP32, path, args.e2e_jobs, local, dist) if args.e2e_jobs > 0 else None
    return {"value": value, "ms_per_step": ms / args.steps, "time_steps_timed": nts, "gpu_launches": int(launches),
            "roofline": roof, "clocks": clk, "e2e": e2e}


def c2_leg(prep, args, local, dist):
    """The dispersive-scattering deck beside the headline: whole 4000-step
    jobs (one warm-up, args.c2_jobs timed), roofline, e2e, FP64 legs."""
    a = argparse.Namespace(**vars(args))
    a.chunk, a.warmup, a.steps = prep.dk.nsteps, 1, args.c2_jobs
    h = headline(prep, a, local, dist, clocks_on=False)
    out = {"workload": workload_name(prep.dk, "dispersive", a.chunk), "grid": [prep.dk.nx] * 3,
           "metric": "Gcell-upd/s", "value": h["value"], "ms_per_step": h["ms_per_step"], "steps": a.steps,
           "roofline": h["roofline"], "e2e": h["e2e"], "gpu_launches": h["gpu_launches"], "dtype": "fp32"}
    if not args.no_fp64:
        a.fp64_chunks = 1
        a.fp64_e2e_steps = prep.dk.nsteps
        out["fp64"] = fp64_legs(prep, a, local, dist)
    return out


def run_ours(args):
    import torch
    world, rank, local, dist = dist_setup()
    import cpsfdtd_b200 as cps  # noqa: F401
    torch.cuda.set_device(local)
    prep = Prepared(args.workload, args.n, args.job_steps)
    h = headline(prep, args, local, dist)
    fp64 = None if args.no_fp64 else fp64_legs(prep, args, local, dist)
    c2 = None
    c2_prep = None
    if args.workload == "laser" and not args.no_c2:
        c2_prep = Prepared("dispersive", 256, 4000)
        c2 = c2_leg(c2_prep, args, local, dist)
    acc = None
    if not args.no_accuracy and world == 1:
        try:
            acc = accuracy_legs(args, local, prep if args.workload == "laser" else None,
                                c2_prep if args.workload == "laser" else prep)
        except Exception as ex:
            acc = {"error": str(ex)}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(prep, args.cpu_steps)
    ens = None
    if args.ens_grids > 0:
        try:
            ens = ensemble(args, local, dist)
        except Exception as ex:
            ens = {"error": str(ex)}
    srv = None
    if args.serve_jobs > 0 and world == 1:
        try:
            srv = serving(args, local)
        except Exception as ex:
            srv = {"error": str(ex)}
    if rank == 0:
        line = {"metric": "Gcell-upd/s", "value": h["value"], "unit": "Gcell-upd/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": h["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
                "data": "synthetic (seeded deck generator)",
                "config": config_of(prep.dk, args.workload, world, args.chunk, args.path),
                "roofline": h["roofline"], "clocks": h["clocks"], "gpu_launches": h["gpu_launches"],
                "e2e": h["e2e"], "fp64": fp64, "c2": c2, "accuracy": acc, "cpu_baseline": cpu,
                "ensemble": ens, "serving": srv}
        print(json.dumps(line), flush=True)
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
