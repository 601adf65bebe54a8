#!/usr/bin/env python
"""Benchmark of the hosono-2DMHD time-step path on B200.

Metric: FP64 zone-updates/s -- interior cells x full RK3 time steps (every
MOOD pass and the CFL reduction included) per second.  A step is one
cfl_computedt + timeStep_advanceSolution on the resident state.

Default workload: Orszag-Tang vortex 2048x2048, GP radius 2 (cascade 2->1->0),
ell/Delta = 12, HLLC, SSP-RK3, CFL 0.8, FLICD on, periodic, FP64, synthetic
initial state generated on the host.  The state (270 MB of U alone) is
larger than the 126 MB L2, so no L2 flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: the path is not partitioned (no domain decomposition exists in
the reference); N ranks run N independent replicas of the workload
("replicas only", weak scaling), value = all ranks' zone-updates / max time.

--impl reference times the reference algorithm on the host cores: the CPU
oracle restatement (the Fortran reference cannot be compiled here), with all
host threads, same metric and workload; rank 0 only.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "tests"))

MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0

WORKLOADS = {
    "ot2048_r2": dict(n=2048, radius=2, ell=12.0, desc="Orszag-Tang 2048x2048, GP-MOOD R=2 (5th->3rd->1st), ell/dx=12"),
    "ot1536_r2": dict(n=1536, radius=2, ell=12.0, desc="Orszag-Tang 1536x1536, GP-MOOD R=2 (5th->3rd->1st), ell/dx=12"),
    "ot1024_r2": dict(n=1024, radius=2, ell=12.0, desc="Orszag-Tang 1024x1024, GP-MOOD R=2 (5th->3rd->1st), ell/dx=12"),
    "ot128_r1": dict(n=128, radius=1, ell=6.0, desc="Orszag-Tang 128x128, GP-MOOD R=1 (3rd->1st), ell/dx=6"),
    "sedov2048_r2": dict(n=2048, radius=2, ell=6.0, problem="sedov",
                         desc="Sedov blast 2048x2048, hydro, outflow, GP-MOOD R=2, CFL 0.6, ell/dx=6"),
}


def load_pkg():
    import pkg
    return pkg.load()


def par_for(workload, d):
    import parfiles
    w = WORKLOADS[workload]
    if w.get("problem") == "sedov":
        kv = parfiles.sedov(w["n"], w["radius"], ell=w["ell"], tmax=0.05, cfl=0.6)
    else:
        kv = parfiles.orszag_tang(w["n"], w["radius"], ell=w["ell"], tmax=0.5, cfl=0.8)
    return parfiles.make(d, workload, kv)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() in ("active", "1", "yes"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks():
    try:
        with open(MEASURED_PEAKS) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


# The ncu capture of one k_face_pass1<2> launch (DRAM bytes, FP64-pipe
# activity) lives in the committed profile summary; its "bench-keys:" line
# holds the numbers this bench scales to its workload by algorithmic bytes.
PASS1_PROFILE_FILE = os.path.join(ROOT, "profiles", "k_face_pass1_ot1536_r2.md")


def pass1_profile():
    """{workload, n, radius, dram_bytes, fp64_pipe_active_frac} from the
    profile summary's bench-keys line, or None when it has none."""
    try:
        with open(PASS1_PROFILE_FILE) as f:
            line = next((ln for ln in f if ln.startswith("bench-keys:")), None)
    except OSError:
        return None
    if not line:
        return None
    kv = dict(tok.split("=", 1) for tok in line.split(":", 1)[1].split())
    return {"workload": kv["workload"], "n": int(kv["n"]), "radius": int(kv["radius"]),
            "dram_bytes": float(kv["dram_bytes"]), "fp64_pipe_active_frac": float(kv["fp64_pipe_active_frac"]),
            "source": os.path.relpath(PASS1_PROFILE_FILE, ROOT)}


# Algorithmic FP64 operations of one pass-1 launch per interior cell: the
# operation-counting build of the oracle (oracle/flopcount.h, `make -C oracle
# count`) counts every double add, multiply, divide and square root of the
# MOOD pass-1 reconstruction and fluxes (GP face states, face CAD/PAD, the
# Riemann solves and their Gauss sums) over the three stages of one step;
# per launch is a third of that.  Counted on each workload's own grid (the
# halo work of a small grid included): Orszag-Tang R=2, ell/dx=12 at 2048^2
# on steps 1 and 13 (15858.3 and 15858.2 flops per zone-update); Sedov R=2
# (hydro) at 2048^2, steps 1-3 (14269.5); Orszag-Tang R=1 at 128^2, steps 1-3
# (7855.4 to 7855.8).
PASS1_FLOPS = {("ot", 2, 12.0): 15858.2 / 3, ("sedov", 2, 6.0): 14269.5 / 3, ("ot", 1, 6.0): 7855.8 / 3}
FP64_LANES_PER_SM = 64  # FP64 FMA lanes per B200 SM (two flops per lane per clock)


def pass1_bytes(n, radius):
    """Algorithmic HBM bytes of one MOOD pass-1 kernel launch (n x n interior):
    read U once over the interior plus NGC guard rings (8 doubles/cell), write
    fluxRaw x/y (16 doubles) and the two corrected-B copies (2 doubles) on the
    (n+3)^2 flux faces, and the per-face admissibility bytes (2 per cell)."""
    ngc = radius + 2
    cells_u = (n + 2 * ngc) ** 2
    faces = (n + 3) ** 2
    return cells_u * 8 * 8 + faces * 18 * 8 + (n + 5) ** 2 * 2


def host_has_avx2_fma():
    try:
        with open("/proc/cpuinfo") as f:
            flags = next((ln for ln in f if ln.startswith("flags")), "").split()
        return "avx2" in flags and "fma" in flags
    except OSError:
        return False


def oracle_build():
    return "-O3 AVX2/FMA contraction" if host_has_avx2_fma() else "-O3 SSE2, no contraction"


def run_cpu_baseline(workload, steps, threads, fast=None, to_end=False):
    """Time the oracle restatement on the host cores: returns (zone-updates/s,
    seconds, steps).  to_end: the whole run from the initial state to t_end.
    fast=None picks the AVX2/FMA build when the host supports it."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    if fast is None:
        fast = host_has_avx2_fma()
    oracle.set_threads(threads, fast=fast)
    w = WORKLOADS[workload]
    with tempfile.TemporaryDirectory() as d:
        par = par_for(workload, d)
        o = oracle.Oracle(par, fast=fast)
        if to_end:
            t0 = time.perf_counter()
            rc, _, steps = o.run()
            el = time.perf_counter() - t0
        else:
            dt = o.cfl()
            o.advance(dt)  # warm-up step (page faults, thread pool)
            t0 = time.perf_counter()
            for _ in range(steps):
                dt = o.cfl()
                o.advance(dt)
            el = time.perf_counter() - t0
        o.close()
    rate = w["n"] * w["n"] * steps / el
    return rate, el, steps


def max_over_ranks(ms, dist, device):
    """The slowest rank's time (replicas: the job ends when the last one does)."""
    if dist is None:
        return ms
    import torch
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replicas_value(world, zones, steps, ms):
    """Whole-job zone-updates/s of `world` replicas, each `steps` steps of
    `zones` cells, over the slowest rank's time."""
    return world * zones * steps / (ms / 1e3)


def bench_reference(args, rank):
    """--impl reference: the reference algorithm on the host cores (rank 0 only)."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    w = WORKLOADS[args.workload]
    # bounded sample: at most ~120 s of CPU time whatever --steps says
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    rate1, el1, _ = run_cpu_baseline(args.workload, 1, threads)
    steps = max(1, min(args.steps, int(120.0 / max(el1, 1e-3))))
    rate, el, _ = run_cpu_baseline(args.workload, steps, threads) if steps > 1 else (rate1, el1, 1)
    line = {
        "metric": "fp64_zone_updates_per_s", "value": rate, "unit": "zone-updates/s", "n_gpus": args.gpus,
        "steps": steps, "warmup": 1, "ms_per_step": el / steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "desc": w["desc"], "fp": "fma (release-like)"},
        "impl": "reference",
        "cpu_baseline": {"value": rate, "unit": "zone-updates/s", "cores": threads, "kind": "port",
                         "sample": f"{steps} full RK3 steps of {args.workload} after 1 warm-up step, "
                                   f"CPU oracle (C++ restatement of the Fortran, OpenMP, {oracle_build()})"},
        "e2e": {"value": rate, "unit": "zone-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def bench_ours(args, rank, world, local):
    import numpy as np
    import torch

    m = load_pkg()
    torch.cuda.set_device(local)
    m.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    w = WORKLOADS[args.workload]
    fp = m.FP_FAST if args.fp == "fast" else m.FP_STRICT
    with tempfile.TemporaryDirectory() as d:
        par = par_for(args.workload, d)
        params, run = m.par_load(par)
        params.fp_mode = fp
        pv, qw, st = m.par_gp(par, params.max_radius)
        U0, V0 = m.ic_set(par, params)
    sol = m.Solver(params, pv, qw, st)
    if args.eager:
        sol.set_graphs(False)
    sol.upload(U0, V0)
    sol.set_time(0.0, run.tmax, 0, run.nstepmax)
    tune = None
    if args.tuning:  # a fixed launch choice (staging,schedule,blocks per SM[,boxes]), e.g. for a profiler
        f = [int(x) for x in args.tuning.split(",")]
        sol.set_tuning(pass1_staging=f[0], pass1_schedule=f[1], pass1_blocks_per_sm=f[2],
                       pass1_boxes=f[3] if len(f) > 3 else 0)
        tune = {"fixed": sol.tuning()}
    elif not args.no_tune:
        tune = sol.autotune(trials=5, force=True)
    stream = torch.cuda.ExternalStream(sol.stream())
    zones = w["n"] * w["n"]

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # warm-up (graph capture happens here; the clock sampler starts here so it
    # has samples under load even when the timed region is short)
    clocks = ClockSampler(local)
    clocks.start()
    sol.step(max(args.warmup, 1))
    barrier()
    # timed region: K steps, each one launch of the step graph (cfl, dt,
    # three MOOD stages, RK3) with CUDA events bracketing the pass-1 kernels
    if not args.eager and not args.to_end:  # the pass-1 events live in the profiled step graph
        sol.profile(True)
    sol.profile_read(reset=True)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    if args.to_end:  # the whole run from the initial state to t_end
        sol.upload(U0, V0)
        sol.set_time(0.0, run.tmax, 0, run.nstepmax)
        e0.record(stream)
        t_sim, n_steps = sol.step(0)
        args.steps = n_steps
    else:
        t_sim, n_steps = sol.step(args.steps)
    e1.record(stream)
    e1.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    p1_ms, p1_n, launches = sol.profile_read(reset=True)
    passes = sol.stats()["mood_passes"]
    sol.profile(False)
    barrier()
    ms = max_over_ranks(ms, dist, "cuda")
    value = replicas_value(world, zones, args.steps, ms)

    # end to end through the reference-facing calls with host buffers, as a
    # Fortran driver that keeps grid_state%U on the host makes them each step:
    # dt = cfl_computedt (hosono_gpu_cfl, dt to the host), then
    # timeStep_advanceSolution on the host array (hosono_gpu_advance_host:
    # U from pinned memory to the device, in row bands that overlap the first
    # stage's pass 1; the step, which rebuilds V; U back to the host)
    Uh = torch.from_numpy(np.ascontiguousarray(U0)).pin_memory().numpy()
    sol.upload(Uh, None)
    e2e_steps = max(1, min(args.steps, 5))
    barrier()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(e2e_steps):
        dt = sol.cfl_computedt()
        sol.advance_host(dt, Uh, None)
    f1.record(stream)
    f1.synchronize()
    e2e_ms = f0.elapsed_time(f1)
    e2e_ms = max_over_ranks(e2e_ms, dist, "cuda")
    barrier()
    e2e = {"value": world * zones * e2e_steps / (e2e_ms / 1e3), "unit": "zone-updates/s",
           "h2d_bytes_per_step": U0.nbytes, "d2h_bytes_per_step": U0.nbytes + 8,
           "steps": e2e_steps, "ms_per_step": e2e_ms / e2e_steps,
           "calls": "per step: hosono_gpu_cfl (dt to the host), hosono_gpu_advance_host(dt, U, NULL): U host->device, "
                    "step, U device->host (V rebuilt on the device)"}
    sol.close()

    # the same workload in fast arithmetic (FMA contraction; results within
    # 1e-12 relative L1 of strict after one step), for comparison only
    other = None
    if fp == m.FP_STRICT and not args.to_end and world == 1:
        params.fp_mode = m.FP_FAST
        solf = m.Solver(params, pv, qw, st)
        solf.upload(U0, V0)
        solf.set_time(0.0, run.tmax, 0, run.nstepmax)
        solf.step(max(args.warmup, 1))
        sf = torch.cuda.ExternalStream(solf.stream())
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(sf)
        solf.step(args.steps)
        g1.record(sf)
        g1.synchronize()
        fms = g0.elapsed_time(g1)
        other = {"fp": "fast", "value": zones * args.steps / (fms / 1e3), "ms_per_step": fms / args.steps,
                 "unit": "zone-updates/s", "note": "FMA contraction allowed; not bit-identical to the oracle"}
        solf.close()
        params.fp_mode = fp

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    hbm, hbm_kind = peaks()
    p1_avg = p1_ms / max(p1_n, 1)
    bytes1 = pass1_bytes(w["n"], w["radius"])
    achieved = bytes1 / (p1_avg / 1e3) / 1e9 if p1_avg > 0 else None
    prof = pass1_profile()
    traffic = None
    if prof and w["radius"] == prof["radius"]:
        traffic = prof["dram_bytes"] * bytes1 / pass1_bytes(prof["n"], prof["radius"])
    roofline = {"bound": "hbm", "kernel": "k_face_pass1", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm if achieved else None, "traffic": traffic, "peak_kind": hbm_kind,
                "kernel_ms": p1_avg, "kernel_launches": p1_n,
                "traffic_source": (f"ncu dram bytes of one launch on {prof['workload']} ({prof['source']}), scaled "
                                   "by algorithmic bytes") if prof else None,
                "fp64_pipe_active_frac": prof["fp64_pipe_active_frac"] if prof else None,
                "note": "FP64 CUDA-core kernel bound by the FP64 pipe and latency (fp64_pipe_active_frac from "
                        "ncu); the HBM line is shown as the contract requires"}
    fpc = PASS1_FLOPS.get((w.get("problem", "ot"), w["radius"], w["ell"]))
    if fpc is not None and p1_avg > 0:
        sms = torch.cuda.get_device_properties(local).multi_processor_count
        mhz = (clk or {}).get("sm_max_mhz") or 1965.0
        peak = sms * FP64_LANES_PER_SM * 2 * mhz * 1e6 / 1e12
        tf = fpc * w["n"] * w["n"] / (p1_avg / 1e3) / 1e12
        roofline["fp64"] = {"achieved": tf, "peak": peak, "unit": "TFLOP/s", "frac": tf / peak,
                            "frac_of_unfused_rate": tf / (peak / 2), "flops_per_cell": fpc,
                            "peak_kind": f"nominal: {sms} SMs x {FP64_LANES_PER_SM} FP64 lanes x 2 (FMA) x "
                                         f"{mhz:.0f} MHz",
                            "note": "strict arithmetic cannot contract to FMA, so one flop per lane per clock "
                                    "(frac_of_unfused_rate) is its ceiling; flops counted by the oracle's "
                                    "operation-counting build"}
    line = {
        "metric": "fp64_zone_updates_per_s", "value": value, "unit": "zone-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "desc": w["desc"], "fp": args.fp, "parallelism": f"replicas{world}",
                   "l2": "inputs larger than L2 (U alone 270 MB at 2048^2)", "mood_passes": passes},
        "gpu_launches": launches, "clocks": clk, "roofline": roofline, "e2e": e2e,
    }
    if tune:
        line["tuning"] = tune
    if other:
        line["fast_fp"] = other
    if world == 1 and not args.no_config0 and args.workload != "ot128_r1":
        line["config0"] = bench_config0(m, fp, torch)
    if world == 1 and not args.no_batched:
        line["batched"] = bench_batched(m, fp, torch, limit=args.batched_limit, eager=args.eager,
                                        tune=not args.no_tune)
    served_kept = {}
    if world == 1 and args.serve_requests > 0:
        import importlib
        srv_mod = importlib.import_module("hosono_2dmhd_b200.serve")
        pols = {"fifo": ("fifo", srv_mod.SERVE_FIFO, {}),
                "shortest": ("shortest", srv_mod.SERVE_SHORTEST, SHORTEST_DEFAULTS)}
        chosen = list(pols.values()) if args.serve_policy == "both" else [pols[args.serve_policy]]
        line["served"], served_kept = bench_served(m, fp, args.serve_requests, args.serve_check,
                                                   args.serve_calibrate, args.serve_sample, args.serve_hashes,
                                                   args.serve_mean_work, args.serve_records, policies=chosen)
    if not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        rate, el, nst = run_cpu_baseline(args.workload, 1, threads, to_end=args.to_end)
        what = f"the whole run to t_end ({nst} steps)" if args.to_end else "1 full RK3 step after 1 warm-up step"
        line["cpu_baseline"] = {"value": rate, "unit": "zone-updates/s", "cores": threads, "kind": "port",
                                "sample": f"{what} of {args.workload}, CPU oracle "
                                          f"(C++ restatement, OpenMP, {oracle_build()}), {el:.1f} s"}
        if served_kept:
            line["served"]["accuracy"] = cpu_baseline_served_check(served_kept)
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def bench_config0(m, fp, torch):
    """The reference's own runnable case: Orszag-Tang 128^2, GP radius 1,
    ell/dx = 6, to t_end = 0.5 as one graph launch (plain single solve, dt on
    the device), after an untimed run that captures the graphs."""
    with tempfile.TemporaryDirectory() as d:
        par = par_for("ot128_r1", d)
        s = m.Solver.from_par(par, fp_mode=fp)
        U0, V0, _ = s.download()
        tune = s.autotune(trials=5, force=True)
        s.run()
        s.upload(U0, V0)
        s.set_time(0.0, s.run_info.tmax, 0, s.run_info.nstepmax)
        stream = torch.cuda.ExternalStream(s.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        t, n = s.step(0)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        passes = s.stats()["mood_passes"]
        s.close()
    return {"workload": "Orszag-Tang 128x128, GP-MOOD R=1 (3rd->1st), ell/dx=6, to t_end=0.5", "steps": n,
            "t_end": t, "value": 128 * 128 * n / (ms / 1e3), "unit": "zone-updates/s", "ms_per_step": ms / n,
            "mood_passes_per_step": passes / n, "tuning": tune["best"]}


def sweep_tuning(args):
    """--sweep-tuning: every pass-1 launch choice on the workload, whole time
    steps (CUDA events around --steps steps after --warmup) and the pass-1
    launches alone, in strict and fast arithmetic; one JSON line per choice."""
    import torch
    m = load_pkg()
    w = WORKLOADS[args.workload]
    choices = ([(st, sc, 2, bx) for bx in (1, 2) for st in (0, 1) for sc in (0, 1)] +
               [(0, 0, 3, 1), (0, 1, 3, 1), (0, 0, 4, 1), (0, 1, 4, 1)])
    for fp in (m.FP_STRICT, m.FP_FAST):
        for st, sc, bl, bx in choices:
            with tempfile.TemporaryDirectory() as d:
                par = par_for(args.workload, d)
                params, run = m.par_load(par)
                params.fp_mode = fp
                pv, qw, stc = m.par_gp(par, params.max_radius)
                U0, V0 = m.ic_set(par, params)
            sol = m.Solver(params, pv, qw, stc)
            sol.upload(U0, V0)
            sol.set_time(0.0, run.tmax, 0, run.nstepmax)
            sol.set_tuning(pass1_staging=st, pass1_schedule=sc, pass1_blocks_per_sm=bl, pass1_boxes=bx)
            sol.step(max(args.warmup, 1))
            stream = torch.cuda.ExternalStream(sol.stream())
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            sol.step(args.steps)
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / args.steps
            sol.profile(True)
            sol.profile_read(reset=True)
            sol.step(3)
            p1, n1, _ = sol.profile_read(reset=True)
            sol.close()
            print(json.dumps({"workload": args.workload, "fp": "fast" if fp else "strict", "pass1_staging": st,
                              "pass1_schedule": sc, "pass1_blocks_per_sm": bl, "pass1_boxes": bx, "ms_per_step": ms,
                              "pass1_ms": p1 / max(n1, 1), "zone_updates_per_s": w["n"] ** 2 / (ms / 1e3)}),
                  flush=True)


def sweep_later_passes(args):
    """--sweep-launch: the step's launch forms -- the later MOOD passes as a
    kernel chain (with and without programmatic dependent launches) and as
    one persistent launch per stage -- on the reference's runnable case to
    t_end, Sedov 1024^2 (10 steps), Orszag-Tang 2048^2 (5 steps) and the
    blast64 batch; one JSON line each."""
    import torch
    m = load_pkg()
    problems = load_problems()

    def timed(stream, fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), r
    forms = [("kernels", dict(later_passes=0, pdl=0)), ("kernels+pdl", dict(later_passes=0, pdl=1)),
             ("persistent", dict(later_passes=1, pdl=0))]
    for name, tune in forms:
        with tempfile.TemporaryDirectory() as d:
            s = m.Solver.from_par(par_for("ot128_r1", d))
            s.set_tuning(**tune)
            U0, V0, _ = s.download()
            s.run()
            s.upload(U0, V0)
            s.set_time(0.0, 0.5, 0, 1 << 30)
            ms, (t, n) = timed(torch.cuda.ExternalStream(s.stream()), lambda: s.step(0))
            s.close()
            print(json.dumps({"later_passes": name, "workload": "ot128_r1 to t_end", "steps": n,
                              "ms_per_step": ms / n}), flush=True)
            import parfiles
            s = m.Solver.from_par(parfiles.make(d, "sedov1024", parfiles.sedov(1024, 2)))
            s.set_tuning(**tune)
            s.set_time(0.0, 1e30, 0, 1 << 30)
            s.step(3)
            ms, _ = timed(torch.cuda.ExternalStream(s.stream()), lambda: s.step(10))
            passes = s.stats()["mood_passes"]
            s.close()
            print(json.dumps({"later_passes": name, "workload": "sedov1024_r2, 10 steps", "ms_per_step": ms / 10,
                              "mood_passes": passes}), flush=True)
            s = m.Solver.from_par(par_for("ot2048_r2", d))
            s.set_tuning(**tune)
            s.set_time(0.0, 1e30, 0, 1 << 30)
            s.step(3)
            ms, _ = timed(torch.cuda.ExternalStream(s.stream()), lambda: s.step(5))
            s.close()
            print(json.dumps({"later_passes": name, "workload": "ot2048_r2, 5 steps", "ms_per_step": ms / 5}),
                  flush=True)
            with open(os.path.join(ROOT, "hosono-2dmhd_b200", "workloads", "blast64_seed0.json")) as f:
                entries = json.load(f)["instances"]
            pars = [problems.make(d, f"i{e['id']}", problems.from_entry(e)) for e in entries]
            b = m.Batch(len(pars), sum(m.Batch.tiles_for(m.par_load(p)[0]) for p in pars))
            b.set_tuning(**tune)
            slots = [b.add_par(p) for p in pars]
            b.run(max_steps=1)
            ms, _ = timed(torch.cuda.ExternalStream(b.stream()), lambda: b.run())
            zu = sum(e["n"] ** 2 * (b.status(k)["nstep"] - 1) for k, e in zip(slots, entries))
            b.close()
            print(json.dumps({"later_passes": name, "workload": "blast64 batch to t_end", "s": ms / 1e3,
                              "zone_updates_per_s": zu / (ms / 1e3)}), flush=True)


def load_problems():
    import importlib
    load_pkg()
    return importlib.import_module("hosono_2dmhd_b200.problems")


def bench_batched(m, fp, torch, manifest="blast64_seed0.json", limit=None, eager=False, tune=True):
    """The 64-instance MHD-blast workload (uneven N in {128..512}) advanced to
    t_end=0.02 as one batch (one graph launch for the whole run) and, for
    comparison, as 64 plain single solves one after the other.  Set-up (host
    initial state, GP tables, upload) and the first step of each (graph
    capture) are outside the timed regions; zone-updates count the timed steps."""
    import time as _t
    problems = load_problems()
    path = os.path.join(ROOT, "hosono-2dmhd_b200", "workloads", manifest)
    with open(path) as f:
        entries = json.load(f)["instances"][:limit]
    with tempfile.TemporaryDirectory() as d:
        pars = [problems.make(d, f"i{e['id']}", problems.from_entry(e)) for e in entries]
        tiles = sum(m.Batch.tiles_for(m.par_load(p)[0]) for p in pars)
        b = m.Batch(len(pars), tiles, fp_mode=fp)
        if eager:
            b.set_graphs(False)
        slots = [b.add_par(p) for p in pars]
        tune_b = b.autotune(trials=3, force=True) if tune else {"fixed": b.tuning()}
        b.run(max_steps=1)
        n0 = {k: b.status(k)["nstep"] for k in slots}
        stream = torch.cuda.ExternalStream(b.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        w0 = _t.perf_counter()
        e0.record(stream)
        b.run()
        e1.record(stream)
        e1.synchronize()
        wall_b = _t.perf_counter() - w0
        ms_b = e0.elapsed_time(e1)
        zu_b = 0
        steps = []
        for k, e in zip(slots, entries):
            st = b.status(k)
            assert st["done"] and st["error"] == 0, st
            zu_b += e["n"] * e["n"] * (st["nstep"] - n0[k])
            steps.append(st["nstep"])
        b.close()
        # plain: one solve after another, each through its own single-instance engine
        ms_p = 0.0
        zu_p = 0
        for p, e in zip(pars, entries):
            s = m.Solver.from_par(p, fp_mode=fp)
            if tune:
                s.autotune(trials=3)  # per size class: timed once, then taken from the cache
            s.set_time(0.0, e["tmax"], 0, 1 << 30)
            s.step(1)
            st_ = torch.cuda.ExternalStream(s.stream())
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record(st_)
            _, n = s.step(0)
            a1.record(st_)
            a1.synchronize()
            ms_p += a0.elapsed_time(a1)
            zu_p += e["n"] * e["n"] * (n - 1)
            s.close()
    rate_b = zu_b / (ms_b / 1e3)
    rate_p = zu_p / (ms_p / 1e3)
    return {"workload": f"blast64: {len(entries)} of 64 MHD blasts, N in {{128..512}} (seed 0), R=2, t_end=0.02",
            "instances": len(entries), "zone_updates": zu_b, "steps_min": min(steps), "steps_max": max(steps),
            "batched_value": rate_b, "batched_s": ms_b / 1e3, "batched_wall_s": wall_b,
            "plain_value": rate_p, "plain_s": ms_p / 1e3, "ratio_batched_over_plain": rate_b / rate_p,
            "unit": "zone-updates/s", "tuning": tune_b}


def bench_served(m, fp, requests, check, calibrate=0, sample=0, hashes_path=None, mean_work=None,
                 records_path=None, policies=None):
    """The served request stream (workloads/served2000_seed1.json, first
    `requests` requests) under both scheduling policies.  Capacity: the
    stream's first `calibrate` requests (all of them when 0) run closed loop
    (all submitted at once, FIFO); their zone-updates/s divided by the
    stream's mean work per request -- measured when every request ran, else
    predicted from the calibration run's step counts (steps ~ k_problem * N *
    t_end, k fitted per problem) -- gives requests/s.  Then the whole stream
    runs open loop, once per policy (FIFO; shortest estimated work first with
    an aging bound), with the manifest's seeded exponential gaps scaled to
    80% of that capacity.  Latency is submit -> final state on the host.  The
    `check` requests with the least predicted work keep their final U, which
    must be the same bits under both policies; they are returned for the
    accuracy check against the CPU oracle.  With `sample`, the SHA-256 of the
    final U of `sample` seeded-random requests is written to `hashes_path`."""
    import hashlib
    import importlib
    import numpy as np
    load_pkg()
    srv = importlib.import_module("hosono_2dmhd_b200.serve")
    if policies is None:
        policies = [("fifo", srv.SERVE_FIFO, {}), ("shortest", srv.SERVE_SHORTEST, SHORTEST_DEFAULTS)]
    path = os.path.join(ROOT, "hosono-2dmhd_b200", "workloads", "served2000_seed1.json")
    with open(path) as f:
        entries = json.load(f)["requests"][:requests]
    cal = entries[:calibrate] if 0 < calibrate < len(entries) else entries
    with srv.Server(fp_mode=fp) as s:
        closed, _, cinfos = srv.run_stream(cal, 1.0, s, fp_mode=fp, closed=True)
    by_id = {e["id"]: e for e in cal}
    ks = {}
    for i in cinfos:
        e = by_id[i["entry"]]
        ks.setdefault(e["problem"], []).append(i["nstep"] / (e["n"] * e["tmax"]))
    k = {p_: float(np.median(v)) for p_, v in ks.items()}
    kall = float(np.median([x for v in ks.values() for x in v]))

    def predicted(e):  # zone-updates of one request
        return e["n"] ** 3 * e["tmax"] * k.get(e["problem"], kall)
    if mean_work:  # known from an earlier run of the same requests (results are deterministic)
        mean_work = float(mean_work)
    elif cal is entries:
        mean_work = closed["zone_updates"] / len(entries)
    else:
        mean_work = float(np.mean([predicted(e) for e in entries]))
    cap = closed["zone_updates_per_s"] / mean_work
    rate = 0.8 * cap
    keep = [e["id"] for e in sorted(entries, key=predicted)[:check]]
    sampled = []
    if sample > 0:
        rng = np.random.Generator(np.random.PCG64(2))
        sampled = sorted(int(x) for x in rng.choice([e["id"] for e in entries], size=min(sample, len(entries)),
                                                    replace=False))
    out = {"workload": f"served2000 (seed 1) requests 0..{len(entries) - 1}: Orszag-Tang / Sedov / MHD blast, "
                       f"N log-uniform in [64,1024], R in {{1,2}}, t_end U[0.1,1] x default",
           "requests": len(entries), "load": 0.8, "calibration_requests": len(cal), "capacity_rps": cap,
           "closed_loop_zone_updates_per_s": closed["zone_updates_per_s"], "rate_per_s": rate,
           "unit": "zone-updates/s", "mean_work_used": mean_work}
    keys = ("zone_updates", "zone_updates_per_s", "makespan_s", "latency_p50_s", "latency_p99_s", "latency_max_s",
            "queue_wait_p50_s", "queue_wait_p99_s", "submit_lag_max_s", "peak_resident", "peak_bytes",
            "budget_bytes", "gpu_busy_frac", "completed", "failed", "failed_status")
    kept_by = {}
    for name, pol, kw in policies:
        with srv.Server(fp_mode=fp, policy=pol, **kw) as s:
            rep, kept, infos = srv.run_stream(entries, rate, s, keep=keep + sampled, fp_mode=fp)
        out[name] = {k_: rep[k_] for k_ in keys}
        out[name]["server"] = dict(policy=name, **kw)
        out[name]["mean_work_measured"] = rep["zone_updates"] / max(rep["completed"], 1)
        # the load the stream actually offered: its arrival rate times the
        # measured work per request, over the closed-loop throughput
        out[name]["offered_load"] = rate * out[name]["mean_work_measured"] / closed["zone_updates_per_s"]
        kept_by[name] = kept
        if name == policies[0][0]:
            for k_ in keys:  # the first policy's figures at the top level
                out[k_] = rep[k_]
            first_infos = infos
    out["policies_identical"] = all(np.array_equal(kept_by[policies[0][0]][i], kept_by[n][i])
                                    for n, _, _ in policies for i in keep + sampled)
    if records_path:
        with open(records_path, "w") as f:
            json.dump([{k_: i[k_] for k_ in ("entry", "status", "nstep", "zone_updates", "submit_s", "admit_s",
                                              "finish_s")} for i in first_infos], f)
    if sampled and hashes_path:
        recs = {}
        for i in first_infos:
            if i["entry"] in sampled:
                U = kept_by[policies[0][0]][i["entry"]]
                recs[str(i["entry"])] = {"sha256": hashlib.sha256(np.ascontiguousarray(U).tobytes()).hexdigest(),
                                         "nstep": i["nstep"], "t": i["t"], "zone_updates": i["zone_updates"]}
        with open(hashes_path, "w") as f:
            json.dump({"manifest": "served2000_seed1.json", "sample_seed": 2, "fp": "strict" if fp == 0 else "fast",
                       "requests": recs}, f, indent=1)
        out["sampled_hashes"] = {"file": os.path.basename(hashes_path), "requests": sampled}
    return out, {e["id"]: (e, kept_by[policies[0][0]][e["id"]]) for e in entries if e["id"] in keep}


# the shortest-first server's settings the bench runs
SHORTEST_DEFAULTS = {}


def cpu_baseline_served_check(kept):
    """Accuracy of served results against the CPU oracle run of the same
    request to its t_end: relative L1 of each conserved variable over the
    interior (the worst one reported) and whether the states are identical."""
    import numpy as np
    import oracle
    problems = load_problems()
    worst, same, checked = 0.0, True, []
    with tempfile.TemporaryDirectory() as d:
        for eid, (e, U) in sorted(kept.items()):
            par = problems.make(d, f"chk{eid}", problems.from_entry(e))
            o = oracle.Oracle(par)
            rc, t, n = o.run()
            Uo = o.U()
            g = o.ngc
            a, b = U[g:-g, g:-g, :], Uo[g:-g, g:-g, :]
            rel = float(max(np.abs(a[..., v] - b[..., v]).sum() / max(np.abs(b[..., v]).sum(), 1e-300)
                            for v in range(8)))
            worst = max(worst, rel)
            same = same and bool(np.array_equal(U, Uo))
            checked.append(eid)
            o.close()
    return {"checked_requests": checked, "max_rel_l1": worst, "identical": same, "tolerance": 1e-8,
            "reference": "CPU oracle (C++ restatement, strict FP) run to the same t_end"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="ot2048_r2", choices=sorted(WORKLOADS))
    ap.add_argument("--fp", default="strict", choices=["strict", "fast"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="keep the default launch choices (no autotuning)")
    ap.add_argument("--sweep-launch", "--sweep-later-passes", dest="sweep_later_passes", action="store_true",
                    help="time the step's launch forms (kernel chain, with programmatic dependent launches, one "
                         "persistent later-pass launch) and exit")
    ap.add_argument("--sweep-tuning", action="store_true",
                    help="time every pass-1 launch choice on the workload (whole steps and pass 1) and exit")
    ap.add_argument("--tuning", default=None,
                    help="fixed pass-1 launch choice 'staging,schedule,blocks_per_sm[,boxes]' instead of autotuning")
    ap.add_argument("--no-batched", action="store_true", help="skip the 64-instance batched-vs-plain measurement")
    ap.add_argument("--no-config0", action="store_true", help="skip the Orszag-Tang 128^2 R=1 to t_end leg")
    ap.add_argument("--eager", action="store_true",
                    help="launch kernels one by one instead of as CUDA graphs (the plain and batched legs; for "
                         "profilers, which do not see inside conditional graph nodes)")
    ap.add_argument("--batched-limit", type=int, default=64, help="instances of the batched workload to run")
    ap.add_argument("--to-end", action="store_true",
                    help="time the whole run from the initial state to t_end instead of --steps steps")
    ap.add_argument("--serve-requests", type=int, default=50,
                    help="requests of the served stream to run (0: skip the served measurement)")
    ap.add_argument("--serve-check", type=int, default=20,
                    help="served requests (least predicted work first) checked against the CPU oracle")
    ap.add_argument("--serve-calibrate", type=int, default=0,
                    help="first requests run closed loop to measure capacity (0: all of them, which measures the "
                         "stream's mean work exactly; fewer predict it, and a poor prediction skews the load)")
    ap.add_argument("--serve-sample", type=int, default=0,
                    help="seeded-random served requests whose final-state SHA-256 is written to --serve-hashes")
    ap.add_argument("--serve-hashes", default=None, help="output JSON of the sampled hashes")
    ap.add_argument("--serve-mean-work", type=float, default=None,
                    help="mean zone-updates per request of the stream when known from an earlier run (the "
                         "results, and so the work, are deterministic); else predicted from the calibration")
    ap.add_argument("--serve-records", default=None, help="output JSON of per-request work and timestamps")
    ap.add_argument("--serve-policy", choices=("both", "fifo", "shortest"), default="both",
                    help="scheduling policies the served stream runs under")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.sweep_tuning:
        sweep_tuning(args)
    elif args.sweep_later_passes:
        sweep_later_passes(args)
    elif args.impl == "reference":
        bench_reference(args, rank)
    else:
        bench_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
