"""Benchmark: FP64 cell-updates/s of the cubed-sphere MHD update on one B200,
batched (served ensemble) vs plain per-solve launches, with the ensemble's
p50/p99 time-to-solution.

One cell-update = one valid cell advanced one full RK4 step (4 operator
evaluations with their stage preparation and RK update), dt = cfl / max CFL
rate computed on the device before every step.

Workloads (synthetic input; the reference ships no data for them), gamma
5/3, r in [21.5, 215] Rsun, radial stretch 1.5, CFL 0.4, Powell on:

  --workload serve (default): the served CME ensemble.  256 requests arrive
      as a seeded Poisson stream whose rate puts about 8 solves in flight;
      each has a grid of {32,48,64,96} radial x {32,48,64}^2 cells per panel,
      the scheme PLM-MC + Rusanov or Berta WENOZ + Roe (50/50) and a
      cone-CME cloud (speed U[500, 2000] km/s, half-width U[20, 60] deg,
      lat/lon U[-30, 30] deg, density ratio U[2, 6]) inserted on the device
      at admission; --steps RK4 steps per request.  The same requests run
      through the continuous-batching server (value) and one after another
      through plain per-solve launches (plain).  e2e: the served run with
      every request's initial state copied from pinned host memory at
      admission.  The same line carries the large single solve
      (large_solve: 256 x 192^2 x 6, WENOZ + Roe + solar gravity, cone of
      1500 km/s and 45 deg), whose operator gives the roofline.
  --workload uniform: one solve advanced --steps RK4 steps (--order 4:
      64 x 64^2 x 6 WENOZ + Roe on the perturbed wind; --order 2: 32 x 32^2
      x 6 PLM-MC + Rusanov on the pressure pulse; --nr/--na/--gravity/--init
      cone for other sizes).
  --workload amr: the AMR-style box batch (boxes of 8^3-32^3 on three
      levels), batched vs per-box launches.
  --workload slabs: one shell (default 256 x 192^2 x 6, WENOZ + Roe + solar
      gravity) split into radial slabs over the N ranks (strong scaling):
      halo layers swapped with the radial neighbours before every RK4 stage,
      dt from an all-reduce of the CFL rate.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--workload ...]

N > 1 (torchrun): every rank runs an independent replica of the workload
(weak scaling; the path has no exchange between replicas), timed on the
device and reduced as the max over ranks; --workload slabs shares one shell
among the ranks instead.  --impl reference times the CPU
restatement of the reference's algorithm (the reference itself cannot be
built: its Proto dependency is absent) on the host cores, on a bounded
sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FP64 cell-updates/s on 1 B200, batched vs plain; ensemble p50/p99 latency"
METRIC_UNIFORM = "FP64 cell-updates/s on 1 B200 (RK4 step of the cubed-sphere MHD update)"
UNIT = "cell-updates/s"
L2_BYTES = 126 * 1024 * 1024
OPERATOR_BYTES_PER_CELL_STAGE = 128  # read 8 FP64 primitives, write 8 FP64 rhs


def operator_launches(args) -> int:
    """Kernels of one fourth-order operator evaluation (hc_level_rhs)."""
    roe, powell = int(args.riemann == 2), 1
    # detector + point values (3); per direction reconstruction, Roe point
    # dissipation, fused face chain and the Powell face chain (3); the radial
    # face averages of the TMA-staged radial chain (1); Powell coefficients,
    # averages and application (3)
    return 3 + 3 * (2 + roe + 3 * powell) + 1 + 3 * powell


def launches_per_step(args) -> int:
    """Kernels of this library launched by one hc_level_advance_cfl step."""
    if args.order == 2:
        return 11  # prim + cfl + 4 x (ghosts, stage) + time (prologue in every 1-step call)
    operator = operator_launches(args)
    per_stage = 4 + int(args.gravity) + operator + 1               # prepare, gravity, operator, update
    return 1 + 4 * per_stage + 2 + 1                               # cfl, stages, reflux, time


def workload_params(args, nr=None, na=None):
    from heliocubed_b200.level import Params
    return Params(nr=nr or args.nr, na=na or args.na, spatial_order=args.order, limiter=args.limiter,
                  riemann_solver=args.riemann, divergence_cleaning=1, sun_gravity=args.gravity, cfl=0.4,
                  berta_fallback_type=0)


def scheme_name(args) -> str:
    solver = "Roe 8-wave" if args.riemann == 2 else "Rusanov"
    if args.order == 4:
        return f"Berta pointwise WENOZ (WENO3 fallback) + {solver}"
    return f"PLM-{'MC' if args.limiter == 3 else args.limiter} + {solver}"


def workload_config(args, flush: bool):
    return {
        "workload": f"cubed-sphere MHD RK4 step, {scheme_name(args)}, {args.nr}x{args.na}^2x6",
        "cells": 6 * args.nr * args.na * args.na,
        "scheme": {"spatial_order": args.order, "limiter": args.limiter if args.order == 2 else None,
                   "riemann_solver": args.riemann, "powell": 1, "gravity": args.gravity, "temporal_order": 4,
                   "cfl": 0.4},
        "init": ("Parker-like wind + finite cone-CME cloud (field model 4) 1500 km/s, 45 deg, 4x density, "
                 "seeded axis, inserted on the device at the inner boundary"
                 if args.init == "cone" else
                 "Parker-like wind + seeded 5% tangential v and B (stream-function curl)" if args.order == 4
                 else "Parker-like wind + seeded Gaussian pressure pulse"),
        "l2": "flushed between timed steps (256 MiB write)" if flush else "working set larger than L2",
        "dt": "device CFL reduction every step",
        "launch": "CUDA graph replay per step" if args.graph else "eager launches",
    }


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic_per_cell_stage(order: int):
    """DRAM bytes per cell-stage of the operator from the committed ncu
    summary of that operator, or None before one exists."""
    path = os.path.join(ROOT, "profiles", "o2_stage_kernel.md" if order == 2 else "o4_operator.md")
    if not os.path.exists(path):
        return None
    m = re.search(r"traffic_bytes_per_cell_stage:\s*([0-9.eE+-]+)", open(path).read())
    return float(m.group(1)) if m else None


def profiled_fp64_flops_per_cell_stage(order: int):
    """FP64 flops (dadd + dmul + 2 dfma thread instructions, ncu counters)
    per cell-stage of the operator from the committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", "o2_stage_kernel.md" if order == 2 else "o4_operator.md")
    if not os.path.exists(path):
        return None
    m = re.search(r"fp64_flops_per_cell_stage:\s*([0-9.eE+-]+)", open(path).read())
    return float(m.group(1)) if m else None


def measure_fp64_peak() -> float:
    """FP64 TFLOP/s of a cuBLAS DGEMM (8192^3, best of 3, CUDA events) on
    this GPU: the denominator of the FP64-pipe roofline."""
    import torch
    a = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    b = torch.randn_like(a)
    c = torch.empty_like(a)
    torch.matmul(a, b, out=c)
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b, out=c)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b, c
    torch.cuda.empty_cache()
    return 2.0 * 8192 ** 3 / (best * 1e-3) / 1e12


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows: list[list[str]] = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except ValueError:
                continue
            for n, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        dist.init_process_group("nccl" if torch.cuda.is_available() else "gloo",
                                timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def dist_max(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def native_oracle() -> str:
    """Build the oracle for this machine's CPU (-march=native) and load it;
    returns how the timed library was built."""
    from oracle import build as ob
    from oracle import pyoracle as po
    path = ob.build_oracle_native(os.path.join(ROOT, "oracle", "_native"))
    if path is None:
        return "g++ -O3 -march=x86-64-v3 (shipped; the native build failed)"
    po.use_library(path)
    return "g++ -O3 -march=native -ffp-contract=off -fopenmp, built on this machine"


def cpu_baseline(args, budget_s: float = 12.0) -> dict:
    """The oracle (CPU restatement of the reference) on the host cores, on a
    bounded number of RK4 steps of the same scheme: the full grid at order 2,
    a 32 x 32^2 x 6 grid at order 4 (one step of the 64^3 grid takes minutes
    on the host)."""
    build = native_oracle()
    from oracle import pyoracle as po
    cores = os.cpu_count() or 1
    nr, na = (args.nr, args.na) if args.order == 2 else (min(args.nr, 32), min(args.na, 32))
    p = po.make_params(nr=nr, na=na, spatial_order=args.order, limiter=args.limiter, riemann_solver=args.riemann,
                       sun_gravity=args.gravity, berta_fallback_type=0)
    if args.order == 4:
        from heliocubed_b200.level import perturbed_wind_state
        L = po.OracleLevelO4(p)
        det = L.base.geometry(4).reshape(6, na, na)
        dvolr = L.base.geometry(0).reshape(nr + 1, 4)[:nr, 3]
        ju = np.ascontiguousarray(perturbed_wind_state(workload_params(args, nr, na), det, dvolr, args.seed).reshape(-1))
    else:
        L = po.OracleLevel(p)
        from heliocubed_b200.level import InitSpec
        spec = InitSpec.seeded(args.seed, nr, na)
        s = po.HcInit()
        s.kind = 1
        for k in ("pulse_block", "pulse_i", "pulse_j", "pulse_k", "rho0", "p0", "vr", "b0", "r_ref", "pulse_amp",
                  "pulse_width"):
            setattr(s, k, getattr(spec, k))
        ju = L.init(s)
    steps, t = 0, 0.0
    t0 = time.perf_counter()
    while True:
        dt = 0.4 / L.inv_dt(ju)
        L.rk4_step(ju, dt, t)
        t += dt
        steps += 1
        if time.perf_counter() - t0 > budget_s or steps >= args.cpu_max_steps:
            break
    el = time.perf_counter() - t0
    value = 6 * nr * na * na * steps / el
    same = "the same" if (nr, na) == (args.nr, args.na) else f"the same scheme on a"
    return {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "build": build,
            "sample": f"{steps} RK4 steps (CFL dt each step) of {same} {nr}x{na}^2x6 grid, "
                      f"OpenMP over {cores} host threads, {el:.1f} s"}


def run_reference(args, world, rank):
    """The CPU arm: the oracle (the reference's algorithm restated; the
    reference itself needs the absent Proto library) on the host cores, on
    a bounded sample of the same workload, with the workload's metric."""
    if rank != 0:
        return
    if args.workload == "serve":
        reqs = serve_requests(args, None)
        cb = cpu_baseline_serve(args, reqs, budget_s=args.ref_budget)
        metric = METRIC
        config = {"workload": "served CME ensemble (config 4): %d requests, %d RK4 steps each"
                              % (len(reqs), args.steps),
                  "requests": len(reqs), "steps_per_request": args.steps,
                  "sample": "CPU oracle on the ensemble's smallest-grid requests (see cpu_baseline.sample)"}
    else:
        cb = cpu_baseline(args, budget_s=args.ref_budget)
        metric = METRIC_UNIFORM
        cfg = workload_config(args, flush=False)
        config = {k: cfg[k] for k in ("workload", "cells", "scheme", "init")}
        config["dt"] = "host CFL reduction every step"
    out = {"impl": "reference", "metric": metric, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
           "scaling": "strong" if args.workload == "slabs" else "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": config, "cpu_baseline": cb,
           "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def cone_request(args):
    """The large-solve workload's input: the wind with a 1500 km/s, 45 deg,
    4x density cone cloud on a seeded axis (lat/lon U[-30, 30] deg)
    inserted at the inner boundary."""
    from heliocubed_b200 import serve
    rng = np.random.default_rng(args.seed)
    cone = serve.Cone(speed_kms=1500.0, half_width_deg=45.0, lat_deg=rng.uniform(-30, 30),
                      lon_deg=rng.uniform(-30, 30), density_ratio=4.0)
    return serve.Request(0, args.nr, args.na, args.order, 0, cone=cone)


def run_b200(args, world, rank, local):
    out = measure_uniform(args, world, rank, local)
    if rank == 0:
        if not args.no_cpu_baseline and world == 1:
            out["cpu_baseline"] = cpu_baseline(args)
        print(json.dumps(out), flush=True)


def measure_uniform(args, world, rank, local, e2e_min_steps: int = 4) -> dict:
    """One solve of the uniform workload of `args` advanced args.steps RK4
    steps (graph replay, device CFL every step): the result line of the
    uniform workload, with the operator's rooflines and the end-to-end rate
    through the public API with host buffers."""
    import torch
    from heliocubed_b200.level import InitSpec, Shell
    torch.cuda.set_device(local)
    params = workload_params(args)
    shell = Shell(params, device=local)
    cells = shell.cells
    if args.init == "cone":
        from heliocubed_b200 import serve
        ju0 = torch.from_numpy(serve.initial_state(shell, cone_request(args))).to(shell._dev)
    elif args.order == 4:
        ju0 = shell.init_perturbed_wind(args.seed)
    else:
        ju0 = shell.init(InitSpec.seeded(args.seed, args.nr, args.na))
    ju = ju0.clone()
    # autotuner: time the candidates on this level, keep the fastest
    if args.order == 2:
        from heliocubed_b200.level import stage_tiles
        (trk, trhs), tms = shell.autotune(ju0)
        shapes = stage_tiles()
        tuning = {"rk_stage_tile": [int(x) for x in shapes[trk]], "operator_tile": [int(x) for x in shapes[trhs]],
                  "candidates": [[int(x) for x in r] for r in shapes],
                  "rk_stage_ms": [round(float(x), 5) for x in tms[0]],
                  "operator_ms": [round(float(x), 5) for x in tms[1]],
                  "tile_fields": "cells x, y, z, min CTAs/SM Rusanov, Roe"}
    else:
        from heliocubed_b200.level import o4_variants
        mb = o4_variants()
        names = ("reconstruction", "roe_point", "face_chain")
        if args.o4_variants:
            # fixed variants (profiling: timings taken under a profiler would
            # steer the tuner to a different choice than the plain run's)
            var = [int(x) for x in args.o4_variants.split(",")]
            shell.set_o4_variants(*var)
            tuning = {"min_ctas_per_sm": {n: int(mb[q, var[q]]) for q, n in enumerate(names)}, "fixed": True}
        else:
            var, vms = shell.autotune(ju0)
            tuning = {"min_ctas_per_sm": {n: int(mb[q, var[q]]) for q, n in enumerate(names)},
                      "candidates": {n: [int(x) for x in mb[q]] for q, n in enumerate(names)},
                      "operator_ms": {n: [round(float(x), 4) for x in vms[q]] for q, n in enumerate(names)}}
    time_dev = torch.zeros(1, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    state_bytes = ju.numel() * 8
    working = state_bytes * 3 + shell.ng * 8
    flush = working < 2 * L2_BYTES
    scratch = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda") if flush else None

    graph = shell.capture_advance(ju, 1, time_dev) if args.graph else None

    def step():
        if graph is not None:
            graph.replay()
        else:
            shell.advance(ju, 1, time_dev)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if not shell.valid(ju):
        raise RuntimeError("warm-up produced an invalid state")

    sampler = ClockSampler(local)
    sampler.start()
    barrier(world)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for s in range(args.steps):
        if flush:
            scratch.zero_()
        ev[s][0].record(stream)
        step()
        ev[s][1].record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    ms = sum(a.elapsed_time(b) for a, b in ev)
    ms = dist_max(ms, world)
    ok = shell.valid(ju)

    # operator kernel alone (hc_level_rhs: read primitives, write rhs) for the roofline
    w = shell.prepare(ju)
    k = shell.new_state()
    for _ in range(3):
        shell.rhs(w, k)
    reps = 20
    kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    for r in range(reps):
        if flush:
            scratch.zero_()
        kev[r][0].record(stream)
        shell.rhs(w, k)
        kev[r][1].record(stream)
    torch.cuda.synchronize()
    kms = statistics.mean(a.elapsed_time(b) for a, b in kev)
    peak, peak_kind = peaks()
    achieved = OPERATOR_BYTES_PER_CELL_STAGE * cells / (kms * 1e-3) / 1e9
    tr = profiled_traffic_per_cell_stage(args.order)
    fl = profiled_fp64_flops_per_cell_stage(args.order)
    fp64_peak = measure_fp64_peak()

    # End to end through the public API with host buffers: every step copies
    # its input from pinned host memory, advances one RK4 step and copies the
    # result back.  Steps are independent solves of the same input; with room
    # for a second context they alternate between two contexts on two
    # streams, so one step's copies overlap the other's compute.
    host_in = ju0.cpu().pin_memory()
    footprint = 40 * state_bytes  # a context's level buffers and operator scratch, generously
    nlanes = 2 if torch.cuda.mem_get_info()[0] > 2 * footprint else 1
    lanes = []
    for q in range(nlanes):
        sh = shell if q == 0 else Shell(params, device=local)
        lanes.append({"shell": sh, "stream": torch.cuda.Stream(), "dev": torch.empty_like(ju0),
                      "out": torch.empty_like(host_in).pin_memory(),
                      "t": torch.zeros(1, dtype=torch.float64, device="cuda")})

    def e2e_step(n):
        lane = lanes[n % nlanes]
        with torch.cuda.stream(lane["stream"]):
            lane["dev"].copy_(host_in, non_blocking=True)
            lane["shell"].advance(lane["dev"], 1, lane["t"])
            lane["out"].copy_(lane["dev"], non_blocking=True)

    # With one context: two device state buffers and a copy stream; step n
    # computes on one buffer while the other returns step n-1's result and
    # takes step n+1's input.
    bufs = [lanes[0]["dev"], torch.empty_like(ju0)] if nlanes == 1 else None
    copy_stream = torch.cuda.Stream() if nlanes == 1 else None
    loaded = [torch.cuda.Event(), torch.cuda.Event()]
    computed = [torch.cuda.Event(), torch.cuda.Event()]

    def e2e_run(nsteps):
        if nlanes > 1:
            for n in range(nsteps):
                e2e_step(n)
            return
        lane = lanes[0]
        with torch.cuda.stream(copy_stream):
            bufs[0].copy_(host_in, non_blocking=True)
            loaded[0].record(copy_stream)
        for n in range(nsteps):
            cur, nxt = n % 2, (n + 1) % 2
            with torch.cuda.stream(lane["stream"]):
                lane["stream"].wait_event(loaded[cur])
                lane["shell"].advance(bufs[cur], 1, lane["t"])
                computed[cur].record(lane["stream"])
            with torch.cuda.stream(copy_stream):
                if n > 0:
                    copy_stream.wait_event(computed[nxt])
                    lane["out"].copy_(bufs[nxt], non_blocking=True)
                if n + 1 < nsteps:
                    bufs[nxt].copy_(host_in, non_blocking=True)
                    loaded[nxt].record(copy_stream)
        with torch.cuda.stream(copy_stream):
            copy_stream.wait_event(computed[(nsteps - 1) % 2])
            lane["out"].copy_(bufs[(nsteps - 1) % 2], non_blocking=True)

    e2e_steps = max(e2e_min_steps, args.steps // 2)
    e2e_run(2 * nlanes)
    torch.cuda.synchronize()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for lane in lanes:
        lane["stream"].wait_stream(stream)
    if copy_stream is not None:
        copy_stream.wait_stream(stream)
    e2e_run(e2e_steps)
    for lane in lanes:
        stream.wait_stream(lane["stream"])
    if copy_stream is not None:
        stream.wait_stream(copy_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = dist_max(e0.elapsed_time(e1) / e2e_steps, world)
    for lane in lanes[1:]:
        lane["shell"].close()

    value = cells * world * args.steps / (ms * 1e-3)
    out = {
            "metric": METRIC_UNIFORM, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(workload_config(args, flush), parallelism=f"replicas x{world}",
                           **({"autotune": tuning} if tuning else {})),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind,
                         "kernel": ("o2StageKernel (operator: read primitives, write rhs)" if args.order == 2 else
                                    "Berta operator launch group (hc_level_rhs, %d kernels): read USph, write rhs"
                                    % operator_launches(args)),
                         "algorithmic_bytes": f"{OPERATOR_BYTES_PER_CELL_STAGE} B/cell-stage x {cells} cells",
                         "kernel_ms": kms,
                         "traffic": None if tr is None else tr * cells},
            # The operator does no contraction; its binding roofline is the
            # FP64 pipe (flops from ncu instruction counters, peak from a
            # DGEMM measured in this run).
            "fp64_roofline": None if fl is None else {
                "bound": "fp64", "flops_per_cell_stage": fl, "achieved": fl * cells / (kms * 1e-3) / 1e12,
                "peak": fp64_peak, "unit": "TFLOP/s", "frac": fl * cells / (kms * 1e-3) / 1e12 / fp64_peak,
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (best of 3)"},
            "e2e": {"value": cells * world / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": state_bytes,
                    "d2h_bytes_per_step": state_bytes,
                    "pipeline": f"{nlanes} context(s) on {nlanes} stream(s); a step's copies overlap the other "
                                "context's compute" if nlanes > 1 else
                                "one context, two device state buffers and a copy stream: step n computes on one "
                                "while the other returns step n-1's result and takes step n+1's input"},
            "gpu_launches": launches_per_step(args) * args.steps,
            "clocks": clocks,
            "valid_state": ok,
    }
    shell.close()
    del lanes, scratch, bufs
    torch.cuda.empty_cache()
    return out


def dist_sum(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
    dist.all_reduce(t)
    return float(t.item())


def run_slabs(args, world, rank, local):
    """One shell split into radial slabs over the ranks (strong scaling): each
    rank owns nr / N radial cells of all six panels plus halo layers, swaps
    them with its neighbours before every RK4 stage (NCCL point-to-point)
    and takes dt from an all-reduce of the CFL rate; dt stays on the device."""
    import torch
    from heliocubed_b200.shard import ShardedShell
    torch.cuda.set_device(local)
    params = workload_params(args)
    from heliocubed_b200 import serve
    sh = ShardedShell(params, rank, world, device=local)
    lvl, plan = sh.levels[0], sh.plans[0]
    # the large-solve input: the wind with the cone cloud inserted, each rank
    # building its own slab (the insertion is pointwise in the shell's radii)
    st0 = lvl.new_state()
    time_dev = torch.zeros(1, dtype=torch.float64, device="cuda")
    serve.admit(lvl, cone_request(args), st0, time_dev, schedule=False)
    states = [st0.clone()]
    stream = torch.cuda.current_stream()
    state_bytes = st0.numel() * 8
    flush = 3 * state_bytes < 2 * L2_BYTES
    scratch = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda") if flush else None
    for _ in range(args.warmup):
        sh.advance(states, 1, time_dev)
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    barrier(world)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for s in range(args.steps):
        if flush:
            scratch.zero_()
        ev[s][0].record(stream)
        sh.advance(states, 1, time_dev)
        ev[s][1].record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    ms = dist_max(sum(a.elapsed_time(b) for a, b in ev), world)
    sh.exchange(states, 0)
    ok = dist_sum(float(lvl.valid(states[0])), world) == world

    # End to end: each step takes the slab's state from pinned host memory
    # and returns the cells the rank owns.
    host_in = st0.cpu().pin_memory()
    owned = sh.owned([st0])[0]
    host_out = torch.empty(owned.shape, dtype=torch.float64).pin_memory()
    dev = torch.empty_like(st0)
    t_e2e = torch.zeros(1, dtype=torch.float64, device="cuda") + time_dev
    e2e_steps = max(2, args.steps // 2)
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        dev.copy_(host_in, non_blocking=True)
        sh.advance([dev], 1, t_e2e)
        host_out.copy_(sh.owned([dev])[0], non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = dist_max(e0.elapsed_time(e1) / e2e_steps, world)
    h2d = dist_sum(state_bytes, world)
    d2h = dist_sum(owned.numel() * 8, world)

    cells = 6 * args.nr * args.na * args.na
    rows = 48 * args.na * args.na if args.order == 4 else 48 * (args.na + 4) ** 2
    halo_bytes = 4 * (world - 1) * 2 * plan.halo * rows * 8
    out = {
        "metric": METRIC_UNIFORM, "value": cells * args.steps / (ms * 1e-3), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(workload_config(args, flush), parallelism=f"radial slabs x{world}",
                       init="Parker-like wind + finite cone-CME cloud (field model 4) 1500 km/s, 45 deg, 4x "
                            "density, seeded axis, inserted on the device (each rank into its own slab)",
                       launch="eager: per stage the halo swap, then hc_level_rk4_stage",
                       slabs={"owned_radial_cells": [list(x) for x in
                                                     (lambda w: [(r * args.nr // w, (r + 1) * args.nr // w)
                                                                 for r in range(w)])(world)],
                              "halo_layers": plan.halo, "halo_bytes_per_step": halo_bytes,
                              "exchange": "before every RK4 stage, point-to-point with the radial neighbours "
                                          "(NCCL); dt from an all-reduce (max) of the CFL rate"}),
        "e2e": {"value": cells / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                "pipeline": "each rank: its slab's state in from pinned host memory, one RK4 step, the cells it "
                            "owns back, on one stream"},
        "gpu_launches": (launches_per_step(args) - 1) * args.steps,
        "clocks": clocks,
        "valid_state": ok,
    }
    if rank == 0:
        if not args.no_cpu_baseline and world == 1:
            out["cpu_baseline"] = cpu_baseline(args)
        print(json.dumps(out), flush=True)
    sh.close()


SERVE_GRIDS = {"radial": (32, 48, 64, 96), "angular": (32, 48, 64)}


def serve_requests(args, rate_hz):
    from heliocubed_b200 import serve
    return serve.synthetic_requests(args.serve_requests, args.seed, rate_hz, args.steps,
                                    radial=SERVE_GRIDS["radial"], angular=SERVE_GRIDS["angular"])


def serve_launches(reqs, cohort_steps: int | None = None) -> int:
    """Kernels of this library launched for `reqs` (admission, steps,
    schedule): per request the wind, the cone insertion and the schedule,
    then each RK4 step's launches of its order.  With a fourth-order cohort
    (cohort_steps = steps of all its chunks) a fourth-order request's steps
    launch everything but the operator, which runs once per stage of every
    cohort step for all members together."""
    total = 0
    for r in reqs:
        a = argparse.Namespace(order=r.order, riemann=2 if r.order == 4 else 1, gravity=0)
        per_step = launches_per_step(a)
        if cohort_steps is not None and r.order == 4:
            per_step -= 4 * operator_launches(a)
        total += 3 + per_step * r.steps
    if cohort_steps:
        total += 4 * operator_launches(argparse.Namespace(riemann=2)) * cohort_steps
    return total


def run_serve(args, world, rank, local):
    """The served CME ensemble (module docstring): continuous batching vs
    plain per-solve launches on the same seeded Poisson stream, then the
    host-staged (e2e) served run, then the large single solve."""
    import torch
    from heliocubed_b200 import serve
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    probe = serve_requests(args, None)
    shapes = sorted({(r.nr, r.na, r.order) for r in probe})
    counts = {shp: sum(1 for r in probe if (r.nr, r.na, r.order) == shp) for shp in shapes}

    # contexts of the plain path, one per shape; W warm-up steps each, timed
    # with CUDA events to set the arrival rate (Little's law: about
    # `serve_inflight` solves in flight at the plain path's service time)
    shells = {shp: serve.Shell(serve.Request(0, *shp, 0).params(), device=local) for shp in shapes}
    step_ms = {}
    for shp, sh in shells.items():
        req = next(r for r in probe if (r.nr, r.na, r.order) == shp)
        ju = torch.from_numpy(serve.initial_state(sh, req)).to(dev)
        t = torch.zeros(1, dtype=torch.float64, device=dev)
        sh.advance(ju, 1, t)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        sh.advance(ju, args.warmup, t)
        e1.record()
        torch.cuda.synchronize()
        step_ms[shp] = e0.elapsed_time(e1) / args.warmup
    service_s = statistics.mean(step_ms[(r.nr, r.na, r.order)] * 1e-3 * args.steps for r in probe)
    rate = args.serve_inflight / service_s
    reqs = serve_requests(args, rate)

    # the server's slots, pooled by shape (contexts, buffers, graphs of
    # `chunk` steps), built before the timed runs as a long-running server has them
    chunk = max(1, min(10, args.steps))
    server = serve.EnsembleServer(hbm_budget=args.serve_budget_gb * 1e9, max_inflight=args.serve_inflight,
                                  chunk=chunk, device=local, keep_states=False, cobatch=not args.no_cobatch)
    for shp in shapes:
        server.warm([r for r in reqs if (r.nr, r.na, r.order) == shp], per_shape=min(counts[shp], 3))
    torch.cuda.synchronize()

    # host-staged copies of the requests (pinned initial states) for e2e
    staged = []
    for r in reqs:
        sh = shells[(r.nr, r.na, r.order)]
        host = torch.from_numpy(serve.initial_state(sh, r)).pin_memory()
        staged.append(serve.Request(r.rid, r.nr, r.na, r.order, r.steps, r.arrival, r.cone, initial=host))

    sampler = ClockSampler(local)
    sampler.start()
    # each rank serves its own copy of the stream; the ranks start each run
    # together and the whole-job rate is all ranks' work over the slowest
    # rank's makespan
    barrier(world)
    plain = serve.run_plain(reqs, device=local, shells=shells, keep_states=False)
    barrier(world)
    batched = server.run(reqs)
    cohort_steps = server.cohort.chunk_steps if server.cohort is not None else None
    # the host-staged run starts, as the batched one did, without cached
    # ensembles: the same arrivals would otherwise find every membership built
    server.forget_ensembles()
    torch.cuda.synchronize()
    barrier(world)
    hosted = server.run(staged)
    barrier(world)
    clocks = sampler.stop()

    same = serve.same_results(plain, batched)
    same_e2e = serve.same_results(batched, hosted)
    finite = sum(int(bool(r.finite)) for r in batched)
    sp, sb, se = serve.summarize(plain), serve.summarize(batched), serve.summarize(hosted)
    for summary in (sp, sb, se):
        summary["makespan_max_over_ranks_s"] = dist_max(summary["makespan_s"], world)
    state_bytes = sum(8 * 8 * r.cells for r in reqs)
    request_steps = sum(r.steps for r in reqs)
    for sh in shells.values():
        sh.close()
    server.close()
    del staged, plain, batched, hosted
    torch.cuda.synchronize()
    torch.cuda.empty_cache()

    large = None
    if not args.no_large:
        la = argparse.Namespace(**vars(args))
        la.order, la.nr, la.na, la.riemann, la.gravity, la.init = 4, 256, 192, 2, 1, "cone"
        la.steps, la.warmup = args.large_steps, 3
        la.graph, la.o4_variants = True, None
        large = measure_uniform(la, world, rank, local, e2e_min_steps=2)

    if rank != 0:
        return
    job = lambda sm: world * sm["cell_updates"] / sm["makespan_max_over_ranks_s"]  # noqa: E731
    out = {"metric": METRIC, "value": job(sb), "unit": UNIT, "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": sb["makespan_max_over_ranks_s"] * 1e3 / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": "served CME ensemble (config 4): %d requests, %d RK4 steps each"
                                  % (len(reqs), args.steps),
                      "requests": len(reqs), "steps_per_request": args.steps,
                      "steps_note": "the configured 500 steps per request shrunk to --steps (a step of this line "
                                    "is one RK4 step of every request)",
                      "grids": "nr in {32,48,64,96} x na in {32,48,64}, scheme 50/50 PLM-MC+Rusanov / "
                               "Berta WENOZ+Roe, cone speed U[500,2000] km/s, half-width U[20,60] deg, "
                               "lat/lon U[-30,30] deg, density ratio U[2,6]",
                      "arrivals": "seeded Poisson, rate %.3f /s (%d in flight at the plain path's mean service "
                                  "time %.3f s)" % (rate, args.serve_inflight, service_s),
                      "max_inflight": args.serve_inflight, "hbm_budget_gb": args.serve_budget_gb,
                      "chunk_steps": chunk, "slots_per_shape": "min(requests of the shape, 3), built before timing",
                      "fourth_order_cohort": "the fourth-order requests in flight step together (hc_ensemble): "
                                             "each operator kernel one launch per stage over all their panels; "
                                             "second-order requests on their own streams",
                      "l2": "working set of the in-flight solves larger than L2",
                      "parallelism": f"replicas x{world}"},
           "batched": sb, "plain": sp,
           "batched_over_plain": job(sb) / job(sp),
           "p50_s": sb["p50_s"], "p99_s": sb["p99_s"],
           "identical_results": same, "finite_results": finite,
           "e2e": {"value": job(se), "unit": UNIT,
                   "h2d_bytes_per_step": state_bytes / request_steps,
                   "d2h_bytes_per_step": state_bytes / request_steps,
                   "p50_s": se["p50_s"], "p99_s": se["p99_s"], "identical_to_device_built": same_e2e,
                   "pipeline": "served run with every request's initial state copied from pinned host memory at "
                               "admission and its result copied back (bytes per request-step)"},
           "gpu_launches": serve_launches(reqs, cohort_steps),
           "clocks": clocks}
    if large is not None:
        out["roofline"] = dict(large["roofline"], workload="large solve 256x192^2x6 (operator launch group)")
        out["fp64_roofline"] = large["fp64_roofline"]
        out["large_solve"] = {k: large[k] for k in ("value", "unit", "ms_per_step", "steps", "config", "e2e",
                                                     "valid_state", "clocks", "gpu_launches")}
    if not args.no_cpu_baseline and world == 1:
        out["cpu_baseline"] = cpu_baseline_serve(args, reqs)
    print(json.dumps(out), flush=True)


def oracle_request(po, req):
    """(oracle level, its state) of a served request, built by the oracle:
    the wind and the request's cone cloud inserted at its insertion time."""
    from heliocubed_b200 import serve
    from heliocubed_b200.level import ConeSpec
    prm = req.params()
    kw = dict(nr=req.nr, na=req.na, spatial_order=req.order, limiter=prm.limiter, riemann_solver=prm.riemann_solver,
              berta_fallback_type=prm.berta_fallback_type, sun_gravity=0)
    p = po.make_params(**kw)
    L = po.OracleLevelO4(p) if req.order == 4 else po.OracleLevel(p)
    base = L.base if req.order == 4 else L
    wind = serve.wind_spec()
    s = po.HcInit()
    s.kind = 1
    for k in ("pulse_block", "pulse_i", "pulse_j", "pulse_k", "rho0", "p0", "vr", "b0", "r_ref", "pulse_amp",
              "pulse_width"):
        setattr(s, k, getattr(wind, k))
    ju = base.init(s)
    c = req.cone
    rho_inner = wind.rho0 * (wind.r_ref / p.inner_radius) ** 2
    spec = ConeSpec.on_inner_boundary(p.inner_radius, lat_deg=c.lat_deg, lon_deg=c.lon_deg,
                                      half_angle_deg=c.half_width_deg, apex_speed=c.speed_kms,
                                      density=c.density_ratio * rho_inner, temperature=c.temperature)
    cs = po.HcConeSpec()
    for k in po.CONE_SPEC_FIELDS:
        setattr(cs, k, getattr(spec, k))
    cone = po.cone_prepare(cs, p.inner_radius)
    base.insert_cone(cone, cone.insertion_time, ju)
    return L, ju, cone.insertion_time


def cpu_baseline_serve(args, reqs, budget_s: float = 20.0) -> dict:
    """The oracle on the host cores on a bounded sample of the ensemble: one
    request of each scheme on the ensemble's smallest grid, each advanced
    with CFL dt until its half of the time budget is spent.  The ensemble
    rate combines the two schemes' rates by their shares of the ensemble's
    cell-updates: total work / sum over schemes of (work / rate)."""
    build = native_oracle()
    from oracle import pyoracle as po
    cores = os.cpu_count() or 1
    small = min((r.nr * r.na * r.na, r.nr, r.na) for r in reqs)
    sample = [r for r in reqs if (r.nr, r.na) == small[1:]]
    picks = [next((r for r in sample if r.order == o), None) for o in (2, 4)]
    picks = [r for r in picks if r is not None]
    rates, notes, el = {}, [], 0.0
    for r in picks:
        L, ju, t = oracle_request(po, r)
        n = 0
        t0 = time.perf_counter()
        while n < args.steps:
            dt = 0.4 / L.inv_dt(ju)
            L.rk4_step(ju, dt, t)
            t += dt
            n += 1
            if time.perf_counter() - t0 > budget_s / len(picks):
                break
        dt_s = time.perf_counter() - t0
        el += dt_s
        rates[r.order] = r.cells * n / dt_s
        notes.append(f"{n} {'WENOZ+Roe' if r.order == 4 else 'PLM-MC+Rusanov'} steps "
                     f"({rates[r.order]:.4g} cell-updates/s)")
    work = {o: sum(r.cells * r.steps for r in reqs if r.order == o) for o in rates}
    value = sum(work.values()) / sum(work[o] / rates[o] for o in rates)
    return {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "build": build,
            "sample": f"one request of each scheme on the ensemble's smallest grid {small[1]}x{small[2]}^2x6 with "
                      f"its cone: {', '.join(notes)}, CFL dt each step, OpenMP over {cores} host threads, "
                      f"{el:.1f} s; combined by the schemes' shares of the ensemble's cell-updates"}


def amr_two_level_step(args, local, seed: int) -> dict:
    """The whole two-level AMR RK4 step on the device (heliocubed_b200.amr):
    a 48 x 48^2 x 6 coarse shell and 8^3 boxes of the 96 x 96^2 x 6 level
    tiling the interiors of panels 0 and 3 (radial 16..79, angular 24..71),
    on the perturbed wind.  Per stage: coarse preparation and operator, the
    fine boxes' coarse-fine fill, exchanges, native conversion and batched
    operator, reflux and restrictions; the state update and averageDown."""
    import torch
    from heliocubed_b200.amr import AmrStep
    from heliocubed_b200.level import Params, Shell, perturbed_wind_state
    kw = dict(spatial_order=4, riemann_solver=2, berta_fallback_type=0)
    nc, nf = 48, 96
    coarse = Shell(Params(nr=nc, na=nc, **kw), device=local)
    fine = Shell(Params(nr=nf, na=nf, **kw), device=local)

    def wind(sh, n):
        det = sh.geometry(4).reshape(6, n, n)
        vol = sh.geometry(0).reshape(n + 1, 4)[:n, 3]
        return perturbed_wind_state(sh.params, det, vol, seed=seed)

    boxes = [(b, (i, j, k), (i + 7, j + 7, k + 7)) for b in (0, 3) for i in range(16, 80, 8)
             for j in range(24, 72, 8) for k in range(24, 72, 8)]
    ju_c = torch.from_numpy(np.ascontiguousarray(wind(coarse, nc).reshape(-1))).to(coarse._dev)
    wf = wind(fine, nf)
    states = [torch.from_numpy(np.ascontiguousarray(wf[b][:, lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1]))
              .to(fine._dev) for b, lo, hi in boxes]
    del wf
    step = AmrStep(coarse, fine, boxes)
    step.load(ju_c, states)
    dt = 0.5 * coarse.params.cfl / float(coarse.inv_dt_max(ju_c).item())
    step.step(dt, 0.0)
    torch.cuda.synchronize()
    reps = 3
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for r in range(reps):
        step.step(dt, (r + 1) * dt)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    valid = bool(torch.isfinite(step.state_c).all().item() and torch.isfinite(step.f["state"][0]).all().item())
    cells_c, cells_f = 6 * nc ** 3, 512 * len(boxes)
    step.close()
    coarse.close()
    fine.close()
    return {"ms_per_step": ms, "cell_updates_per_s": (cells_c + cells_f) / (ms * 1e-3), "coarse_cells": cells_c,
            "fine_boxes": len(boxes), "fine_cells": cells_f, "steps_timed": reps, "finite": valid,
            "what": "coarse 48x48^2x6 shell + 8^3 fine boxes (ratio 2) tiling panels 0 and 3 (radial 16..79, "
                    "angular 24..71 of 96): per stage the coarse preparation and operator with seam "
                    "reconciliation, the fine boxes' coarse-fine fill, <JU>/<U> recovery, exchanges, native "
                    "conversion and batched operator, reflux and restrictions; then the update and averageDown"}


def run_amr(args, world, rank, local):
    """Batched AMR-style operator evaluation (config-3 style, scaled): boxes
    of 8^3-32^3 on three refinement levels (48^3, 96^3 and 192^3 per panel,
    ratio 2), fourth-order WENOZ + Roe + Powell.  The batched path evaluates
    each level's boxes with one launch per operator kernel (hc_o4_batch_rhs);
    the plain path calls the operator once per box, as the reference's level
    evaluation does per patch.  Metric: cell-stage evaluations per second."""
    import torch
    from heliocubed_b200.level import Params, Shell, make_box, wind_box_state
    torch.cuda.set_device(local)
    rng = np.random.default_rng(args.seed)
    plan = [(48, [(16, None)]), (96, [(16, args.amr_l1)]), (192, [(8, int(0.6 * args.amr_l2)),
                                                             (16, int(0.3 * args.amr_l2)),
                                                             (32, args.amr_l2 - int(0.6 * args.amr_l2) - int(0.3 * args.amr_l2))])]
    levels = []
    for n, groups in plan:
        sh = Shell(Params(nr=n, na=n, spatial_order=4, riemann_solver=2, berta_fallback_type=0), device=local)
        specs = []
        for size, count in groups:
            if count is None:  # tile the whole level
                for b in range(6):
                    for k0 in range(0, n, size):
                        for j0 in range(0, n, size):
                            for i0 in range(0, n, size):
                                specs.append((b, (i0, j0, k0), size))
            else:
                for _ in range(count):
                    lo = tuple(int(rng.integers(0, n - size + 1)) for _ in range(3))
                    specs.append((int(rng.integers(0, 6)), lo, size))
        works = []
        for q, (b, lo, size) in enumerate(specs):
            hi = tuple(x + size - 1 for x in lo)
            u = torch.from_numpy(wind_box_state(sh.params, lo, hi, 5, args.seed + q)).to(sh._dev)
            rhs = torch.zeros(8 * size ** 3, dtype=torch.float64, device=sh._dev)
            works.append((make_box(lo, hi, 5, b), u, rhs, None))
        batch = sh.o4_batch(works)
        singles = [sh.o4_batch([w]) for w in works]
        levels.append((n, sh, works, batch, singles))
    cells = sum(sum(int(w[2].numel()) // 8 for w in lv[2]) for lv in levels)
    nboxes = sum(len(lv[2]) for lv in levels)
    stream = torch.cuda.current_stream()

    def batched():
        for _, _, _, batch, _ in levels:
            batch.rhs()

    def plain():
        for _, _, _, _, singles in levels:
            for one in singles:
                one.rhs()

    def timed(fn, reps):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    # the RK4 stage logic of the same boxes (all levels, one plan): each box's
    # valid state, stage state and four stage right-hand sides (the operator
    # output of stage s is rk[s]); one combine launch per stage
    from heliocubed_b200.level import AmrPlan
    rk_boxes = []
    for _, sh, works, _, _ in levels:
        for w in works:
            nv = w[2].numel()
            rk_boxes.append((torch.zeros(nv, dtype=torch.float64, device=sh._dev),
                             torch.zeros(nv, dtype=torch.float64, device=sh._dev),
                             [w[2]] + [torch.zeros(nv, dtype=torch.float64, device=sh._dev) for _ in range(3)]))
    plan = AmrPlan(levels[0][1], rk_boxes)

    def stage_logic():
        for s in range(5):
            plan.rk_stage(4, s, 1.0e-3)

    def batched_step():
        for s in range(4):
            batched()
            plan.rk_stage(4, s, 1.0e-3)
        plan.rk_stage(4, 4, 1.0e-3)

    # the fourth-order coarse-fine ghost interpolation of every box of the
    # refined levels: each box's ghosted storage (a copy, so the operator
    # inputs stay as they are) from a coarse array over its parents'
    # stencil footprint (synthetic averages in [1, 2)), one launch for all
    cf_boxes, ghost_cells = [], 0
    for _, sh, works, _, _ in levels[1:]:
        for w in works:
            box = w[0]
            flo = [box.lo[d] - box.ghost for d in range(3)]
            fhi = [box.hi[d] + box.ghost for d in range(3)]
            clo = [flo[d] // 2 - 2 for d in range(3)]
            cn = [fhi[d] // 2 + 2 - clo[d] + 1 for d in range(3)]
            coarse = torch.rand(8 * cn[0] * cn[1] * cn[2], dtype=torch.float64, device=sh._dev) + 1.0
            fn = [fhi[d] - flo[d] + 1 for d in range(3)]
            ghost_cells += fn[0] * fn[1] * fn[2] - (box.hi[0] - box.lo[0] + 1) ** 3
            cf_boxes.append({"coarse": coarse, "fine": w[1].clone(), "coarse_lo": clo, "coarse_n": cn, "fine_lo": flo,
                             "fine_n": fn, "valid_lo": list(box.lo), "valid_hi": list(box.hi), "ratio": (2, 2, 2),
                             "ncomp": 8})
    cf_plan = AmrPlan(levels[0][1], [])
    cf_plan.set_cf_interp(cf_boxes)

    def cf_fill():
        cf_plan.cf_interpolate(0, len(cf_boxes))

    sampler = ClockSampler(local)
    sampler.start()
    ms_b = timed(batched, args.amr_reps)
    ms_p = timed(plain, max(1, args.amr_reps // 4))
    ms_rk = timed(stage_logic, args.amr_reps)
    ms_step = timed(batched_step, max(1, args.amr_reps // 4))
    ms_cf = timed(cf_fill, args.amr_reps)
    clocks = sampler.stop()
    plan.close()
    cf_plan.close()
    # identical results
    for _, _, works, _, _ in levels:
        for w in works:
            w[2].zero_()
    batched()
    ref = [w[2].clone() for lv in levels for w in lv[2]]
    for _, _, works, _, _ in levels:
        for w in works:
            w[2].zero_()
    plain()
    torch.cuda.synchronize()
    same = all(torch.equal(a, w[2]) for a, w in zip(ref, [w for lv in levels for w in lv[2]]))
    nop = operator_launches(argparse.Namespace(riemann=2))
    if rank == 0:
        out = {"metric": "FP64 cell-stage evaluations/s, batched AMR boxes vs plain per-box launches",
               "value": cells / (ms_b * 1e-3) * world, "unit": "cell-stage evaluations/s", "n_gpus": world,
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
               "data": "synthetic",
               "config": {"workload": "AMR-style box batch (scaled config 3), Berta WENOZ + Roe + Powell",
                          "levels": [{"n": n, "boxes": len(w)} for n, _, w, _, _ in levels], "boxes": nboxes,
                          "cells": cells, "ghost": 5},
               "batched": {"ms_per_evaluation": ms_b, "launches": len(levels) * nop},
               "plain": {"ms_per_evaluation": ms_p, "cell_stage_per_s": cells / (ms_p * 1e-3),
                         "launches": nop * nboxes},
               "batched_over_plain": ms_p / ms_b, "identical_results": same,
               "rk4_stage_logic": {"ms_per_step": ms_rk, "launches": 5,
                                   "what": "tableau combine of every box of every level, 4 stages + final"},
               "rk4_step_without_ghost_fill": {"ms": ms_step, "cell_updates_per_s": cells / (ms_step * 1e-3),
                                               "what": "4 x (batched operator of each level + stage combine) + "
                                                       "final combine; coarse-fine ghost fill and registers are "
                                                       "the caller's"},
               "coarse_fine_interpolation": {"ms": ms_cf, "boxes": len(cf_boxes), "ghost_cells": ghost_cells,
                                             "launches": 1,
                                             "what": "fourth-order quartic interpolation of the 5 ghost layers of "
                                                     "every box of the two refined levels from coarse averages, "
                                                     "8 components, one launch"},
               "clocks": clocks}
    for _, sh, _, batch, singles in levels:
        batch.close()
        for one in singles:
            one.close()
        sh.close()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    two = amr_two_level_step(args, local, args.seed)
    if rank == 0:
        out["two_level_rk4_step"] = two
        print(json.dumps(out), flush=True)


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--order", type=int, choices=[2, 4], default=None,
                    help="uniform workload: spatial order (default 4); implies --workload uniform")
    ap.add_argument("--nr", type=int, default=None)
    ap.add_argument("--na", type=int, default=None)
    ap.add_argument("--limiter", type=int, default=3)
    ap.add_argument("--riemann", type=int, default=None)
    ap.add_argument("--gravity", type=int, default=None, help="solar gravity (default: 1 for slabs, else 0)")
    ap.add_argument("--init", choices=["default", "cone"], default="default",
                    help="cone: the wind with a 1500 km/s, 45 deg cone-CME cloud (the large-solve workload)")
    ap.add_argument("--seed", type=int, default=20261204)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-graph", dest="graph", action="store_false",
                    help="launch the step eagerly instead of replaying a captured CUDA graph")
    ap.add_argument("--o4-variants", default=None, metavar="R,P,F",
                    help="order 4: use these register-cap variants of the reconstruction, Roe point and final-flux "
                         "kernels instead of timing them (for profiler runs)")
    ap.add_argument("--cpu-max-steps", type=int, default=60)
    ap.add_argument("--ref-budget", type=float, default=20.0)
    ap.add_argument("--workload", choices=["serve", "uniform", "amr", "slabs"], default=None,
                    help="serve (default): the served CME ensemble with the large solve; uniform: one solve; "
                         "amr: the AMR-style box batch; slabs: one shell split into radial slabs over the ranks")
    ap.add_argument("--serve", action="store_true", help="same as --workload serve")
    ap.add_argument("--amr", action="store_true", help="same as --workload amr")
    ap.add_argument("--no-large", action="store_true", help="serve: leave out the large single solve")
    ap.add_argument("--large-steps", type=int, default=5, help="serve: RK4 steps of the large single solve")
    ap.add_argument("--amr-l1", type=int, default=600)
    ap.add_argument("--amr-l2", type=int, default=1200)
    ap.add_argument("--amr-reps", type=int, default=8)
    ap.add_argument("--serve-requests", type=int, default=256)
    ap.add_argument("--serve-inflight", type=int, default=8)
    ap.add_argument("--serve-budget-gb", type=float, default=120.0)
    ap.add_argument("--no-cobatch", action="store_true",
                    help="serve: fourth-order requests on their own streams instead of one cohort")
    args = ap.parse_args()
    # --order, --nr, --na or --init cone without --workload select the uniform workload
    uniform_opts = args.order is not None or args.nr is not None or args.na is not None or args.init != "default"
    args.workload = args.workload or ("amr" if args.amr else "serve" if args.serve or not uniform_opts
                                      else "uniform")
    args.order = args.order or 4
    o4 = args.order == 4
    slabs = args.workload == "slabs"
    args.nr = args.nr or (256 if slabs and o4 else 64 if o4 else 32)
    args.na = args.na or (192 if slabs and o4 else 64 if o4 else 32)
    args.riemann = args.riemann or (2 if o4 else 1)
    args.gravity = (1 if slabs else 0) if args.gravity is None else args.gravity
    args.steps = args.steps or (20 if args.workload == "serve" else 10 if slabs else 100 if o4 else 2000)
    if args.warmup < 3:
        ap.error("--warmup must be at least 3")
    if args.impl == "reference" and int(os.environ.get("RANK", "0")) != 0:
        return 0  # the CPU reference arm runs on rank 0 only
    if args.impl == "reference":
        run_reference(args, 1, 0)
        return 0
    world, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        elif args.workload == "serve":
            run_serve(args, world, rank, local)
        elif args.workload == "amr":
            run_amr(args, world, rank, local)
        elif args.workload == "slabs":
            run_slabs(args, world, rank, local)
        else:
            run_b200(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
