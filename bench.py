"""Benchmark of the time-step hot path (one JSON line on rank 0).

Workload: the viscous hot-gas plume (methalox products, gamma 1.2, T0 3500 K,
p0 70 bar, 80 % bell with expansion 20, sea level) on a 512 x 192 grid:
Sutherland + eddy viscosity, wall model, afterburning scalars. Synthetic and
deterministic: every input comes from the setup pipeline.

One bench step = one ``GPUSolver.step(n, P)`` call with n = SOLVER_STEPS time
steps (the reference's frame loop calls ``step(n, P)`` the same way). The L2
cache is flushed (a 512 MiB write on the solver's stream) before every timed
bench step. ``value`` = cell updates per second over the timed steps, device
time from CUDA events on the solver's stream, max over ranks; ``e2e`` = the
same through the public API with the parameter upload and the read-out
read-back (step info, exit column, chamber cell) in the timed region, host
clock. With --gpus N every rank runs its own instance (replicas: one grid does
not shard).

--impl reference times the CPU oracle (the restatement of the reference's
shader passes; the reference itself needs WebGL2) on all host cores.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
import __graft_entry__ as ge  # noqa: E402

SOLVER_STEPS = 100          # time steps per bench step
FLUSH_BYTES = 512 << 20     # > 126 MB L2
WORKLOAD = "viscous plume 512x192 (methalox gamma 1.2, T0 3500 K, p0 70 bar, bell eps 20, sea level)"
# algorithmic HBM bytes per cell for each kernel kind (fused design): state
# planes are 32 B per cell (A 16 + B 16), geometry 49 B (geoA, geoG, geoM 16
# each + mask 1); spray parcels 112 B each.
BYTES_PER_CELL = {"stage1": 32 + 49 + 32, "stage2": 32 + 32 + 49 + 32, "stage2_physics": 32 + 32 + 49 + 32,
                  "apply": 32 + 16 + 33 + 32, "reduce": 32 + 1}
THROTTLE_BITS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
                 0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
                 0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting"}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(kind):
    """DRAM bytes per cell of a kernel from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "traffic_per_cell.txt")
    try:
        with open(path) as f:
            for line in f:
                parts = line.split()
                if len(parts) >= 2 and parts[0] == kind:
                    return float(parts[1])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons, every 20 ms while
    it runs. Started before the warm-up (nvidia-smi takes a while to start);
    mark() brackets the timed region and summary() keeps the samples taken
    inside it (the nearest later one if the region was shorter than a
    sampling interval)."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None
        self.window = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active",
                 "--format=csv,noheader,nounits", "-lms", "20"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 3:
                try:
                    self.samples.append((time.monotonic(), float(parts[0]), float(parts[1]), int(parts[2], 16)))
                except ValueError:
                    pass

    def wait_first(self, timeout_s=5.0):
        """Waits (bounded) until nvidia-smi has produced its first sample."""
        t0 = time.monotonic()
        while self.proc is not None and not self.samples and time.monotonic() - t0 < timeout_s:
            time.sleep(0.01)

    def mark(self, t0, t1):
        self.window = (t0, t1)

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        samples = self.samples
        if self.window is not None:
            t0, t1 = self.window
            inside = [q for q in samples if t0 <= q[0] <= t1]
            if not inside:
                later = [q for q in samples if q[0] > t1]
                inside = later[:1]
            samples = inside
        if not samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [q[1] for q in samples]
        reasons = set()
        for q in samples:
            for bit, name in THROTTLE_BITS.items():
                if q[3] & bit and name != "gpu_idle":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(q[2] for q in samples),
                "reasons": sorted(reasons), "samples": len(sm), "interval_ms": 20}


GRID = (512, 192)


def make_setup(rn):
    from rocket_nozzle_cfd_solver_b200.configs import viscous_plume
    cfg, _ = viscous_plume(Nx=GRID[0], Nr=GRID[1])
    return rn.build_sim_setup(cfg)


def cpu_sample(setup, seconds=12.0, threads=None, start=2):
    """Oracle (FP32 port of the shader passes) on the host cores: cell-updates/s,
    timed from time step `start` (reached untimed) of the solve."""
    oracle = ge.load_oracle()
    threads = threads or os.cpu_count() or 1
    oracle.set_threads(threads)
    o = oracle.OracleSolver(setup.Nx, setup.Nr)
    o.setGeometry(setup.geo)
    init = setup.initialState()
    o.setState(init["A"], init["B"])
    o.step(start, setup.P)
    steps, t0 = 0, time.perf_counter()
    while True:
        o.step(1, setup.P)
        steps += 1
        el = time.perf_counter() - t0
        if el >= seconds or steps >= 2000:
            break
    o.close()
    return setup.Nx * setup.Nr * steps / el, threads, steps, el


def run_reference(args, rank, world):
    """The reference arm: the CPU oracle on all host cores, timed over the
    stretch of the solve where our arm's timed region starts (our arm times
    time steps W*SOLVER_STEPS .. (W+K)*SOLVER_STEPS after W warm-up bench
    steps; the oracle steps untimed to W*SOLVER_STEPS, then times K steps,
    one per bench step: the per-step cost drifts a few percent as the plume
    develops)."""
    if rank != 0:
        return
    rn = ge.load_package()
    setup = make_setup(rn)
    oracle = ge.load_oracle()
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    o = oracle.OracleSolver(setup.Nx, setup.Nr)
    o.setGeometry(setup.geo)
    init = setup.initialState()
    o.setState(init["A"], init["B"])
    start = args.warmup * SOLVER_STEPS
    o.step(start, setup.P)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o.step(1, setup.P)
    el = time.perf_counter() - t0
    cells = setup.Nx * setup.Nr
    value = cells * args.steps / el
    sample = (f"time steps {start}..{start + args.steps} of the {setup.Nx}x{setup.Nr} viscous plume (the start of "
              f"our arm's timed window, steps {start}..{start + args.steps * SOLVER_STEPS}), one per bench step")
    line = {"impl": "reference", "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "solver_steps_per_bench_step": 1,
                       "window": [start, start + args.steps],
                       "implementation": "CPU oracle: C++ restatement of the reference's WebGL2 passes "
                                         "(the reference itself needs a graphics stack)"},
            "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local_rank):
    import torch
    rn = ge.load_package()
    from rocket_nozzle_cfd_solver_b200 import replicas
    torch.cuda.set_device(local_rank)
    setup = make_setup(rn)
    cells = setup.Nx * setup.Nr
    g = rn.GPUSolver(setup.Nx, setup.Nr)
    if args.tile:
        g.setTile(args.tile)
    g.setGeometry(setup.geo)
    init = setup.initialState()
    g.setState(init["A"], init["B"])
    params = rn.params_from_P(setup.P)
    # tile shape: the autotuner's pick (timed on this state, which it restores)
    tile_name = g.tile if args.tile else g.autotune(params, steps=100)
    stream = torch.cuda.ExternalStream(g.stream())
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{local_rank}")

    def flush_l2():
        with torch.cuda.stream(stream):
            flush.fill_(1.0)

    clk = ClockSampler(local_rank)
    clk.__enter__()                             # sampling from the warm-up on; the timed window is marked below
    clk.wait_first()
    for _ in range(args.warmup):
        flush_l2()
        g.step(SOLVER_STEPS, params)
    g.sync()
    torch.cuda.synchronize()
    launches0 = g.kernelLaunches()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()

    # ---- timed region: device time per bench step, L2 flushed before each
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t_clk0 = time.monotonic()
    for k in range(args.steps):
        flush_l2()
        with torch.cuda.stream(stream):
            evs[k][0].record(stream)
        g.step(SOLVER_STEPS, params)
        with torch.cuda.stream(stream):
            evs[k][1].record(stream)
    g.sync()
    torch.cuda.synchronize()
    clk.mark(t_clk0, time.monotonic())
    time.sleep(0.05)                            # the sample after a region shorter than the interval
    clk.__exit__(None, None, None)
    launches = g.kernelLaunches() - launches0
    ms = sum(a.elapsed_time(b) for a, b in evs)
    dev = f"cuda:{local_rank}"
    ms = replicas.max_over_ranks(ms, dev)
    value = world * cells * SOLVER_STEPS * args.steps / (ms * 1e-3)

    # ---- end to end through the public API: params up, step, read-outs down
    # (right after the timed region, so that both cover the same stretch of the
    # solve: the per-step cost grows a few percent as the plume develops)
    reqs = [{"name": "step", "tex": g.stepInfoTex, "x": 0, "y": 0, "w": 1, "h": 1},
            {"name": "colA", "tex": g.state["A"], "x": setup.iExit, "y": 0, "w": 1, "h": setup.Nr},
            {"name": "colB", "tex": g.state["B"], "x": setup.iExit, "y": 0, "w": 1, "h": setup.Nr},
            {"name": "chA", "tex": g.state["A"], "x": setup.iChamber, "y": 0, "w": 1, "h": 1},
            {"name": "chB", "tex": g.state["B"], "x": setup.iChamber, "y": 0, "w": 1, "h": 1}]
    d2h = sum(r["w"] * r["h"] * 16 for r in reqs)
    import ctypes
    h2d = ctypes.sizeof(params)
    if world > 1:
        torch.distributed.barrier()
    # The app's frame loop: queue the next step(n, P) before waiting for the
    # previous read-back, then turn that read-back into the read-outs while
    # the GPU runs (requestAsync / pollAsync keep one read in flight). Run 3
    # times; the median run is reported, all three are listed.
    def frame_loop():
        t0 = time.perf_counter()
        perf, iters = None, []
        g.step(SOLVER_STEPS, setup.P)              # parameter block converted and passed every call
        g.requestAsync(reqs, 0)
        for k in range(args.steps):
            ta = time.perf_counter()
            if k + 1 < args.steps:
                g.step(SOLVER_STEPS, setup.P)
            res = None
            while res is None:
                res = g.pollAsync()
            d = res["data"]
            perf = rn.exit_performance(setup, {"A": d["colA"], "B": d["colB"]})
            if k + 1 < args.steps:
                g.requestAsync(reqs, k + 1)
            iters.append(time.perf_counter() - ta)
        g.sync()
        return replicas.max_over_ranks(time.perf_counter() - t0, dev), perf, iters

    runs = [frame_loop() for _ in range(3)]
    e2e_runs = [world * cells * SOLVER_STEPS * args.steps / r[0] for r in runs]
    e2e_s, perf, iters = sorted(runs, key=lambda r: r[0])[1]
    e2e = world * cells * SOLVER_STEPS * args.steps / e2e_s
    # ---- per-kernel profile over the same number of bench steps (roofline):
    # CUDA events around each kernel inside replays of the step graph (the
    # kernels back to back, as in the timed region), and launch by launch
    # (each kernel between two host-side event records: it includes the gaps
    # in which the GPU waits for the host's next launch)
    def kernel_profile(in_graph):
        g.profile(True, in_graph=in_graph)
        for k in range(args.steps):
            flush_l2()
            g.step(SOLVER_STEPS, params)
        p = g.profileRead()
        g.profile(False)
        return p
    prof = kernel_profile(True)
    prof_lbl = kernel_profile(False)
    kind, (kms, kn) = max(((k, v) for k, v in prof.items() if v[1] > 0), key=lambda kv: kv[1][0])
    ev_ms = kms / kn
    lbl_ms = prof_lbl[kind][0] / max(prof_lbl[kind][1], 1)
    total_ms = sum(v[0] for v in prof.values())
    # An event pair around a kernel also holds its launch processing, which
    # back-to-back launches overlap with the kernel before (the event-timed
    # kernels of a step add up to more than the step takes in the timed
    # region). The kernel's time in the timed region: the region's device time
    # per solver step times the kernel's share of the step's kernel time.
    step_ms = ms / (args.steps * SOLVER_STEPS)
    launches_per_step = kn / (args.steps * SOLVER_STEPS)
    avg_ms = step_ms * (kms / total_ms) / launches_per_step
    peak, peak_kind = measured_peak()
    bpc = BYTES_PER_CELL.get(kind)
    achieved = bpc * cells / (avg_ms * 1e-3) / 1e9 if bpc else None
    traffic_pc = profiled_traffic(kind)

    def frac_of(t_ms):
        return bpc * cells / (t_ms * 1e-3) / 1e9 / peak if bpc else None
    resident_mb = cells * (3 * 32 + 49) / 1e6      # state ring + geometry
    roofline = {"bound": "hbm", "kernel": kind, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak if achieved else None, "peak_source": peak_kind,
                "bytes_per_launch": bpc * cells if bpc else None, "avg_launch_us": avg_ms * 1e3,
                "timing": "timed-region device time per solver step (CUDA events on the solver's stream) x the "
                          "kernel's share of the step's kernel time (CUDA events around each kernel inside the "
                          "replayed step graph)",
                "step_us": step_ms * 1e3,
                "avg_launch_us_event_pair_in_graph": ev_ms * 1e3, "frac_event_pair_in_graph": frac_of(ev_ms),
                "avg_launch_us_launch_by_launch": lbl_ms * 1e3, "frac_launch_by_launch": frac_of(lbl_ms),
                "traffic": traffic_pc * cells if traffic_pc else None,
                "share": {k: round(v[0] / total_ms, 4) for k, v in prof.items() if v[1] > 0},
                "l2_note": (f"{setup.Nx}x{setup.Nr} state + geometry (~{resident_mb:.0f} MB) fits in the 126 MB L2: "
                            "within a bench step the kernels run mostly from L2, so achieved can exceed the HBM "
                            "copy bandwidth") if resident_mb < 126 else
                           f"{setup.Nx}x{setup.Nr} state + geometry (~{resident_mb:.0f} MB) exceeds the 126 MB L2"}

    # ---- steady state: back-to-back steps, no flush (for reference)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
    g.step(SOLVER_STEPS * args.steps, params)
    with torch.cuda.stream(stream):
        e1.record(stream)
    g.sync()
    steady = cells * SOLVER_STEPS * args.steps / (e0.elapsed_time(e1) * 1e-3)

    g.close()
    del flush
    torch.cuda.empty_cache()
    batched = serving = large = spray = None
    if world == 1 and not args.no_large:
        spray = run_spray(args, local_rank)
    if world == 1 and not args.no_large:
        large = run_large_grid(args)
        torch.cuda.empty_cache()
    if args.batch_instances > 0:
        batched = run_batched(args, local_rank, rank, world)
    if world == 1 and args.serve_requests > 0:
        serving = run_serving(args)

    if rank != 0:
        return
    cpu = None
    fp64 = run_fp64_check(args) if world == 1 and not args.no_cpu else None
    if world == 1 and not args.no_cpu:
        start = args.warmup * SOLVER_STEPS
        cv, threads, nst, el = cpu_sample(setup, start=start)
        cpu = {"value": cv, "unit": "cell-updates/s", "cores": threads, "kind": "port",
               "sample": f"{nst} time steps of the {setup.Nx}x{setup.Nr} viscous plume from step {start}, the "
                         f"start of the timed window ({el:.1f} s, FP32 oracle, OpenMP over rows)"}
    line = {"metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "grid": [setup.Nx, setup.Nr], "cells": cells,
                       "solver_steps_per_bench_step": SOLVER_STEPS, "l2": "flushed before every bench step",
                       "parallelism": f"replicas x{world}", "physics": "viscous+wall model+afterburning",
                       "tile": tile_name},
            "roofline": roofline, "cpu_baseline": cpu,
            "e2e": {"value": e2e, "unit": "cell-updates/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "exit_thrust_N": perf["F"] if perf else None, "runs": e2e_runs,
                    "frame_ms_median": 1e3 * float(np.median(iters)), "frame_ms_max": 1e3 * float(max(iters))},
            "steady_state_value": steady,
            "gpu_launches": launches, "clocks": clk.summary(), "fp64_error": fp64, "spray": spray, "large_grid": large,
            "batched": batched, "serving": serving}
    print(json.dumps(line), flush=True)


def run_batched(args, local_rank, rank=0, world=1):
    """The batched workload: `--batch-instances` seeded nozzles (grids drawn
    from 128x48 .. 1024x384, expansion 4-40, p0 10-100 bar, gamma 1.2/1.4,
    altitude 0-30 km, all viscous) stepped by one SolverBatch (one launch per
    kernel kind per step, 6-step periods replayed from a CUDA graph, tile shape
    from the batch autotuner), against the same handles stepped one at a time
    with rn_step. Both are device times from CUDA events; the batch's state
    (~1 GB with geometry) is far larger than L2, so no flush is needed."""
    import torch
    rn = ge.load_package()
    from rocket_nozzle_cfd_solver_b200 import configs
    from rocket_nozzle_cfd_solver_b200 import replicas
    cfgs = configs.batched(args.batch_instances, seed=2024)
    if world > 1:
        # instances shard across ranks by grid cells (no data-path collective)
        cells_of = [c["Nx"] * round(c["aspect"] * c["Nx"]) for c in cfgs]
        cfgs = [cfgs[k] for k in replicas.partition_by_cost(cells_of, rank, world)]
    t0 = time.perf_counter()
    setups = [rn.build_sim_setup(c) for c in cfgs]
    t_setup = time.perf_counter() - t0
    handles = []
    for s in setups:
        g = rn.GPUSolver(s.Nx, s.Nr)
        g.setGeometry(s.geo)
        init = s.initialState()
        g.setState(init["A"], init["B"])
        handles.append(g)
    cells = sum(s.Nx * s.Nr for s in setups)
    batch = rn.SolverBatch()
    for g, s in zip(handles, setups):
        batch.add(g, s.P)
    tile = batch.autotune(steps=12)
    stream = torch.cuda.ExternalStream(batch.stream())
    nsteps = args.batch_steps
    for _ in range(args.warmup):
        batch.step(nsteps)
    batch.sync()
    l0 = batch.kernelLaunches()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            evs[k][0].record(stream)
        batch.step(nsteps)
        with torch.cuda.stream(stream):
            evs[k][1].record(stream)
    batch.sync()
    launches = batch.kernelLaunches() - l0
    dev = f"cuda:{local_rank}"
    ms = replicas.max_over_ranks(sum(a.elapsed_time(b) for a, b in evs), dev)
    my_cells = cells
    cells = int(replicas.sum_over_ranks(cells, dev))
    value = cells * nsteps * args.steps / (ms * 1e-3)
    # FP64 read-outs of every member after the batch run (thrust, mass flow)
    F = [g.integrals(s) for g, s in zip(handles, setups)]
    finite = all(math.isfinite(x["F"]) and math.isfinite(x["mdot"]) for x in F)
    # the same handles one at a time (rn_step per instance, its own stream)
    for g in handles:
        batch.remove(g)
    batch.close()
    rounds = max(1, min(args.steps, 5))
    p_list = [rn.params_from_P(s.P) for s in setups]
    for g, p in zip(handles, p_list):
        g.step(nsteps, p)
    for g in handles:
        g.sync()
    single_ms = 0.0
    t0 = time.perf_counter()
    for _ in range(rounds):
        for g, p in zip(handles, p_list):
            st = torch.cuda.ExternalStream(g.stream())
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(st):
                a.record(st)
            g.step(nsteps, p)
            with torch.cuda.stream(st):
                b.record(st)
            b.synchronize()
            single_ms += a.elapsed_time(b)
    single_wall = replicas.max_over_ranks(time.perf_counter() - t0, dev)
    single_ms = replicas.max_over_ranks(single_ms, dev)
    single = cells * nsteps * rounds / (single_ms * 1e-3)
    for g in handles:
        g.close()
    sizes = {}
    for s in setups:
        sizes[f"{s.Nx}x{s.Nr}"] = sizes.get(f"{s.Nx}x{s.Nr}", 0) + 1
    peak, src = measured_peak()
    bpc = BYTES_PER_CELL["stage1"] + BYTES_PER_CELL["stage2_physics"]
    instances = int(replicas.sum_over_ranks(len(setups), dev))
    classes = None
    if world == 1 and not args.no_classes:
        classes = [class_solves(rn, size, n, fp64_samples=(2 if size[0] <= 256 else 0))
                   for size, n in CLASS_COUNTS.items()]
    return {"metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "instances": instances,
            "ranks": world, "cells_this_rank": my_cells,
            "achieved_gbs": value * bpc / 1e9, "bytes_per_cell_step": bpc, "frac": value * bpc / 1e9 / peak,
            "peak_source": src,
            "cells": cells, "grids": sizes, "solver_steps_per_bench_step": nsteps, "steps": args.steps,
            "ms_per_step": ms / args.steps, "tile": tile, "gpu_launches": launches,
            "launches_per_solver_step": launches / (nsteps * args.steps),
            "one_at_a_time": {"value": single, "unit": "cell-updates/s", "wall_value":
                              cells * nsteps * rounds / single_wall, "rounds": rounds},
            "speedup_vs_one_at_a_time": value / single, "fp64_readouts_finite": finite,
            "setup_s": t_setup, "l2": "state ~1 GB > L2: no flush",
            "solves_per_class": classes}


CLASS_COUNTS = {(128, 48): 64, (256, 96): 64, (512, 192): 8, (1024, 384): 4}


def class_solves(rn, size, count, t_end_s=2e-3, K=60, seed=64, fp64_samples=0):
    """Solves/s of `count` seeded nozzles of one grid class (configs.
    batched_instance: expansion 4-40, p0 10-100 bar, gamma 1.2/1.4, altitude
    0-30 km, viscous), each run to 2 ms of simulated time in chunks of K steps
    (`while t < t_end: step(K)`), one at a time (rn_step per solve, in turn,
    default tile) and batched (one SolverBatch, tile shape from its autotuner,
    rn_batch_run: every member stops on the device at its own chunk). Host
    clock around the stepping, setups and the autotuner excluded. Final exit
    thrust and mass flow of every solve; the first `fp64_samples` solves of
    both forms checked against the oracle run in FP64 for the same steps (the
    FP64-scheme error; also for the FP32 oracle, the scheme's own FP32 error)."""
    import torch
    from rocket_nozzle_cfd_solver_b200 import configs
    rng = np.random.default_rng(seed + size[0])
    setups = [rn.build_sim_setup(configs.batched_instance(rng, size)) for _ in range(count)]

    def start(s):
        g = rn.GPUSolver(s.Nx, s.Nr)
        g.setGeometry(s.geo)
        init = s.initialState()
        g.setState(init["A"], init["B"])
        return g

    def finish(g, s):
        col = g.readColumn(s.iExit)
        perf = rn.exit_performance(s, col)
        return {"steps": g.stepCount, "F": perf["F"], "mdot": perf["mdot"], "A": g.readAll()}

    t_end = [t_setups_end(s, t_end_s) for s in setups]
    # one at a time
    hs = [start(s) for s in setups]
    ps = [rn.params_from_P(s.P) for s in setups]
    single_tile = hs[0].tile
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for g, te, p in zip(hs, t_end, ps):
        while float(g.readStepInfo()[2]) < te:
            g.step(K, p)
    t_single = time.perf_counter() - t0
    single_res = [finish(g, s) for g, s in zip(hs, setups)]
    for g in hs:
        g.close()
    # batched
    hs = [start(s) for s in setups]
    batch = rn.SolverBatch()
    for g, s in zip(hs, setups):
        batch.add(g, s.P)
    tile = batch.autotune(steps=12)
    batch.sync()
    torch.cuda.synchronize()
    launches0 = batch.kernelLaunches()
    t0 = time.perf_counter()
    batch.run(t_end, chunk=K)
    t_batch = time.perf_counter() - t0
    launches = batch.kernelLaunches() - launches0
    batch.close()
    batch_res = [finish(g, s) for g, s in zip(hs, setups)]
    for g in hs:
        g.close()
    same_steps = all(a["steps"] == b["steps"] for a, b in zip(single_res, batch_res))
    diff = max(float(np.linalg.norm(a["A"]["A"].astype(np.float64) - b["A"]["A"]) /
                     max(np.linalg.norm(a["A"]["A"].astype(np.float64)), 1e-30))
               for a, b in zip(single_res, batch_res))

    def rel(x, y):
        return abs(x - y) / max(abs(y), 1e-30)

    fp64 = []
    if fp64_samples:
        oracle = ge.load_oracle()
        oracle.set_threads(os.cpu_count() or 1)
        for s, r1, rb in list(zip(setups, single_res, batch_res))[:fp64_samples]:
            ref = {}
            for dbl in (True, False):
                o = oracle.OracleSolver(s.Nx, s.Nr, fp64=dbl)
                o.setGeometry(s.geo)
                init = s.initialState()
                o.setState(init["A"], init["B"])
                o.step(rb["steps"], s.P)
                ref[dbl] = rn.exit_performance(s, exit_column(o.readAll(), s))
                o.close()
            op = ref[True]
            fp64.append({"steps": rb["steps"],
                         "batched": {"thrust_rel_err": rel(rb["F"], op["F"]), "mdot_rel_err": rel(rb["mdot"], op["mdot"])},
                         "one_at_a_time": {"thrust_rel_err": rel(r1["F"], op["F"]),
                                           "mdot_rel_err": rel(r1["mdot"], op["mdot"])},
                         "fp32_oracle": {"thrust_rel_err": rel(ref[False]["F"], op["F"]),
                                         "mdot_rel_err": rel(ref[False]["mdot"], op["mdot"])}})
    steps = [r["steps"] for r in batch_res]
    return {"grid": f"{size[0]}x{size[1]}", "solves": count, "steps_to_2ms": [min(steps), max(steps)],
            "one_at_a_time_solves_per_s": count / t_single, "batched_solves_per_s": count / t_batch,
            "speedup": t_single / t_batch, "tile": {"one_at_a_time": single_tile, "batched": tile},
            "batched_launches": launches, "same_steps": same_steps,
            "state_rel_l2_batched_vs_one_at_a_time": diff, "fp64_error": fp64}


def t_setups_end(s, t_end_s):
    return t_end_s / s.tScale


def run_large_grid(args):
    """HBM-resident sweep point: the plain cold-gas nozzle on a 4096 x 1536
    grid (6.3 M cells; one state copy is 201 MB, beyond the 126 MB L2), two
    kernels per step. Achieved GB/s = algorithmic bytes per cell-step (258 B:
    stage 1 reads 32 + 49, writes 32; stage 2 reads 32 + 32 + 49, writes 32)
    x cell-steps/s, device time from CUDA events."""
    import torch
    rn = ge.load_package()
    from rocket_nozzle_cfd_solver_b200.configs import plain_small
    s = rn.build_sim_setup(plain_small(4096, 1536)[0])
    g = rn.GPUSolver(s.Nx, s.Nr)
    g.setGeometry(s.geo)
    init = s.initialState()
    g.setState(init["A"], init["B"])
    p = rn.params_from_P(s.P)
    tile = g.autotune(p, steps=10)
    stream = torch.cuda.ExternalStream(g.stream())
    n = 20
    for _ in range(max(args.warmup, 1)):
        g.step(n, p)
    g.sync()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    g.profile(True)
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            evs[k][0].record(stream)
        g.step(n, p)
        with torch.cuda.stream(stream):
            evs[k][1].record(stream)
    g.sync()
    prof = g.profileRead()
    g.profile(False)
    ms = sum(a.elapsed_time(b) for a, b in evs)
    cells = s.Nx * s.Nr
    rate = cells * n * args.steps / (ms * 1e-3)
    peak, src = measured_peak()
    bpc = BYTES_PER_CELL["stage1"] + BYTES_PER_CELL["stage2"]
    kern = {}
    for k in ("stage1", "stage2"):
        kms, kn = prof[k]
        if kn:
            gbs = BYTES_PER_CELL[k] * cells / (kms / kn * 1e-3) / 1e9
            kern[k] = {"avg_launch_us": 1e3 * kms / kn, "achieved_gbs": gbs, "frac": gbs / peak}
    g.close()
    return {"workload": "plain cold-gas nozzle 4096x1536 (inviscid, 2 kernels per step)", "cells": cells,
            "value": rate, "unit": "cell-updates/s", "bytes_per_cell_step": bpc,
            "achieved_gbs": rate * bpc / 1e9, "peak_gbs": peak, "peak_source": src,
            "frac": rate * bpc / 1e9 / peak, "kernels": kern, "tile": tile}


def run_spray(args, local_rank, t_end_s=2e-3, chunk=50):
    """Injector + spray chamber, the configuration as stated: coaxial methalox
    at 70 bar (preset injCoax), 512 x 192, the 65,536-slot parcel ring
    pre-populated with 65,536 seeded parcels (configs.prepopulated_parcels:
    lognormal diameters, median 60 um, sigma 0.4, on the injector elements,
    30 / 120 m/s +-10 %) and spawning 4 per step from the injector table, run
    to about 2 ms of simulated time. Device time of the stepping (CUDA events
    around each chunk of steps; the chunk boundaries read the step info to
    stop at 2 ms). Reported beside each other: live parcel-steps/s (live
    parcels summed over the steps, counted on the device, per second) and
    slot-steps/s (all 65,536 ring slots every step, what the reference's spray
    pass draws)."""
    import torch
    rn = ge.load_package()
    from rocket_nozzle_cfd_solver_b200 import configs
    s = rn.build_sim_setup(configs.injector_spray(512, 192)[0])
    PA, PB, head = configs.prepopulated_parcels(s, 65536)
    g = rn.GPUSolver(s.Nx, s.Nr)
    g.setGeometry(s.geo)
    init = s.initialState()
    g.setState(init["A"], init["B"])
    rn.GPUSpray(g).resize()
    g.spray.setInjector(s.injector)
    g.spray.setParcels(PA, PB, head)
    live0 = g.spray.stats()["parcels"]
    p = rn.params_from_P(s.P)
    st = torch.cuda.ExternalStream(g.stream())
    t_end = t_end_s / s.tScale
    ms, steps, t = 0.0, 0, 0.0
    while t < t_end:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(st):
            e0.record(st)
        g.step(chunk, p)
        with torch.cuda.stream(st):
            e1.record(st)
        t = float(g.readStepInfo()[2])
        ms += e0.elapsed_time(e1)
        steps += chunk
    live_steps = g.spray.parcelSteps()
    live = g.spray.stats()["parcels"]
    g.profile(True)
    g.step(chunk, p)
    prof = g.profileRead()
    g.profile(False)
    total = sum(v[0] for v in prof.values())
    g.close()
    sec = ms * 1e-3
    return {"workload": "injector + spray chamber 512x192 (injCoax, methalox 70 bar), ring pre-populated with "
                        "65,536 parcels (lognormal d, median 60 um, sigma 0.4), about 2 ms simulated",
            "steps": steps, "simulated_ms": t * s.tScale * 1e3, "ms_per_step": ms / steps,
            "steps_per_s": steps / sec, "cell_updates_per_s": s.Nx * s.Nr * steps / sec,
            "live_parcel_steps_per_s": live_steps / sec, "slot_steps_per_s": 65536 * steps / sec,
            "live_parcel_steps": live_steps, "live_parcels_at_start": live0, "live_parcels_at_end": live,
            "deposit": "fixed-point sums per cell (fast precision; scale from the ring's largest mass and speed)",
            "share": {k: round(v[0] / total, 4) for k, v in prof.items() if v[1]}}


def exit_column(state, s):
    """The exit-plane column (iExit) of a full state, as exit_performance reads it."""
    A = np.asarray(state["A"]).reshape(s.Nr, s.Nx, 4)[:, s.iExit].ravel()
    B = np.asarray(state["B"]).reshape(s.Nr, s.Nx, 4)[:, s.iExit].ravel()
    return {"A": A, "B": B}


def run_fp64_check(args):
    """Thrust and exhaust mass flow of the CUDA path (FP32, default precision)
    against an FP64 run of the same scheme (the oracle in double precision),
    after the same number of steps: the plain cold-gas cone 256x96 at its full 2000 steps and the
    viscous plume over a bounded 1000-step sample (its 10k steps take minutes
    in FP64 on the host)."""
    rn = ge.load_package()
    oracle = ge.load_oracle()
    oracle.set_threads(os.cpu_count() or 1)
    from rocket_nozzle_cfd_solver_b200 import configs
    out = {}
    for name, cfg, n in (("plain cold-gas cone 256x96, 2000 steps", configs.plain_small()[0], 2000),
                         ("viscous plume 512x192", configs.viscous_plume()[0], 1000)):
        s = rn.build_sim_setup(cfg)
        g = rn.GPUSolver(s.Nx, s.Nr)
        g.setGeometry(s.geo)
        init = s.initialState()
        g.setState(init["A"], init["B"])
        g.step(n, s.P)
        gp = rn.exit_performance(s, exit_column(g.readAll(), s))
        g.close()
        o = oracle.OracleSolver(s.Nx, s.Nr, fp64=True)
        o.setGeometry(s.geo)
        o.setState(init["A"], init["B"])
        o.step(n, s.P)
        op = rn.exit_performance(s, exit_column(o.readAll(), s))
        o.close()
        out[name] = {"steps": n, "thrust_N": gp["F"], "mdot_kg_s": gp["mdot"],
                     "thrust_rel_err": abs(gp["F"] - op["F"]) / max(abs(op["F"]), 1e-30),
                     "mdot_rel_err": abs(gp["mdot"] - op["mdot"]) / max(abs(op["mdot"]), 1e-30)}
    return out


def serving_requests(rn, count, seed=7, spray_frac=0.2):
    """Seeded serving workload: nozzles drawn as in the batched workload; a
    fraction are injector chambers with the spray whose parcel ring starts with
    U{16,384 .. 65,536} seeded parcels (configs.prepopulated_parcels) and keeps
    spawning from the injector, 4 parcels per step, as the reference does.
    Entries: (kind, setup, parcels or None)."""
    from rocket_nozzle_cfd_solver_b200 import configs
    rng = np.random.default_rng(seed)
    out = []
    for q in range(count):
        if rng.uniform() < spray_frac:
            Nx, Nr = configs.BATCH_SIZES[int(rng.integers(len(configs.BATCH_SIZES)))]
            s = rn.build_sim_setup(configs.injector_spray(Nx, Nr)[0])
            # the parcel count has its own stream, so the request mix is that of rng alone
            npar = int(np.random.default_rng(seed * 1000 + q).integers(16384, 65537))
            out.append(("spray", s, configs.prepopulated_parcels(s, npar, seed=20261203 + q)))
        else:
            out.append(("nozzle", rn.build_sim_setup(configs.batched_instance(rng)), None))
    return out


def serve_once(rn, reqs, arrivals, max_active, check_every, drop, t_end_s, max_cells=0):
    """Submits reqs at their arrival times (s) to a SolveServer; returns the results."""
    srv = rn.SolveServer(max_active=max_active, check_every=check_every, max_active_cells=max_cells)
    ids = []
    t0 = time.perf_counter()
    for (kind, s, parcels), ta in zip(reqs, arrivals):
        delay = ta - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        ids.append(srv.submit(s, drop=drop, t_end_s=t_end_s, parcels=parcels))
    res = [srv.wait(i, timeout_s=1800) for i in ids]
    st = srv.stats()
    srv.close()
    return res, st


def latency_summary(res):
    lat = np.array([r["latency_ms"] for r in res])
    span = max(r["done_ms"] for r in res) - min(r["submit_ms"] for r in res)
    return {"solves_per_s": len(res) / (span * 1e-3), "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "makespan_s": span * 1e-3}


def run_serving(args):
    """Serving: Poisson arrivals of whole solves (stop at a density-residual
    drop of 1e-4 or 2 ms of simulated time) into the continuous-batching
    SolveServer, against the same arrivals served one solve at a time
    (max_active=1, the plain form), at every rate of --serve-rates (the
    configuration's 1-50 req/s). The same seeded request mix at every rate."""
    rn = ge.load_package()
    t0 = time.perf_counter()
    reqs = serving_requests(rn, args.serve_requests)
    t_setup = time.perf_counter() - t0
    K, drop, t_end = 60, 1e-4, 2e-3
    sweep = []
    for rate in (float(r) for r in args.serve_rates.split(",")):
        rng = np.random.default_rng(11)
        arrivals = np.cumsum(rng.exponential(1.0 / rate, size=len(reqs)))
        arrivals -= arrivals[0]
        served, st = serve_once(rn, reqs, arrivals, 0, K, drop, t_end, args.serve_max_cells)
        plain, _ = serve_once(rn, reqs, arrivals, 1, K, drop, t_end)
        same = all(a["integrals"] == b["integrals"] and a["steps"] == b["steps"] for a, b in zip(served, plain))
        status = {}
        for r in served:
            status[r["status"]] = status.get(r["status"], 0) + 1
        cells = sum(s.Nx * s.Nr * r["steps"] for (_, s, _), r in zip(reqs, served))
        sv, pl = latency_summary(served), latency_summary(plain)
        sweep.append({"rate_per_s": rate, "solves_per_s": sv["solves_per_s"], "p50_ms": sv["p50_ms"],
                      "p99_ms": sv["p99_ms"], "makespan_s": sv["makespan_s"],
                      "cell_updates_per_s": cells / sv["makespan_s"], "status": status, "ticks": st["ticks"],
                      "one_at_a_time": pl, "speedup_solves_per_s": sv["solves_per_s"] / pl["solves_per_s"],
                      "results_identical_in_mix_and_alone": same})
    top = max(sweep, key=lambda e: e["rate_per_s"])
    return {"metric": "solves/s", "value": top["solves_per_s"], "unit": "solves/s", "rate_per_s": top["rate_per_s"],
            "requests": len(reqs), "spray_requests": sum(1 for k, _, _ in reqs if k == "spray"),
            "spray_parcels": [int((np.asarray(pc[1]).reshape(-1, 4)[:, 1] > 0).sum()) for k, _, pc in reqs if pc],
            "grids": [f"{s.Nx}x{s.Nr}" for _, s, _ in reqs],
            "stop": "density residual drop 1e-4 or 2 ms simulated", "check_every": K,
            "max_active_cells": args.serve_max_cells, "sweep": sweep, "setup_s": t_setup}


def main():
    global GRID, SOLVER_STEPS, WORKLOAD
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline sample")
    ap.add_argument("--batch-instances", type=int, default=64,
                    help="instances of the batched workload measured after the main line's (0: skip)")
    ap.add_argument("--batch-steps", type=int, default=30, help="time steps per batched bench step")
    ap.add_argument("--grid", default="512x192",
                    help="grid of the main viscous-plume leg (other sizes are for profiling; the bench line's "
                         "workload is 512x192)")
    ap.add_argument("--solver-steps", type=int, default=SOLVER_STEPS, help="time steps per bench step")
    ap.add_argument("--tile", default=None, help="tile shape of the main leg (default: the library's)")
    ap.add_argument("--no-large", action="store_true",
                    help="skip the 4096x1536 HBM-resident sweep point and the spray chamber leg")
    ap.add_argument("--only-spray", action="store_true",
                    help="run only the spray chamber leg and print its JSON object (for profiling)")
    ap.add_argument("--serve-requests", type=int, default=12,
                    help="requests of the serving leg at each arrival rate (0: skip)")
    ap.add_argument("--serve-rates", default="1,2,5,10,20,50",
                    help="Poisson arrival rates of the serving leg (1/s), comma-separated")
    ap.add_argument("--serve-max-cells", type=int, default=2000000,
                    help="admission cap on the grid cells the server steps at once (0: memory budget only)")
    ap.add_argument("--no-classes", action="store_true",
                    help="skip the batched leg's solves-per-grid-class comparison (for profiling)")
    args = ap.parse_args()
    GRID = tuple(int(v) for v in args.grid.lower().split("x"))
    SOLVER_STEPS = args.solver_steps
    if GRID != (512, 192):
        WORKLOAD = WORKLOAD.replace("512x192", f"{GRID[0]}x{GRID[1]}")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.only_spray:
        import torch
        torch.cuda.set_device(local_rank)
        print(json.dumps(run_spray(args, local_rank)), flush=True)
        return
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
