#!/usr/bin/env python
"""Benchmark of the SPH fluid step: particle-steps/s of the DFSPH dam break
with 1,048,576 particles (128 x 64 x 128 lattice at r = 0.005 m in a
2 x 1 x 2 m box container) and 4 two-way coupled rigid bodies (2 spheres of
radius 0.05 m, 2 boxes of side 0.08 m, seeded, 64^3 cubic-Lagrange distance
grids and volume maps), at 0.1 % density / divergence tolerance.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

One step = one SolverDf step (solver_df.hpp:74-359) over the whole scene.
Multi-GPU runs are independent replicas of the scene (weak scaling): the
step has no data-path exchange.  Rank 0 prints one JSON line.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s at 0.1% avg density error"
UNIT = "particle-steps/s"
WORKLOAD = ("DFSPH dam break, 1,048,576 particles (128x64x128 lattice, r=0.005 m) in a "
            "2x1x2 m box, 4 rigid bodies (2 spheres r=0.05, 2 boxes 0.08 m) with 64^3 "
            "cubic-Lagrange SDF + volume maps, two-way coupled")
LATTICE = (128, 64, 128)
RADIUS = 0.005
CONTAINER = (2.0, 1.0, 2.0)
SEED = 0

# Compulsory per-particle state traffic per pass, float32 ("Model A": every
# per-particle array read/written once per pass, neighbor gathers served
# on chip, the stored neighbor list counted only in the pass that writes
# it).  (bytes per particle, bytes per active boundary pair)
MODEL_A = {
    "sort": (104, 0),            # hash + counting sort + reorder (x, v, kappa, kappa_v)
    "boundary": (0, 48),         # boundary sample
    "neighbors": (148 + 24, 16),  # neighbor build (4 B indices, K ~ 32) + density + factor
    "div_warm": (100, 32),       # divergence warm start + rho_dot
    "div_iteration": (68, 32),   # divergence iteration (fused residual)
    "viscosity": (68, 32),
    "cfl_integrate": (80, 0),    # CFL + v += a dt
    "press_warm": (110, 32),     # pressure warm start + rho_adv
    "press_iteration": (72, 32),  # pressure iteration (fused residual)
    "finish": (48, 0),           # integrate x
}
# engine launch groups -> Model A pass
GROUP_PASS = {
    "grid_sort": "sort", "gather_state": "sort", "boundary": "boundary",
    "neighbors": "neighbors", "div_warm0": "div_warm", "div_warm1": "div_warm",
    "div_rho_adv": "div_warm", "div_iter": "div_iteration", "div_residual": "div_iteration",
    "viscosity": "viscosity", "integrate_np": "cfl_integrate", "press_warm0": "press_warm",
    "press_warm1": "press_warm", "press_rho_adv": "press_warm", "press_iter": "press_iteration",
    "press_residual": "press_iteration", "finish": "finish",
}
# how many times a pass runs per step: iteration passes once per iteration
PASS_PER_STEP = {"div_iteration": "div", "press_iteration": "den"}


def parse_args():
    p = argparse.ArgumentParser(description=__doc__,
                                formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["engine", "reference"], default="engine")
    p.add_argument("--cpu-seconds", type=float, default=20.0,
                   help="budget of the CPU-baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--rigid-bodies", type=int, default=4, choices=[0, 4],
                   help="0 drops the 4 rigid bodies (profiling case)")
    p.add_argument("--container-resolution", type=int, default=64,
                   help="volume-map resolution of the container")
    p.add_argument("--eager", action="store_true",
                   help="launch every kernel from the host (no captured step graph)")
    return p.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.QUERY,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
            return
        # wait (bounded) until nvidia-smi has written its first sample
        for _ in range(100):
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.05)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        smax = [num(r[2]) for r in rows if num(r[2]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4)
                          if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(rows)}


def build_scene(engine, dtype=np.float32, rigid_bodies=4, container_resolution=64):
    from alluvion_b200 import scenes
    bodies = []
    if rigid_bodies:
        bodies = scenes.seeded_rigid_bodies(SEED, CONTAINER, RADIUS, resolution=64)
    return scenes.dam_break(engine, dtype, LATTICE, RADIUS, CONTAINER, bodies, seed=SEED,
                            volume_resolution=container_resolution)


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def committed_traffic():
    """DRAM bytes per particle of the dominant pass from the committed ncu
    summary (profiles/traffic.json), or None."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return None


def timed_steps(scene, sp, dt, steps, torch, on_step=None):
    """Runs `steps` steps between CUDA events on the launching (default)
    stream, synchronised on both sides.  Returns (ms, dt, reports)."""
    reps = []
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(steps):
        if on_step:
            on_step("before")
        dt, rep = scene.step("df", sp, dt)
        if on_step:
            on_step("after")
        reps.append((rep.num_divergence_solve, rep.num_density_solve,
                     rep.mean_density_error, rep.num_active_boundary_pairs))
    stop.record()
    torch.cuda.synchronize()
    return start.elapsed_time(stop), dt, reps


def max_over_ranks(value, world, torch):
    if world == 1:
        return value
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_baseline(scene, sp, dt, budget_s, host_state, host_bodies):
    """The oracle's DFSPH step on the host cores on a bounded sample of the
    same scene (same initial state and grids)."""
    from oracle import binding as orc
    hb, keep, rigid = host_bodies
    nb = scene.num_boundaries
    bodies = (type(hb[0]) * nb)(*[hb[b] for b in range(nb)])
    state = {k: np.ascontiguousarray(host_state[k]).copy()
             for k in ("x", "v", "kappa", "kappa_v", "density", "density_adv", "a")}
    rig = rigid.copy()
    steps = 0
    t0 = time.perf_counter()
    while True:
        dt, _ = orc.run("df", scene.cn, scene.cni, bodies, rig, state, sp, dt, 1)
        steps += 1
        el = time.perf_counter() - t0
        # stop at the budget, or before a step that would overrun it by half
        if el > budget_s or steps >= 100 or el * (steps + 1) / steps > 1.5 * budget_s:
            break
    return {"value": scene.n * steps / el, "unit": UNIT, "cores": orc.num_threads(),
            "kind": "port",
            "sample": "%d step(s) of the 1,048,576-particle scene from the same initial state "
                      "(grids built by the engine, untimed), %.1f s" % (steps, el)}


def engine_arm(args):
    import torch
    from alluvion_b200 import _capi, scenes
    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    engine = _capi.Engine(local)
    engine.set_graph_mode(not args.eager)
    scene = build_scene(engine, rigid_bodies=args.rigid_bodies,
                        container_resolution=args.container_resolution)
    sp = scenes.solver_params()
    dt = float(sp.max_dt)
    host_state = scene.state() if rank == 0 and world == 1 else None
    host_bodies = scene.host_bodies() if host_state is not None else None
    # warm-up
    for _ in range(args.warmup):
        dt, _ = scene.step("df", sp, dt)
    # ---- device-resident timed region (value)
    barrier(world)
    clocks = ClockSampler(local)
    clocks.start()
    launches0 = engine.launch_count()
    graphs0 = engine.graph_stats()
    ms, dt, reps = timed_steps(scene, sp, dt, args.steps, torch)
    launches = engine.launch_count() - launches0
    graphs1 = engine.graph_stats()
    clk = clocks.stop()
    barrier(world)
    ms = max_over_ranks(ms, world, torch)
    total_particles = scene.n * world
    value = total_particles * args.steps / (ms / 1e3)
    # ---- end to end: host buffers in pinned memory, H2D + step + D2H per step
    n = scene.n
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    hx, hv = pin(scene.x.cpu().numpy()), pin(scene.v.cpu().numpy())
    hk, hkv = pin(scene.kappa.cpu().numpy()), pin(scene.kappa_v.cpu().numpy())
    h2d = (hx.numel() + hv.numel() + hk.numel() + hkv.numel()) * 4
    d2h = (hx.numel() + hv.numel()) * 4

    def io(phase):
        if phase == "before":
            scene.x.copy_(hx, non_blocking=True)
            scene.v.copy_(hv, non_blocking=True)
            scene.kappa.copy_(hk, non_blocking=True)
            scene.kappa_v.copy_(hkv, non_blocking=True)
        else:
            hx.copy_(scene.x, non_blocking=True)
            hv.copy_(scene.v, non_blocking=True)
    barrier(world)
    ms_e2e, dt, _ = timed_steps(scene, sp, dt, args.steps, torch, on_step=io)
    barrier(world)
    ms_e2e = max_over_ranks(ms_e2e, world, torch)
    e2e = total_particles * args.steps / (ms_e2e / 1e3)
    # ---- per-pass device times (profiling pass after the timed region)
    engine.reset_stats()
    engine.set_profiling(True)
    prof_steps = 3
    _, dt, preps = timed_steps(scene, sp, dt, prof_steps, torch)
    engine.set_profiling(False)
    stats = engine.kernel_stats()
    iters_div = sum(r[0] for r in preps) / prof_steps
    iters_den = sum(r[1] for r in preps) / prof_steps
    pairs = sum(r[3] for r in preps) / prof_steps
    pass_ms = {}
    for name, (tot, cnt) in stats.items():
        p = GROUP_PASS.get(name)
        if p:
            pass_ms[p] = pass_ms.get(p, 0.0) + tot / prof_steps
    per_launch = {}
    for p, t in pass_ms.items():
        runs = {"div": iters_div, "den": iters_den}.get(PASS_PER_STEP.get(p), 1.0)
        if runs > 0:
            per_launch[p] = t / runs
    dominant = max(pass_ms, key=pass_ms.get)
    peak, peak_kind = measured_peaks()
    bpp, bpair = MODEL_A[dominant]
    alg_bytes = bpp * n + bpair * pairs
    achieved = alg_bytes / (per_launch[dominant] / 1e3) / 1e9
    traffic = committed_traffic()
    tr = None
    if traffic and traffic.get("pass") == dominant:
        tr = traffic.get("dram_bytes_per_particle", 0) * n
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": tr,
                "kernel": dominant, "peak_kind": peak_kind,
                "algorithmic_bytes_per_launch": int(alg_bytes),
                "launch_ms": round(per_launch[dominant], 4)}
    steps_reps = reps
    workload = WORKLOAD
    if args.rigid_bodies == 0 or args.container_resolution != 64:
        workload += " [variant: %d rigid bodies, %d^3 container map]" % (
            args.rigid_bodies, args.container_resolution)
    result = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded jittered lattice, seeded rigid bodies)",
        "config": {"workload": workload, "particles_per_gpu": n, "global_particles":
                   total_particles, "parallelism": "replicas" if world > 1 else "single",
                   "l2": "working set > 126 MB L2 (inputs larger than L2, no flush)",
                   "mean_divergence_iterations": round(sum(r[0] for r in steps_reps) /
                                                       len(steps_reps), 3),
                   "mean_density_iterations": round(sum(r[1] for r in steps_reps) /
                                                    len(steps_reps), 3),
                   "active_boundary_pairs": int(pairs),
                   "launch": "eager" if args.eager else "step graph (conditional WHILE loops)",
                   "graph_replays_timed": graphs1[1] - graphs0[1],
                   "pass_ms_per_step": {k: round(v, 4) for k, v in pass_ms.items()}},
        "e2e": {"value": round(e2e, 1), "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": int(launches),
        "roofline": roofline,
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        result["cpu_baseline"] = cpu_baseline(scene, sp, float(sp.max_dt), args.cpu_seconds,
                                              host_state, host_bodies)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result), flush=True)


def reference_arm(args):
    """The reference's CPU formulation of the path (the oracle port: the
    reference itself needs Eigen/GLFW/glm and does not build here), timed on
    all host cores.  Rank 0 only."""
    world, rank, local = dist_env()
    if rank != 0:
        return
    import torch
    from alluvion_b200 import _capi, scenes
    from oracle import binding as orc
    torch.cuda.set_device(local)
    engine = _capi.Engine(local)
    scene = build_scene(engine)  # setup only: grids built on the device, untimed
    hb, keep, rigid = scene.host_bodies()
    nb = scene.num_boundaries
    bodies = (type(hb[0]) * nb)(*[hb[b] for b in range(nb)])
    st = scene.state()
    state = {k: np.ascontiguousarray(st[k]).copy()
             for k in ("x", "v", "kappa", "kappa_v", "density", "density_adv", "a")}
    sp = scenes.solver_params()
    dt = float(sp.max_dt)
    # each benchmark step is one full oracle step; warm-up steps are shortened
    # to one so the run stays within minutes
    for _ in range(min(args.warmup, 1)):
        dt, _ = orc.run("df", scene.cn, scene.cni, bodies, rigid, state, sp, dt, 1)
    steps = max(1, min(args.steps, 5))
    t0 = time.perf_counter()
    dt, _ = orc.run("df", scene.cn, scene.cni, bodies, rigid, state, sp, dt, steps)
    el = time.perf_counter() - t0
    value = scene.n * steps / el
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 1), "unit": UNIT,
        "n_gpus": world, "steps": steps, "warmup": min(args.warmup, 1),
        "ms_per_step": round(el * 1e3 / steps, 2), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded jittered lattice, seeded rigid bodies)",
        "config": {"workload": WORKLOAD, "particles_per_gpu": scene.n},
        "cpu_baseline": {"value": round(value, 1), "unit": UNIT, "cores": orc.num_threads(),
                         "kind": "port",
                         "sample": "%d full steps of the 1,048,576-particle scene" % steps},
        "e2e": {"value": round(value, 1), "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    args = parse_args()
    if args.impl == "reference":
        reference_arm(args)
    else:
        engine_arm(args)


if __name__ == "__main__":
    main()
