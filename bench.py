#!/usr/bin/env python
"""Benchmark of the SPH fluid step: particle-steps/s of the DFSPH dam break
with 1,048,576 particles (128 x 64 x 128 lattice at r = 0.005 m in a
2 x 1 x 2 m box container) and 4 two-way coupled rigid bodies (2 spheres of
radius 0.05 m, 2 boxes of side 0.08 m, seeded, 64^3 cubic-Lagrange distance
grids and volume maps), at 0.1 % density / divergence tolerance.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]
                  [--workload dambreak-1m|dambreak-32k|dambreak-8m] [--method df|ii|i]

One step = one SolverDf step (solver_df.hpp:74-359), one SolverIi step
(solver_ii.hpp:76-243) with --method ii, or one SolverI step (implicit SPH,
solver_i.hpp:79-327) with --method i, over the whole scene.  The default
workload is the 1M-particle scene; dambreak-32k (32^3 lattice, r = 0.01 m,
no rigid bodies) and dambreak-8m (256 x 128 x 256 lattice, r = 0.0025 m,
sphere + box + torus with 128^3 grids) are the small and large variants.
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
SEED = 0
# Seeded synthetic dam breaks (a jittered lattice block in a box container
# with two-way coupled rigid bodies above it); no dataset is involved.
WORKLOADS = {
    "dambreak-1m": dict(
        lattice=(128, 64, 128), radius=0.005, container=(2.0, 1.0, 2.0), bodies="2s2b",
        grid_resolution=64, container_resolution=64,
        desc="dam break, 1,048,576 particles (128x64x128 lattice, r=0.005 m) in a 2x1x2 m box, "
             "4 rigid bodies (2 spheres r=0.05, 2 boxes 0.08 m) with 64^3 cubic-Lagrange SDF + "
             "volume maps, two-way coupled"),
    "dambreak-32k": dict(
        lattice=(32, 32, 32), radius=0.01, container=(1.0, 0.7, 0.7), bodies="none",
        grid_resolution=64, container_resolution=64,
        desc="dam break, 32,768 particles (32^3 lattice, r=0.01 m) in a 1.0x0.7x0.7 m box with "
             "a 64^3 volume map"),
    "dambreak-8m": dict(
        lattice=(256, 128, 256), radius=0.0025, container=(2.0, 1.0, 2.0), bodies="sbt",
        grid_resolution=128, container_resolution=128,
        desc="dam break, 8,388,608 particles (256x128x256 lattice, r=0.0025 m) in a 2x1x2 m "
             "tank, sphere r=0.1 + box 0.16 m + torus R=0.1 r=0.04 with 128^3 cubic-Lagrange "
             "SDF + volume maps, two-way coupled"),
}
BATCH_WORKLOADS = {
    "batch64": dict(
        scenes=64, radius=0.01,
        desc="batched dam breaks: 64 scenes, particle counts log-uniform in [8,192, 262,144] "
             "(cubic lattices, r=0.01 m, seeded), boxes scaled with the count from 1.0x0.7x0.7 m, "
             "0-2 seeded rigid spheres per scene, 32^3 volume maps, one graph launch per step"),
}
# Post-processing variants (the reference's statistics kernels): their own
# metric, not the headline.
POSTPROC_WORKLOADS = {
    "histogram-256m": dict(
        n=1 << 28, metric="values/s (histogram256 with mask)", unit="values/s",
        desc="histogram256 with mask of 268,435,456 seeded uniform float32 values (1 GiB, and "
             "a 1 GiB mask, both larger than L2) in 256 bins"),
    "sampling-1m": dict(
        n=1 << 20, metric="samples/s (density, velocity, vorticity)", unit="samples/s",
        desc="density, velocity and vorticity at 1,048,576 seeded samples in a jittered "
             "1,000,000-particle lattice (r = 0.01 m, 100^3), no bodies"),
}
METHOD_NAME = {"df": "DFSPH", "ii": "IISPH", "i": "implicit SPH (SolverI)"}
# the large coupled scene: 8,388,608 particles, three bodies on 128^3 grids
DEFAULT_WORKLOAD = "dambreak-8m"

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
    # IISPH, the same accounting: predict_advection0 reads x, rho, a, v, p and
    # writes v, p_last, d_ii (92 B + 16 B per pair); predict_advection1 reads
    # x, v, d_ii, rho and writes rho_adv, a_ii (60 B + 32 B per pair); one
    # Jacobi iteration (both kernels fused) ~110 B; pressure accelerations +
    # integration read x, rho, p, v, a and write x, v (80 B + 32 B per pair)
    "ii_predict": (152, 48),
    "ii_iteration": (110, 16),
    "ii_finish": (80, 32),
    # implicit SPH (SolverI): advect_and_init_pressure reads v, a, p and
    # writes v, p_last (56 B); the diagonal pass reads x, v, rho and writes
    # diag, rho_adv (48 B + 32 B per pair); one Jacobi iteration reads x,
    # rho, p_last, diag, rho_adv and writes p, err (56 B); the final copy of
    # an even iteration count moves p (8 B)
    "i_advect": (56, 0),
    "i_diag": (48, 32),
    "i_iteration": (56, 0),
    "i_final": (8, 0),
}
# engine launch groups -> Model A pass
GROUP_PASS = {
    "grid_sort": "sort", "gather_state": "sort", "boundary": "boundary",
    "neighbors": "neighbors", "div_warm0": "div_warm", "div_warm1": "div_warm",
    "div_rho_adv": "div_warm", "div_iter": "div_iteration", "div_residual": "div_iteration",
    "viscosity": "viscosity", "integrate_np": "cfl_integrate", "press_warm0": "press_warm",
    "press_warm1": "press_warm", "press_rho_adv": "press_warm", "press_iter": "press_iteration",
    "press_residual": "press_iteration", "finish": "finish",
    "ii_predict0": "ii_predict", "ii_predict1": "ii_predict", "ii_iter0": "ii_iteration",
    "ii_iter1": "ii_iteration", "i_advect": "i_advect", "i_diag": "i_diag",
    "i_iter": "i_iteration", "i_final": "i_final",
}
# the write-back group of the pressure methods is their acceleration pass
FINISH_PASS = {"df": "finish", "ii": "ii_finish", "i": "ii_finish"}
# how many times a pass runs per step: iteration passes once per iteration
PASS_PER_STEP = {"div_iteration": "div", "press_iteration": "den", "ii_iteration": "den",
                 "i_iteration": "den"}


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
    p.add_argument("--rigid-bodies", type=int, default=None, choices=[0],
                   help="0 drops the workload's rigid bodies (profiling case)")
    p.add_argument("--container-resolution", type=int, default=None,
                   help="volume-map resolution of the container (default: the workload's)")
    p.add_argument("--eager", action="store_true",
                   help="launch every kernel from the host (no captured step graph)")
    p.add_argument("--workload", choices=sorted(WORKLOADS) + sorted(BATCH_WORKLOADS) +
                   sorted(POSTPROC_WORKLOADS), default=DEFAULT_WORKLOAD)
    p.add_argument("--method", choices=["df", "ii", "i"], default="df")
    p.add_argument("--warm-start", choices=["auto", "plain", "learned", "both"], default="auto",
                   help="learned: DFSPH with the learned warm start; both: plain and learned "
                        "arms from the same initial state, the learned one reported as the "
                        "value; auto: both on the default workload's DFSPH, else plain")
    p.add_argument("--warm-net", default=None,
                   help="network file (default: the committed alluvion_b200/data/"
                        "warm_start_dambreak.npz); 'train': fit one now (untimed)")
    p.add_argument("--fp64-steps", type=int, default=None,
                   help="steps of the float32-vs-float64 error statement (default 20 on the "
                        "default workload, else 0)")
    p.add_argument("--autotune", choices=["auto", "on", "off"], default="auto",
                   help="sweep the pass groups' launch shapes before timing (untimed; "
                        "alluvion_b200.autotune); auto: on for single scenes (the sweep keeps "
                        "the defaults when its table is slower in the step graph) and for "
                        "batched workloads run as branches")
    p.add_argument("--batch-form", choices=["fused", "branches"], default="fused",
                   help="batched workloads: fused (one launch per solver pass over all "
                        "scenes) or one graph branch per scene; the line also times the "
                        "other form for comparison")
    p.add_argument("--max-dt", type=float, default=None,
                   help="time-step cap (default 2e-4 s)")
    a = p.parse_args()
    if a.fp64_steps is None:
        a.fp64_steps = 20 if a.workload == DEFAULT_WORKLOAD and a.impl == "engine" else 0
    return a


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


def workload_bodies(wl):
    """Rigid bodies of a workload (seeded positions above the fluid block)."""
    from alluvion_b200 import _capi, scenes
    if wl["bodies"] == "2s2b":
        return scenes.seeded_rigid_bodies(SEED, wl["container"], wl["radius"],
                                          resolution=wl["grid_resolution"])
    if wl["bodies"] == "sbt":
        rng = np.random.Generator(np.random.PCG64(SEED + 2000))
        size = np.asarray(wl["container"], dtype=np.float64)
        res = wl["grid_resolution"]
        out = []
        for k in range(3):
            rho = rng.uniform(500.0, 2000.0)
            pos = (rng.uniform(0.25, 0.75) * size[0], rng.uniform(0.75, 0.85) * size[1],
                   rng.uniform(0.25, 0.75) * size[2])
            if k == 0:
                r = 0.1
                mass = rho * 4.0 / 3.0 * np.pi * r ** 3
                out.append(dict(shape=_capi.SHAPE_SPHERE, params=[r], sign=1.0, resolution=res,
                                use_distance_grid=True, mass=mass,
                                inertia=scenes.sphere_inertia(mass, r), x=pos))
            elif k == 1:
                w = (0.16,) * 3
                mass = rho * 0.16 ** 3
                out.append(dict(shape=_capi.SHAPE_BOX, params=scenes.box_params(w), sign=1.0,
                                resolution=res, use_distance_grid=True, mass=mass,
                                inertia=scenes.box_inertia(mass, w), x=pos))
            else:
                R, r = 0.1, 0.04
                mass = rho * 2.0 * np.pi ** 2 * R * r * r
                iy = mass * (R * R + 0.75 * r * r)
                ixz = mass * (0.5 * R * R + 0.625 * r * r)
                out.append(dict(shape=_capi.SHAPE_TORUS, params=[R, r], sign=1.0,
                                resolution=res, use_distance_grid=True, mass=mass,
                                inertia=(ixz, iy, ixz), x=pos))
        return out
    return []


def build_scene_spec(workload="dambreak-1m", dtype=np.float32, rigid_bodies=None,
                     container_resolution=None, seed=SEED):
    """Host description of a workload's seeded scene (no engine involved)."""
    from alluvion_b200 import scenes
    wl = WORKLOADS[workload]
    bodies = [] if rigid_bodies == 0 else workload_bodies(wl)
    res = container_resolution or wl["container_resolution"]
    return scenes.dam_break_spec(dtype, wl["lattice"], wl["radius"], wl["container"], bodies,
                                 seed=seed, volume_resolution=res)


def build_scene(engine, workload="dambreak-1m", dtype=np.float32, rigid_bodies=None,
                container_resolution=None, seed=SEED):
    return build_scene_spec(workload, dtype, rigid_bodies, container_resolution,
                            seed).device(engine)


def oracle_scene(spec, dilate=2):
    """The scene's grids built by the oracle on the host cores, for the CPU
    arms that must not load the engine: distance nodes sampled from the
    analytic shapes, volume maps filled lazily (same node values as the
    eager build), with every node the particles can reach within `dilate`
    cells computed up front.  Returns (bodies, keep-alive arrays, rigid,
    seconds)."""
    from oracle import binding as orc
    t0 = time.perf_counter()
    bodies, rigid = spec.bodies()
    keep = []
    for b in range(spec.num_boundaries):
        body = bodies[b]
        assert "mesh" not in spec.body_specs[b], "oracle_scene: analytic shapes only"
        if body.use_distance_grid:
            dist = orc.distance_grid(body, spec.dtype)
            keep.append(dist)
            body.distance_nodes = dist.ctypes.data
        vol = orc.lazy_volume_field(spec.cn, body, spec.dtype)
        keep.append(vol)
        body.volume_nodes = vol.ctypes.data
        orc.lazy_volume_touch(body, rigid[b], spec.x, dilate)
    return bodies, keep, rigid, time.perf_counter() - t0


def lazy_nodes_computed(keep):
    """Volume-map nodes computed so far by the oracle's lazy maps."""
    from oracle import binding as orc
    return sum(sum(orc.lazy_volume_counts(a)) for a in keep)


def release_oracle_scene(spec, keep):
    from oracle import binding as orc
    for a in keep:
        orc.lazy_volume_release(a)


TRAIN_STEPS, TRAIN_PER_STEP, FIT_STEPS = 300, 32768, 5000


def train_warm_start(engine, args, sp):
    """Untimed setup of --warm-start learned: plain steps of the workload at
    seed SEED + 1 provide (features, converged kappa) pairs; the network is
    fitted with the engine's own kernels."""
    from alluvion_b200 import warm_start
    sc = build_scene(engine, args.workload, rigid_bodies=args.rigid_bodies,
                     container_resolution=args.container_resolution, seed=SEED + 1)
    x, t = warm_start.collect(sc, sp, TRAIN_STEPS, TRAIN_PER_STEP, seed=SEED + 1)
    net, losses = warm_start.fit(engine, x, t, steps=FIT_STEPS, seed=SEED + 1)
    info = {"samples": int(x.shape[0]), "adam_steps": FIT_STEPS,
            "loss_first_last": [round(float(np.mean(losses[:50])), 4),
                                round(float(np.mean(losses[-50:])), 4)]}
    del sc, x, t
    return net, info


def workload_name(args, warm_mode="plain"):
    wl = WORKLOADS[args.workload]
    name = METHOD_NAME[args.method] + " " + wl["desc"]
    if args.rigid_bodies == 0 or args.container_resolution:
        name += " [variant: %s rigid bodies, %d^3 container map]" % (
            "no" if args.rigid_bodies == 0 else "with",
            args.container_resolution or wl["container_resolution"])
    if warm_mode == "learned":
        name += ", learned warm start"
    elif warm_mode == "both":
        name += ", learned warm start (plain DFSPH beside it)"
    if getattr(args, "max_dt", None):
        name += ", max_dt %g s" % args.max_dt
    return name


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def committed_traffic(workload, pass_name):
    """DRAM bytes per launch of `pass_name` on `workload` from the committed
    ncu captures (profiles/traffic.json), or None when that workload and
    pass were not captured."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        entry = json.load(f).get("workloads", {}).get(workload, {}).get(pass_name)
    return None if entry is None else float(entry["dram_bytes_per_launch"])


L2_BYTES = 126 * 2 ** 20
# device bytes a step touches per particle (records, positions, scalars,
# ~33-entry neighbor list, boundary state); below L2 the bench flushes
STEP_BYTES_PER_PARTICLE = 300


def timed_steps(scene, sp, dt, steps, torch, on_step=None, method="df", flush=None, warm=None):
    """Runs `steps` steps between CUDA events on the launching (default)
    stream, synchronised on both sides.  With `flush` (a device buffer
    larger than L2), every step is timed alone after the buffer is
    rewritten (untimed), so no step starts with the previous one's data in
    L2.  Returns (ms, dt, reports)."""
    reps = []
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    total = 0.0
    if flush is None:
        start.record()
    for _ in range(steps):
        if flush is not None:
            flush.add_(1)
            start.record()
        if on_step:
            on_step("before")
        dt, rep = scene.step(method, sp, dt, warm=warm)
        if on_step:
            on_step("after")
        if flush is not None:
            stop.record()
            torch.cuda.synchronize()
            total += start.elapsed_time(stop)
        reps.append((rep.num_divergence_solve, rep.num_density_solve,
                     rep.mean_density_error, rep.num_active_boundary_pairs,
                     rep.mean_density_change))
    if flush is None:
        stop.record()
        torch.cuda.synchronize()
        total = start.elapsed_time(stop)
    return total, dt, reps


def accuracy_summary(reps):
    """Iteration counts and achieved errors of a run's steps.  reps: tuples
    (divergence iterations, density iterations, mean density error, active
    boundary pairs, mean density change) per step.  The density error is
    the density solve's final mean (rho_adv - rho0) / rho0, held below the
    0.1 % tolerance; the density change is the divergence solve's final
    mean drho/dt / rho0 in 1/s, held below 0.1 % / dt."""
    a = np.asarray([r[:5] for r in reps], dtype=np.float64)
    return {"mean_divergence_iterations": round(float(a[:, 0].mean()), 3),
            "mean_density_iterations": round(float(a[:, 1].mean()), 3),
            "max_density_iterations": int(a[:, 1].max()),
            "density_error_mean": float("%.4g" % a[:, 2].mean()),
            "density_error_max": float("%.4g" % a[:, 2].max()),
            "density_change_mean_per_s": float("%.4g" % a[:, 4].mean()),
            "density_change_max_per_s": float("%.4g" % a[:, 4].max()),
            "density_error_tolerance": 1e-3}


def max_over_ranks(value, world, torch):
    """The largest of the ranks' values (device times: the job ends with its
    slowest rank).  The tensor lives where the process group's backend
    reduces: on the GPU for nccl, on the host for gloo."""
    if world == 1:
        return value
    import torch.distributed as dist
    device = "cpu" if dist.get_backend() == "gloo" else "cuda"
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(units_per_rank, world, steps, ms_max):
    """Whole-job units per second: every rank advances its own replica of
    units_per_rank for `steps` steps; the job takes the slowest rank's time."""
    return units_per_rank * world * steps / (ms_max / 1e3)


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# per-particle state a step reads and writes besides x and v
STATE = {"df": ("kappa", "kappa_v"), "ii": ("pressure",), "i": ("pressure",)}


def oracle_state(host_state, method):
    keys = ("x", "v", "density", "density_adv", "a") + STATE[method]
    return {k: np.ascontiguousarray(host_state[k]).copy() for k in keys}


def cpu_baseline(scene, sp, dt, budget_s, host_state, host_bodies, method="df"):
    """The oracle's step on the host cores on a bounded sample of the same
    scene (same initial state and grids)."""
    from oracle import binding as orc
    hb, keep, rigid = host_bodies
    nb = scene.num_boundaries
    bodies = (type(hb[0]) * nb)(*[hb[b] for b in range(nb)])
    state = oracle_state(host_state, method)
    rig = rigid.copy()
    steps = 0
    t0 = time.perf_counter()
    while True:
        dt, _ = orc.run(method, scene.cn, scene.cni, bodies, rig, state, sp, dt, 1)
        steps += 1
        el = time.perf_counter() - t0
        # stop at the budget, or before a step that would overrun it by half
        if el > budget_s or steps >= 100 or el * (steps + 1) / steps > 1.5 * budget_s:
            break
    return {"value": scene.n * steps / el, "unit": UNIT, "cores": orc.num_threads(),
            "kind": "port",
            "sample": "%d step(s) of the %s-particle scene from the same initial state "
                      "(grids built by the engine, untimed), %.1f s" % (steps, format(scene.n, ","),
                                                                      el)}


def batch_scene_list(engine, spec, seed=SEED):
    """The batch workload's scenes (seeded), on the device."""
    return [sp.device(engine) for sp in batch_scene_specs(spec, seed)]


def batch_scene_specs(spec, seed=SEED):
    """Host descriptions of the batch workload's scenes (seeded)."""
    from alluvion_b200 import _capi, scenes
    rng = np.random.Generator(np.random.PCG64(seed + 3000))
    r = spec["radius"]
    h = 4 * r
    out = []
    for _ in range(spec["scenes"]):
        target = np.exp(rng.uniform(np.log(8192), np.log(262144)))
        a = max(4, int(round(target ** (1.0 / 3.0))))
        s = (a ** 3 / 32768.0) ** (1.0 / 3.0)
        block = 2 * r * a
        box = np.array([max(1.0 * s, 1.6 * block + 2 * h), max(0.7 * s, block + 3 * h),
                        max(0.7 * s, block + 2 * h)])
        bodies = []
        for _ in range(int(rng.integers(0, 3))):
            rad = 0.05 * s
            y = block + h + rad + 0.5 * h
            if y + rad + h > box[1]:
                continue
            rho = rng.uniform(500.0, 2000.0)
            mass = rho * 4.0 / 3.0 * np.pi * rad ** 3
            pos = (rng.uniform(0.3, 0.7) * box[0], y, rng.uniform(0.3, 0.7) * box[2])
            bodies.append(dict(shape=_capi.SHAPE_SPHERE, params=[rad], sign=1.0, resolution=32,
                               use_distance_grid=True, mass=mass,
                               inertia=scenes.sphere_inertia(mass, rad), x=pos))
        seed_k = int(rng.integers(0, 2 ** 31))
        out.append(scenes.dam_break_spec(np.float32, (a, a, a), r, tuple(box), bodies,
                                         seed=seed_k, volume_resolution=32))
    return out


def pack_scenes(scene_list, keys, torch):
    """Rebinds each scene's per-particle arrays `keys` to views into one
    device tensor per key (the scenes' data copied in, every view starting on
    a 256-byte boundary), as a host that owns many scenes would lay them out:
    its host copies then move each array of the whole batch at once.
    Returns {key: tensor}."""
    out = {}
    for k in keys:
        parts = [getattr(sc, k) for sc in scene_list]
        offs, off = [], 0
        for p in parts:
            offs.append(off)
            off += (p.numel() + 63) // 64 * 64
        big = torch.zeros(off, dtype=parts[0].dtype, device=parts[0].device)
        for sc, p, o in zip(scene_list, parts, offs):
            view = big[o:o + p.numel()].view(p.shape)
            view.copy_(p)
            setattr(sc, k, view)
        out[k] = big
    return out


def batch_arm(args):
    """Config-3 style batch: every step advances all scenes with one
    al_df_batch_step_f32 call (one graph launch from the second step on),
    fused (one launch per solver pass over all scenes) or as one graph
    branch per scene (--batch-form)."""
    import torch
    from alluvion_b200 import _capi, scenes
    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    spec = BATCH_WORKLOADS[args.workload]
    engine = _capi.Engine(local)
    engine.set_graph_mode(not args.eager)
    sl = batch_scene_list(engine, spec)
    packed = pack_scenes(sl, ("x", "v", "kappa", "kappa_v"), torch)
    sp = scenes.solver_params()
    if args.max_dt:
        sp.max_dt = args.max_dt
    total_n = sum(sc.n for sc in sl)

    def tune():
        if args.autotune == "off":
            return None
        from alluvion_b200 import autotune
        t0 = time.perf_counter()
        tb = autotune.tune_batch(engine, sl, sp)
        tb["seconds"] = round(time.perf_counter() - t0, 1)
        return {k: tb[k] for k in ("batch_ms_default", "batch_ms_uniform", "uniform_shape",
                                   "batch_ms_tuned", "buckets", "seconds")}
    fused = args.batch_form == "fused"
    engine.set_batch_fused(fused)
    # the fused form's pair passes have one launch shape; the branches are tuned
    tuning = None if fused else tune()
    host_state = [sc.state() for sc in sl] if rank == 0 and world == 1 else None
    host_bodies = [sc.host_bodies() for sc in sl] if host_state is not None else None
    dts = [float(sp.max_dt)] * len(sl)
    for _ in range(args.warmup):
        dts, _, _ = scenes.batch_step(engine, sl, sp, dts)

    def run(steps, on_step=None):
        torch.cuda.synchronize()
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        nonlocal dts
        its = []
        start.record()
        for _ in range(steps):
            if on_step:
                on_step("before")
            dts, reps, _ = scenes.batch_step(engine, sl, sp, dts)
            if on_step:
                on_step("after")
            its.append([(r.num_divergence_solve, r.num_density_solve) for r in reps])
        stop.record()
        torch.cuda.synchronize()
        return start.elapsed_time(stop), np.asarray(its, dtype=np.float64)
    barrier(world)
    clocks = ClockSampler(local)
    clocks.start()
    launches0 = engine.launch_count()
    graphs0 = engine.graph_stats()
    ms, its = run(args.steps)
    launches = engine.launch_count() - launches0
    graphs1 = engine.graph_stats()
    clk = clocks.stop()
    barrier(world)
    ms = max_over_ranks(ms, world, torch)
    value = job_throughput(total_n, world, args.steps, ms)
    # host copies of all scenes' x, v, kappa, kappa_v (one pinned buffer per
    # array): uploaded before and x, v read back after every batched step
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    dev_in = [packed[k] for k in ("x", "v", "kappa", "kappa_v")]
    host_in = [pin(t.cpu().numpy()) for t in dev_in]
    dev_out = [packed["x"], packed["v"]]
    host_out = [pin(t.cpu().numpy()) for t in dev_out]
    h2d = sum(t.numel() * t.element_size() for t in host_in)
    d2h = sum(t.numel() * t.element_size() for t in host_out)

    def io(phase):
        if phase == "before":
            for d, hh in zip(dev_in, host_in):
                d.copy_(hh, non_blocking=True)
        else:
            for d, hh in zip(dev_out, host_out):
                hh.copy_(d, non_blocking=True)
    barrier(world)
    ms_e2e, _ = run(args.steps, io)
    ms_e2e = max_over_ranks(ms_e2e, world, torch)
    e2e = job_throughput(total_n, world, args.steps, ms_e2e)
    peak, peak_kind = measured_peaks()
    result = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded jittered lattices, seeded rigid spheres)",
        "config": {"workload": "DFSPH " + spec["desc"], "scenes": len(sl),
                   "particles_per_gpu": total_n, "global_particles": total_n * world,
                   "scene_particles_min_max": [min(sc.n for sc in sl), max(sc.n for sc in sl)],
                   "parallelism": "replicas" if world > 1 else "single",
                   "l2": "working set > 126 MB L2 (inputs larger than L2, no flush)",
                   "launch": ("eager" if args.eager else "batch graph") + (
                       ": fused, every pass one launch over all scenes (one counting sort "
                       "over all scenes' cells; pair passes one thread per particle in "
                       "128-thread blocks)" if fused else ": one branch per scene"),
                   "autotune": tuning,
                   "graph_replays_timed": graphs1[1] - graphs0[1],
                   "mean_divergence_iterations": round(float(its[:, :, 0].mean()), 3),
                   "mean_density_iterations": round(float(its[:, :, 1].mean()), 3)},
        "e2e": {"value": round(e2e, 1), "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": int(launches),
        "roofline": None,
        "clocks": clk,
    }
    # roofline of the dominant pass from the eager per-pass times (fused: each
    # pass one launch over all scenes; branches: the scenes in turn)
    engine.reset_stats()
    engine.set_profiling(True)
    run(2)
    engine.set_profiling(False)
    pass_ms = {}
    for name, (tot, cnt) in engine.kernel_stats().items():
        pp = GROUP_PASS.get(name)
        if pp:
            pass_ms[pp] = pass_ms.get(pp, 0.0) + tot / 2
    dominant = max(pass_ms, key=pass_ms.get)
    runs = {"div_iteration": float(its[:, :, 0].mean()),
            "press_iteration": float(its[:, :, 1].mean())}.get(dominant, 1.0)
    bpp, bpair = MODEL_A[dominant]
    alg = bpp * total_n
    per_launch = pass_ms[dominant] / max(runs, 1e-9)
    achieved = alg / (per_launch / 1e3) / 1e9
    result["config"]["pass_ms_per_step_sequential"] = {k: round(v, 4) for k, v in pass_ms.items()}
    # the other form on the same scenes, for comparison (untimed tuning first)
    other = "branches" if fused else "fused"
    engine.set_batch_fused(not fused)
    other_tuning = tune() if fused else None
    for _ in range(args.warmup):
        dts, _, _ = scenes.batch_step(engine, sl, sp, dts)
    barrier(world)
    ms_o, its_o = run(args.steps)
    ms_o = max_over_ranks(ms_o, world, torch)
    result["config"]["other_form"] = {
        "form": other, "ms_per_step": round(ms_o / args.steps, 4),
        "value": round(job_throughput(total_n, world, args.steps, ms_o), 1),
        "mean_density_iterations": round(float(its_o[:, :, 1].mean()), 3),
        "autotune": other_tuning}
    engine.set_batch_fused(fused)
    result["roofline"] = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                          "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": None,
                          "kernel": dominant, "peak_kind": peak_kind,
                          "algorithmic_bytes_per_launch": int(alg),
                          "launch_ms": round(per_launch, 4),
                          "note": "per-pass times from eager steps (%s)" % (
                              "each pass one launch over all scenes" if fused
                              else "scenes in turn")}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import binding as orc
        t0 = time.perf_counter()
        done = 0
        k = 0
        while time.perf_counter() - t0 < args.cpu_seconds and k < len(sl):
            sc = sl[k]
            hb, keep, rigid = host_bodies[k]
            nb = sc.num_boundaries
            bodies = (type(hb[0]) * nb)(*[hb[b] for b in range(nb)])
            state = oracle_state(host_state[k], "df")
            orc.run("df", sc.cn, sc.cni, bodies, rigid.copy(), state, sp, float(sp.max_dt), 1)
            done += sc.n
            k += 1
        el = time.perf_counter() - t0
        result["cpu_baseline"] = {"value": round(done / el, 1), "unit": UNIT,
                                  "cores": orc.num_threads(), "kind": "port",
                                  "sample": "one step of each of the first %d scenes, %.1f s"
                                            % (k, el)}
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result), flush=True)


def load_warm_net(engine, args, sp):
    """The committed network (alluvion_b200/data/warm_start_dambreak.npz,
    trained by alluvion_b200.train_warm_start on 200 seeded 1M-particle dam
    breaks), or one trained now on a differently seeded scene of the
    workload when --warm-net train."""
    from alluvion_b200 import warm_start
    if args.warm_net == "train":
        return train_warm_start(engine, args, sp)
    path = args.warm_net or os.path.join(ROOT, "alluvion_b200", "data",
                                         "warm_start_dambreak.npz")
    net = warm_start.WarmStartNet.load(path)
    info = {"network": os.path.relpath(path, ROOT)}
    ev = os.path.splitext(path)[0] + "_eval.json"
    if os.path.exists(ev):
        with open(ev) as f:
            info["trained"] = json.load(f).get("training")
    return net, info


def time_arm(engine, scene, sp, args, warm, world, local, torch, want_e2e, clocks_on):
    """Warm-up, the device-resident timed region, optionally the end-to-end
    region, and a profiling pass of one arm; returns a dict."""
    dt = float(sp.max_dt)
    for _ in range(args.warmup):
        dt, _ = scene.step(args.method, sp, dt, warm=warm)
    barrier(world)
    clocks = ClockSampler(local) if clocks_on else None
    if clocks:
        clocks.start()
    launches0 = engine.launch_count()
    graphs0 = engine.graph_stats()
    flush = None
    if scene.n * STEP_BYTES_PER_PARTICLE < L2_BYTES:
        flush = torch.zeros(2 * L2_BYTES // 4, dtype=torch.int32, device="cuda")
    ms, dt, reps = timed_steps(scene, sp, dt, args.steps, torch, method=args.method, flush=flush,
                               warm=warm)
    out = {"launches": engine.launch_count() - launches0,
           "graph_replays": engine.graph_stats()[1] - graphs0[1],
           "clocks": clocks.stop() if clocks else None, "flush": flush is not None}
    barrier(world)
    out["ms"] = max_over_ranks(ms, world, torch)
    out["value"] = job_throughput(scene.n, world, args.steps, out["ms"])
    out["reps"] = reps
    if want_e2e:
        # host copies of the step's inputs (x, v and the warm-start state) in
        # pinned memory: uploaded before and x, v read back after every step
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        dev_in = [scene.x, scene.v] + [getattr(scene, k) for k in STATE[args.method]]
        host_in = [pin(t.cpu().numpy()) for t in dev_in]
        out["h2d"] = sum(t.numel() * t.element_size() for t in host_in)
        out["d2h"] = sum(t.numel() * t.element_size() for t in host_in[:2])

        def io(phase):
            if phase == "before":
                for d, h in zip(dev_in, host_in):
                    d.copy_(h, non_blocking=True)
            else:
                for d, h in zip(dev_in[:2], host_in[:2]):
                    h.copy_(d, non_blocking=True)
        barrier(world)
        ms_e2e, dt, _ = timed_steps(scene, sp, dt, args.steps, torch, on_step=io,
                                    method=args.method, flush=flush, warm=warm)
        barrier(world)
        out["ms_e2e"] = max_over_ranks(ms_e2e, world, torch)
        out["e2e"] = job_throughput(scene.n, world, args.steps, out["ms_e2e"])
    # per-pass device times (profiling pass after the timed regions)
    engine.reset_stats()
    engine.set_profiling(True)
    prof_steps = 3
    _, dt, preps = timed_steps(scene, sp, dt, prof_steps, torch, method=args.method, warm=warm)
    engine.set_profiling(False)
    pass_ms = {}
    for name, (tot, cnt) in engine.kernel_stats().items():
        p = FINISH_PASS[args.method] if name == "finish" else GROUP_PASS.get(
            name, "warm_start" if name.startswith("warm") else None)
        if p:
            pass_ms[p] = pass_ms.get(p, 0.0) + tot / prof_steps
    out["pass_ms"] = pass_ms
    out["iters"] = (sum(r[0] for r in preps) / prof_steps, sum(r[1] for r in preps) / prof_steps)
    out["pairs"] = sum(r[3] for r in preps) / prof_steps
    return out


def fp64_error(engine, args, sp, steps):
    """Per-quantity error of the float32 plain method against a float64 run
    of the plain method from the same initial positions, after `steps`
    steps: L2-relative and max-relative (of each quantity's scale)."""
    f32 = build_scene(engine, args.workload, np.float32, args.rigid_bodies,
                      args.container_resolution)
    f64 = build_scene(engine, args.workload, np.float64, args.rigid_bodies,
                      args.container_resolution)
    f64.x.copy_(f32.x.double())
    d32 = d64 = float(sp.max_dt)
    for _ in range(steps):
        d32, _ = f32.step(args.method, sp, d32)
        d64, _ = f64.step(args.method, sp, d64)
    a, b = f32.state(), f64.state()
    out = {"steps": steps}
    for k in ("x", "v", "density") + STATE[args.method]:
        x = np.asarray(a[k], np.float64)
        y = np.asarray(b[k], np.float64)
        out[k] = {"l2_rel": float("%.3g" % (np.sqrt(((x - y) ** 2).sum() /
                                                     max((y ** 2).sum(), 1e-300)))),
                  "max_rel": float("%.3g" % (np.abs(x - y).max() /
                                             max(np.abs(y).max(), 1e-300)))}
    del f32, f64
    return out


def roofline_of(out, n, flush, workload):
    """Roofline of the arm's dominant pass: Model-A bytes of one launch over
    its CUDA-event time per launch."""
    per_launch = {}
    for p, t in out["pass_ms"].items():
        runs = {"div": out["iters"][0], "den": out["iters"][1]}.get(PASS_PER_STEP.get(p), 1.0)
        if runs > 0 and p in MODEL_A:
            per_launch[p] = t / runs
    dominant = max((p for p in out["pass_ms"] if p in MODEL_A), key=out["pass_ms"].get)
    peak, peak_kind = measured_peaks()
    bpp, bpair = MODEL_A[dominant]
    alg_bytes = bpp * n + bpair * out["pairs"]
    achieved = alg_bytes / (per_launch[dominant] / 1e3) / 1e9
    # the capture of this workload's own dominant pass (no L2 flush variant)
    tr = None if flush else committed_traffic(workload, dominant)
    return {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": tr, "kernel": dominant,
            "peak_kind": peak_kind, "algorithmic_bytes_per_launch": int(alg_bytes),
            "launch_ms": round(per_launch[dominant], 4)}


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
    sp = scenes.solver_params()
    if args.max_dt:
        sp.max_dt = args.max_dt
    warm_mode = args.warm_start
    if warm_mode == "auto":
        warm_mode = "both" if args.method == "df" and args.workload == DEFAULT_WORKLOAD \
            else "plain"
    if warm_mode != "plain" and args.method != "df":
        raise SystemExit("--warm-start learned: DFSPH only")
    net, warm_info = (None, None)
    if warm_mode != "plain":
        net, warm_info = load_warm_net(engine, args, sp)
    scene = build_scene(engine, args.workload, rigid_bodies=args.rigid_bodies,
                        container_resolution=args.container_resolution)
    n = scene.n
    host_state = scene.state() if rank == 0 and world == 1 else None
    host_bodies = scene.host_bodies() if host_state is not None else None
    tuning = None
    if args.autotune == "on" or (args.autotune == "auto" and not args.eager):
        from alluvion_b200 import autotune
        t0 = time.perf_counter()
        tuning = autotune.tune_scene(engine, scene, sp, method=args.method)
        tuning["seconds"] = round(time.perf_counter() - t0, 1)
    snap = scene.snapshot()
    arms = ([("plain", None)] if warm_mode in ("plain", "both") else []) + \
           ([("learned", net.warm_start())] if warm_mode in ("learned", "both") else [])
    primary = arms[-1][0]
    res = {}
    for name, warm in arms:
        scene.restore(snap)
        res[name] = time_arm(engine, scene, sp, args, warm, world, local, torch,
                             want_e2e=name == primary, clocks_on=name == primary)
    main_ = res[primary]
    roofline = roofline_of(main_, n, main_["flush"], args.workload)
    if args.rigid_bodies == 0 or args.container_resolution or args.method != "df":
        roofline["traffic"] = None  # the captures are of the default DFSPH scenes
    bodies_desc = ", seeded rigid bodies" if scene.num_boundaries > 1 else ""
    l2 = ("working set > 126 MB L2 (inputs larger than L2, no flush)" if not main_["flush"] else
          "working set < L2: a 252 MB buffer is rewritten before every timed step (untimed)")
    config = {"workload": workload_name(args, warm_mode), "particles_per_gpu": n,
              "global_particles": n * world,
              "parallelism": "replicas" if world > 1 else "single", "l2": l2,
              **accuracy_summary(main_["reps"]),
              "active_boundary_pairs": int(main_["pairs"]),
              "launch": "eager" if args.eager else "step graph (conditional WHILE loops)",
              "max_dt": float(sp.max_dt), "warm_start": primary,
              "graph_replays_timed": main_["graph_replays"],
              "pass_ms_per_step": {k: round(v, 4) for k, v in main_["pass_ms"].items()}}
    if warm_info is not None:
        arm_rows = {}
        for name, r in res.items():
            arm_rows[name] = dict({"value": round(r["value"], 1),
                                   "ms_per_step": round(r["ms"] / args.steps, 4)},
                                  **accuracy_summary(r["reps"]))
        warm_info["arms"] = arm_rows
        warm_info["gate"] = ("the network runs on a scene's first step, then after a step "
                             "whose solves went beyond their minimum iteration counts if its "
                             "last outcome was no worse than the plain start's (or it has not "
                             "run for 64 steps); at the minimum counts no warm start can save "
                             "an iteration")
        config["learned_warm_start"] = warm_info
    if tuning is not None:
        config["autotune"] = {"seconds": tuning["seconds"], "kept": tuning["kept"],
                              "graph_ms_per_step": tuning["graph_ms"], "shapes": {
            e["group"]: [e["block"], e["tpp"]] for e in tuning["entries"]}}
    if args.fp64_steps and rank == 0:
        config["error_vs_fp64_plain"] = fp64_error(engine, args, sp, args.fp64_steps)
    result = {
        "metric": METRIC, "value": round(main_["value"], 1), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(main_["ms"] / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded jittered lattice%s)" % bodies_desc,
        "config": config,
        "e2e": {"value": round(main_["e2e"], 1), "unit": UNIT,
                "h2d_bytes_per_step": main_["h2d"], "d2h_bytes_per_step": main_["d2h"]},
        "gpu_launches": int(main_["launches"]),
        "roofline": roofline,
        "clocks": main_["clocks"],
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        result["cpu_baseline"] = cpu_baseline(scene, sp, float(sp.max_dt), args.cpu_seconds,
                                              host_state, host_bodies, args.method)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result), flush=True)


def reference_batch(args):
    """Reference arm of a batch workload: the oracle port advances every
    scene of the batch by one step per benchmark step (scenes in turn, all
    host cores), on grids the oracle builds."""
    from alluvion_b200 import scenes
    from oracle import binding as orc
    spec = BATCH_WORKLOADS[args.workload]
    specs = batch_scene_specs(spec)
    sp = scenes.solver_params()
    items = []
    setup_s = 0.0
    for sc in specs:
        bodies, keep, rigid, t = oracle_scene(sc)
        setup_s += t
        items.append([sc, bodies, keep, rigid, zero_state(sc, "df"), float(sp.max_dt)])
    total_n = sum(sc.n for sc in specs)
    reps = []
    el = 0.0
    steps = 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        for it in items:
            sc, bodies, _, rigid, state, dt = it
            it[5], r = orc.run("df", sc.cn, sc.cni, bodies, rigid, state, sp, dt, 1)
            reps += r
        el += time.perf_counter() - t0
        steps += 1
        if el * (steps + 1) / steps > REFERENCE_SECONDS:
            break
    for it in items:
        release_oracle_scene(it[0], it[2])
    value = total_n * steps / el
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 1), "unit": UNIT,
        "n_gpus": 1, "steps": steps, "warmup": 0, "ms_per_step": round(el * 1e3 / steps, 2),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded jittered lattices, seeded rigid spheres)",
        "config": dict({"workload": "DFSPH " + spec["desc"], "particles_per_gpu": total_n,
                        "grids": "built by the oracle on the host cores (untimed, %.1f s)"
                                 % setup_s},
                       **accuracy_summary([(r.num_divergence_solve, r.num_density_solve,
                                            r.mean_density_error, r.num_active_boundary_pairs,
                                            r.mean_density_change) for r in reps])),
        "cpu_baseline": {"value": round(value, 1), "unit": UNIT, "cores": orc.num_threads(),
                         "kind": "port",
                         "sample": "%d step(s) of all %d scenes" % (steps, len(specs))},
        "e2e": {"value": round(value, 1), "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


REFERENCE_SECONDS = 150.0


def zero_state(spec, method):
    n, T = spec.n, spec.dtype
    st = {"x": np.ascontiguousarray(spec.x).copy(), "v": np.zeros((n, 3), T),
          "density": np.zeros(n, T), "density_adv": np.zeros(n, T), "a": np.zeros((n, 3), T)}
    for k in STATE[method]:
        st[k] = np.zeros(n, T)
    return st


def reference_arm(args):
    """The reference's CPU formulation of the path (the oracle port: the
    reference itself needs Eigen/GLFW/glm and does not build here), timed on
    all host cores.  Nothing here loads the engine: grids are built by the
    oracle.  Rank 0 only."""
    world, rank, local = dist_env()
    if rank != 0:
        return
    from alluvion_b200 import scenes
    from oracle import binding as orc
    if args.workload in BATCH_WORKLOADS:
        return reference_batch(args)
    spec = build_scene_spec(args.workload, rigid_bodies=args.rigid_bodies,
                            container_resolution=args.container_resolution)
    bodies, keep, rigid, setup_s = oracle_scene(spec)
    nodes_setup = lazy_nodes_computed(keep)
    state = zero_state(spec, args.method)
    sp = scenes.solver_params()
    if args.max_dt:
        sp.max_dt = args.max_dt
    dt = float(sp.max_dt)
    t_w = time.perf_counter()
    warm = 0
    for _ in range(args.warmup):
        dt, _ = orc.run(args.method, spec.cn, spec.cni, bodies, rigid, state, sp, dt, 1)
        warm += 1
        if time.perf_counter() - t_w > 0.25 * REFERENCE_SECONDS:
            break
    nodes_before = lazy_nodes_computed(keep)
    reps = []
    el = 0.0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        dt, r = orc.run(args.method, spec.cn, spec.cni, bodies, rigid, state, sp, dt, 1)
        el += time.perf_counter() - t0
        reps += r
        if el * (len(reps) + 1) / len(reps) > REFERENCE_SECONDS:
            break
    steps = len(reps)
    nodes_timed = lazy_nodes_computed(keep) - nodes_before
    release_oracle_scene(spec, keep)
    value = spec.n * steps / el
    sample = "%d full steps of the %s-particle scene after %d warm-up step(s)" % (
        steps, format(spec.n, ","), warm)
    if steps < args.steps:
        sample += " (%d requested; stopped at the %.0f s budget)" % (args.steps,
                                                                    REFERENCE_SECONDS)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 1), "unit": UNIT,
        "n_gpus": world, "steps": steps, "warmup": warm,
        "ms_per_step": round(el * 1e3 / steps, 2), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded jittered lattice%s)" % (
            ", seeded rigid bodies" if spec.num_boundaries > 1 else ""),
        "config": dict({"workload": workload_name(args), "particles_per_gpu": spec.n,
                        "grids": "built by the oracle on the host cores (untimed, %.1f s): "
                                 "analytic distance nodes, lazily filled volume maps; %d volume "
                                 "nodes computed before the timed steps, %d during them"
                                 % (setup_s, nodes_before, nodes_timed)},
                       **accuracy_summary([(r.num_divergence_solve, r.num_density_solve,
                                            r.mean_density_error, r.num_active_boundary_pairs,
                                            r.mean_density_change) for r in reps])),
        "cpu_baseline": {"value": round(value, 1), "unit": UNIT, "cores": orc.num_threads(),
                         "kind": "port", "sample": sample},
        "e2e": {"value": round(value, 1), "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)
    del nodes_setup


def postproc_inputs(spec, name, torch, device):
    """Seeded inputs of a post-processing workload (on `device`)."""
    g = torch.Generator(device=device)
    g.manual_seed(SEED)
    if name == "histogram-256m":
        v = torch.rand(spec["n"], device=device, generator=g)
        m = (torch.rand(spec["n"], device=device, generator=g) < 0.5).float()
        return dict(v=v, mask=m)
    side = 100
    idx = torch.arange(side ** 3, device=device)
    lat = torch.stack([idx // (side * side), (idx // side) % side, idx % side], 1).float()
    x = (lat + 0.5) * 0.02 + (torch.rand(lat.shape, device=device, generator=g) - 0.5) * 0.002
    rho = 1000.0 + 10.0 * torch.rand(side ** 3, device=device, generator=g)
    v = torch.randn(side ** 3, 3, device=device, generator=g)
    sx = torch.rand(spec["n"], 3, device=device, generator=g) * 1.96 + 0.02
    return dict(x=x.contiguous(), rho=rho, v=v.contiguous(), sx=sx.contiguous())


def postproc_arm(args):
    """Post-processing variants: histogram256 with mask, and sampling."""
    import ctypes
    import torch
    from alluvion_b200 import _capi, scenes
    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    engine = _capi.Engine(local)
    spec = POSTPROC_WORKLOADS[args.workload]
    lib = _capi.lib()
    inp = postproc_inputs(spec, args.workload, torch, "cuda")
    hist = torch.zeros(256, dtype=torch.int32, device="cuda")
    if args.workload == "histogram-256m":
        n = spec["n"]
        def run(v, m):
            _capi.check(lib.al_histogram256_f32(engine.handle, v.data_ptr(), m.data_ptr(), n,
                                                ctypes.c_float(0.0), ctypes.c_float(1.0),
                                                hist.data_ptr(), None), "histogram")
        call = lambda: run(inp["v"], inp["mask"])
        units = n
        alg_bytes = 8 * n  # values and mask, read once
    else:
        cn = scenes.make_const(np.float32, 0.01)
        cni = scenes.make_consti((0.0, 0.0, 0.0), (2.0, 2.0, 2.0), float(cn.kernel_radius))
        s = spec["n"]
        outs = [torch.zeros(s, device="cuda"), torch.zeros(s, 3, device="cuda"),
                torch.zeros(s, 3, device="cuda")]
        req = _capi.SampleF32()
        req.sample_x, req.num_samples = inp["sx"].data_ptr(), s
        req.particle_density, req.particle_v = inp["rho"].data_ptr(), inp["v"].data_ptr()
        req.sample_density, req.sample_v = outs[0].data_ptr(), outs[1].data_ptr()
        req.sample_vorticity = outs[2].data_ptr()
        npart = inp["x"].shape[0]
        def call():
            _capi.check(lib.al_sample_fluid_f32(engine.handle, _capi.ptr(cn), _capi.ptr(cni),
                                                inp["x"].data_ptr(), npart, None, _capi.ptr(req),
                                                None), "sample")
        units = s
        # particle x, rho, v read once; samples read, three outputs written
        alg_bytes = npart * (12 + 4 + 12) + s * (12 + 4 + 12 + 12)
    for _ in range(args.warmup):
        call()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(args.steps):
        call()
    b.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = a.elapsed_time(b)
    value = units * args.steps / (ms / 1e3)
    # per-launch device time of the dominant launch group
    engine.reset_stats()
    engine.set_profiling(True)
    call()
    engine.synchronize()
    engine.set_profiling(False)
    stats = engine.kernel_stats()
    dom = max(stats, key=lambda k: stats[k][0])
    launch_ms = stats[dom][0] / max(stats[dom][1], 1)
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (ms / args.steps / 1e3) / 1e9
    # end to end: inputs from pinned host memory, results back, every step
    if args.workload == "histogram-256m":
        hv = inp["v"].cpu().pin_memory()
        hm = inp["mask"].cpu().pin_memory()
        hh = torch.zeros(256, dtype=torch.int32).pin_memory()
        def e2e_step():
            inp["v"].copy_(hv, non_blocking=True)
            inp["mask"].copy_(hm, non_blocking=True)
            call()
            hh.copy_(hist, non_blocking=True)
        h2d, d2h = 8 * spec["n"], 1024
    else:
        hs = inp["sx"].cpu().pin_memory()
        hx = inp["x"].cpu().pin_memory()
        ho = [o.cpu().pin_memory() for o in outs]
        def e2e_step():
            inp["sx"].copy_(hs, non_blocking=True)
            inp["x"].copy_(hx, non_blocking=True)
            call()
            for h, o in zip(ho, outs):
                h.copy_(o, non_blocking=True)
        h2d = hs.numel() * 4 + hx.numel() * 4
        d2h = sum(o.numel() * 4 for o in outs)
    e2e_step()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e_steps = max(3, min(args.steps, 10))
    for _ in range(e_steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e = units * e_steps / (time.perf_counter() - t0)
    result = {
        "metric": spec["metric"], "value": round(value, 1), "unit": spec["unit"], "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded)",
        "config": {"workload": spec["desc"], "l2": "inputs larger than L2 (no flush)",
                   "launch_groups_ms": {k: round(v[0], 4) for k, v in stats.items()}},
        "e2e": {"value": round(e2e, 1), "unit": spec["unit"], "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(engine.launch_count()),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": None,
                     "kernel": dom, "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": int(alg_bytes),
                     "launch_ms": round(launch_ms, 4)},
        "clocks": clk,
    }
    if not args.no_cpu_baseline:
        result["cpu_baseline"] = postproc_cpu(args, spec, inp)
    print(json.dumps(result), flush=True)


def postproc_cpu(args, spec, inp):
    """The oracle on a bounded sample of the same workload, host threads."""
    from oracle import binding as orc
    if args.workload == "histogram-256m":
        m = 1 << 24
        v = inp["v"][:m].cpu().numpy()
        mk = inp["mask"][:m].cpu().numpy()
        t0 = time.perf_counter()
        orc.histogram256(v, 0.0, 1.0, mk)
        dt = time.perf_counter() - t0
        return {"value": round(m / dt, 1), "unit": spec["unit"], "cores": 1, "kind": "port",
                "sample": "the oracle's histogram of the first %d values and mask" % m}
    from alluvion_b200 import scenes
    cn = scenes.make_const(np.float32, 0.01)
    cni = scenes.make_consti((0.0, 0.0, 0.0), (2.0, 2.0, 2.0), float(cn.kernel_radius))
    m = 1 << 16
    t0 = time.perf_counter()
    orc.sample_fluid(cn, cni, inp["x"].cpu().numpy(), None, inp["sx"][:m].cpu().numpy(),
                     inp["rho"].cpu().numpy(), inp["v"].cpu().numpy(),
                     outputs=("density", "v", "vorticity"))
    dt = time.perf_counter() - t0
    return {"value": round(m / dt, 1), "unit": spec["unit"], "cores": orc.lib().orc_num_threads(),
            "kind": "port",
            "sample": "the oracle's sampling of the first %d samples (grid sort of all "
                      "particles included)" % m}


def postproc_reference(args):
    """Reference arm of the post-processing variants: the oracle port."""
    world, rank, local = dist_env()
    if rank != 0:
        return
    import torch
    spec = POSTPROC_WORKLOADS[args.workload]
    inp = postproc_inputs(spec, args.workload, torch, "cpu")
    for _ in range(max(args.warmup, 1)):
        base = postproc_cpu(args, spec, inp)
    vals = [postproc_cpu(args, spec, inp)["value"] for _ in range(max(1, min(args.steps, 3)))]
    v = float(np.median(vals))
    print(json.dumps({"impl": "reference", "metric": spec["metric"], "value": round(v, 1),
                      "unit": spec["unit"], "n_gpus": world, "steps": len(vals),
                      "warmup": args.warmup, "higher_is_better": True,
                      "config": {"workload": spec["desc"]},
                      "cpu_baseline": dict(base, value=round(v, 1)),
                      "e2e": {"value": round(v, 1), "unit": spec["unit"],
                              "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}), flush=True)


def main():
    args = parse_args()
    if args.workload in POSTPROC_WORKLOADS:
        if args.impl == "reference":
            postproc_reference(args)
        else:
            postproc_arm(args)
        return
    if args.impl == "reference":
        reference_arm(args)
    elif args.workload in BATCH_WORKLOADS:
        batch_arm(args)
    else:
        engine_arm(args)


if __name__ == "__main__":
    main()
