"""Trains and evaluates the learned DFSPH warm start at full scale, on a CUDA
device, with the engine's own kernels (no counterpart in the reference).

Training set: converged solves of 200 seeded dam breaks of 1,048,576
particles (128 x 64 x 128 lattice, r = 0.005 m, 2 x 1 x 2 m box with a 64^3
volume map, two rigid spheres and two boxes on 64^3 grids at seeded
positions): each scene runs `--steps` plain DFSPH steps at max_dt 2e-4 s and
contributes `--per-step` random particles of every step after the first 5
(features of the step's start, converged kappa_v / dt and kappa / dt^2).
Fit: Adam, lr 1e-3 with a step-down schedule, 20,000 steps of 65,536
samples.  Evaluation: 20 held-out seeds of the same scene family, plain
against learned warm start over `--eval-steps` steps each, at the
reference's minimum iteration counts (1 divergence, 2 density) and at the
0.1 % tolerances.

Writes the network to alluvion_b200/data/warm_start_dambreak.npz (loaded by
warm_start.WarmStartNet.load) and the evaluation next to it as JSON.

Usage: python -m alluvion_b200.train_warm_start [--scenes 200] [--fit-steps 20000]
"""
import argparse
import json
import os
import time

import numpy as np

from . import _capi, scenes, warm_start

DATA_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
WEIGHTS = os.path.join(DATA_DIR, "warm_start_dambreak.npz")
EVALUATION = os.path.join(DATA_DIR, "warm_start_dambreak_eval.json")

LATTICE, RADIUS, CONTAINER = (128, 64, 128), 0.005, (2.0, 1.0, 2.0)
TRAIN_SEED0, EVAL_SEED0 = 10_000, 20_000


def scene_spec(seed):
    """One scene of the family: jitter and body placement seeded by `seed`."""
    bodies = scenes.seeded_rigid_bodies(seed, CONTAINER, RADIUS, resolution=64)
    return scenes.dam_break_spec(np.float32, LATTICE, RADIUS, CONTAINER, bodies, seed=seed,
                                 volume_resolution=64)


def run_iterations(engine, spec, sp, steps, warm=None):
    """Steps a fresh device copy of `spec`; returns per-step (divergence,
    density) iterations, mean density errors and the device time in ms."""
    import torch
    sc = spec.device(engine)
    dt = float(sp.max_dt)
    its, errs = [], []
    ws = warm.warm_start() if warm is not None else None
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(steps):
        dt, rep = sc.step("df", sp, dt, warm=ws)
        its.append((rep.num_divergence_solve, rep.num_density_solve))
        errs.append(rep.mean_density_error)
    t1.record()
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1)
    del sc
    return np.asarray(its), np.asarray(errs), ms


def net_used(its, sp):
    """Steps on which the engine's gate runs the network (the rule of
    warm_gate_update in the engine, replayed on the iteration record)."""
    w = [0, 0, 0, 0]
    used = []
    for d, r in its:
        u = w[0] == 0
        used.append(u)
        w[2 if u else 3] = d + r
        w[1] = 0 if u else w[1] + 1
        at_floor = d <= sp.min_divergence_solve and r <= sp.min_density_solve
        w[0] = 0 if (not at_floor and (w[2] <= w[3] or w[1] >= 64)) else 1
    return np.asarray(used)


def main():
    ap = argparse.ArgumentParser(description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--scenes", type=int, default=200)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--per-step", type=int, default=4096)
    ap.add_argument("--fit-steps", type=int, default=20000)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--eval-scenes", type=int, default=20)
    ap.add_argument("--eval-steps", type=int, default=200)
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--eval-out", default=EVALUATION)
    ap.add_argument("--eval-only", action="store_true",
                    help="evaluate the network in --out again (its training record is kept)")
    args = ap.parse_args()
    import torch
    torch.cuda.set_device(0)
    engine = _capi.Engine(0)
    sp = scenes.solver_params()
    if args.eval_only:
        net = warm_start.WarmStartNet.load(args.out)
        with open(args.eval_out) as f:
            training = json.load(f)["training"]
        evaluate(engine, net, sp, args, training)
        engine.close()
        return
    t_start = time.perf_counter()
    xs, ts = [], []
    for k in range(args.scenes):
        sc = scene_spec(TRAIN_SEED0 + k).device(engine)
        x, t = warm_start.collect(sc, sp, args.steps, args.per_step, seed=TRAIN_SEED0 + k)
        xs.append(x)
        ts.append(t)
        del sc
    feats = torch.cat(xs)
    targs = torch.cat(ts)
    del xs, ts
    t_collect = time.perf_counter() - t_start
    t0 = time.perf_counter()
    net, losses = warm_start.fit(engine, feats, targs, steps=args.fit_steps, batch=args.batch,
                                 lr=args.lr, seed=1)
    torch.cuda.synchronize()
    t_fit = time.perf_counter() - t0
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    net.save(args.out)
    training = {"scenes": args.scenes, "steps_per_scene": args.steps,
                "samples": int(feats.shape[0]), "adam_steps": args.fit_steps,
                "batch": args.batch, "lr": args.lr,
                "loss_first_last": [round(float(np.mean(losses[:100])), 5),
                                    round(float(np.mean(losses[-100:])), 5)],
                "collect_s": round(t_collect, 1), "fit_s": round(t_fit, 1)}
    del feats, targs
    evaluate(engine, net, sp, args, training)
    engine.close()


def evaluate(engine, net, sp, args, training):
    """Plain against learned warm start on the held-out seeds; writes the
    evaluation JSON (with the training record) and prints its summary."""
    rows = []
    for k in range(args.eval_scenes):
        spec = scene_spec(EVAL_SEED0 + k)
        ip, ep, mp = run_iterations(engine, spec, sp, args.eval_steps)
        il, el, ml = run_iterations(engine, spec, sp, args.eval_steps, warm=net)
        used = net_used(il, sp)
        rows.append({
            "seed": EVAL_SEED0 + k,
            "plain_iterations": [round(float(v), 4) for v in ip.mean(0)],
            "learned_iterations": [round(float(v), 4) for v in il.mean(0)],
            "plain_ms_per_step": round(mp / args.eval_steps, 4),
            "learned_ms_per_step": round(ml / args.eval_steps, 4),
            "learned_steps_using_net": int(used.sum()),
            "plain_iterations_steps_1_10": [round(float(v), 3) for v in ip[:10].mean(0)],
            "learned_iterations_steps_1_10": [round(float(v), 3) for v in il[:10].mean(0)],
            "max_density_error": [float(ep.max()), float(el.max())],
        })
    pi = np.array([r["plain_iterations"] for r in rows])
    li = np.array([r["learned_iterations"] for r in rows])
    pm = np.array([r["plain_ms_per_step"] for r in rows])
    lm = np.array([r["learned_ms_per_step"] for r in rows])
    n = scene_spec(EVAL_SEED0).n
    summary = {
        "training": training,
        "evaluation": {"scenes": args.eval_scenes, "steps": args.eval_steps,
                       "particles": n, "max_dt": float(sp.max_dt),
                       "min_iterations": [int(sp.min_divergence_solve),
                                          int(sp.min_density_solve)],
                       "plain_iterations_per_step": [round(float(v), 4) for v in pi.mean(0)],
                       "learned_iterations_per_step": [round(float(v), 4) for v in li.mean(0)],
                       "plain_particle_steps_per_s": round(n / (pm.mean() / 1e3), 1),
                       "learned_particle_steps_per_s": round(n / (lm.mean() / 1e3), 1),
                       "learned_steps_using_net": int(sum(r["learned_steps_using_net"]
                                                          for r in rows))},
        "per_scene": rows,
    }
    with open(args.eval_out, "w") as f:
        json.dump(summary, f, indent=1)
    print(json.dumps({k: summary[k] for k in ("training", "evaluation")}, indent=1))


if __name__ == "__main__":
    main()
