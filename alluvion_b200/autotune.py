"""Launch-shape autotuner for the step's pass groups.

The counterpart of the reference's block-size sweep (bin/block_scan:15-36,
which times every kernel at each block size and writes the best to
.alcache/<kernel>.yaml) and of its table loaded at start-up
(Runner::load_optimal_block_size, runner.hpp:4922-4937).  Here the shape of
a pass group is (threads per block, threads per particle) and the table is
keyed by the scene's particle-count bucket floor(log2 N) and by context
(single step or a scene of a batched step), because the best shape depends
on how many threads the pass has to fill the GPU with.

  tune_scene(engine, scene, sp)   every group of one scene's step, timed per
                                  launch with the engine's CUDA-event
                                  statistics (each candidate from the same
                                  state); single-step context
  tune_batch(engine, scenes, sp)  whole batched steps timed (graph replays,
                                  scenes side by side): the best shape for
                                  all buckets alike, then coordinate descent
                                  over the buckets; batch context
  save(table, path), load(engine, path), apply(engine, table)

A table is a dict {"device": ..., "entries": [{"group", "bucket", "batch",
"block", "tpp", "ms"}]} and is stored as JSON.
"""
import json

import numpy as np

from . import _capi

# (threads per block, threads per particle) tried for pair passes; the
# neighbor build (one thread per particle) tries the block sizes only
PAIR_CANDIDATES = [(64, 1), (128, 1), (256, 1), (64, 2), (128, 2), (256, 2), (128, 4),
                   (256, 4), (128, 8), (256, 8)]
BLOCK_CANDIDATES = [(64, 1), (128, 1), (256, 1)]


def bucket_of(n):
    return int(n).bit_length() - 1 if n > 0 else 0


def _candidates(pair):
    return PAIR_CANDIDATES if pair else BLOCK_CANDIDATES


def apply(engine, table):
    for e in table["entries"]:
        engine.set_launch_shape(e["group"], e["bucket"], e["batch"], e["block"], e["tpp"])


def clear(engine, table):
    for e in table["entries"]:
        engine.set_launch_shape(e["group"], e["bucket"], e["batch"], 0, 0)


def validate(table):
    """Checks a table's entries (names, ranges); returns it."""
    names = {}
    for e in table["entries"]:
        for k in ("group", "bucket", "batch", "block", "tpp"):
            if k not in e:
                raise ValueError("launch-shape entry without %r: %r" % (k, e))
        if e["block"] not in (64, 128, 256) or e["tpp"] not in (1, 2, 4, 8):
            raise ValueError("launch-shape entry out of range: %r" % e)
        if not 0 <= e["bucket"] < 32 or e["batch"] not in (0, 1):
            raise ValueError("launch-shape entry out of range: %r" % e)
        key = (e["group"], e["bucket"], e["batch"])
        if key in names:
            raise ValueError("duplicate launch-shape entry %r" % (key,))
        names[key] = e
    return table


def save(table, path):
    with open(path, "w") as f:
        json.dump(validate(table), f, indent=1)


def load(engine, path):
    """Reads a table written by save() and applies it to `engine`."""
    with open(path) as f:
        table = validate(json.load(f))
    apply(engine, table)
    return table


def _group_ms(engine, steps):
    """{group: ms per launch} of the last profiled steps."""
    return {name: tot / cnt for name, (tot, cnt) in engine.kernel_stats().items() if cnt}


def _graph_step_ms(scene, sp, method, snap, steps, warm):
    """ms per step of `steps` captured steps from the restored state (two
    untimed steps first: the eager one and the capture)."""
    import torch
    scene.restore(snap)
    dt = float(sp.max_dt)
    for _ in range(2):
        dt, _ = scene.step(method, sp, dt, warm=warm)
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(steps):
        dt, _ = scene.step(method, sp, dt, warm=warm)
    t1.record()
    torch.cuda.synchronize()
    return t0.elapsed_time(t1) / steps


def tune_scene(engine, scene, sp, method="df", steps=3, warm=None, check_steps=10):
    """Sweeps every tunable group's shape on `scene` (its state is put back
    after each trial and at the end), timing each group per launch; then
    times whole captured steps with the fastest shape per group and with the
    defaults, and keeps the faster of the two (per-launch times of small
    scenes do not show how the launches overlap in the step graph).  Applies
    and returns the table for the scene's bucket, single-step context; its
    "graph_ms" records both step times and "kept" which won."""
    import torch
    groups = _capi.tunable_groups()
    b = bucket_of(scene.n)
    snap = scene.snapshot()
    trials = {}
    ncand = len(PAIR_CANDIDATES)
    for ci in range(ncand):
        for name, pair in groups:
            cands = _candidates(pair)
            blk, tpp = cands[ci % len(cands)]
            engine.set_launch_shape(name, b, 0, blk, tpp)
        scene.restore(snap)
        dt = float(sp.max_dt)
        dt, _ = scene.step(method, sp, dt, warm=warm)  # first use of the shapes, untimed
        engine.reset_stats()
        engine.set_profiling(True)
        for _ in range(steps):
            dt, _ = scene.step(method, sp, dt, warm=warm)
        engine.set_profiling(False)
        torch.cuda.synchronize()
        ms = _group_ms(engine, steps)
        for name, pair in groups:
            cands = _candidates(pair)
            if ci >= len(cands) or name not in ms:
                continue
            trials.setdefault(name, []).append((ms[name], cands[ci]))
    entries = []
    for name, pair in groups:
        engine.set_launch_shape(name, b, 0, 0, 0)
        if name not in trials:
            continue
        best_ms, (blk, tpp) = min(trials[name])
        entries.append({"group": name, "bucket": b, "batch": 0, "block": blk, "tpp": tpp,
                        "ms": round(best_ms, 5),
                        "default_ms": round(dict((c, t) for t, c in trials[name]).get(
                            engine.launch_shape(name, scene.n, 0), float("nan")), 5)})
    table = {"device": torch.cuda.get_device_name(), "entries": entries}
    default_ms = _graph_step_ms(scene, sp, method, snap, check_steps, warm)
    apply(engine, table)
    tuned_ms = _graph_step_ms(scene, sp, method, snap, check_steps, warm)
    table["graph_ms"] = {"default": round(default_ms, 4), "tuned": round(tuned_ms, 4)}
    table["kept"] = "tuned" if tuned_ms < default_ms else "default"
    if table["kept"] == "default":
        clear(engine, table)
        table["entries"] = []
    scene.restore(snap)
    return table


def tune_batch(engine, scene_list, sp, steps=8, candidates=None, step_fn=None):
    """Shapes for a batch, timed on whole batched steps (graph replays,
    every trial from the same restored state), in two stages: the best
    shape applied to every particle-count bucket alike, then coordinate
    descent over the buckets from there, keeping a change only when it
    saves more than 1 % of the batch step.  Returns and applies the table;
    `step_fn(dts)` steps the batch (default scenes.batch_step)."""
    import torch
    from . import scenes as _scenes
    cands = candidates or PAIR_CANDIDATES
    groups = _capi.tunable_groups()
    snaps = [sc.snapshot() for sc in scene_list]
    if step_fn is None:
        step_fn = lambda dts: _scenes.batch_step(engine, scene_list, sp, dts)[0]
    buckets = sorted({bucket_of(sc.n) for sc in scene_list})

    def set_bucket(b, shape):
        for name, pair in groups:
            engine.set_launch_shape(name, b, 1, shape[0], shape[1] if pair else 1)

    def trial():
        for sc, sn in zip(scene_list, snaps):
            sc.restore(sn)
        dts = [float(sp.max_dt)] * len(scene_list)
        for _ in range(2):  # eager first call, then the capture
            dts = step_fn(dts)
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        for _ in range(steps):
            dts = step_fn(dts)
        t1.record()
        torch.cuda.synchronize()
        return t0.elapsed_time(t1) / steps

    base_ms = trial()
    uniform = None
    for shape in cands:
        for b in buckets:
            set_bucket(b, shape)
        ms = trial()
        if uniform is None or ms < uniform[0]:
            uniform = (ms, shape)
    current = {b: uniform[1] for b in buckets}
    for b in buckets:
        set_bucket(b, uniform[1])
    best = trial()
    for b in buckets:
        for shape in cands:
            if shape == current[b]:
                continue
            set_bucket(b, shape)
            ms = trial()
            if ms < 0.99 * best:
                best, current[b] = ms, shape
        set_bucket(b, current[b])
    for sc, sn in zip(scene_list, snaps):
        sc.restore(sn)
    entries = [{"group": name, "bucket": b, "batch": 1, "block": current[b][0],
                "tpp": current[b][1] if pair else 1, "ms": round(best, 5)}
               for b in buckets for name, pair in groups]
    table = {"device": torch.cuda.get_device_name(), "entries": entries,
             "batch_ms_default": round(base_ms, 4), "batch_ms_uniform": round(uniform[0], 4),
             "uniform_shape": list(uniform[1]), "batch_ms_tuned": round(best, 4),
             "buckets": {str(b): {"block": current[b][0], "tpp": current[b][1],
                                  "scenes": int(np.sum([bucket_of(sc.n) == b
                                                        for sc in scene_list]))}
                         for b in buckets}}
    apply(engine, table)
    return table
