"""Captured step graphs against eager steps, through the C ABI.

With graph mode on, repeated al_*_step calls with the same configuration
replay one CUDA graph whose solver loops are conditional WHILE nodes.  The
graph runs the same kernels with the same launch shapes in the same order
as the eager path, so every output must be bit-identical to it, including
when dt, the solver parameters and the rigid state change between calls
(they are staged through pinned memory, not baked into the graph).
"""
import numpy as np
import pytest
import torch

from alluvion_b200 import _capi, scenes

pytestmark = pytest.mark.gpu


def _scene(engine, dtype, seed=5):
    extra = [
        dict(shape=_capi.SHAPE_SPHERE, params=[0.035], sign=1.0, resolution=16,
             use_distance_grid=True, mass=0.12, inertia=scenes.sphere_inertia(0.12, 0.035),
             x=(0.14, 0.32, 0.13), v=(0.0, -0.3, 0.0)),
    ]
    scene = scenes.dam_break(engine, dtype, (14, 12, 12), 0.01, (0.45, 0.4, 0.35), extra,
                             seed=seed, volume_resolution=16)
    rng = np.random.default_rng(seed)
    v0 = rng.normal(0, 0.02, size=(scene.n, 3)).astype(dtype)
    scene.v.copy_(torch.from_numpy(v0).cuda())
    return scene


def _params(k):
    """Solver parameters that vary from call to call."""
    sp = scenes.solver_params()
    if k == 2:
        sp.max_density_solve = 0  # density loop skipped on the device
    if k == 3:
        sp.min_density_solve = 5
        sp.min_divergence_solve = 3
    if k == 4:
        sp.enable_divergence_solve = 1
        sp.max_divergence_solve = 1
    return sp


def _run(engine, method, dtype, graph, steps=6):
    engine.set_graph_mode(graph)
    engine.synchronize()
    scene = _scene(engine, dtype)
    c0, r0 = engine.graph_stats()
    n0 = engine.launch_count()
    dt = 1e-4
    reps = []
    for k in range(steps):
        dt_out, rep = scene.step(method, _params(k), dt * (1.0 + 0.1 * (k % 3)))
        reps.append((dt_out, rep.num_divergence_solve, rep.num_density_solve,
                     rep.mean_density_change, rep.mean_density_error,
                     np.array(rep.force).copy(), np.array(rep.torque).copy()))
    torch.cuda.synchronize()
    c1, r1 = engine.graph_stats()
    rigid = np.array([list(r.x) + list(r.v) + list(r.q) + list(r.omega)
                      for r in scene.rigid[:scene.num_boundaries]])
    out = dict(state=scene.state(), rigid=rigid, reps=reps,
               launches=engine.launch_count() - n0, captures=c1 - c0, replays=r1 - r0)
    engine.set_graph_mode(True)
    return out


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("method", ["df", "ii", "i"])
def test_graph_matches_eager(engine, method, dtype):
    eager = _run(engine, method, dtype, graph=False)
    graph = _run(engine, method, dtype, graph=True)
    assert eager["replays"] == 0 and eager["captures"] == 0
    # first call eager, second captures, the rest replay
    assert graph["replays"] >= 4, (graph["captures"], graph["replays"])
    for k in eager["state"]:
        np.testing.assert_array_equal(graph["state"][k], eager["state"][k], err_msg=k)
    np.testing.assert_array_equal(graph["rigid"], eager["rigid"])
    for a, b in zip(graph["reps"], eager["reps"]):
        assert a[:5] == b[:5]
        np.testing.assert_array_equal(a[5], b[5])
        np.testing.assert_array_equal(a[6], b[6])
    assert graph["launches"] == eager["launches"]


def test_graph_respects_profiling(engine):
    """Profiling runs eagerly (launch groups are timed one by one)."""
    scene = _scene(engine, np.float32, seed=11)
    sp = scenes.solver_params()
    engine.set_profiling(True)
    engine.reset_stats()
    try:
        c0, r0 = engine.graph_stats()
        for _ in range(3):
            scene.step("df", sp, 1e-4)
        c1, r1 = engine.graph_stats()
        stats = engine.kernel_stats()
    finally:
        engine.set_profiling(False)
        engine.reset_stats()
    assert (c1 - c0, r1 - r0) == (0, 0)
    assert stats["neighbors"][1] == 3


def test_learned_warm_start_graph_matches_eager(engine):
    """The learned warm start's inference sits in a conditional IF node of
    the captured step (launched only when the per-scene gate is open); the
    eager path launches the kernels, which return at once when it is closed.
    Both take the same gate decisions, so every output is bit-identical, and
    a captured step launches at most one kernel more than an eager one (the
    node's condition) and two fewer when the gate is closed."""
    import os
    from alluvion_b200 import warm_start
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                        "alluvion_b200", "data", "warm_start_dambreak.npz")
    net = warm_start.WarmStartNet.load(path)
    out = {}
    for graph in (False, True):
        engine.set_graph_mode(graph)
        scene = _scene(engine, np.float32, seed=13)
        n0 = engine.launch_count()
        c0, r0 = engine.graph_stats()
        dt = 1e-4
        reps = []
        for k in range(8):
            sp = scenes.solver_params(max_dt=4e-4 if k < 4 else 2e-4)
            dt, rep = scene.step("df", sp, dt, warm=net.warm_start())
            reps.append((dt, rep.num_divergence_solve, rep.num_density_solve,
                         rep.mean_density_change, rep.mean_density_error))
        torch.cuda.synchronize()
        out[graph] = dict(state=scene.state(), reps=reps, launches=engine.launch_count() - n0,
                          replays=engine.graph_stats()[1] - r0)
    engine.set_graph_mode(True)
    assert out[True]["replays"] >= 4
    assert out[False]["reps"] == out[True]["reps"]
    for k in out[False]["state"]:
        np.testing.assert_array_equal(out[True]["state"][k], out[False]["state"][k], err_msg=k)
    assert out[True]["launches"] <= out[False]["launches"] + 8
