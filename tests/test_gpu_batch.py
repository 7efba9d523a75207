"""Batched scenes (al_df_batch_step_f32) against the same scenes stepped
one at a time with al_df_step_f32.  Each batch branch runs the scene's own
kernels; with the default launch-shape tables (the same shapes in the
single and the batch context: threads per particle from the scene's own
particle count) the launch shapes are the same too, so the results are
bit-identical, whether the batch runs eagerly (first call) or as one
replayed graph.  Tuned tables that give a scene another shape in a batch
change its float results in the last bits (tests/test_gpu_launch_shapes.py
covers that case against the oracle)."""
import numpy as np
import pytest

from alluvion_b200 import _capi, scenes

pytestmark = pytest.mark.gpu

SIZES = [(10, 8, 10), (16, 12, 16), (8, 8, 8), (20, 10, 12), (12, 12, 12)]


def _scenes(engine):
    out = []
    for k, lat in enumerate(SIZES):
        bodies = []
        if k % 2 == 1:
            bodies = [dict(shape=_capi.SHAPE_SPHERE, params=[0.03], sign=1.0, resolution=16,
                           use_distance_grid=True, mass=0.1,
                           inertia=scenes.sphere_inertia(0.1, 0.03),
                           x=(0.12, 0.3, 0.12), v=(0.0, -0.2, 0.0))]
        out.append(scenes.dam_break(engine, np.float32, lat, 0.01, (0.5, 0.4, 0.4), bodies,
                                    seed=k, volume_resolution=16))
    return out


def test_batch_matches_single_steps(engine):
    sp = scenes.solver_params()
    batch = _scenes(engine)
    single = _scenes(engine)
    c0, r0 = engine.graph_stats()
    dts_b = [2e-4] * len(batch)
    dts_s = [2e-4] * len(single)
    for step in range(4):
        dts_b, reps_b, status = scenes.batch_step(engine, batch, sp, dts_b)
        assert status == [0] * len(batch)
        for k, sc in enumerate(single):
            dts_s[k], rep = sc.step("df", sp, dts_s[k])
            assert rep.num_density_solve == reps_b[k].num_density_solve
            assert rep.num_divergence_solve == reps_b[k].num_divergence_solve
            assert rep.mean_density_error == reps_b[k].mean_density_error
        assert dts_b == dts_s
    c1, r1 = engine.graph_stats()
    assert r1 - r0 >= 2 + 2 * len(single)  # batch replays + the single scenes' replays
    for b, s in zip(batch, single):
        sb, ss = b.state(), s.state()
        for key in ("x", "v", "kappa", "kappa_v", "density"):
            np.testing.assert_array_equal(sb[key], ss[key], err_msg=key)
        nb = b.num_boundaries
        for i in range(nb):
            assert list(b.rigid[i].x) == list(s.rigid[i].x)
            assert list(b.rigid[i].q) == list(s.rigid[i].q)


def test_batch_rejects_too_many_scenes(engine):
    arr = (_capi.SceneF32 * 1)()
    st = _capi.lib().al_df_batch_step_f32(engine.handle, arr, 257, None)
    assert st == 2  # AL_ERR_INVALID


@pytest.mark.parametrize("shape", [None, (256, 1)])
def test_batch_of_benchmark_scenes_matches_oracle(engine, shape):
    """The four smallest scenes of the 64-scene benchmark batch (seeded, with
    their rigid spheres), stepped as one batch, each against the oracle's
    step of the same scene: equal iteration counts and the float32 one-step
    tolerances of the single-step parity tests (the jittered start's
    pressure kick amplifies rounding from the second step on).  With shape
    set, the batch context runs a tuned table (other threads per particle
    than a single step would use)."""
    import bench
    from alluvion_b200 import autotune
    from test_gpu_step import TOL, _close, _oracle_run
    specs = bench.batch_scene_specs(bench.BATCH_WORKLOADS["batch64"])
    chosen = sorted(specs, key=lambda s: s.n)[:4]
    batch = [s.device(engine) for s in chosen]
    groups = _capi.tunable_groups()
    buckets = sorted({autotune.bucket_of(sc.n) for sc in batch})
    try:
        if shape:
            for b in buckets:
                for name, pair in groups:
                    engine.set_launch_shape(name, b, 1, shape[0], shape[1] if pair else 1)
        sp = scenes.solver_params()
        oracle = [_oracle_run(sc, "df", sp, 2e-4, 1) for sc in batch]
        dts, reps, status = scenes.batch_step(engine, batch, sp, [2e-4] * len(batch))
        assert status == [0] * len(batch)
        tol = TOL[(np.float32, 1)]
        for k, sc in enumerate(batch):
            ostate, origid, odt, oreps = oracle[k]
            assert reps[k].num_density_solve == oreps[0].num_density_solve
            assert reps[k].num_divergence_solve == oreps[0].num_divergence_solve
            g = sc.state()
            _close(g["x"], ostate["x"], tol["x"], "x")
            _close(g["v"], ostate["v"], tol["v"], "v")
            _close(g["density"], ostate["density"], tol["density"], "density")
    finally:
        for b in buckets:
            for name, _ in groups:
                engine.set_launch_shape(name, b, 1, 0, 0)
