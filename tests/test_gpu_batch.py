"""Batched scenes (al_df_batch_step_f32).

Branch form (one graph branch per scene, al_engine_set_batch_fused(0)):
each branch runs the scene's own kernels; with the default launch-shape
tables (the same shapes in the single and the batch context: threads per
particle from the scene's own particle count) the results equal the same
scenes stepped one at a time with al_df_step_f32 bit for bit, whether the
batch runs eagerly (first call) or as one replayed graph.  Tuned tables that give a scene another shape in a
batch change its float results in the last bits
(tests/test_gpu_launch_shapes.py covers that case against the oracle).

Fused form (one launch per solver pass over all scenes, the default): pair
passes run one thread per particle in 128-thread blocks, so with those
shapes in the batch context the two forms agree bit for bit, including
scenes whose solves take different iteration counts; against the oracle
both meet the single-step tolerances."""
import numpy as np
import pytest

from alluvion_b200 import _capi, autotune, scenes

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


def _uniform_batch_shapes(engine, scene_list, block, tpp):
    """Sets (block, tpp) for every pass group in the batch context of the
    scenes' buckets (0, 0: back to the defaults)."""
    for b in sorted({autotune.bucket_of(sc.n) for sc in scene_list}):
        for name, pair in _capi.tunable_groups():
            engine.set_launch_shape(name, b, 1, block, tpp if pair or not tpp else 1)


def test_batch_matches_single_steps(engine):
    engine.set_batch_fused(False)
    try:
        _batch_matches_single_steps(engine)
    finally:
        engine.set_batch_fused(True)


def _batch_matches_single_steps(engine):
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


def _states_equal(a, b):
    sa, sb = a.state(), b.state()
    for key in ("x", "v", "kappa", "kappa_v", "density", "a"):
        np.testing.assert_array_equal(sa[key], sb[key], err_msg=key)
    for i in range(a.num_boundaries):
        for f in ("x", "v", "omega", "q"):
            assert list(getattr(a.rigid[i], f)) == list(getattr(b.rigid[i], f)), (i, f)


def test_fused_batch_matches_branch_batch(engine):
    """Fused against branch form with 128-thread blocks and one thread per
    particle in the batch context: equal dts, iteration counts, reports and
    states bit for bit over four steps (the first eager, then captured).
    The second scene is held to at least five density iterations, so the
    others sit out iterations of the fused loop; the third runs a smaller
    time-step cap and the fourth keeps its rigid body fixed."""
    fused, branch = _scenes(engine), _scenes(engine)
    sps = [scenes.solver_params() for _ in fused]
    sps[1] = scenes.solver_params(min_density_solve=5)
    sps[2] = scenes.solver_params(max_dt=1e-4)
    sps[3] = scenes.solver_params(integrate_rigids=0)
    _uniform_batch_shapes(engine, fused, 128, 1)
    try:
        c0, r0 = engine.graph_stats()
        dts_f = [2e-4] * len(fused)
        dts_b = [2e-4] * len(branch)
        for step in range(4):
            engine.set_batch_fused(True)
            dts_f, reps_f, st_f = scenes.batch_step(engine, fused, sps, dts_f)
            engine.set_batch_fused(False)
            dts_b, reps_b, st_b = scenes.batch_step(engine, branch, sps, dts_b)
            assert st_f == st_b == [0] * len(fused)
            assert dts_f == dts_b
            for rf, rb in zip(reps_f, reps_b):
                assert rf.num_divergence_solve == rb.num_divergence_solve
                assert rf.num_density_solve == rb.num_density_solve
                assert rf.mean_density_error == rb.mean_density_error
                assert rf.mean_density_change == rb.mean_density_change
                assert rf.num_active_boundary_pairs == rb.num_active_boundary_pairs
                for b in range(len(rf.force)):
                    assert list(rf.force[b]) == list(rb.force[b])
                    assert list(rf.torque[b]) == list(rb.torque[b])
            assert reps_f[1].num_density_solve >= 5
            assert min(r.num_density_solve for r in reps_f) < reps_f[1].num_density_solve
        c1, r1 = engine.graph_stats()
        assert r1 - r0 >= 4  # both forms replayed from the second step on
        for f, b in zip(fused, branch):
            _states_equal(f, b)
    finally:
        engine.set_batch_fused(True)
        _uniform_batch_shapes(engine, fused, 0, 0)


def test_two_fused_batches_alternate(engine):
    """Two fused batches of different scenes, stepped in turn (each replays
    its own graph over the shared arena tables): each equals its branch-form
    twin bit for bit."""
    mk = lambda seed0: [scenes.dam_break(engine, np.float32, lat, 0.01, (0.5, 0.4, 0.4), [],
                                         seed=seed0 + k, volume_resolution=16)
                        for k, lat in enumerate(SIZES[:3])]
    a_f, a_b, b_f, b_b = mk(10), mk(10), mk(20), mk(20)
    b_f, b_b = b_f[:2], b_b[:2]
    sp = scenes.solver_params()
    _uniform_batch_shapes(engine, a_f + b_f, 128, 1)
    try:
        dts = {id(x): [2e-4] * len(x) for x in (a_f, a_b, b_f, b_b)}
        for step in range(3):
            for fused, batch in ((True, a_f), (True, b_f), (False, a_b), (False, b_b)):
                engine.set_batch_fused(fused)
                dts[id(batch)], _, st = scenes.batch_step(engine, batch, sp, dts[id(batch)])
                assert st == [0] * len(batch)
        for f, b in zip(a_f + b_f, a_b + b_b):
            _states_equal(f, b)
    finally:
        engine.set_batch_fused(True)
        _uniform_batch_shapes(engine, a_f + b_f, 0, 0)


def test_fused_batch_reports_each_scenes_anomalies(engine):
    """Anomalies stay with their scene in the fused form: a particle outside
    one scene's grid (AL_ERR_OUT_OF_GRID), a cell cap of 4 in another
    (AL_ERR_CELL_OVERFLOW) and a neighbor cap of 16 in a third
    (AL_ERR_NEIGHBOR_OVERFLOW: its lists keep the first 16 canonical
    neighbors) give the same per-scene statuses, reports and states as the
    branch form (128-thread blocks, one thread per particle), and the other
    scene AL_OK."""
    def mk():
        out = _scenes(engine)[:4]
        out[1].x[0] = out[1].x.new_tensor([50.0, 50.0, 50.0])
        out[2].cni.max_num_particles_per_cell = 4
        out[3].cni.max_num_neighbors_per_particle = 16
        return out
    fused, branch = mk(), mk()
    sp = scenes.solver_params()
    _uniform_batch_shapes(engine, fused, 128, 1)
    try:
        dts_f, dts_b = [2e-4] * 4, [2e-4] * 4
        for step in range(2):
            engine.set_batch_fused(True)
            dts_f, reps_f, st_f = scenes.batch_step(engine, fused, sp, dts_f,
                                                    allow=_capi.ANOMALY_STATUSES)
            engine.set_batch_fused(False)
            dts_b, reps_b, st_b = scenes.batch_step(engine, branch, sp, dts_b,
                                                    allow=_capi.ANOMALY_STATUSES)
            assert st_f == st_b == [0, _capi.AL_ERR_OUT_OF_GRID, _capi.AL_ERR_CELL_OVERFLOW,
                                    _capi.AL_ERR_NEIGHBOR_OVERFLOW]
            assert dts_f == dts_b
            for rf, rb in zip(reps_f, reps_b):
                assert list(rf.grid_anomaly) == list(rb.grid_anomaly)
                assert rf.num_density_solve == rb.num_density_solve
        for f, b in zip(fused, branch):
            _states_equal(f, b)
    finally:
        engine.set_batch_fused(True)
        _uniform_batch_shapes(engine, fused, 0, 0)


def test_fused_batch_falls_back_for_mixed_constants(engine):
    """A batch whose scenes have different constants (particle radii) runs as
    branches: equal to the same scenes stepped alone, bit for bit."""
    mk = lambda: [scenes.dam_break(engine, np.float32, (10, 8, 10), 0.01, (0.5, 0.4, 0.4), [],
                                   seed=1, volume_resolution=16),
                  scenes.dam_break(engine, np.float32, (12, 10, 12), 0.008, (0.5, 0.4, 0.4), [],
                                   seed=2, volume_resolution=16)]
    batch, single = mk(), mk()
    sp = scenes.solver_params()
    engine.set_batch_fused(True)
    try:
        dts_b, reps_b, status = scenes.batch_step(engine, batch, sp, [2e-4, 2e-4])
    finally:
        engine.set_batch_fused(True)
    assert status == [0, 0]
    for k, sc in enumerate(single):
        dt, rep = sc.step("df", sp, 2e-4)
        assert dt == dts_b[k]
        assert rep.num_density_solve == reps_b[k].num_density_solve
    for b, s in zip(batch, single):
        _states_equal(b, s)


def test_batch_rejects_too_many_scenes(engine):
    arr = (_capi.SceneF32 * 1)()
    st = _capi.lib().al_df_batch_step_f32(engine.handle, arr, 257, None)
    assert st == 2  # AL_ERR_INVALID


@pytest.mark.parametrize("fused,shape", [(True, None), (False, None), (False, (256, 1))])
def test_batch_of_benchmark_scenes_matches_oracle(engine, fused, shape):
    """The four smallest scenes of the 64-scene benchmark batch (seeded, with
    their rigid spheres), stepped as one batch (fused, or as branches), each
    against the oracle's step of the same scene: equal iteration counts and
    the float32 one-step tolerances of the single-step parity tests (the
    jittered start's pressure kick amplifies rounding from the second step
    on).  With shape set, the batch context runs a tuned table (other threads
    per particle than a single step would use)."""
    import bench
    from alluvion_b200 import autotune
    from test_gpu_step import TOL, _close, _oracle_run
    specs = bench.batch_scene_specs(bench.BATCH_WORKLOADS["batch64"])
    chosen = sorted(specs, key=lambda s: s.n)[:4]
    batch = [s.device(engine) for s in chosen]
    groups = _capi.tunable_groups()
    buckets = sorted({autotune.bucket_of(sc.n) for sc in batch})
    engine.set_batch_fused(fused)
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
        engine.set_batch_fused(True)
        for b in buckets:
            for name, _ in groups:
                engine.set_launch_shape(name, b, 1, 0, 0)
