"""Launch-shape table of the step's pass groups (al_engine_set_launch_shape)
and the autotuner over it (alluvion_b200.autotune), the counterpart of the
reference's per-kernel block sizes (runner.hpp:4922-4937, bin/block_scan).

Bars: any shape gives the oracle's iteration counts and the float32
one-step tolerances of the step parity tests; at one thread per particle
the block size changes no particle result (bit-identical x, v, density);
batched scenes equal single steps bit for bit when both contexts use the
same shapes."""
import numpy as np
import pytest

from alluvion_b200 import _capi, autotune, scenes
from test_gpu_step import TOL, _close, _oracle_run, _scene

pytestmark = pytest.mark.gpu


def test_shape_api(engine):
    groups = dict(_capi.tunable_groups())
    assert groups["press_iter"] and not groups["neighbors"]
    n = 5000
    b = autotune.bucket_of(n)
    assert engine.launch_shape("press_iter", n) == (128, 8)  # default below 2^17 threads
    engine.set_launch_shape("press_iter", b, 0, 256, 2)
    assert engine.launch_shape("press_iter", n) == (256, 2)
    assert engine.launch_shape("press_iter", n, batch=1) == (128, 8)
    assert engine.launch_shape("press_iter", 40000) == (128, 4)  # another bucket
    engine.set_launch_shape("press_iter", b, 0, 0, 0)
    assert engine.launch_shape("press_iter", n) == (128, 8)
    lib = _capi.lib()
    for args in [(b"no_such_group", 0, 0, 128, 1), (b"press_iter", 0, 0, 96, 1),
                 (b"press_iter", 0, 0, 128, 3), (b"neighbors", 0, 0, 128, 2),
                 (b"press_iter", 32, 0, 128, 1), (b"press_iter", 0, 2, 128, 1)]:
        assert lib.al_engine_set_launch_shape(engine.handle, *args) == _capi.AL_ERR_INVALID


@pytest.mark.parametrize("shape", [(64, 1), (256, 1), (256, 2), (64, 4), (128, 8)])
@pytest.mark.parametrize("method", ["df", "ii", "i"])
def test_step_matches_oracle_under_shapes(engine, shape, method):
    dtype = np.float32
    scene = _scene(engine, dtype)
    b = autotune.bucket_of(scene.n)
    groups = _capi.tunable_groups()
    try:
        for name, pair in groups:
            engine.set_launch_shape(name, b, 0, shape[0], shape[1] if pair else 1)
        sp = scenes.solver_params()
        ostate, _, odt, oreps = _oracle_run(scene, method, sp, 1e-4, 1)
        dt, rep = scene.step(method, sp, 1e-4)
        assert rep.num_density_solve == oreps[0].num_density_solve
        assert rep.num_divergence_solve == oreps[0].num_divergence_solve
        tol = TOL[(dtype, 1)]
        g = scene.state()
        _close(g["x"], ostate["x"], tol["x"], "x")
        _close(g["v"], ostate["v"], tol["v"], "v")
        _close(g["density"], ostate["density"], tol["density"], "density")
        for k in range(1, scene.num_boundaries):
            _close(np.array(rep.force[k]), np.array(oreps[0].force[k]), tol["force"], "force")
    finally:
        for name, _ in groups:
            engine.set_launch_shape(name, b, 0, 0, 0)


def test_block_size_changes_no_particle_result(engine):
    """One thread per particle: every particle sums its list in list order
    whatever the block size, so particle results are bit-identical."""
    groups = _capi.tunable_groups()
    out = []
    for block in (64, 128, 256):
        scene = _scene(engine, np.float32)
        b = autotune.bucket_of(scene.n)
        for name, pair in groups:
            engine.set_launch_shape(name, b, 0, block, 1)
        scene.step("df", scenes.solver_params(), 1e-4)
        out.append(scene.state())
        for name, _ in groups:
            engine.set_launch_shape(name, b, 0, 0, 0)
    for key in ("x", "v", "density", "kappa", "kappa_v"):
        assert np.array_equal(out[0][key], out[1][key]) and np.array_equal(out[0][key],
                                                                           out[2][key]), key


def _batch_scenes(engine):
    out = []
    for k, lat in enumerate([(10, 8, 10), (16, 12, 16), (20, 10, 12)]):
        out.append(scenes.dam_break(engine, np.float32, lat, 0.01, (0.5, 0.4, 0.4), [], seed=k,
                                    volume_resolution=16))
    return out


@pytest.mark.parametrize("fused,shape", [(False, (256, 2)), (True, (128, 1))])
def test_batch_equals_single_steps_with_the_same_shapes(engine, fused, shape):
    """A batch equals its scenes' single steps bit for bit when both run the
    same launch shapes: as branches with any shape set in both contexts; fused
    (whose pair passes always run one thread per particle in 128-thread
    blocks) when the single steps run that shape too."""
    groups = _capi.tunable_groups()
    batch = _batch_scenes(engine)
    single = _batch_scenes(engine)
    buckets = sorted({autotune.bucket_of(sc.n) for sc in batch})
    engine.set_batch_fused(fused)
    try:
        for b in buckets:
            for name, pair in groups:
                for ctx in (0, 1):
                    engine.set_launch_shape(name, b, ctx, shape[0], shape[1] if pair else 1)
        sp = scenes.solver_params()
        dts_b = [2e-4] * 3
        dts_s = [2e-4] * 3
        for _ in range(3):
            dts_b, reps_b, status = scenes.batch_step(engine, batch, sp, dts_b)
            assert status == [0] * 3
            for k, sc in enumerate(single):
                dts_s[k], rep = sc.step("df", sp, dts_s[k])
                assert rep.num_density_solve == reps_b[k].num_density_solve
        for a, s in zip(batch, single):
            sa, ss = a.state(), s.state()
            for key in ("x", "v", "kappa", "kappa_v", "density"):
                np.testing.assert_array_equal(sa[key], ss[key], err_msg=key)
    finally:
        engine.set_batch_fused(True)
        for b in buckets:
            for name, _ in groups:
                for ctx in (0, 1):
                    engine.set_launch_shape(name, b, ctx, 0, 0)


def test_autotune_scene_and_batch(engine, tmp_path):
    """The tuners run, apply their tables (the step then uses the tuned
    shapes; the scene tuner keeps the defaults when its table is slower in
    the step graph) and the table survives a save / load round trip."""
    scene = _scene(engine, np.float32)
    sp = scenes.solver_params()
    table = autotune.tune_scene(engine, scene, sp, steps=2)
    try:
        g = table["graph_ms"]
        if table["kept"] == "tuned":
            assert g["tuned"] < g["default"]
            names = {e["group"] for e in table["entries"]}
            assert {"neighbors", "div_iter", "press_iter", "viscosity"} <= names
        else:
            assert table["kept"] == "default" and g["tuned"] >= g["default"]
            assert table["entries"] == []
        for e in table["entries"]:
            assert engine.launch_shape(e["group"], scene.n) == (e["block"], e["tpp"])
        ostate, _, _, oreps = _oracle_run(scene, "df", sp, 1e-4, 1)
        _, rep = scene.step("df", sp, 1e-4)
        assert rep.num_density_solve == oreps[0].num_density_solve
        _close(scene.state()["x"], ostate["x"], TOL[(np.float32, 1)]["x"], "x")
        path = str(tmp_path / "shapes.json")
        autotune.save(table, path)
        autotune.clear(engine, table)
        assert autotune.load(engine, path)["entries"] == table["entries"]
    finally:
        autotune.clear(engine, table)
    batch = _batch_scenes(engine)
    bt = autotune.tune_batch(engine, batch, sp, steps=2, candidates=[(128, 1), (128, 4)])
    try:
        assert bt["batch_ms_tuned"] <= bt["batch_ms_default"] * 1.5
        assert set(bt["buckets"]) == {str(autotune.bucket_of(sc.n)) for sc in batch}
        dts, reps, status = scenes.batch_step(engine, batch, sp, [2e-4] * 3)
        assert status == [0] * 3
    finally:
        autotune.clear(engine, bt)
