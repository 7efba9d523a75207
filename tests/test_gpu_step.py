"""GPU parity of whole solver steps against the oracle, through the C ABI:
SolverDf::step<0> (solver_df.hpp:74-359), SolverIi::step<0>
(solver_ii.hpp:76-243) and SolverI::step<0> (solver_i.hpp:79-327), all
without contacts, on seeded dam-break scenes with a container and two-way
coupled rigid bodies.

Tolerances (stated per quantity, relative to the quantity's scale; float32
differences come from FMA contraction and summation order of the same
formulas, amplified by the Jacobi solves):
  float32 after 1 step: x 1e-5, v / density 1e-3, kappa 1e-2, rigid force 1e-2
  float32 after 4 steps: x 5e-5, v 1e-2, kappa 5e-2
  float64 after 1..4 steps: 1e-11 .. 1e-6 (see TOL)
Iteration counts must match exactly; the engine reduces the convergence
means deterministically in double, the oracle sequentially in double.
"""
import numpy as np
import pytest
import torch

from alluvion_b200 import _capi, scenes
from oracle import binding as orc

pytestmark = pytest.mark.gpu


def _scene(engine, dtype, seed=3, bodies=True, lattice=(14, 12, 12)):
    container = (0.45, 0.4, 0.35)
    extra = []
    if bodies:
        extra = [
            dict(shape=_capi.SHAPE_SPHERE, params=[0.035], sign=1.0, resolution=16,
                 use_distance_grid=True, mass=0.12, inertia=scenes.sphere_inertia(0.12, 0.035),
                 x=(0.14, 0.32, 0.13), v=(0.0, -0.3, 0.0)),
            dict(shape=_capi.SHAPE_BOX, params=scenes.box_params((0.05, 0.04, 0.06)), sign=1.0,
                 resolution=16, use_distance_grid=True, mass=0.1,
                 inertia=scenes.box_inertia(0.1, (0.05, 0.04, 0.06)),
                 x=(0.3, 0.33, 0.24), omega=(0.5, 0.0, 1.0)),
        ]
    scene = scenes.dam_break(engine, dtype, lattice, 0.01, container, extra, seed=seed,
                             volume_resolution=16)
    # a little initial motion so every term is exercised
    rng = np.random.default_rng(seed)
    v0 = rng.normal(0, 0.02, size=(scene.n, 3)).astype(dtype)
    scene.v.copy_(torch.from_numpy(v0).cuda())
    return scene


def _oracle_run(scene, method, sp, dt, steps):
    hb, keep, rigid = scene.host_bodies()
    st = scene.state()
    state = {k: np.ascontiguousarray(st[k]) for k in ("x", "v", "kappa", "kappa_v", "density",
                                                       "density_adv", "a", "pressure")}
    nb = scene.num_boundaries
    bodies = (type(hb[0]) * max(nb, 1))(*[hb[b] for b in range(nb)]) if nb else hb
    dt_out, reps = orc.run(method, scene.cn, scene.cni, bodies if nb else [], rigid, state, sp,
                           dt, steps)
    return state, rigid, dt_out, reps


def _close(a, b, rel, what):
    scale = max(np.abs(b).max(), 1e-30)
    err = np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)).max() / scale
    assert err <= rel, "%s: max error %.3e of scale %.3e (bound %.1e)" % (what, err, scale, rel)


TOL = {
    (np.float32, 1): dict(x=1e-5, v=1e-3, density=1e-3, kappa=1e-2, force=1e-2, dt=1e-5),
    (np.float32, 4): dict(x=5e-5, v=1e-2, density=5e-3, kappa=5e-2, force=5e-2, dt=1e-4),
    (np.float64, 1): dict(x=1e-12, v=1e-9, density=1e-11, kappa=1e-8, force=1e-7, dt=1e-9),
    (np.float64, 4): dict(x=1e-11, v=1e-8, density=1e-10, kappa=1e-7, force=1e-6, dt=1e-9),
}


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("steps", [1, 4])
@pytest.mark.parametrize("method", ["df", "ii", "i"])
def test_step_parity(engine, dtype, steps, method):
    scene = _scene(engine, dtype)
    sp = scenes.solver_params()
    dt0 = 1e-4
    ostate, origid, odt, oreps = _oracle_run(scene, method, sp, dt0, steps)
    dt = dt0
    reps = []
    for _ in range(steps):
        dt, rep = scene.step(method, sp, dt)
        reps.append(rep)
    g = scene.state()
    tol = TOL[(dtype, steps)]
    for r, o in zip(reps, oreps):
        assert r.num_density_solve == o.num_density_solve
        assert r.num_divergence_solve == o.num_divergence_solve
        assert list(r.grid_anomaly) == [0, 0, 0]
        assert r.dt == pytest.approx(o.dt, rel=tol["dt"])
    assert dt == pytest.approx(odt, rel=tol["dt"])
    _close(g["x"], ostate["x"], tol["x"], "x")
    _close(g["v"], ostate["v"], tol["v"], "v")
    _close(g["density"], ostate["density"], tol["density"], "density")
    if method == "df":
        _close(g["kappa"], ostate["kappa"], tol["kappa"], "kappa")
        _close(g["kappa_v"], ostate["kappa_v"], tol["kappa"], "kappa_v")
    else:
        _close(g["pressure"], ostate["pressure"], tol["kappa"], "pressure")
    grig = scenes.rigid_array(dtype, [scene.rigid[b] for b in range(scene.num_boundaries)])
    _close(grig[:, :3], origid[:, :3], tol["x"] * 10, "rigid x")
    for b in range(1, scene.num_boundaries):
        _close(np.array(reps[-1].force[b]), np.array(oreps[-1].force[b]), tol["force"],
               "rigid force %d" % b)


@pytest.mark.parametrize("method", ["df", "ii", "i"])
def test_step_without_bodies_conserves_momentum(engine, method):
    """Free blob, g = 0, no boundaries, viscosity 0: the pressure pair terms are
    antisymmetric, so total momentum is conserved (the reference's viscosity
    weights by 1/rho_j and is not antisymmetric, runner.hpp:2168-2173)."""
    dtype = np.float64
    cn = scenes.make_const(dtype, 0.01, gravity=(0.0, 0.0, 0.0), viscosity=0.0)
    x = scenes.fluid_block((10, 10, 10), (0, 0, 0), 0.01, dtype, seed=1)
    cni = scenes.make_consti(x.min(0) - 0.1, x.max(0) + 0.1, cn.kernel_radius, 0)
    scene = scenes.DeviceScene(engine, dtype, cn, cni, x, [])
    rng = np.random.default_rng(2)
    v0 = rng.normal(0, 0.2, size=(scene.n, 3))
    scene.v.copy_(torch.from_numpy(v0).cuda())
    p0 = v0.sum(0)
    sp = scenes.solver_params()
    dt = 1e-4
    for _ in range(3):
        dt, rep = scene.step(method, sp, dt)
    p1 = scene.state()["v"].sum(0)
    assert np.abs(p1 - p0).max() < 1e-9 * np.abs(v0).sum()


def test_iteration_caps_and_disabled_solves(engine):
    dtype = np.float32
    scene = _scene(engine, dtype, bodies=False)
    sp = scenes.solver_params(max_density_solve=3, min_density_solve=3,
                              max_divergence_solve=2, min_divergence_solve=2)
    ostate, _, _, oreps = _oracle_run(scene, "df", sp, 1e-4, 1)
    _, rep = scene.step("df", sp, 1e-4)
    assert rep.num_density_solve == 3 == oreps[0].num_density_solve
    assert rep.num_divergence_solve == 2 == oreps[0].num_divergence_solve
    _close(scene.state()["x"], ostate["x"], 1e-5, "x")
    scene2 = _scene(engine, dtype, bodies=False)
    sp2 = scenes.solver_params(enable_divergence_solve=0, enable_density_solve=0)
    ostate2, _, _, oreps2 = _oracle_run(scene2, "df", sp2, 1e-4, 1)
    _, rep2 = scene2.step("df", sp2, 1e-4)
    assert rep2.num_density_solve == 0 and rep2.num_divergence_solve == 0
    _close(scene2.state()["v"], ostate2["v"], 1e-3, "v")


@pytest.mark.parametrize("iterations", [0, 1, 2, 3])
def test_implicit_sph_iteration_counts(engine, iterations):
    """SolverI with exactly K Jacobi iterations: the engine alternates its two
    pressure arrays by iteration parity, the reference copies; K = 0 keeps
    the previous step's pressure for the accelerations."""
    dtype = np.float32
    scene = _scene(engine, dtype)
    scene.pressure.copy_(torch.linspace(0.0, 50.0, scene.n, device="cuda"))
    sp = scenes.solver_params(min_density_solve=iterations, max_density_solve=iterations)
    ostate, _, _, oreps = _oracle_run(scene, "i", sp, 1e-4, 1)
    _, rep = scene.step("i", sp, 1e-4)
    assert rep.num_density_solve == iterations == oreps[0].num_density_solve
    g = scene.state()
    _close(g["pressure"], ostate["pressure"], 1e-2, "pressure")
    _close(g["x"], ostate["x"], 1e-5, "x")
    _close(g["v"], ostate["v"], 1e-3, "v")


def test_empty_fluid_step(engine):
    dtype = np.float32
    cn = scenes.make_const(dtype, 0.01)
    x = np.zeros((0, 3), dtype)
    cni = scenes.make_consti((0, 0, 0), (0.2, 0.2, 0.2), cn.kernel_radius, 0)
    scene = scenes.DeviceScene(engine, dtype, cn, cni, x, [])
    dt, rep = scene.step("df", scenes.solver_params(), 1e-4)
    assert dt == pytest.approx(1e-4)


@pytest.mark.parametrize("method", ["df", "ii", "i"])
def test_step_parity_with_truncated_neighbor_lists(engine, method):
    """max_num_neighbors_per_particle below the lattice's ~30 neighbors: the
    reference keeps the first `cap` candidates in its scan order and flags
    grid_anomaly[2] (runner.hpp:1896-1909); every pass of the step then
    sums over the truncated (asymmetric) lists.  The engine keeps the same
    entries, reports AL_ERR_NEIGHBOR_OVERFLOW after writing its outputs, and
    the step matches the oracle's truncated step within the float32
    four-step bounds."""
    dtype = np.float32
    extra = [dict(shape=_capi.SHAPE_SPHERE, params=[0.035], sign=1.0, resolution=16,
                  use_distance_grid=True, mass=0.12, inertia=scenes.sphere_inertia(0.12, 0.035),
                  x=(0.14, 0.32, 0.13), v=(0.0, -0.3, 0.0))]
    scene = scenes.dam_break(engine, dtype, (12, 10, 10), 0.01, (0.45, 0.4, 0.35), extra,
                             seed=9, volume_resolution=16, max_num_neighbors_per_particle=20)
    sp = scenes.solver_params()
    steps = 2
    ostate, origid, odt, oreps = _oracle_run(scene, method, sp, 1e-4, steps)
    dt = 1e-4
    reps = []
    for _ in range(steps):
        dt, rep = scene.step(method, sp, dt, allow=(_capi.AL_ERR_NEIGHBOR_OVERFLOW,))
        reps.append(rep)
    for r, o in zip(reps, oreps):
        assert list(r.grid_anomaly) == [0, 0, 1] and list(o.grid_anomaly) == [0, 0, 1]
        assert r.num_density_solve == o.num_density_solve
        assert r.num_divergence_solve == o.num_divergence_solve
    tol = TOL[(dtype, 4)]
    g = scene.state()
    _close(g["x"], ostate["x"], tol["x"], "x")
    _close(g["v"], ostate["v"], tol["v"], "v")
    _close(g["density"], ostate["density"], tol["density"], "density")
