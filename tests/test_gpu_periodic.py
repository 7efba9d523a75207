"""Periodic-in-y steps (the solvers' step<1>, al_solver_params.wrap_y) against
the oracle: a pipe flow -- fluid inside a y-invariant infinite cylinder
(sign -1, sampled with body-frame y = 0 as compute_volume_and_boundary_x_analytic<1>
does), gravity along the pipe axis, a period of 8 cells, and particles that
cross the seam y = -L/2 during the run.  Bounds as for the non-periodic
steps (tests/test_gpu_step.py).  Also: momentum conservation of a slab
periodic in y, without bodies, gravity or viscosity (the pair terms stay
antisymmetric across the seam)."""
import numpy as np
import pytest
import torch

from alluvion_b200 import _capi, scenes
from test_gpu_step import TOL, _close, _oracle_run

pytestmark = pytest.mark.gpu

PERIOD_CELLS = 8


def _pipe(engine, dtype, r=0.01):
    cn = scenes.make_const(dtype, r)
    h = float(cn.kernel_radius)
    L = PERIOD_CELLS * h
    R = 0.12
    centre = 0.15
    g = 2 * r
    a = np.arange(centre - R + 1.5 * r, centre + R - r, g)
    ys = -L / 2 + 1e-4 + g * np.arange(int(round(L / g)))
    X, Y, Z = np.meshgrid(a, ys, a, indexing="ij")
    x = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
    keep = np.hypot(x[:, 0] - centre, x[:, 2] - centre) < R - h  # one h off the wall
    x = x[keep].astype(dtype)
    cni = scenes.make_consti((0.0, -L / 2, 0.0), (0.3, L / 2, 0.3), h)
    cni.grid_offset[1] = -PERIOD_CELLS // 2
    cni.grid_res[1] = PERIOD_CELLS
    pipe = dict(shape=_capi.SHAPE_INFINITE_CYLINDER, params=[R], sign=-1.0, resolution=16,
                use_distance_grid=False, mass=0.0, x=(centre, 0.0, centre))
    scene = scenes.DeviceScene(engine, dtype, cn, cni, x, [pipe])
    # flow down the pipe, fast enough that the lowest layer crosses the seam
    v0 = np.zeros((scene.n, 3), dtype)
    v0[:, 1] = -2.0
    scene.v.copy_(torch.from_numpy(v0).cuda())
    return scene, L


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("method", ["df", "ii", "i"])
def test_periodic_pipe_parity(engine, dtype, method):
    scene, L = _pipe(engine, dtype)
    sp = scenes.solver_params(wrap_y=1, wrap_length=L)
    steps = 3
    dt0 = 1e-4
    ostate, _, odt, oreps = _oracle_run(scene, method, sp, dt0, steps)
    y0 = scene.state()["x"][:, 1].copy()
    dt = dt0
    reps = []
    for _ in range(steps):
        dt, rep = scene.step(method, sp, dt)
        reps.append(rep)
    g = scene.state()
    tol = TOL[(dtype, steps if steps in (1, 4) else 4)]
    for r, o in zip(reps, oreps):
        assert r.num_density_solve == o.num_density_solve
        assert r.num_divergence_solve == o.num_divergence_solve
        assert list(r.grid_anomaly) == [0, 0, 0]
    # particles crossed the seam and came back in at the top
    crossed = (y0 < -L / 2 + 1e-3) & (g["x"][:, 1] > L / 2 - 3e-3)
    assert crossed.sum() > 20
    assert g["x"][:, 1].min() >= -L / 2 and g["x"][:, 1].max() < L / 2
    # positions compare modulo the period (a particle within rounding of the
    # seam may sit on either side)
    dx = g["x"].astype(np.float64) - ostate["x"]
    dx[:, 1] -= L * np.round(dx[:, 1] / L)
    assert np.abs(dx).max() <= tol["x"] * np.abs(ostate["x"]).max()
    _close(g["v"], ostate["v"], tol["v"], "v")
    _close(g["density"], ostate["density"], tol["density"], "density")
    if method == "df":
        _close(g["kappa"], ostate["kappa"], tol["kappa"], "kappa")
    else:
        _close(g["pressure"], ostate["pressure"], tol["kappa"], "pressure")


@pytest.mark.parametrize("method", ["df", "ii", "i"])
def test_periodic_slab_conserves_momentum(engine, method):
    dtype = np.float64
    cn = scenes.make_const(dtype, 0.01, gravity=(0.0, 0.0, 0.0), viscosity=0.0)
    h = float(cn.kernel_radius)
    L = PERIOD_CELLS * h
    x = scenes.fluid_block((10, 16, 10), (0.0, -L / 2 - 0.02 + 0.005, 0.0), 0.01, dtype, seed=3)
    cni = scenes.make_consti((-0.1, -L / 2, -0.1), (0.4, L / 2, 0.4), h, 0)
    cni.grid_offset[1] = -PERIOD_CELLS // 2
    cni.grid_res[1] = PERIOD_CELLS
    scene = scenes.DeviceScene(engine, dtype, cn, cni, x, [])
    rng = np.random.default_rng(5)
    v0 = rng.normal(0, 0.2, size=(scene.n, 3))
    scene.v.copy_(torch.from_numpy(v0).cuda())
    sp = scenes.solver_params(wrap_y=1, wrap_length=L)
    dt = 1e-4
    for _ in range(3):
        dt, rep = scene.step(method, sp, dt)
        assert list(rep.grid_anomaly) == [0, 0, 0]
    p1 = scene.state()["v"].sum(0)
    assert np.abs(p1 - v0.sum(0)).max() < 1e-9 * np.abs(v0).sum()
    # the seam is invisible: the lattice fills the period exactly, so away
    # from the slab's free x / z faces the layers next to the seam have the
    # density of the middle ones
    st = scene.state()
    xs, rho = st["x"], st["density"]
    inner = (np.abs(xs[:, 0] - 0.1) < 0.03) & (np.abs(xs[:, 2] - 0.1) < 0.03)
    seam = inner & (np.abs(xs[:, 1]) > 0.12)
    mid = inner & (np.abs(xs[:, 1]) < 0.05)
    assert seam.sum() > 10 and mid.sum() > 10
    assert abs(rho[seam].mean() / rho[mid].mean() - 1) < 0.01


def test_periodic_step_rejects_bad_length(engine):
    scene, L = _pipe(engine, np.float32)
    sp = scenes.solver_params(wrap_y=1, wrap_length=0.0)
    with pytest.raises(_capi.EngineError):
        scene.step("df", sp, 1e-4)
