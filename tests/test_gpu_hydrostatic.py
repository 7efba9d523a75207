"""Physical invariant: a water column at rest in a box container (the
hydrostatic column test).  No reference test covers the steps' physics;
this pins them beyond the oracle restatement.

Scene: an unjittered 10 x 20 x 10 lattice at spacing 2r (its interior
density is rho0 to 3e-5) whose outer layers sit 2.9 r from the walls, where
the volume-map wall term (update_volume_field, runner.hpp:1617-1658) plus
the half-lattice sum gives rho0, so the column starts close to rest.  A
jittered or wall-offset start is far from equilibrium: DFSPH removes a
density error in one step, so a 4 % error becomes a kick of metres per
second at dt = 2e-4.

After 1500 steps (0.3 s) the column is near rest and its interior at rho0.
For IISPH (SolverIi) and implicit SPH (SolverI) the stored pressure grows
linearly with depth at rate g: compute_pressure_accels
(runner.hpp:2774-2817) scales -sum m (p_i/rho_i^2 + p_j/rho_j^2) gradW by
density0, so the stored p is the physical pressure over rho0.  The fitted
slope is about 8 % above g at this resolution (the oracle gives 10.6 for
IISPH and 10.7 for implicit SPH); the bound is 15 %.  DFSPH's kappa is a
stiffness, so for it the rest state and density are checked."""
import numpy as np
import pytest

from alluvion_b200 import _capi, scenes

pytestmark = pytest.mark.gpu

R = 0.01
LATTICE = (10, 20, 10)
WALL_GAP = 2.9 * R


def _column(engine, dtype=np.float32):
    cn = scenes.make_const(dtype, R)
    h = float(cn.kernel_radius)
    x = scenes.fluid_block(LATTICE, (WALL_GAP - 2 * R,) * 3, R, dtype, jitter=0.0)
    size = 2 * R * (np.asarray(LATTICE) - 1) + 2 * WALL_GAP
    size[1] += 0.2
    cont = dict(shape=_capi.SHAPE_BOX, params=scenes.box_params(size), sign=-1.0,
                resolution=32, use_distance_grid=False, mass=0.0, x=tuple(size / 2))
    cni = scenes.make_consti(-0.5 * h * np.ones(3), size + 0.5 * h, h, 1)
    return scenes.DeviceScene(engine, dtype, cn, cni, x, [cont])


@pytest.mark.parametrize("method", ["ii", "i", "df"])
def test_hydrostatic_column(engine, method):
    sc = _column(engine)
    sp = scenes.solver_params()
    dt = 2e-4
    for _ in range(1500):
        dt, rep = sc.step(method, sp, dt)
        assert list(rep.grid_anomaly) == [0, 0, 0]
    st = sc.state()
    x, v, rho = st["x"], st["v"], st["density"]
    speed = np.linalg.norm(v, axis=1)
    # near rest: only the particles on the vertical edges still slide
    assert np.percentile(speed, 95) < 0.1, np.percentile(speed, 95)
    assert speed.max() < 0.5
    # the interior is at rest density; the free surface and edges are below
    dense = rho > 990.0
    assert dense.mean() > 0.9
    assert abs(rho[dense].mean() / 1000.0 - 1) < 2e-3
    assert rho.max() < 1010.0
    if method == "df":
        return
    p = st["pressure"]
    depth = x[:, 1].max() - x[:, 1]
    cx, cz = x[:, 0].mean(), x[:, 2].mean()
    inner = (np.abs(x[:, 0] - cx) < 0.05) & (np.abs(x[:, 2] - cz) < 0.05) & \
            (depth > 0.08) & (x[:, 1] > x[:, 1].min() + 0.05)
    assert inner.sum() > 200
    slope, intercept = np.polyfit(depth[inner], p[inner], 1)
    assert slope == pytest.approx(9.81, rel=0.15), (slope, intercept)
