"""CPU checks of the oracle itself, before it is trusted as the checker.

Pins: the Peirce m=14 tables against the reference's literals
(tests/golden/peirce_m14.json, extracted by tests/golden/make_golden.py);
the cubic Lagrange element's defining properties; the cubic spline's
normalisation and gradient; node positions of the reference's own
known-answer setup (tests/field_op.cu:17-58).
"""
import json
import os

import numpy as np
import pytest

from oracle import binding as orc
from alluvion_b200 import scenes, _capi

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_peirce_tables_match_reference_literals():
    ref = json.load(open(os.path.join(GOLDEN, "peirce_m14.json")))["tables"]
    got = orc.peirce_tables()
    for name in ("cosphi", "sinphi", "b", "r", "c"):
        np.testing.assert_allclose(got[name], ref[name], rtol=0, atol=1e-15, err_msg=name)
        # identical once rounded to the solver's float32 constant tables
        assert np.array_equal(np.float32(got[name]), np.float32(ref[name])), name


def test_peirce_rule_integrates_polynomials_on_ball():
    t = orc.peirce_tables()
    # sum over theta of w_theta (2 pi / 60) * b_j * c_k * f(r u) = integral over unit ball
    theta = 2 * np.pi * (np.arange(60) + 1) / 60
    vol = 0.0
    second = 0.0
    for ct, st in zip(np.cos(theta), np.sin(theta)):
        for j in range(30):
            u = np.array([t["sinphi"][j] * ct, t["sinphi"][j] * st, t["cosphi"][j]])
            for k in range(15):
                w = 2 * np.pi * t["b"][j] * t["c"][k] / 60
                p = t["r"][k] * u
                vol += w
                second += w * p[0] ** 2
    assert vol == pytest.approx(4 * np.pi / 3, rel=1e-13)
    assert second == pytest.approx(4 * np.pi / 15, rel=1e-12)


def _node_coords():
    pts = []
    for j in range(8):
        pts.append([1 if j & 1 else -1, 1 if j & 2 else -1, 1 if j & 4 else -1])
    # x-edges: bit0 -> -1/3 | +1/3, bit1 -> z, bit2 -> y
    for e in range(8):
        pts.append([(1 if e & 1 else -1) / 3, 1 if e & 4 else -1, 1 if e & 2 else -1])
    # y-edges: bit1 -> x, bit2 -> z
    for e in range(8):
        pts.append([1 if e & 2 else -1, (1 if e & 1 else -1) / 3, 1 if e & 4 else -1])
    # z-edges: bit1 -> y, bit2 -> x
    for e in range(8):
        pts.append([1 if e & 4 else -1, 1 if e & 2 else -1, (1 if e & 1 else -1) / 3])
    return np.array(pts, dtype=np.float64)


def test_shape_functions_kronecker_and_partition_of_unity():
    nodes = _node_coords()
    for k, p in enumerate(nodes):
        N, _ = orc.shape_functions(p)
        expect = np.zeros(32)
        expect[k] = 1
        np.testing.assert_allclose(N, expect, atol=1e-14)
    rng = np.random.default_rng(1)
    for _ in range(50):
        xi = rng.uniform(-1, 1, 3)
        N, dN = orc.shape_functions(xi)
        assert N.sum() == pytest.approx(1.0, abs=1e-14)
        np.testing.assert_allclose(dN.sum(axis=1), 0, atol=1e-13)


def test_shape_functions_reproduce_cubics_and_gradients():
    nodes = _node_coords()
    rng = np.random.default_rng(2)

    def f(p):
        x, y, z = p
        return 1 + 2 * x - y + 0.5 * z + x * y - 3 * y * z + x * x * z + 2 * x ** 3 - y * y * x

    def grad(p):
        x, y, z = p
        return np.array([2 + y + 2 * x * z + 6 * x * x - y * y,
                         -1 + x - 3 * z - 2 * x * y,
                         0.5 - 3 * y + x * x])

    vals = np.array([f(p) for p in nodes])
    for _ in range(50):
        xi = rng.uniform(-1, 1, 3)
        N, dN = orc.shape_functions(xi)
        assert N @ vals == pytest.approx(f(xi), abs=1e-12)
        np.testing.assert_allclose(dN @ vals, grad(xi), atol=1e-11)


def test_cell_nodes_are_the_reference_corner_and_edge_slots():
    res = np.array([3, 4, 5], np.uint32)
    dmin = np.array([-1.0, 2.0, 0.5])
    cs = np.array([0.5, 0.25, 0.125])
    pos = orc.node_positions(dmin, res, cs, np.float64)
    ref_nodes = _node_coords()
    for ip in ([0, 0, 0], [2, 3, 4], [1, 2, 3]):
        cells = orc.cell_nodes(res, ip)
        lo = dmin + cs * np.array(ip)
        for k in range(32):
            expect = lo + (ref_nodes[k] + 1) / 2 * cs
            np.testing.assert_allclose(pos[cells[k]], expect, atol=1e-12)


def test_node_positions_known_answer():
    """tests/field_op.cu:17-58 setup: domain (-23.1, 12.23, -31.44) ..
    (45.1, 103.2, 12.4), 11^3 cells; every node lies on the vertex/third-point
    lattice of its cell and all nodes are distinct."""
    dmin = np.array([-23.1, 12.23, -31.44])
    dmax = np.array([45.1, 103.2, 12.4])
    res = np.array([11, 11, 11], np.uint32)
    cs = (dmax - dmin) / res
    pos = orc.node_positions(dmin, res, cs, np.float64)
    assert pos.shape[0] == 12 ** 3 + 2 * 3 * 11 * 12 * 12
    frac = (pos - dmin) / cs * 3
    np.testing.assert_allclose(frac, np.round(frac), atol=1e-9)
    assert len({tuple(np.round(f).astype(int)) for f in frac}) == pos.shape[0]
    assert np.all(pos >= dmin - 1e-9) and np.all(pos <= dmax + 1e-9)


def test_cubic_spline_normalised_and_gradient(tmp_path):
    cn = scenes.make_const(np.float64, 0.01)
    h = cn.kernel_radius
    k = cn.cubic_kernel_k

    def W(r):
        q = r / h
        return np.where(q <= 0.5, (6 * q - 6) * q * q + 1,
                        np.where(q <= 1, 2 * (1 - q) ** 3, 0.0)) * k

    r = np.linspace(0, h, 200001)
    integral = np.trapezoid(4 * np.pi * r * r * W(r), r)
    assert integral == pytest.approx(1.0, rel=1e-6)


def _host_scene(dtype, lattice=(6, 6, 6), r=0.01, container=(0.2, 0.2, 0.2), res=8,
                gravity=(0.0, -9.81, 0.0), bodies=True, seed=1):
    cn = scenes.make_const(dtype, r, gravity=gravity)
    x = scenes.fluid_block(lattice, (0, 0, 0), r, dtype, seed=seed)
    size = np.asarray(container, np.float64)
    keep, blist, rig = [], [], []
    if bodies:
        body = scenes.make_body(dtype, cn, _capi.SHAPE_BOX, scenes.box_params(size), res,
                                sign=-1.0)
        vol = orc.volume_field(cn, body, dtype)
        keep.append(vol)
        body.volume_nodes = vol.ctypes.data
        blist.append(body)
        rig.append(scenes.rigid_state(dtype, x=tuple(size / 2)))
    cni = scenes.make_consti(-0.5 * np.asarray(cn.kernel_radius) * np.ones(3),
                             size + 0.5 * cn.kernel_radius, cn.kernel_radius, len(blist))
    arr = (type(blist[0]) * len(blist))(*blist) if blist else []
    n = len(x)
    z = lambda *s: np.zeros(s, dtype)
    state = dict(x=x.copy(), v=z(n, 3), a=z(n, 3), kappa=z(n), kappa_v=z(n), density=z(n),
                 density_adv=z(n), pressure=z(n))
    return cn, cni, arr, scenes.rigid_array(dtype, rig).reshape(-1, 13), state, keep


@pytest.mark.parametrize("method", ["df", "ii", "i"])
def test_oracle_step_conserves_momentum_without_boundaries(method):
    dtype = np.float64
    # pressure terms are pairwise antisymmetric; the reference's viscosity
    # (m / rho_j weighting, runner.hpp:2168-2173) is not, so it is off here
    cn, cni, bodies, rigid, state, keep = _host_scene(dtype, bodies=False,
                                                      gravity=(0.0, 0.0, 0.0))
    cn.viscosity = 0.0
    cni.grid_offset[:] = [-3, -3, -3]
    cni.grid_res[:] = [12, 12, 12]
    rng = np.random.default_rng(0)
    state["v"][:] = rng.normal(0, 0.2, state["v"].shape)
    p0 = state["v"].sum(0)
    dt, reps = orc.run(method, cn, cni, bodies, rigid, state, scenes.solver_params(), 1e-4, 2)
    assert np.abs(state["v"].sum(0) - p0).max() < 1e-10 * np.abs(state["v"]).sum()
    assert all(r.num_density_solve >= 2 for r in reps)


@pytest.mark.parametrize("method", ["df", "ii", "i"])
def test_oracle_step_in_container(method):
    dtype = np.float32
    cn, cni, bodies, rigid, state, keep = _host_scene(dtype)
    sp = scenes.solver_params()
    dt, reps = orc.run(method, cn, cni, bodies, rigid, state, sp, 2e-4, 3)
    for r in reps:
        assert list(r.grid_anomaly) == [0, 0, 0]
        assert 2 <= r.num_density_solve <= 100
        assert 0 < r.dt <= 2e-4
        assert r.num_active_boundary_pairs > 0
    # near-wall particles feel the boundary: no particle leaves the box
    assert state["x"].min() > 0 and state["x"].max() < 0.2
    # the density solve brought the mean density error under the tolerance
    assert reps[-1].mean_density_error <= 1e-3 or reps[-1].num_density_solve == 100


def test_oracle_float32_tracks_float64():
    """The error of the float32 path against the float64 plain method after
    three steps of the 216-particle container scene: positions within 1e-6 m,
    velocities within 1e-3 of their scale."""
    out = {}
    for dtype in (np.float32, np.float64):
        cn, cni, bodies, rigid, state, keep = _host_scene(dtype)
        orc.run("df", cn, cni, bodies, rigid, state, scenes.solver_params(), 2e-4, 3)
        out[dtype] = state
    dx = np.abs(out[np.float32]["x"] - out[np.float64]["x"]).max()
    dv = np.abs(out[np.float32]["v"] - out[np.float64]["v"]).max()
    assert dx < 1e-6
    assert dv < 1e-3 * max(np.abs(out[np.float64]["v"]).max(), 1e-3)


def test_neighbor_list_matches_brute_force():
    cn = scenes.make_const(np.float32, 0.01)
    x = scenes.fluid_block((6, 5, 7), (0, 0, 0), 0.01, np.float32, seed=3)
    cni = scenes.make_consti(x.min(0), x.max(0), cn.kernel_radius)
    density, count, index, nbrs, flags = orc.update_particle_neighbors(cn, cni, x)
    assert not flags.any()
    h2 = np.float32(cn.kernel_radius_sqr)
    d = x[:, None, :] - x[None, :, :]
    d2 = (d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]) + d[..., 2] * d[..., 2]
    for i in range(x.shape[0]):
        expect = set(np.nonzero((d2[i] < h2) & (np.arange(len(x)) != i))[0].tolist())
        got = set(index[i, :count[i]].tolist())
        assert got == expect


@pytest.mark.parametrize("method", ["ii", "i", "df"])
def test_oracle_hydrostatic_column(method):
    """The oracle's steps on the resting water column of
    test_gpu_hydrostatic.py (unjittered 10 x 20 x 10 lattice, outer layers
    2.9 r from the box walls, 1500 steps at dt 2e-4): the column stays near
    rest, its interior at rho0, and for the pressure solvers the stored
    pressure (physical pressure over rho0) grows with depth at about g."""
    dtype = np.float32
    r = 0.01
    lattice = (10, 20, 10)
    gap = 2.9 * r
    cn = scenes.make_const(dtype, r)
    h = float(cn.kernel_radius)
    x = scenes.fluid_block(lattice, (gap - 2 * r,) * 3, r, dtype, jitter=0.0)
    size = 2 * r * (np.asarray(lattice) - 1) + 2 * gap
    size[1] += 0.2
    body = scenes.make_body(dtype, cn, _capi.SHAPE_BOX, scenes.box_params(size), 32, sign=-1.0)
    vol = orc.volume_field(cn, body, dtype)
    body.volume_nodes = vol.ctypes.data
    bodies = (type(body) * 1)(body)
    rigid = scenes.rigid_array(dtype, [scenes.rigid_state(dtype, x=tuple(size / 2))])
    cni = scenes.make_consti(-0.5 * h * np.ones(3), size + 0.5 * h, h, 1)
    n = len(x)
    z = lambda *s: np.zeros(s, dtype)
    st = dict(x=x.copy(), v=z(n, 3), a=z(n, 3), kappa=z(n), kappa_v=z(n), density=z(n),
              density_adv=z(n), pressure=z(n))
    dt, reps = orc.run(method, cn, cni, bodies, rigid.reshape(-1, 13), st,
                       scenes.solver_params(), 2e-4, 1500)
    speed = np.linalg.norm(st["v"], axis=1)
    assert np.percentile(speed, 95) < 0.1
    rho = st["density"]
    dense = rho > 990.0
    assert dense.mean() > 0.9 and abs(rho[dense].mean() / 1000.0 - 1) < 2e-3
    if method == "df":
        return
    xx, p = st["x"], st["pressure"]
    depth = xx[:, 1].max() - xx[:, 1]
    inner = (np.abs(xx[:, 0] - xx[:, 0].mean()) < 0.05) & \
            (np.abs(xx[:, 2] - xx[:, 2].mean()) < 0.05) & (depth > 0.08) & \
            (xx[:, 1] > xx[:, 1].min() + 0.05)
    slope = np.polyfit(depth[inner], p[inner], 1)[0]
    assert slope == pytest.approx(9.81, rel=0.15)


@pytest.mark.parametrize("case", ["container_box", "sphere_analytic", "box_grid"])
def test_lazy_volume_map_equals_eager_build(case):
    """The lazily filled volume map (nodes computed on first use; analytic
    bodies skip nodes 2h outside / h inside the shape) returns the eager
    build's values bit for bit: boundary samples over particles in every
    Lagrange cell are identical, and so is every node they touched."""
    dtype = np.float32
    cn = scenes.make_const(dtype, 0.01)
    h = float(cn.kernel_radius)
    if case == "container_box":
        size = np.array([0.3, 0.2, 0.25])
        body = scenes.make_body(dtype, cn, _capi.SHAPE_BOX, scenes.box_params(size), 10,
                                sign=-1.0)
        rigid_x = size / 2
    elif case == "sphere_analytic":
        body = scenes.make_body(dtype, cn, _capi.SHAPE_SPHERE, [0.05], 8, sign=1.0)
        rigid_x = np.zeros(3)
    else:
        body = scenes.make_body(dtype, cn, _capi.SHAPE_BOX, scenes.box_params((0.06, 0.05, 0.08)),
                                8, sign=1.0, use_distance_grid=True)
        rigid_x = np.zeros(3)
    keep = []
    if body.use_distance_grid:
        dist = orc.distance_grid(body, dtype)
        keep.append(dist)
        body.distance_nodes = dist.ctypes.data
    eager = orc.volume_field(cn, body, dtype)
    lazy = orc.lazy_volume_field(cn, body, dtype)
    try:
        res = np.array(list(body.resolution))
        dmin = np.array(list(body.domain_min), np.float64)
        cs = np.array(list(body.cell_size), np.float64)
        # one particle per cell (cell centre + a small seeded offset), in world coordinates
        idx = np.stack(np.meshgrid(*[np.arange(r) for r in res], indexing="ij"), -1).reshape(-1, 3)
        rng = np.random.default_rng(3)
        local = dmin + (idx + 0.5 + rng.uniform(-0.3, 0.3, idx.shape)) * cs
        x = (local + rigid_x).astype(dtype)
        rigid = np.zeros((1, 13), dtype)
        rigid[0, :3] = rigid_x
        rigid[0, 9] = 1.0
        Body = type(body)
        b_eager = (Body * 1)(body)
        b_eager[0].volume_nodes = eager.ctypes.data
        b_lazy = (Body * 1)(body)
        b_lazy[0].volume_nodes = lazy.ctypes.data
        bnd_e, bk_e = orc.boundary(cn, b_eager, rigid, x)
        bnd_l, bk_l = orc.boundary(cn, b_lazy, rigid, x)
        assert np.array_equal(bnd_e.view(np.uint32), bnd_l.view(np.uint32))
        assert np.array_equal(bk_e.view(np.uint32), bk_l.view(np.uint32))
        # every node belongs to some cell, so every node was computed
        assert np.array_equal(eager.view(np.uint32), lazy.view(np.uint32))
        sampled, skipped = orc.lazy_volume_counts(lazy)
        assert sampled + skipped == body.num_nodes
        if case == "container_box":
            assert skipped > 0  # interior nodes far from the walls need no sampling
        if case == "box_grid":
            assert skipped == 0  # grid distances are always sampled
        assert np.abs(eager).max() > 0.5 * h ** 3
    finally:
        orc.lazy_volume_release(lazy)
