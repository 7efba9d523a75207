"""GPU parity of the Lagrange-grid machinery and boundary sampling against
the oracle, through the C ABI.

Known-answer setups of the reference's own tests are re-run on the engine:
  * tests/field_op.cu:17-58  -- node positions of an 11^3 grid
  * tests/field_gen.cu:16-105 -- volume map of an ellipsoid pseudo-SDF on an
    11^3 grid (h = 1.25, r = 0.25, margin 4h) against host Peirce
    integration, with the reference's doctest::Approx tolerance
    (eps = 100 * FLT_EPSILON, scale 1).
"""
import ctypes

import numpy as np
import pytest
import torch

from alluvion_b200 import _capi, scenes
from oracle import binding as orc
from conftest import dev, host

pytestmark = pytest.mark.gpu

APPROX_EPS = 100 * np.finfo(np.float32).eps


def approx_equal(a, b):
    """doctest::Approx(b) == a with default epsilon and scale 1."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) < APPROX_EPS * (1.0 + np.maximum(np.abs(a), np.abs(b)))


def _lib(name, dtype):
    return getattr(_capi.lib(), name + "_" + _capi.suffix(dtype))


def _grid_body(dtype, dmin, dmax, res, **kw):
    _, BodyT, _, _ = _capi.real_types(dtype)
    b = BodyT()
    b.shape = kw.get("shape", _capi.SHAPE_SPHERE)
    b.use_distance_grid = kw.get("use_distance_grid", 1)
    b.sign = kw.get("sign", 1.0)
    for i, v in enumerate(kw.get("params", [1.0])):
        b.shape_params[i] = v
    T = np.dtype(dtype).type
    for i in range(3):
        b.domain_min[i] = T(dmin[i])
        b.domain_max[i] = T(dmax[i])
        b.cell_size[i] = (T(dmax[i]) - T(dmin[i])) / T(res[i])
        b.resolution[i] = res[i]
    b.num_nodes = scenes.num_grid_nodes(res)
    return b


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_node_positions_field_op(engine, dtype):
    body = _grid_body(dtype, (-23.1, 12.23, -31.44), (45.1, 103.2, 12.4), (11, 11, 11))
    out = torch.zeros(body.num_nodes, 3, dtype=torch.float32 if dtype == np.float32
                      else torch.float64, device="cuda")
    assert _lib("al_node_positions", dtype)(engine.handle, _capi.ptr(body), _capi.ptr(out),
                                            None) == 0
    got = host(out)
    ref = orc.node_positions(np.array(body.domain_min), np.array(body.resolution),
                             np.array(body.cell_size), dtype)
    assert approx_equal(got, ref).all()
    if dtype == np.float64:
        np.testing.assert_allclose(got, ref, rtol=1e-14, atol=1e-12)


def test_volume_field_field_gen(engine):
    """tests/field_gen.cu: ellipsoid pseudo-SDF x^2/25^2 + y^2/15^2 + z^2/35^2 - 1
    sampled on an 11^3 grid; volume map from that distance grid."""
    dtype = np.float32
    r, h = 0.25, 1.25
    margin = 4 * h
    dmin = (-30 - margin, -20 - margin, -40 - margin)
    dmax = (30 + margin, 20 + margin, 40 + margin)
    body = _grid_body(dtype, dmin, dmax, (11, 11, 11), use_distance_grid=1, sign=1.0)
    pos = orc.node_positions(np.array(body.domain_min), np.array(body.resolution),
                             np.array(body.cell_size), dtype)
    dist = (pos[:, 0] ** 2 / 625 + pos[:, 1] ** 2 / 225 + pos[:, 2] ** 2 / 1225 - 1.0)
    dist = dist.astype(dtype)
    cn = scenes.make_const(dtype, r, kernel_radius=h, density0=1.0, particle_mass=0.2)
    dist_d = dev(dist)
    vol_d = torch.zeros(body.num_nodes, dtype=torch.float32, device="cuda")
    body.distance_nodes = dist_d.data_ptr()
    assert _lib("al_build_volume_field", dtype)(engine.handle, _capi.ptr(cn), _capi.ptr(body),
                                                _capi.ptr(vol_d), None) == 0
    got = host(vol_d)
    hb = _grid_body(dtype, dmin, dmax, (11, 11, 11), use_distance_grid=1, sign=1.0)
    hb.distance_nodes = dist.ctypes.data
    ref = orc.volume_field(cn, hb, dtype)
    ok = approx_equal(got, ref)
    assert ok.all(), (np.argwhere(~ok)[:5], got[~ok][:5], ref[~ok][:5])
    assert got.max() > 1.0  # the map is not trivially zero
    # full-ball nodes deep inside integrate the whole kernel support
    assert got.max() == pytest.approx(4.0 / 3.0 * np.pi * h ** 3, rel=1e-3)


@pytest.mark.parametrize("shape,params,sign", [
    (_capi.SHAPE_BOX, [0.3, 0.2, 0.25, 0.0], -1.0),
    (_capi.SHAPE_SPHERE, [0.05], 1.0),
    (_capi.SHAPE_BOX_SHELL, [0.2, 0.15, 0.2, 0.22, 0.17, 0.22, 0.0], 1.0),
    (_capi.SHAPE_TORUS, [0.06, 0.02], 1.0),
    (_capi.SHAPE_CYLINDER, [0.04, 0.1, 0.01], 1.0),
    (_capi.SHAPE_CAPSULE, [0.03, 0.08], 1.0),
    (_capi.SHAPE_INFINITE_CYLINDER, [0.05], -1.0),
    (_capi.SHAPE_INFINITE_TUBE, [0.04, 0.07, 0.05], 1.0),
])
def test_analytic_volume_and_distance_grid(engine, shape, params, sign):
    dtype = np.float32
    cn = scenes.make_const(dtype, 0.005)
    body = scenes.make_body(dtype, cn, shape, params, 12, sign=sign)
    vol_d = torch.zeros(body.num_nodes, device="cuda")
    dist_d = torch.zeros(body.num_nodes, device="cuda")
    assert _lib("al_build_distance_grid", dtype)(engine.handle, _capi.ptr(body),
                                                 _capi.ptr(dist_d), None) == 0
    assert _lib("al_build_volume_field", dtype)(engine.handle, _capi.ptr(cn), _capi.ptr(body),
                                                _capi.ptr(vol_d), None) == 0
    np.testing.assert_allclose(host(dist_d), orc.distance_grid(body, dtype), rtol=1e-5,
                               atol=1e-7)
    ref = orc.volume_field(cn, body, dtype)
    assert approx_equal(host(vol_d), ref).all()


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_particle_boundary_parity(engine, dtype):
    """compute_all_boundaries for a container box (analytic, sign -1) and
    rotated grid-sampled sphere and box bodies."""
    container = (0.4, 0.3, 0.3)
    bodies = [
        dict(shape=_capi.SHAPE_SPHERE, params=[0.04], sign=1.0, resolution=16,
             use_distance_grid=True, mass=1.0, x=(0.15, 0.12, 0.15)),
        dict(shape=_capi.SHAPE_BOX, params=scenes.box_params((0.06, 0.05, 0.07)), sign=1.0,
             resolution=16, use_distance_grid=True, mass=1.0, x=(0.28, 0.1, 0.14),
             q=(0.1, 0.3, -0.2, 0.927)),
    ]
    q = np.array(bodies[1]["q"])
    bodies[1]["q"] = tuple(q / np.linalg.norm(q))
    scene = scenes.dam_break(engine, dtype, (16, 14, 14), 0.01, container, bodies, seed=5,
                             volume_resolution=16)
    n, nb = scene.n, scene.num_boundaries
    T = scene.tdtype
    bnd = torch.zeros(nb, n, 4, dtype=T, device="cuda")
    bk = torch.zeros(nb, n, 4, dtype=T, device="cuda")
    status = _lib("al_compute_particle_boundary", dtype)(
        engine.handle, _capi.ptr(scene.cn), nb, _capi.ptr(scene.bodies), _capi.ptr(scene.rigid),
        _capi.ptr(scene.x), n, _capi.ptr(bnd), _capi.ptr(bk), None)
    assert status == 0
    hb, keep, rigid = scene.host_bodies()
    o_bnd, o_bk = orc.boundary(scene.cn, (type(hb[0]) * nb)(*[hb[b] for b in range(nb)]),
                               rigid, host(scene.x))
    g_bnd, g_bk = host(bnd), host(bk)
    tol = 1e-5 if dtype == np.float32 else 1e-11
    for b in range(nb):
        np.testing.assert_allclose(g_bnd[b], o_bnd[b], rtol=tol, atol=tol * 0.5)
        scale = np.abs(o_bk[b]).max() + 1e-30
        np.testing.assert_allclose(g_bk[b], o_bk[b], rtol=tol * 10, atol=tol * scale)
        # active sets (V != 0) agree exactly
        assert np.array_equal(g_bnd[b][:, 3] != 0, o_bnd[b][:, 3] != 0)
    assert (o_bnd[0][:, 3] != 0).sum() > 100  # the walls are felt
    assert (o_bnd[1][:, 3] != 0).sum() > 10 and (o_bnd[2][:, 3] != 0).sum() > 10


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_particle_boundary_new_shapes(engine, dtype):
    """Cylinder and capsule (grid-sampled and analytic), and the y-invariant
    infinite cylinder (a pipe, fluid inside) and infinite tube, sampled as
    compute_volume_and_boundary_x_analytic<1> does (body-frame y set to 0)."""
    bodies = [
        dict(shape=_capi.SHAPE_CYLINDER, params=[0.035, 0.08, 0.005], sign=1.0, resolution=16,
             use_distance_grid=True, mass=1.0, x=(0.1, 0.1, 0.1), q=(0.0, 0.0, 0.38268343,
                                                                    0.92387953)),
        dict(shape=_capi.SHAPE_CAPSULE, params=[0.03, 0.06], sign=1.0, resolution=16,
             use_distance_grid=False, mass=1.0, x=(0.27, 0.12, 0.2)),
        dict(shape=_capi.SHAPE_INFINITE_CYLINDER, params=[0.14], sign=-1.0, resolution=12,
             use_distance_grid=False, mass=0.0, x=(0.15, 0.15, 0.15)),
        dict(shape=_capi.SHAPE_INFINITE_TUBE, params=[0.02, 0.035, 0.05], sign=1.0,
             resolution=12, use_distance_grid=False, mass=0.0, x=(0.2, 0.2, 0.1)),
    ]
    scene = scenes.dam_break(engine, dtype, (14, 14, 14), 0.01, (0.3, 0.3, 0.3), bodies,
                             seed=6, volume_resolution=12)
    n, nb = scene.n, scene.num_boundaries
    T = scene.tdtype
    bnd = torch.zeros(nb, n, 4, dtype=T, device="cuda")
    bk = torch.zeros(nb, n, 4, dtype=T, device="cuda")
    status = _lib("al_compute_particle_boundary", dtype)(
        engine.handle, _capi.ptr(scene.cn), nb, _capi.ptr(scene.bodies), _capi.ptr(scene.rigid),
        _capi.ptr(scene.x), n, _capi.ptr(bnd), _capi.ptr(bk), None)
    assert status == 0
    hb, keep, rigid = scene.host_bodies()
    o_bnd, o_bk = orc.boundary(scene.cn, (type(hb[0]) * nb)(*[hb[b] for b in range(nb)]),
                               rigid, host(scene.x))
    g_bnd, g_bk = host(bnd), host(bk)
    tol = 1e-5 if dtype == np.float32 else 1e-11
    for b in range(1, nb):
        # boundary points of particles the body does not reach (V = 0) come
        # from finite-difference normals far from the surface, noisy in
        # float32; the active ones are compared at the full bound
        act = o_bnd[b][:, 3] != 0
        np.testing.assert_allclose(g_bnd[b][act], o_bnd[b][act], rtol=tol, atol=tol * 0.5,
                                   err_msg="body %d" % b)
        np.testing.assert_allclose(g_bnd[b][~act], o_bnd[b][~act], rtol=1e-3, atol=1e-4,
                                   err_msg="body %d (inactive)" % b)
        scale = np.abs(o_bk[b]).max() + 1e-30
        np.testing.assert_allclose(g_bk[b], o_bk[b], rtol=tol * 10, atol=tol * scale,
                                   err_msg="body %d" % b)
        assert np.array_equal(g_bnd[b][:, 3] != 0, o_bnd[b][:, 3] != 0)
        assert (o_bnd[b][:, 3] != 0).sum() > 10, b
    # the pipe's boundary points lie on its cylinder (radius 0.14 about the
    # body's y axis) for particles that feel it
    act = o_bnd[3][:, 3] != 0
    r = np.hypot(g_bnd[3][act, 0] - 0.15, g_bnd[3][act, 2] - 0.15)
    np.testing.assert_allclose(r, 0.14, atol=1e-4)


def test_y_invariant_shapes_reject_distance_grids(engine):
    dtype = np.float32
    cn = scenes.make_const(dtype, 0.01)
    body = scenes.make_body(dtype, cn, _capi.SHAPE_INFINITE_CYLINDER, [0.1], 8,
                            use_distance_grid=True)
    out = torch.zeros(body.num_nodes, device="cuda")
    body.volume_nodes = out.data_ptr()
    body.distance_nodes = out.data_ptr()
    assert _lib("al_build_volume_field", dtype)(engine.handle, _capi.ptr(cn), _capi.ptr(body),
                                                _capi.ptr(out), None) == _capi.AL_ERR_INVALID
