"""Pellet relaxation (al_relax_pellets_*, SolverPellet<TF>::step) against the
oracle's restatement, through the C ABI: particles spread inside a sphere
(analytic branch, sign -1 so the inside is the allowed side) and inside a
closed cube mesh (distance-grid branch).  Bounds relative to the scene
size: positions within 2e-5 after 1 step and 2e-4 after 3 (float32; the
device uses the hardware reciprocal square root where the oracle divides),
displacements within 1e-3 of their scale, densities within 1e-5.  Known
property of move_and_avoid_boundary: after a step every particle is at
least one particle radius inside the body (up to rounding)."""
import ctypes

import numpy as np
import pytest
import torch

from alluvion_b200 import _capi, scenes
from oracle import binding as orc

pytestmark = pytest.mark.gpu


def _lattice_in_sphere(R, spacing, seed):
    m = int(np.ceil(R / spacing))
    a = spacing * (np.arange(-m, m + 1) + 0.25)
    g = np.stack(np.meshgrid(a, a, a, indexing="ij"), -1).reshape(-1, 3)
    g = g[np.linalg.norm(g, axis=1) < R - 1.5 * spacing]
    rng = np.random.Generator(np.random.PCG64(seed))
    return (g + rng.uniform(-0.2, 0.2, g.shape) * spacing).astype(np.float32)


def _run(engine, cn, cni, body, x, params, steps):
    X = torch.from_numpy(x.copy()).cuda()
    DX = torch.zeros_like(X)
    RHO = torch.zeros(len(x), device="cuda")
    st = _capi.lib().al_relax_pellets_f32(engine.handle, _capi.ptr(cn), _capi.ptr(cni),
                                          _capi.ptr(body), X.data_ptr(), len(x),
                                          _capi.ptr(params), steps, DX.data_ptr(),
                                          RHO.data_ptr(), None)
    _capi.check(st, "al_relax_pellets_f32")
    return X.cpu().numpy(), DX.cpu().numpy(), RHO.cpu().numpy()


@pytest.mark.parametrize("steps,tol", [(1, 2e-5), (3, 2e-4)])
def test_relax_in_sphere_matches_oracle(engine, steps, tol):
    dtype = np.float32
    cn = scenes.make_const(dtype, 0.01)
    R = 0.2
    body = scenes.make_body(dtype, cn, _capi.SHAPE_SPHERE, [R], 8, sign=-1.0)
    cni = scenes.make_consti((-R - 0.05,) * 3, (R + 0.05,) * 3, float(cn.kernel_radius))
    x = _lattice_in_sphere(R, 0.02, seed=2)
    p = _capi.pellet_relax_params()
    gx, gdx, grho = _run(engine, cn, cni, body, x, p, steps)
    ox, odx, orho, over = orc.relax_pellets(cn, cni, body, x, p, steps)
    assert not over
    assert np.abs(gx - ox).max() <= tol * R, np.abs(gx - ox).max()
    assert np.abs(gdx - odx).max() <= 1e-3 * np.abs(odx).max() + 1e-7
    np.testing.assert_allclose(grho, orho, rtol=1e-5)
    # the particles moved, and every one stays r inside the sphere
    assert np.abs(gx - x).max() > 1e-4
    r = float(cn.particle_radius)
    assert (R - np.linalg.norm(gx, axis=1)).min() >= r - 1e-5


def test_relax_in_mesh_cube_matches_oracle(engine):
    dtype = np.float32
    cn = scenes.make_const(dtype, 0.01)
    half = 0.15
    verts, faces = scenes.cube_mesh(half)
    # the fluid side is the inside: sign -1 on the mesh distance
    body = scenes.make_body(dtype, cn, _capi.SHAPE_MESH, [], 20, sign=-1.0,
                            use_distance_grid=True, aabb=scenes.mesh_aabb(verts))
    nodes = torch.zeros(body.num_nodes, device="cuda")
    v = np.ascontiguousarray(verts, np.float32)
    f = np.ascontiguousarray(faces, np.uint32)
    _capi.check(_capi.lib().al_build_mesh_distance_grid_f32(
        engine.handle, _capi.ptr(body), v.ctypes.data, len(v), f.ctypes.data, len(f),
        ctypes.c_float(0.0), _capi.ptr(nodes), None), "mesh grid")
    body.distance_nodes = nodes.data_ptr()
    cni = scenes.make_consti((-half - 0.05,) * 3, (half + 0.05,) * 3, float(cn.kernel_radius))
    rng = np.random.Generator(np.random.PCG64(4))
    x = rng.uniform(-half + 0.02, half - 0.02, size=(2500, 3)).astype(np.float32)
    p = _capi.pellet_relax_params()
    gx, gdx, grho = _run(engine, cn, cni, body, x, p, 1)
    # the oracle reads the same grid from host memory
    hb = type(body).from_buffer_copy(body)
    hn = nodes.cpu().numpy()
    hb.distance_nodes = hn.ctypes.data
    ox, odx, orho, over = orc.relax_pellets(cn, cni, hb, x, p, 1)
    assert np.abs(gx - ox).max() <= 2e-5 * half
    np.testing.assert_allclose(grho, orho, rtol=1e-5)
    r = float(cn.particle_radius)
    assert (half - np.abs(gx).max(axis=1)).min() >= r - 1e-4


def test_relax_rejects_unknown_shape(engine):
    dtype = np.float32
    cn = scenes.make_const(dtype, 0.01)
    body = scenes.make_body(dtype, cn, _capi.SHAPE_SPHERE, [0.1], 8)
    body.shape = 99
    cni = scenes.make_consti((-0.2,) * 3, (0.2,) * 3, float(cn.kernel_radius))
    x = _lattice_in_sphere(0.1, 0.02, 1)
    X = torch.from_numpy(x).cuda()
    st = _capi.lib().al_relax_pellets_f32(engine.handle, _capi.ptr(cn), _capi.ptr(cni),
                                          _capi.ptr(body), X.data_ptr(), len(x),
                                          _capi.ptr(_capi.pellet_relax_params()), 1, None, None,
                                          None)
    assert st == _capi.AL_ERR_INVALID
