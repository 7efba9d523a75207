"""Distance grids of triangle-mesh bodies built on the device
(al_build_mesh_distance_grid_f32) against the oracle's restatement of
MeshDistance::signedDistance and against analytic shapes.

Bounds: engine vs oracle within 1e-6 + 1e-5 |d| (float32, same algorithm;
FMA contraction on the device).  A closed cube mesh has exactly the box's
signed distance: within 1e-6 of the analytic box SDF.  A subdivided
icosahedron (1280 faces) stays within its chord error (the deepest face
plane below the sphere, < 5e-3 r) of the sphere.  A DFSPH step with a mesh box as a body matches the step with the
analytic box body to the interpolation accuracy of the two grids.
"""
import ctypes

import numpy as np
import pytest
import torch

from alluvion_b200 import _capi, scenes
from oracle import binding as orc

pytestmark = pytest.mark.gpu


def _grid(engine, body, v, f, offset=0.0):
    out = torch.zeros(body.num_nodes, dtype=torch.float32, device="cuda")
    _capi.check(_capi.lib().al_build_mesh_distance_grid_f32(
        engine.handle, _capi.ptr(body), np.ascontiguousarray(v).ctypes.data, len(v),
        np.ascontiguousarray(f).ctypes.data, len(f), ctypes.c_float(offset), _capi.ptr(out),
        None), "al_build_mesh_distance_grid_f32")
    return out.cpu().numpy()


def _positions(engine, body):
    out = torch.zeros((body.num_nodes, 3), dtype=torch.float32, device="cuda")
    _capi.check(_capi.lib().al_node_positions_f32(engine.handle, _capi.ptr(body),
                                                 _capi.ptr(out), None), "positions")
    return out.cpu().numpy().astype(np.float64)


def _body(v, res, offset=0.0):
    cn = scenes.make_const(np.float32, 0.005)
    return scenes.make_body(np.float32, cn, _capi.SHAPE_MESH, [], res, use_distance_grid=True,
                            aabb=scenes.mesh_aabb(v, offset))


def test_cube_mesh_is_the_box_sdf(engine):
    v, f = scenes.cube_mesh(0.05)
    body = _body(v, 12)
    got = _grid(engine, body, v, f)
    ref = orc.mesh_distance_grid(body, v, f)
    np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-6)
    p = _positions(engine, body)
    q = np.abs(p) - 0.05
    box = np.linalg.norm(np.maximum(q, 0), axis=1) + np.minimum(q.max(1), 0)
    np.testing.assert_allclose(got, box, atol=1e-6)
    # the offset shifts every value
    np.testing.assert_allclose(_grid(engine, body, v, f, 0.01), got - 0.01, atol=1e-7)


def test_icosphere_mesh_matches_oracle_and_sphere(engine):
    v, f = scenes.icosphere(0.05, 3)
    body = _body(v, 16)
    got = _grid(engine, body, v, f)
    ref = orc.mesh_distance_grid(body, v, f)
    np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-6)
    p = _positions(engine, body)
    sphere = np.linalg.norm(p, axis=1) - 0.05
    # chord error: the deepest face plane's distance below the sphere
    vv = v.astype(np.float64)
    nrm = np.cross(vv[f[:, 1]] - vv[f[:, 0]], vv[f[:, 2]] - vv[f[:, 0]])
    nrm /= np.linalg.norm(nrm, axis=1)[:, None]
    sagitta = 0.05 - np.einsum("ij,ij->i", nrm, vv[f[:, 0]]).min()
    assert sagitta < 5e-3 * 0.05
    assert np.abs(got - sphere).max() <= sagitta + 1e-6
    assert np.all(np.sign(got[np.abs(sphere) > 1e-3]) == np.sign(sphere[np.abs(sphere) > 1e-3]))


def test_step_with_mesh_body_matches_analytic_body(engine):
    half = 0.04
    v, f = scenes.cube_mesh(half)
    common = dict(sign=1.0, resolution=24, mass=0.2, inertia=scenes.box_inertia(0.2, (0.08,) * 3),
                  x=(0.2, 0.34, 0.16), v=(0.0, -0.2, 0.0))
    mesh_body = dict(shape=_capi.SHAPE_MESH, mesh=(v, f), **common)
    box_body = dict(shape=_capi.SHAPE_BOX, params=scenes.box_params((2 * half,) * 3),
                    use_distance_grid=True, **common)
    sp = scenes.solver_params()
    out = []
    for b in (mesh_body, box_body):
        sc = scenes.dam_break(engine, np.float32, (16, 12, 14), 0.01, (0.45, 0.4, 0.35), [b],
                              seed=4, volume_resolution=16)
        dt = 2e-4
        for _ in range(3):
            dt, rep = sc.step("df", sp, dt)
        out.append((sc.state(), np.array(rep.force[1]), rep.num_active_boundary_pairs))
    (s_m, f_m, n_m), (s_b, f_b, n_b) = out
    assert n_m > 0 and abs(n_m - n_b) <= 0.02 * n_b
    scale = np.abs(s_b["v"]).max()
    assert np.abs(s_m["v"] - s_b["v"]).max() <= 5e-2 * scale
    assert np.linalg.norm(f_m - f_b) <= 5e-2 * np.linalg.norm(f_b) + 1e-6
