"""Rigid-rigid contacts on the device (al_find_contacts_f32,
al_solve_contacts_f32) against the oracle's restatement of
collision_test / Pile::find_contacts / Pile::solve_contacts, on a
container holding an analytic sphere, a sphere and a box with distance
grids, pressed into the floor and into each other.

Both list contacts in (i, j, vertex) order.  Bounds: identical contact
pairs and count; contact points, normals, tangents and congruent matrices
within 1e-4 relative (float32 arithmetic, FMA contraction on the device);
nkninv, goalu within 1e-3, pmax within 1e-2 (1 / t.K.t is ill-conditioned
for short tangents, as the reference notes); velocities after the five
impulse sweeps within 1e-3 of their scale.
"""
import ctypes

import numpy as np
import pytest
import torch

from alluvion_b200 import _capi, scenes
from oracle import binding as orc

pytestmark = pytest.mark.gpu


def _sphere_points(r, n=400):
    k = np.arange(n) + 0.5
    phi = np.arccos(1 - 2 * k / n)
    th = np.pi * (1 + 5 ** 0.5) * k
    return (r * np.stack([np.cos(th) * np.sin(phi), np.cos(phi), np.sin(th) * np.sin(phi)],
                         1)).astype(np.float32)


def _box_points(h, m=10):
    g = np.linspace(-h, h, m)
    pts = []
    for axis in range(3):
        for s in (-h, h):
            a, b = np.meshgrid(g, g)
            p = np.zeros((m * m, 3))
            p[:, axis] = s
            p[:, (axis + 1) % 3] = a.ravel()
            p[:, (axis + 2) % 3] = b.ravel()
            pts.append(p)
    return np.concatenate(pts).astype(np.float32)


def _setup(engine):
    half = 0.04
    bodies = [
        dict(shape=_capi.SHAPE_SPHERE, params=[0.05], sign=1.0, resolution=16,
             use_distance_grid=False, mass=0.5, inertia=scenes.sphere_inertia(0.5, 0.05),
             x=(0.10, 0.045, 0.10), v=(0.0, -0.5, 0.1)),
        dict(shape=_capi.SHAPE_SPHERE, params=[0.05], sign=1.0, resolution=24,
             use_distance_grid=True, mass=0.4, inertia=scenes.sphere_inertia(0.4, 0.05),
             x=(0.185, 0.06, 0.11), v=(-0.3, 0.0, 0.0), omega=(0.0, 1.0, 0.0)),
        dict(shape=_capi.SHAPE_BOX, params=scenes.box_params((0.08, 0.08, 0.08)), sign=1.0,
             resolution=24, use_distance_grid=True, mass=0.3,
             inertia=scenes.box_inertia(0.3, (0.08, 0.08, 0.08)),
             x=(0.33, 0.036, 0.22), v=(0.0, -0.2, 0.0), omega=(0.5, 0.0, 0.2)),
    ]
    sc = scenes.dam_break(engine, np.float32, (4, 4, 4), 0.01, (0.5, 0.4, 0.4), bodies,
                          seed=0, volume_resolution=16)
    verts = [np.zeros((0, 3), np.float32), _sphere_points(0.05), _sphere_points(0.05),
             _box_points(half)]
    return sc, verts


def _contact_bodies(ptrs, counts):
    out = []
    for p, n in zip(ptrs, counts):
        cb = _capi.ContactBodyF32()
        cb.vertices = p
        cb.num_vertices = n
        cb.restitution = 0.8
        cb.friction = 0.1
        out.append(cb)
    return out


def test_contacts_match_oracle(engine):
    sc, verts = _setup(engine)
    nb = sc.num_boundaries
    dev = [torch.from_numpy(v.copy()).cuda() if len(v) else None for v in verts]
    cbs = _contact_bodies([d.data_ptr() if d is not None else None for d in dev],
                          [len(v) for v in verts])
    cb_arr = (_capi.ContactBodyF32 * nb)(*cbs)
    max_c = 4096
    buf = torch.zeros((max_c, _capi.CONTACT_FLOATS), dtype=torch.float32, device="cuda")
    found = ctypes.c_uint32()
    st = _capi.lib().al_find_contacts_f32(engine.handle, _capi.ptr(sc.bodies),
                                          _capi.ptr(sc.rigid), cb_arr, nb, ctypes.c_float(0.0),
                                          max_c, _capi.ptr(buf), ctypes.byref(found), None)
    _capi.check(st, "al_find_contacts_f32")
    n = found.value
    got = (_capi.ContactF32 * n).from_buffer_copy(buf[:n].cpu().numpy().tobytes())
    # oracle with host vertices and nodes
    hb, keep, rigid = sc.host_bodies()
    hbodies = (type(hb[0]) * nb)(*[hb[b] for b in range(nb)])
    hcb = _contact_bodies([v.ctypes.data if len(v) else None for v in verts],
                          [len(v) for v in verts])
    n_ref, ref = orc.find_contacts(hbodies, rigid, hcb, 0.0, max_c)
    assert n == n_ref and n > 20, (n, n_ref)
    pairs = {(c.i, c.j) for c in got[:n]}
    assert {(1, 0), (3, 0), (1, 2), (2, 1)} <= pairs, pairs
    for k in range(n):
        a, b = got[k], ref[k]
        assert (a.i, a.j) == (b.i, b.j), k
        for f in ("cp_i", "cp_j", "n", "t", "iiwi_diag", "iiwi_off_diag"):
            np.testing.assert_allclose(list(getattr(a, f)), list(getattr(b, f)), rtol=1e-4,
                                       atol=1e-5, err_msg="%s of contact %d" % (f, k))
        if b.j != 0:  # the container's inverse inertia is infinite
            for f in ("iiwj_diag", "iiwj_off_diag"):
                np.testing.assert_allclose(list(getattr(a, f)), list(getattr(b, f)),
                                           rtol=1e-4, atol=1e-5, err_msg=f)
        for f, tol in (("nkninv", 1e-3), ("goalu", 1e-3), ("pmax", 1e-2), ("friction", 0)):
            x, y = getattr(a, f), getattr(b, f)
            assert abs(x - y) <= tol * max(abs(y), 1e-6) + 1e-7, (f, k, x, y)
    # five impulse sweeps
    rig_dev = (type(sc.rigid[0]) * nb)(*[sc.rigid[b] for b in range(nb)])
    st = _capi.lib().al_solve_contacts_f32(engine.handle, _capi.ptr(sc.bodies),
                                           ctypes.cast(rig_dev, ctypes.c_void_p), nb,
                                           _capi.ptr(buf), n, None)
    _capi.check(st, "al_solve_contacts_f32")
    rig_ref = rigid.copy()
    orc.solve_contacts(hbodies, rig_ref, ref, n_ref)
    for b in range(1, nb):
        v_ref, w_ref = rig_ref[b][3:6], rig_ref[b][10:13]
        scale = max(np.abs(v_ref).max(), np.abs(w_ref).max(), 1e-3)
        np.testing.assert_allclose(list(rig_dev[b].v), v_ref, atol=1e-3 * scale)
        np.testing.assert_allclose(list(rig_dev[b].omega), w_ref, atol=1e-3 * scale)
    # the solve changed the bodies pressed into the floor
    assert abs(rig_dev[1].v[1] - (-0.5)) > 1e-2


def test_contacts_empty_and_capacity(engine):
    sc, verts = _setup(engine)
    nb = sc.num_boundaries
    dev = [torch.from_numpy(v.copy()).cuda() if len(v) else None for v in verts]
    cbs = _contact_bodies([d.data_ptr() if d is not None else None for d in dev],
                          [len(v) for v in verts])
    cb_arr = (_capi.ContactBodyF32 * nb)(*cbs)
    buf = torch.zeros((8, _capi.CONTACT_FLOATS), dtype=torch.float32, device="cuda")
    found = ctypes.c_uint32()
    # capacity 8: the count still reports every contact found
    _capi.check(_capi.lib().al_find_contacts_f32(
        engine.handle, _capi.ptr(sc.bodies), _capi.ptr(sc.rigid), cb_arr, nb,
        ctypes.c_float(0.0), 8, _capi.ptr(buf), ctypes.byref(found), None), "find")
    assert found.value > 8
    # a large negative tolerance finds nothing
    _capi.check(_capi.lib().al_find_contacts_f32(
        engine.handle, _capi.ptr(sc.bodies), _capi.ptr(sc.rigid), cb_arr, nb,
        ctypes.c_float(-1.0), 8, _capi.ptr(buf), ctypes.byref(found), None), "find")
    assert found.value == 0
