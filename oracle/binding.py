"""ctypes binding of the CPU oracle (test infrastructure only).

All arrays are host numpy arrays in the reference's layouts.  The library is
compiled on first use when missing (g++ is part of the image).
"""
import ctypes

import numpy as np

from . import build as _build

_lib = None
_P = ctypes.c_void_p
_U = ctypes.c_uint32


def lib():
    global _lib
    if _lib is None:
        handle = ctypes.CDLL(_build.build())
        sig = {
            "orc_num_threads": (ctypes.c_int, []),
            "orc_set_num_threads": (None, [ctypes.c_int]),
            "orc_peirce_tables": (None, [_P] * 5),
            "orc_num_grid_nodes": (_U, [_P]),
            "orc_shape_functions_f64": (None, [_P, _P, _P]),
            "orc_cell_nodes": (None, [_P, _P, _P]),
            # bodies, rigid, contact bodies, nb, tolerance, max, out -> count
            "orc_find_contacts_f32": (_U, [_P, _P, _P, _U, ctypes.c_float, _U, _P]),
            "orc_solve_contacts_f32": (None, [_P, _P, _U, _P, _U]),
            "orc_mesh_distance_grid_f32": (None, [_P, _P, _U, _P, _U, ctypes.c_float, _P]),
        }
        for s in ("f32", "f64"):
            sig["orc_grid_sort_" + s] = (ctypes.c_int, [_P, _P, _P, _U, _P, _P, _P, _P])
            sig["orc_update_particle_neighbors_" + s] = (
                ctypes.c_int, [_P, _P, _P, _U, _P, _P, _P, _P, _P, _P])
            sig["orc_node_positions_" + s] = (None, [_P, _P, _P, _P])
            sig["orc_distance_grid_" + s] = (None, [_P, _P])
            sig["orc_volume_field_" + s] = (None, [_P, _P, _P])
            sig["orc_boundary_" + s] = (None, [_P, _P, _P, _U, _P, _U, _P, _P])
            # cn, cni, bodies, rigid, n, x, v, kappa, kappa_v, density, density_adv, a,
            # params, dt, steps, reports (IISPH: pressure instead of kappa, kappa_v)
            sig["orc_df_run_" + s] = (ctypes.c_int, [_P] * 4 + [_U] + [_P] * 9 + [_U, _P])
            sig["orc_ii_run_" + s] = (ctypes.c_int, [_P] * 4 + [_U] + [_P] * 8 + [_U, _P])
        for name, (res, args) in sig.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def _p(a):
    if a is None:
        return None
    if isinstance(a, (ctypes.Structure, ctypes.Array, ctypes._SimpleCData)):
        return ctypes.cast(ctypes.pointer(a), ctypes.c_void_p)
    assert a.flags["C_CONTIGUOUS"], "oracle arrays must be C-contiguous"
    return ctypes.c_void_p(a.ctypes.data)


def _sfx(dtype):
    return "f32" if np.dtype(dtype) == np.float32 else "f64"


def set_threads(n):
    lib().orc_set_num_threads(int(n))


def num_threads():
    return lib().orc_num_threads()


def peirce_tables():
    out = [np.zeros(30), np.zeros(30), np.zeros(30), np.zeros(15), np.zeros(15)]
    lib().orc_peirce_tables(*[_p(a) for a in out])
    return dict(zip(["cosphi", "sinphi", "b", "r", "c"], out))


def shape_functions(xi):
    xi = np.ascontiguousarray(xi, dtype=np.float64)
    N = np.zeros(32)
    dN = np.zeros((3, 32))
    lib().orc_shape_functions_f64(_p(xi), _p(N), _p(dN))
    return N, dN


def cell_nodes(res, ipos):
    res = np.ascontiguousarray(res, dtype=np.uint32)
    ip = np.ascontiguousarray(ipos, dtype=np.int32)
    out = np.zeros(32, dtype=np.uint32)
    lib().orc_cell_nodes(_p(res), _p(ip), _p(out))
    return out


def num_grid_nodes(res):
    return int(lib().orc_num_grid_nodes(_p(np.ascontiguousarray(res, dtype=np.uint32))))


def node_positions(domain_min, res, cell_size, dtype):
    dmin = np.ascontiguousarray(domain_min, dtype=dtype)
    cs = np.ascontiguousarray(cell_size, dtype=dtype)
    r = np.ascontiguousarray(res, dtype=np.uint32)
    out = np.zeros((num_grid_nodes(r), 3), dtype=dtype)
    getattr(lib(), "orc_node_positions_" + _sfx(dtype))(_p(dmin), _p(r), _p(cs), _p(out))
    return out


def grid_sort(cn, cni, x):
    x = np.ascontiguousarray(x)
    n = x.shape[0]
    ncells = cni.grid_res[0] * cni.grid_res[1] * cni.grid_res[2]
    cell = np.zeros(n, np.uint32)
    perm = np.zeros(n, np.uint32)
    start = np.zeros(ncells + 1, np.uint32)
    flags = np.zeros(4, np.uint32)
    getattr(lib(), "orc_grid_sort_" + _sfx(x.dtype))(
        _p(cn), _p(cni), _p(x), n, _p(cell), _p(perm), _p(start), _p(flags))
    return cell, perm, start, flags[:2]


def update_particle_neighbors(cn, cni, x, boundary_kernel=None):
    """Returns density [n], count [n], index [n, cap] (original indices,
    canonical order, 0xffffffff padding), neighbors [n, cap, 4], flags[3]."""
    x = np.ascontiguousarray(x)
    n = x.shape[0]
    cap = cni.max_num_neighbors_per_particle
    density = np.zeros(n, x.dtype)
    count = np.zeros(n, np.uint32)
    index = np.zeros((n, cap), np.uint32)
    nbrs = np.zeros((n, cap, 4), x.dtype)
    flags = np.zeros(4, np.uint32)
    bk = None if boundary_kernel is None else np.ascontiguousarray(boundary_kernel, x.dtype)
    getattr(lib(), "orc_update_particle_neighbors_" + _sfx(x.dtype))(
        _p(cn), _p(cni), _p(x), n, _p(bk), _p(density), _p(count), _p(index), _p(nbrs),
        _p(flags))
    return density, count, index, nbrs, flags[:3]


def distance_grid(body, dtype):
    out = np.zeros(body.num_nodes, dtype)
    getattr(lib(), "orc_distance_grid_" + _sfx(dtype))(_p(body), _p(out))
    return out


def volume_field(cn, body, dtype):
    """Volume-map node values; body.distance_nodes must be a HOST pointer
    when body.use_distance_grid is set."""
    out = np.zeros(body.num_nodes, dtype)
    getattr(lib(), "orc_volume_field_" + _sfx(dtype))(_p(cn), _p(body), _p(out))
    return out


def boundary(cn, bodies, rigid, x):
    """bodies: ctypes array of al_body (host node pointers); rigid (nb, 13)."""
    x = np.ascontiguousarray(x)
    n = x.shape[0]
    nb = len(bodies)
    rigid = np.ascontiguousarray(rigid, x.dtype)
    bnd = np.zeros((nb, n, 4), x.dtype)
    bk = np.zeros((nb, n, 4), x.dtype)
    getattr(lib(), "orc_boundary_" + _sfx(x.dtype))(
        _p(cn), _p(bodies) if nb else None, _p(rigid), nb, _p(x), n, _p(bnd), _p(bk))
    return bnd, bk


def run(method, cn, cni, bodies, rigid, state, sp, dt, steps):
    """Advances `state` (dict of host arrays: x, v, kappa, kappa_v | pressure,
    density, density_adv, a) by `steps` steps in place; returns (dt, reports).
    method: 'df' or 'ii'."""
    from alluvion_b200 import _capi
    x = state["x"]
    T = x.dtype
    n = x.shape[0]
    dt_arr = np.array([dt], dtype=T)
    reports = (_capi.StepReport * steps)()
    nb = len(bodies)
    if method == "df":
        status = getattr(lib(), "orc_df_run_" + _sfx(T))(
            _p(cn), _p(cni), _p(bodies) if nb else None, _p(rigid), n, _p(x), _p(state["v"]),
            _p(state["kappa"]), _p(state["kappa_v"]), _p(state["density"]),
            _p(state["density_adv"]), _p(state["a"]), _p(sp), _p(dt_arr), steps,
            _p(reports))
    else:
        status = getattr(lib(), "orc_ii_run_" + _sfx(T))(
            _p(cn), _p(cni), _p(bodies) if nb else None, _p(rigid), n, _p(x), _p(state["v"]),
            _p(state["pressure"]), _p(state["density"]), _p(state["density_adv"]),
            _p(state["a"]), _p(sp), _p(dt_arr), steps, _p(reports))
    assert status == 0
    return float(dt_arr[0]), list(reports)


def find_contacts(bodies, rigid, contact_bodies, tolerance, max_contacts):
    """Pile::find_contacts restated: (count found, ContactF32 array) with HOST
    pointers in bodies (node arrays) and contact_bodies (vertices)."""
    from alluvion_b200 import _capi
    out = (_capi.ContactF32 * max(max_contacts, 1))()
    nb = len(contact_bodies)
    cb = (_capi.ContactBodyF32 * max(nb, 1))(*contact_bodies)
    n = lib().orc_find_contacts_f32(_p(bodies), _p(rigid), _p(cb), nb, float(tolerance),
                                    max_contacts, _p(out))
    return int(n), out


def solve_contacts(bodies, rigid, contacts, num):
    """Pile::solve_contacts restated: updates rigid (RigidF32 array) in place."""
    lib().orc_solve_contacts_f32(_p(bodies), _p(rigid), len(rigid), _p(contacts), num)


def mesh_distance_grid(body, vertices, faces, offset=0.0):
    """MeshDistance::signedDistance at the nodes of `body` (al_body_f32)."""
    v = np.ascontiguousarray(vertices, np.float32)
    f = np.ascontiguousarray(faces, np.uint32)
    out = np.zeros(body.num_nodes, np.float32)
    lib().orc_mesh_distance_grid_f32(_p(body), _p(v), len(v), _p(f), len(f), float(offset),
                                     _p(out))
    return out
