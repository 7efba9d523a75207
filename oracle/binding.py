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
            # cn, cni, particle_x, n, rigid, request -> overflow
            "orc_sample_fluid_f32": (ctypes.c_int, [_P, _P, _P, _U, _P, _P]),
            "orc_sample_fluid_f64": (ctypes.c_int, [_P, _P, _P, _U, _P, _P]),
            "orc_boundary_mask_f32": (None, [_P, _P, _P, _U, ctypes.c_float, _P]),
            "orc_boundary_mask_f64": (None, [_P, _P, _P, _U, ctypes.c_double, _P]),
            "orc_histogram256_f32": (None, [_P, _P, _U, ctypes.c_float, ctypes.c_float, _P]),
            "orc_histogram256_f64": (None, [_P, _P, _U, ctypes.c_double, ctypes.c_double, _P]),
            "orc_kl_divergence": (ctypes.c_double, [_P, _P, _U, _U, ctypes.c_double, _U]),
            "orc_relax_pellets_f32": (ctypes.c_int, [_P, _P, _P, _P, _U, _P, _U, _P, _P]),
            "orc_lazy_volume_release": (None, [_P]),
        }
        for s in ("f32", "f64"):
            sig["orc_grid_sort_" + s] = (ctypes.c_int, [_P, _P, _P, _U, _P, _P, _P, _P])
            sig["orc_update_particle_neighbors_" + s] = (
                ctypes.c_int, [_P, _P, _P, _U, _P, _P, _P, _P, _P, _P])
            sig["orc_update_particle_neighbors_periodic_" + s] = (
                ctypes.c_int, [_P, _P, _P, _U, _P, _P, _P, _P, _P, _P, ctypes.c_double])
            sig["orc_node_positions_" + s] = (None, [_P, _P, _P, _P])
            sig["orc_distance_grid_" + s] = (None, [_P, _P])
            sig["orc_volume_field_" + s] = (None, [_P, _P, _P])
            sig["orc_lazy_volume_register_" + s] = (None, [_P, _P, _P])
            sig["orc_lazy_volume_counts_" + s] = (None, [_P, _P])
            sig["orc_lazy_volume_touch_" + s] = (None, [_P, _P, _P, _U, _U])
            sig["orc_boundary_" + s] = (None, [_P, _P, _P, _U, _P, _U, _P, _P])
            # cn, cni, bodies, rigid, n, x, v, kappa, kappa_v, density, density_adv, a,
            # params, dt, steps, reports (IISPH: pressure instead of kappa, kappa_v)
            sig["orc_df_run_" + s] = (ctypes.c_int, [_P] * 4 + [_U] + [_P] * 9 + [_U, _P])
            sig["orc_ii_run_" + s] = (ctypes.c_int, [_P] * 4 + [_U] + [_P] * 8 + [_U, _P])
            sig["orc_i_run_" + s] = (ctypes.c_int, [_P] * 4 + [_U] + [_P] * 8 + [_U, _P])
            # ... a, pellet_local, counts, num_pellets, sp, dt, steps, reports, pellet_x, pellet_p
            sig["orc_i_run_pellets_" + s] = (
                ctypes.c_int, [_P] * 4 + [_U] + [_P] * 8 + [_U, _P, _P, _U, _P, _P, _P])
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


def update_particle_neighbors(cn, cni, x, boundary_kernel=None, wrap_length=None):
    """Returns density [n], count [n], index [n, cap] (original indices,
    canonical order, 0xffffffff padding), neighbors [n, cap, 4], flags[3].
    wrap_length: periodic in y (update_particle_neighbors<1>)."""
    x = np.ascontiguousarray(x)
    n = x.shape[0]
    cap = cni.max_num_neighbors_per_particle
    density = np.zeros(n, x.dtype)
    count = np.zeros(n, np.uint32)
    index = np.zeros((n, cap), np.uint32)
    nbrs = np.zeros((n, cap, 4), x.dtype)
    flags = np.zeros(4, np.uint32)
    bk = None if boundary_kernel is None else np.ascontiguousarray(boundary_kernel, x.dtype)
    args = (_p(cn), _p(cni), _p(x), n, _p(bk), _p(density), _p(count), _p(index), _p(nbrs),
            _p(flags))
    if wrap_length is None:
        getattr(lib(), "orc_update_particle_neighbors_" + _sfx(x.dtype))(*args)
    else:
        getattr(lib(), "orc_update_particle_neighbors_periodic_" + _sfx(x.dtype))(
            *args, float(wrap_length))
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


def lazy_volume_field(cn, body, dtype):
    """A volume map whose nodes the oracle computes on first use (same values
    as volume_field at every node it reads).  Point body.volume_nodes at the
    returned array; body.distance_nodes (HOST) must outlive it.  Release
    with lazy_volume_release."""
    out = np.zeros(body.num_nodes, dtype)
    getattr(lib(), "orc_lazy_volume_register_" + _sfx(dtype))(_p(cn), _p(body), _p(out))
    return out


def lazy_volume_counts(out):
    """(nodes computed by sampling, nodes set by the analytic shortcuts)."""
    c = np.zeros(2, np.uint64)
    getattr(lib(), "orc_lazy_volume_counts_" + _sfx(out.dtype))(_p(out), _p(c))
    return int(c[0]), int(c[1])


def lazy_volume_touch(body, rigid_row, x, dilate=1):
    """Computes now the lazy map's nodes that particles x (n, 3), within
    `dilate` cells, will read; body.volume_nodes must be a lazy map."""
    x = np.ascontiguousarray(x)
    r = np.ascontiguousarray(rigid_row, x.dtype)
    getattr(lib(), "orc_lazy_volume_touch_" + _sfx(x.dtype))(_p(body), _p(r), _p(x), x.shape[0],
                                                             int(dilate))


def lazy_volume_release(out):
    lib().orc_lazy_volume_release(_p(out))


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
    method: 'df' (DFSPH), 'ii' (IISPH) or 'i' (implicit SPH, SolverI)."""
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
        status = getattr(lib(), "orc_%s_run_%s" % (method, _sfx(T)))(
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


def sample_fluid(cn, cni, particle_x, rigid, sample_x, particle_density=None, particle_v=None,
                 particle_quantity=None, sample_boundary=None, sample_boundary_kernel=None,
                 outputs=("density", "position_density", "quantity", "v", "vorticity"),
                 wrap_length=None, pellet_x=None, pellet_v=None):
    """sample_fluid / sample_fluid_density / sample_position_density /
    compute_sample_velocity / compute_sample_vorticity restated on host
    arrays of particle_x's real type (float32 or float64; cn, rigid and the
    other arrays follow it); wrap_length: periodic in y
    (make_neighbor_list<1>).  Returns (dict of outputs, neighbor overflow
    flag)."""
    from alluvion_b200 import _capi
    T = np.float64 if np.asarray(particle_x).dtype == np.float64 else np.float32
    f32 = lambda a: None if a is None else np.ascontiguousarray(a, T)
    px, sx = f32(particle_x), f32(sample_x)
    rho, pv, pq = f32(particle_density), f32(particle_v), f32(particle_quantity)
    sb, sbk = f32(sample_boundary), f32(sample_boundary_kernel)
    s = len(sx)
    qdim = 0 if pq is None else (1 if pq.ndim == 1 else pq.shape[1])
    out = {}
    shapes = {"density": (s,), "position_density": (s,), "quantity": (s, qdim) if qdim > 1
              else (s,), "v": (s, 3), "vorticity": (s, 3)}
    for k in outputs:
        out[k] = np.zeros(shapes[k], T)
    req = _capi.sample_struct(T)()
    req.sample_x = sx.ctypes.data
    req.num_samples = s
    req.quantity_dim = qdim
    if wrap_length is not None:
        req.wrap_y = 1
        req.wrap_length = float(wrap_length)
    pxh, pvh = f32(pellet_x), f32(pellet_v)
    if pxh is not None and len(pxh):
        req.pellet_x = pxh.ctypes.data
        req.pellet_v = pvh.ctypes.data if pvh is not None else None
        req.num_pellets = len(pxh)
    for name, arr in (("particle_density", rho), ("particle_v", pv), ("particle_quantity", pq),
                      ("sample_boundary", sb), ("sample_boundary_kernel", sbk)):
        setattr(req, name, None if arr is None else arr.ctypes.data)
    for k, name in (("density", "sample_density"), ("position_density", "sample_position_density"),
                    ("quantity", "sample_quantity"), ("v", "sample_v"),
                    ("vorticity", "sample_vorticity")):
        setattr(req, name, out[k].ctypes.data if k in out else None)
    flag = getattr(lib(), "orc_sample_fluid_" + _sfx(T))(_p(cn), _p(cni), _p(px), len(px),
                                                        _p(rigid), _p(req))
    return out, bool(flag)


def boundary_mask(body, rigid, sample_x, threshold, mask):
    """compute_boundary_mask restated: mask *= (sign d >= threshold), in the
    real type of mask (float32 or float64)."""
    T = mask.dtype.type
    sx = np.ascontiguousarray(sample_x, T)
    getattr(lib(), "orc_boundary_mask_" + _sfx(T))(_p(body), _p(rigid), _p(sx), len(sx),
                                                   float(threshold), _p(mask))
    return mask


def histogram256(v, v_min, v_max, mask=None):
    """launch_histogram256[_with_mask] restated: 256 uint32 counts, in v's
    real type (float32 or float64)."""
    T = np.float64 if np.asarray(v).dtype == np.float64 else np.float32
    v = np.ascontiguousarray(v, T)
    m = None if mask is None else np.ascontiguousarray(mask, T)
    h = np.zeros(256, np.uint32)
    getattr(lib(), "orc_histogram256_" + _sfx(T))(_p(v), _p(m), len(v), float(v_min),
                                                  float(v_max), _p(h))
    return h


def kl_divergence(p, q, n_p, n_q, q_lower_bound):
    """calculate_kl_divergence restated in double."""
    p = np.ascontiguousarray(p, np.uint32)
    q = np.ascontiguousarray(q, np.uint32)
    return lib().orc_kl_divergence(_p(p), _p(q), n_p, n_q, float(q_lower_bound), len(p))


def run_pellets(cn, cni, bodies, rigid, state, pellet_local, counts, sp, dt, steps):
    """SolverI with the pellet boundary model: advances `state` (x, v,
    pressure, density, density_adv, a) by `steps` steps in place.  Returns
    (dt, reports, pellet world positions, pellet pressures) of the last step."""
    from alluvion_b200 import _capi
    x = state["x"]
    T = x.dtype
    n = x.shape[0]
    local = np.ascontiguousarray(pellet_local, T).reshape(-1, 3)
    npl = len(local)
    cnt = np.ascontiguousarray(counts, np.uint32)
    dt_arr = np.array([dt], dtype=T)
    reports = (_capi.StepReport * steps)()
    px = np.zeros((npl, 3), T)
    pp = np.zeros(npl, T)
    nb = len(bodies)
    status = getattr(lib(), "orc_i_run_pellets_" + _sfx(T))(
        _p(cn), _p(cni), _p(bodies) if nb else None, _p(rigid), n, _p(x), _p(state["v"]),
        _p(state["pressure"]), _p(state["density"]), _p(state["density_adv"]), _p(state["a"]),
        _p(local) if npl else None, _p(cnt), npl, _p(sp), _p(dt_arr), steps, _p(reports),
        _p(px), _p(pp))
    assert status == 0
    return float(dt_arr[0]), list(reports), px, pp


def relax_pellets(cn, cni, body, x, params, steps):
    """SolverPellet<float>::step restated: returns (x, dx, density) after
    `steps` steps and the neighbor-overflow flag."""
    xs = np.ascontiguousarray(x, np.float32).copy()
    dx = np.zeros_like(xs)
    rho = np.zeros(len(xs), np.float32)
    over = lib().orc_relax_pellets_f32(_p(cn), _p(cni), _p(body), _p(xs), len(xs), _p(params),
                                       steps, _p(dx), _p(rho))
    return xs, dx, rho, bool(over)
