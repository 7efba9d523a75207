"""Physical constants, grid sizing, bodies and seeded synthetic scenes.

Constants are derived in the solver's real type with the operation order of
Const<TF>::set_kernel_radius / set_particle_attr (constants.hpp:100-128), so
float32 scenes see exactly the float32 values the reference would.
"""
import ctypes
import math

import numpy as np

from . import _capi

PI = 3.14159265358979323846264338327950288


def make_const(dtype, particle_radius, density0=1000.0, viscosity=0.01,
               boundary_viscosity=0.01, dfsph_factor_epsilon=1e-6,
               gravity=(0.0, -9.81, 0.0), kernel_radius=None, particle_mass=None):
    """Returns an al_const_{f32,f64} for a particle radius r.

    Defaults follow the benchmark scenes: h = 4r, m = rho0 (2r)^3 so that
    V = (2r)^3, viscosity 0.01, boundary_viscosity 0.01,
    dfsph_factor_epsilon 1e-6 (both unset in the reference, whose default is
    0), g = (0, -9.81, 0).
    """
    T = np.dtype(dtype).type
    ConstT, _, _, _ = _capi.real_types(dtype)
    r = T(particle_radius)
    h = T(kernel_radius) if kernel_radius is not None else T(4) * r
    # Const::set_kernel_radius
    h2 = h * h
    h3 = h2 * h
    h4 = h2 * h2
    k = T(8.0) / h3 / T(PI)
    l = T(48.0) / h4 / T(PI)
    # Const::set_particle_attr
    rho0 = T(density0)
    if particle_mass is None:
        d = T(2) * r
        mass = rho0 * (d * d * d)
    else:
        mass = T(particle_mass)
    vol = mass / rho0
    c = ConstT()
    c.kernel_radius = h
    c.kernel_radius_sqr = h2
    c.cubic_kernel_k = k
    c.cubic_kernel_l = l
    c.cubic_kernel_zero = k
    c.particle_radius = r
    c.particle_vol = vol
    c.particle_mass = mass
    c.density0 = rho0
    c.viscosity = T(viscosity)
    c.boundary_viscosity = T(boundary_viscosity)
    c.dfsph_factor_epsilon = T(dfsph_factor_epsilon)
    for i in range(3):
        c.gravity[i] = T(gravity[i])
    return c


def make_consti(domain_min, domain_max, kernel_radius, num_boundaries=0,
                max_num_particles_per_cell=64, max_num_neighbors_per_particle=64):
    """Uniform grid of cell size h covering [domain_min, domain_max].

    grid_offset = floor(domain_min / h) - 1 and the resolution spans the
    domain plus one cell of margin on each side.
    """
    g = _capi.ConstI()
    h = float(kernel_radius)
    for i in range(3):
        lo = math.floor(domain_min[i] / h) - 1
        hi = math.floor(domain_max[i] / h) + 1
        g.grid_offset[i] = lo
        g.grid_res[i] = hi - lo + 1
    g.max_num_particles_per_cell = max_num_particles_per_cell
    g.max_num_neighbors_per_particle = max_num_neighbors_per_particle
    g.num_boundaries = num_boundaries
    return g


def fluid_block(num, box_min, particle_radius, dtype=np.float32, jitter=0.1, seed=0):
    """Lattice block of num = (nx, ny, nz) particles at spacing 2r starting at
    box_min + 2r, the mode-0 layout of index_to_position_in_fluid_block
    (runner.hpp:971-995), plus seeded uniform jitter of +-jitter*r per
    coordinate (numpy PCG64)."""
    nx, ny, nz = num
    r = float(particle_radius)
    n = nx * ny * nz
    p = np.arange(n, dtype=np.int64)
    j = (p % (nx * nz)) // nz
    k = p // (nx * nz)
    l = p % nz
    pos = np.stack([2 * r * j, 2 * r * k, 2 * r * l], axis=1).astype(np.float64)
    pos += np.asarray(box_min, dtype=np.float64) + 2 * r
    if jitter:
        rng = np.random.Generator(np.random.PCG64(seed))
        pos += rng.uniform(-jitter * r, jitter * r, size=pos.shape)
    return pos.astype(dtype)


# ----------------------------------------------------------------- bodies
def shape_aabb(shape, params):
    """(aabb_min, aabb_max, max_distance) of an analytic shape in its frame
    (dg/box_distance.hpp:13-17, dg/sphere_distance.hpp:11-13,
    dg/box_shell_distance.hpp:13-21 and the constructors of the cylinder,
    capsule, infinite cylinder and infinite tube distances; the torus is new).
    The infinite tube's optional third parameter is its box half length in y."""
    p = [float(v) for v in params]
    if shape == _capi.SHAPE_BOX:
        hw = np.array(p[:3])
        out = p[3]
        return -hw - out, hw + out, float(np.linalg.norm(hw)) + out
    if shape == _capi.SHAPE_SPHERE:
        rr = p[0]
        return np.full(3, -rr), np.full(3, rr), rr
    if shape == _capi.SHAPE_BOX_SHELL:
        outer = np.array(p[3:6])
        out = p[6]
        return -outer - out, outer + out, float(np.linalg.norm(outer)) + out
    if shape == _capi.SHAPE_TORUS:
        R, rr = p[0], p[1]
        e = np.array([R + rr, rr, R + rr])
        return -e, e, R + rr
    if shape == _capi.SHAPE_CYLINDER:  # dg/cylinder_distance.hpp:13-22
        rr, hh, com = p[0], 0.5 * p[1], p[2]
        return (np.array([-rr, -hh - com, -rr]), np.array([rr, hh - com, rr]),
                float(np.sqrt(rr * rr + (hh + abs(com)) ** 2)))
    if shape == _capi.SHAPE_CAPSULE:  # dg/capsule_distance.hpp:13-19
        rr, hh = p[0], 0.5 * p[1]
        return np.array([-rr, -hh - rr, -rr]), np.array([rr, hh + rr, rr]), hh + rr
    if shape == _capi.SHAPE_INFINITE_CYLINDER:  # finite box (infinite_cylinder_distance.hpp:13-16)
        rr = p[0]
        return np.full(3, -rr), np.full(3, rr), rr
    if shape == _capi.SHAPE_INFINITE_TUBE:  # infinite_tube_distance.hpp:15-28
        ro, half = p[1], (p[2] if len(p) > 2 and p[2] else p[1])
        return (np.array([-ro, -half, -ro]), np.array([ro, half, ro]), max(half, ro))
    raise ValueError("unknown shape %r (mesh bodies pass aabb= to make_body)" % shape)


def box_params(widths, outset=0.0):
    w = [0.5 * float(v) for v in widths]
    return w + [outset]


def box_shell_params(inner_widths, thickness, outset=0.0):
    hi = [0.5 * float(v) for v in inner_widths]
    ho = [v + float(thickness) for v in hi]
    return hi + ho + [outset]


def make_body(dtype, cn, shape, params, resolution, sign=1.0, margin=None,
              use_distance_grid=False, mass=0.0, inertia=(1.0, 1.0, 1.0), aabb=None):
    """al_body_{f32,f64} with the domain of Pile::calculate_domain_and_resolution
    (pile.hpp:40-65; margin defaults to h for sign < 0, 2h otherwise) and the
    grid attributes of Pile::calculate_grid_attributes (pile.hpp:66-78).
    Node pointers are left NULL.  aabb: (min, max, max_distance) of a mesh
    body (AL_SHAPE_MESH), whose extent does not follow from params."""
    T = np.dtype(dtype).type
    _, BodyT, _, _ = _capi.real_types(dtype)
    h = T(cn.kernel_radius)
    if margin is None:
        margin = h if sign < 0 else h * T(2)
    margin = T(margin)
    lo, hi, maxd = shape_aabb(shape, params) if aabb is None else aabb
    b = BodyT()
    b.shape = shape
    b.use_distance_grid = int(bool(use_distance_grid))
    b.sign = T(sign)
    padded = list(params) + [0.0] * (8 - len(params))
    for i in range(8):
        b.shape_params[i] = T(padded[i])
    res = [int(v) for v in (resolution if np.ndim(resolution) else [resolution] * 3)]
    for i in range(3):
        dmin = T(lo[i]) - margin
        dmax = T(hi[i]) + margin
        b.domain_min[i] = dmin
        b.domain_max[i] = dmax
        b.cell_size[i] = (dmax - dmin) / T(res[i])
        b.resolution[i] = res[i]
    b.num_nodes = num_grid_nodes(res)
    b.max_distance = T(maxd)
    b.mass = T(mass)
    for i in range(3):
        b.inertia[i] = T(inertia[i])
    return b


def num_grid_nodes(res):
    nx, ny, nz = res
    return ((nx + 1) * (ny + 1) * (nz + 1) + 2 * (nx * (ny + 1) * (nz + 1) +
            (nx + 1) * ny * (nz + 1) + (nx + 1) * (ny + 1) * nz))


def rigid_state(dtype, x=(0, 0, 0), v=(0, 0, 0), q=(0, 0, 0, 1), omega=(0, 0, 0)):
    _, _, RigidT, _ = _capi.real_types(dtype)
    s = RigidT()
    for i in range(3):
        s.x[i], s.v[i], s.omega[i] = x[i], v[i], omega[i]
    for i in range(4):
        s.q[i] = q[i]
    return s


def rigid_array(dtype, states):
    """Packs rigid states into an (nb, 13) array: x, v, q, omega."""
    T = np.dtype(dtype).type
    out = np.zeros((len(states), 13), dtype=T)
    for b, s in enumerate(states):
        out[b, 0:3] = list(s.x)
        out[b, 3:6] = list(s.v)
        out[b, 6:10] = list(s.q)
        out[b, 10:13] = list(s.omega)
    return out


def sphere_inertia(mass, radius):
    i = 0.4 * mass * radius * radius
    return (i, i, i)


def box_inertia(mass, widths):
    wx, wy, wz = widths
    return (mass * (wy * wy + wz * wz) / 12, mass * (wx * wx + wz * wz) / 12,
            mass * (wx * wx + wy * wy) / 12)


def body_from_spec(dtype, cn, spec):
    """al_body_{f32,f64} (node pointers NULL) of a body spec dict: keys shape,
    params, sign, resolution, use_distance_grid, mass, inertia, optional
    margin, and mesh = (vertices, faces) with offset for AL_SHAPE_MESH."""
    mesh = spec.get("mesh")
    aabb = mesh_aabb(mesh[0], spec.get("offset", 0.0)) if mesh is not None else None
    return make_body(dtype, cn, spec["shape"], spec.get("params", []), spec["resolution"],
                     sign=spec.get("sign", 1.0), margin=spec.get("margin"),
                     use_distance_grid=mesh is not None or spec.get("use_distance_grid", False),
                     mass=spec.get("mass", 0.0), inertia=spec.get("inertia", (1, 1, 1)),
                     aabb=aabb)


def rigid_from_spec(dtype, spec):
    return rigid_state(dtype, x=spec.get("x", (0, 0, 0)), v=spec.get("v", (0, 0, 0)),
                       q=spec.get("q", (0, 0, 0, 1)), omega=spec.get("omega", (0, 0, 0)))


class SceneSpec:
    """Host description of a seeded scene: constants (cn, cni), particle
    positions x [n][3] and body spec dicts (see body_from_spec), with no
    device memory and no call into the engine library."""

    def __init__(self, dtype, cn, cni, x, bodies):
        self.dtype = np.dtype(dtype)
        self.cn = cn
        self.cni = cni
        self.x = x
        self.body_specs = list(bodies)
        self.cni.num_boundaries = len(self.body_specs)

    @property
    def n(self):
        return int(self.x.shape[0])

    @property
    def num_boundaries(self):
        return len(self.body_specs)

    def bodies(self):
        """ctypes array of al_body (node pointers NULL) and rigid (nb, 13)."""
        _, BodyT, _, _ = _capi.real_types(self.dtype)
        nb = self.num_boundaries
        arr = (BodyT * max(nb, 1))()
        for b, spec in enumerate(self.body_specs):
            arr[b] = body_from_spec(self.dtype, self.cn, spec)
        rigid = rigid_array(self.dtype, [rigid_from_spec(self.dtype, s) for s in self.body_specs])
        return arr, rigid

    def device(self, engine, device="cuda"):
        """The scene on a CUDA device (grids built by the engine)."""
        return DeviceScene(engine, self.dtype, self.cn, self.cni, self.x, self.body_specs,
                           device=device)


class DeviceScene:
    """A seeded scene held on one CUDA device: constants, grid dimensions,
    bodies with device-built distance grids and volume maps, and the
    reference-layout particle buffers.  Steps go through the C ABI.

    bodies: list of dicts with keys shape, params, sign, resolution,
    use_distance_grid, mass, inertia, x, q (optional v, omega, margin).
    """

    def __init__(self, engine, dtype, cn, cni, x, bodies=(), device="cuda",
                 pile_gravity=(0.0, -9.81, 0.0)):
        import torch
        self.torch = torch
        self.engine = engine
        self.dtype = np.dtype(dtype)
        self.tdtype = torch.float32 if self.dtype == np.float32 else torch.float64
        self.sfx = _capi.suffix(dtype)
        self.cn = cn
        self.cni = cni
        self.device = device
        self.n = int(x.shape[0])
        zeros = lambda *s: torch.zeros(*s, dtype=self.tdtype, device=device)
        self.x = torch.from_numpy(np.ascontiguousarray(x, dtype=self.dtype)).to(device)
        self.v = zeros(self.n, 3)
        self.a = zeros(self.n, 3)
        self.density = zeros(self.n)
        self.dfsph_factor = zeros(self.n)
        self.kappa = zeros(self.n)
        self.kappa_v = zeros(self.n)
        self.density_adv = zeros(self.n)
        self.pressure = zeros(self.n)
        self.pile_gravity = pile_gravity
        self.body_specs = list(bodies)
        self.distance_nodes = []
        self.volume_nodes = []
        _, BodyT, RigidT, _ = _capi.real_types(dtype)
        nb = len(self.body_specs)
        self.bodies = (BodyT * max(nb, 1))()
        self.rigid = (RigidT * max(nb, 1))()
        for b, spec in enumerate(self.body_specs):
            mesh = spec.get("mesh")  # (vertices [nv][3], faces [nf][3]) for SHAPE_MESH
            body = body_from_spec(dtype, cn, spec)
            dist = zeros(body.num_nodes) if body.use_distance_grid else None
            vol = zeros(body.num_nodes)
            if mesh is not None:
                assert self.sfx == "f32", "mesh bodies: float32 scenes"
                v = np.ascontiguousarray(mesh[0], np.float32)
                f = np.ascontiguousarray(mesh[1], np.uint32)
                body.distance_nodes = dist.data_ptr()
                _capi.check(_capi.lib().al_build_mesh_distance_grid_f32(
                    engine.handle, _capi.ptr(body), v.ctypes.data, len(v), f.ctypes.data, len(f),
                    ctypes.c_float(spec.get("offset", 0.0)), _capi.ptr(dist), None),
                    "al_build_mesh_distance_grid_f32")
            elif dist is not None:
                body.distance_nodes = dist.data_ptr()
                _capi.check(getattr(_capi.lib(), "al_build_distance_grid_" + self.sfx)(
                    engine.handle, _capi.ptr(body), _capi.ptr(dist), None),
                    "al_build_distance_grid")
            body.volume_nodes = vol.data_ptr()
            _capi.check(getattr(_capi.lib(), "al_build_volume_field_" + self.sfx)(
                engine.handle, _capi.ptr(cn), _capi.ptr(body), _capi.ptr(vol), None),
                "al_build_volume_field")
            self.bodies[b] = body
            self.distance_nodes.append(dist)
            self.volume_nodes.append(vol)
            self.rigid[b] = rigid_from_spec(dtype, spec)
        self.cni.num_boundaries = nb
        torch.cuda.synchronize()

    @property
    def num_boundaries(self):
        return len(self.body_specs)

    def fluid(self, export_boundary=None):
        bufs = dict(particle_x=self.x, particle_v=self.v, particle_a=self.a,
                    particle_density=self.density, particle_dfsph_factor=self.dfsph_factor,
                    particle_kappa=self.kappa, particle_kappa_v=self.kappa_v,
                    particle_density_adv=self.density_adv, particle_pressure=self.pressure)
        if export_boundary is not None:
            bufs["particle_boundary"], bufs["particle_boundary_kernel"] = export_boundary
        return _capi.make_fluid(self.n, **bufs)

    def step(self, method, sp, dt, report=None, stream=None, allow=(), warm=None):
        """One DFSPH ('df') or IISPH ('ii') step; returns (dt_out, report).
        warm: an _capi.WarmStart for the float32 DFSPH step with the learned
        warm start and/or feature output (al_df_step_warm_f32)."""
        T = self.dtype.type
        dt_c = (ctypes_real(self.dtype))(T(dt))
        rep = report if report is not None else _capi.StepReport()
        fluid = self.fluid()
        bodies = _capi.ptr(self.bodies) if self.num_boundaries else None
        rigid = _capi.ptr(self.rigid) if self.num_boundaries else None
        if warm is not None:
            assert method == "df" and self.sfx == "f32", "learned warm start: float32 DFSPH"
            status = _capi.lib().al_df_step_warm_f32(
                self.engine.handle, _capi.ptr(self.cn), _capi.ptr(self.cni), _capi.ptr(fluid),
                bodies, rigid, _capi.ptr(sp), _capi.ptr(warm), _capi.ptr(dt_c), _capi.ptr(rep),
                stream)
            _capi.check(status, "al_df_step_warm_f32", allow=allow)
            return float(dt_c.value), rep
        fn = getattr(_capi.lib(), "al_%s_step_%s" % (method, self.sfx))
        status = fn(self.engine.handle, _capi.ptr(self.cn), _capi.ptr(self.cni), _capi.ptr(fluid),
                    bodies, rigid, _capi.ptr(sp), _capi.ptr(dt_c), _capi.ptr(rep), stream)
        _capi.check(status, "al_%s_step" % method, allow=allow)
        return float(dt_c.value), rep

    def host_bodies(self):
        """(bodies with HOST node pointers, keep-alive arrays, rigid (nb,13))
        for CPU consumers of the same grids."""
        _, BodyT, _, _ = _capi.real_types(self.dtype)
        nb = self.num_boundaries
        hb = (BodyT * max(nb, 1))()
        keep = []
        for b in range(nb):
            src = self.bodies[b]
            ctypes_copy(hb, b, src)
            vol = self.volume_nodes[b].cpu().numpy()
            keep.append(vol)
            hb[b].volume_nodes = vol.ctypes.data
            if self.distance_nodes[b] is not None:
                dist = self.distance_nodes[b].cpu().numpy()
                keep.append(dist)
                hb[b].distance_nodes = dist.ctypes.data
        rigid = rigid_array(self.dtype, [self.rigid[b] for b in range(nb)])
        return hb, keep, rigid

    STATE_KEYS = ("x", "v", "a", "density", "dfsph_factor", "kappa", "kappa_v", "density_adv",
                  "pressure")

    def snapshot(self):
        """Device copies of the mutable state (particles and rigid bodies)."""
        dev = {k: getattr(self, k).clone() for k in self.STATE_KEYS}
        rig = []
        for b in range(self.num_boundaries):
            r = type(self.rigid[b])()
            ctypes.memmove(ctypes.addressof(r), ctypes.addressof(self.rigid[b]), ctypes.sizeof(r))
            rig.append(r)
        return dev, rig

    def restore(self, snap):
        """Puts back a snapshot() (same scene, same buffers)."""
        dev, rig = snap
        for k, t in dev.items():
            getattr(self, k).copy_(t)
        for b, r in enumerate(rig):
            ctypes.memmove(ctypes.addressof(self.rigid[b]), ctypes.addressof(r), ctypes.sizeof(r))

    def state(self):
        """Host copies of the particle state."""
        g = lambda t: t.cpu().numpy()
        return {"x": g(self.x), "v": g(self.v), "a": g(self.a), "density": g(self.density),
                "kappa": g(self.kappa), "kappa_v": g(self.kappa_v),
                "density_adv": g(self.density_adv), "pressure": g(self.pressure),
                "dfsph_factor": g(self.dfsph_factor)}


def ctypes_real(dtype):
    import ctypes
    return ctypes.c_float if np.dtype(dtype) == np.float32 else ctypes.c_double


def ctypes_copy(dst_array, index, src):
    import ctypes
    ctypes.memmove(ctypes.addressof(dst_array) + index * ctypes.sizeof(src),
                   ctypes.addressof(src), ctypes.sizeof(src))


def dam_break(engine, dtype, lattice, particle_radius, container, bodies=(), seed=0,
              volume_resolution=64, jitter=0.1, max_num_particles_per_cell=64,
              max_num_neighbors_per_particle=64, **const_kw):
    """Dam break: a jittered lattice block in the low corner of a box
    container (analytic box distance, sign -1, fluid inside) centred at
    container/2, plus extra bodies.  Returns a DeviceScene.

    The block's outer particles start one kernel radius h from the three
    walls.  (The reference's mode-0 block starts 2r = h/2 from its box; with
    the volume-map boundary term, runner.hpp:1982-2072, a particle at h/2
    from a wall sees rho ~ 2 rho0, so that layout starts far from
    equilibrium.  At h the wall term is exactly zero.)"""
    return dam_break_spec(dtype, lattice, particle_radius, container, bodies, seed=seed,
                          volume_resolution=volume_resolution, jitter=jitter,
                          max_num_particles_per_cell=max_num_particles_per_cell,
                          max_num_neighbors_per_particle=max_num_neighbors_per_particle,
                          **const_kw).device(engine)


def dam_break_spec(dtype, lattice, particle_radius, container, bodies=(), seed=0,
                   volume_resolution=64, jitter=0.1, max_num_particles_per_cell=64,
                   max_num_neighbors_per_particle=64, **const_kw):
    """The host description (SceneSpec) of dam_break's scene."""
    cn = make_const(dtype, particle_radius, **const_kw)
    h = float(cn.kernel_radius)
    gap = h - 2 * float(particle_radius)
    x = fluid_block(lattice, (gap, gap, gap), particle_radius, dtype, jitter=jitter, seed=seed)
    size = np.asarray(container, dtype=np.float64)
    cont = dict(shape=_capi.SHAPE_BOX, params=box_params(size), sign=-1.0,
                resolution=volume_resolution, use_distance_grid=False, mass=0.0,
                x=tuple(size / 2))
    all_bodies = [cont] + list(bodies)
    cni = make_consti(-0.5 * h * np.ones(3), size + 0.5 * h, h, len(all_bodies),
                      max_num_particles_per_cell, max_num_neighbors_per_particle)
    return SceneSpec(dtype, cn, cni, x, all_bodies)


def seeded_rigid_bodies(seed, container, particle_radius, spheres=2, boxes=2,
                        sphere_radius=0.05, box_side=0.08, resolution=64,
                        y_range=(0.75, 0.9), density_range=(500.0, 2000.0)):
    """Rigid spheres and boxes at seeded positions above the fluid block,
    densities uniform in density_range, analytic mass and inertia, sampled
    onto cubic-Lagrange distance grids (use_distance_grid)."""
    rng = np.random.Generator(np.random.PCG64(seed + 1000))
    size = np.asarray(container, dtype=np.float64)
    out = []
    for k in range(spheres + boxes):
        rho = rng.uniform(*density_range)
        pos = (rng.uniform(0.2, 0.8) * size[0], rng.uniform(*y_range) * size[1],
               rng.uniform(0.2, 0.8) * size[2])
        if k < spheres:
            r = sphere_radius
            mass = rho * 4.0 / 3.0 * PI * r ** 3
            out.append(dict(shape=_capi.SHAPE_SPHERE, params=[r], sign=1.0,
                            resolution=resolution, use_distance_grid=True, mass=mass,
                            inertia=sphere_inertia(mass, r), x=pos))
        else:
            w = (box_side,) * 3
            mass = rho * box_side ** 3
            out.append(dict(shape=_capi.SHAPE_BOX, params=box_params(w), sign=1.0,
                            resolution=resolution, use_distance_grid=True, mass=mass,
                            inertia=box_inertia(mass, w), x=pos))
    return out


def solver_params(**kw):
    """al_solver_params with the reference defaults (solver_df.hpp:60-67) and
    the benchmark's cfl 0.4, max_dt 2e-4."""
    p = _capi.SolverParams()
    p.density_change_tolerance = 1e-3
    p.density_error_tolerance = 1e-3
    p.min_density_solve = 2
    p.max_density_solve = 100
    p.min_divergence_solve = 1
    p.max_divergence_solve = 100
    p.enable_divergence_solve = 1
    p.enable_density_solve = 1
    p.cfl = 0.4
    p.max_dt = 2e-4
    p.min_dt = 0.0
    p.pile_gravity[:] = (0.0, -9.81, 0.0)
    p.integrate_rigids = 1
    for k, v in kw.items():
        if k == "pile_gravity":
            p.pile_gravity[:] = v
        else:
            setattr(p, k, v)
    return p


def batch_step(engine, scene_list, sp, dts, stream=None, allow=()):
    """One DFSPH step of every float32 scene in one call
    (al_df_batch_step_f32).  sp: solver parameters for all scenes, or a list
    with one per scene; dts: per-scene time steps.  Returns (new dts,
    reports, per-scene statuses)."""
    k = len(scene_list)
    sps = list(sp) if isinstance(sp, (list, tuple)) else [sp] * k
    arr = (_capi.SceneF32 * k)()
    keep = []
    dt_c = [ctypes.c_float(float(d)) for d in dts]
    reps = [_capi.StepReport() for _ in range(k)]
    for i, sc in enumerate(scene_list):
        assert sc.sfx == "f32", "batched steps: float32 scenes"
        fl = sc.fluid()
        keep.append(fl)
        a = arr[i]
        a.cn = _capi.ptr(sc.cn).value
        a.cni = _capi.ptr(sc.cni).value
        a.fluid = _capi.ptr(fl).value
        a.bodies = _capi.ptr(sc.bodies).value if sc.num_boundaries else None
        a.rigid = _capi.ptr(sc.rigid).value if sc.num_boundaries else None
        a.params = _capi.ptr(sps[i]).value
        a.dt = ctypes.addressof(dt_c[i])
        a.report = ctypes.addressof(reps[i])
    status = _capi.lib().al_df_batch_step_f32(engine.handle, arr, k, stream)
    _capi.check(status, "al_df_batch_step_f32", allow=allow)
    return [d.value for d in dt_c], reps, [arr[i].status for i in range(k)]


# ------------------------------------------------------------------ meshes
def mesh_aabb(vertices, offset=0.0):
    """(min, max, max_distance) of a mesh, as MeshDistance computes them
    (dg/mesh_distance.hpp:105-125): the vertex box grown by the offset, and
    the largest vertex radius plus the offset."""
    v = np.asarray(vertices, np.float64)
    return (v.min(0) - offset, v.max(0) + offset,
            float(np.sqrt((v * v).sum(1).max())) + offset)


def cube_mesh(half):
    """Closed box mesh [-half, half]^3 (12 triangles, outward winding)."""
    h = np.broadcast_to(np.asarray(half, np.float64), (3,))
    v = np.array([[x, y, z] for x in (-1, 1) for y in (-1, 1) for z in (-1, 1)]) * h
    faces = [(0, 1, 3), (0, 3, 2), (4, 6, 7), (4, 7, 5), (0, 4, 5), (0, 5, 1),
             (2, 3, 7), (2, 7, 6), (0, 2, 6), (0, 6, 4), (1, 5, 7), (1, 7, 3)]
    return v.astype(np.float32), np.asarray(faces, np.uint32)


def icosphere(radius, subdivisions=2):
    """Closed sphere mesh: an icosahedron subdivided `subdivisions` times
    with the new vertices projected to the sphere (outward winding)."""
    t = (1 + 5 ** 0.5) / 2
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t),
         (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    v = [np.asarray(p, np.float64) / np.linalg.norm(p) for p in v]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
         (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
         (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdivisions):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = v[a] + v[b]
                v.append(m / np.linalg.norm(m))
                cache[key] = len(v) - 1
            return cache[key]
        nf = []
        for a, b, c in f:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        f = nf
    return (np.asarray(v) * radius).astype(np.float32), np.asarray(f, np.uint32)


def load_obj(path):
    """Vertices [nv][3] and triangles [nf][3] of a Wavefront OBJ file (the
    format Mesh reads for MeshDistance bodies); polygons are fanned into
    triangles, `v/vt/vn` face entries and negative indices are accepted."""
    verts, faces = [], []
    with open(path) as fh:
        for line in fh:
            parts = line.split()
            if not parts:
                continue
            if parts[0] == "v":
                verts.append([float(x) for x in parts[1:4]])
            elif parts[0] == "f":
                idx = []
                for p in parts[1:]:
                    k = int(p.split("/")[0])
                    idx.append(k - 1 if k > 0 else len(verts) + k)
                for j in range(1, len(idx) - 1):
                    faces.append((idx[0], idx[j], idx[j + 1]))
    return np.asarray(verts, np.float32), np.asarray(faces, np.uint32)


# ------------------------------------------------------------------ pellets
def box_shell_pellets(inner_size, spacing, layers=3):
    """Boundary particles of a box container in its frame (centred): lattice
    points of the given spacing in `layers` layers outside the interior box
    of size inner_size (the fluid side), for the pellet boundary model."""
    half = 0.5 * np.asarray(inner_size, np.float64)
    lo = -half - (layers - 0.5) * spacing
    counts = np.floor((2 * half + (2 * layers - 1) * spacing) / spacing).astype(int) + 1
    axes = [lo[k] + spacing * np.arange(counts[k]) for k in range(3)]
    g = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 3)
    outside = np.any(np.abs(g) > half, axis=1)
    return g[outside]


def sphere_pellets(radius, spacing, thickness):
    """Boundary particles of a sphere in its frame: lattice points of the
    given spacing with radius - thickness < |x| <= radius."""
    m = int(np.ceil(radius / spacing))
    a = spacing * np.arange(-m, m + 1)
    g = np.stack(np.meshgrid(a, a, a, indexing="ij"), -1).reshape(-1, 3)
    r = np.linalg.norm(g, axis=1)
    return g[(r <= radius) & (r > radius - thickness)]
