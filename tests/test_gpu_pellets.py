"""The implicit SPH step on the pellet boundary model (al_i_step_pellets_*)
against the oracle's restatement of SolverI<TF>::step<0> with
VolumeMethod::pellets, through the C ABI.

Scene: a jittered fluid block in a box container represented by three
layers of pellets, and a moving, spinning sphere of pellets beside the
block (two-way coupled).  Bounds relative to each quantity's scale, as for
the volume-map steps: float32 after 1 step x 1e-5, v / density 1e-3,
pressure 1e-2, rigid force 1e-2 (5e-5 / 1e-2 / 5e-3 / 5e-2 / 5e-2 after 3);
float64 1e-11 .. 1e-6.  Iteration counts identical.

Known answers of the pressure extrapolation (extrapolate_pressure_to_pellet,
runner.hpp:2543-2607), run through a step without Jacobi iterations so the
beads keep the given pressure field: at r = 0.01 m every eigenvalue of the
weighted second moment is below the reference's 1e-2 cut, so a pellet gets
the Shepard average of its bead neighbors; at r = 0.5 m the linear term is
active and a linear pressure field is reproduced exactly at the pellets.
"""
import ctypes

import numpy as np
import pytest
import torch

from alluvion_b200 import _capi, scenes
from oracle import binding as orc

pytestmark = pytest.mark.gpu

TOL = {
    (np.float32, 1): dict(x=1e-5, v=1e-3, density=1e-3, p=1e-2, force=1e-2),
    (np.float32, 3): dict(x=5e-5, v=1e-2, density=5e-3, p=5e-2, force=5e-2),
    (np.float64, 1): dict(x=1e-12, v=1e-9, density=1e-11, p=1e-8, force=1e-7),
    (np.float64, 3): dict(x=1e-11, v=1e-8, density=1e-10, p=1e-7, force=1e-6),
}


def _body(dtype, mass, inertia, max_distance):
    _, BodyT, _, _ = _capi.real_types(dtype)
    b = BodyT()
    b.shape = _capi.SHAPE_SPHERE
    b.sign = 1.0
    b.mass = mass
    for k in range(3):
        b.inertia[k] = inertia[k]
        b.resolution[k] = 1
    b.max_distance = max_distance
    return b


def _scene(dtype, r=0.01, lattice=(10, 8, 10), seed=4, sphere=True, container=True,
           sphere_at=(23.5, 8.0, 15.0)):
    """Positions in units of r: the container's interior is 30 r wide."""
    cn = scenes.make_const(dtype, r)
    size = 30 * r
    x = scenes.fluid_block(lattice, (-r, -r, -r), r, dtype, seed=seed)
    local, bodies, rig = [], [], []
    if container:
        local.append(scenes.box_shell_pellets((size,) * 3, 2 * r, layers=3))
        bodies.append(_body(dtype, 0.0, (1, 1, 1), 0.0))
        rig.append(scenes.rigid_state(dtype, x=(size / 2,) * 3))
    if sphere:
        rad = 4 * r
        ball = scenes.sphere_pellets(rad, 2 * r, 3 * r)
        local.append(ball)
        m = 0.2
        bodies.append(_body(dtype, m, scenes.sphere_inertia(m, rad), rad))
        rig.append(scenes.rigid_state(dtype, x=tuple(r * np.asarray(sphere_at)),
                                      v=(-0.2, 0.0, 0.0), omega=(0.0, 0.0, 1.0)))
    counts = [len(p) for p in local]
    local = np.concatenate(local).astype(dtype)
    h = float(cn.kernel_radius)
    cni = scenes.make_consti((-0.2 * size,) * 3, (1.2 * size,) * 3, h, len(bodies))
    BodyT = type(bodies[0])
    barr = (BodyT * len(bodies))(*bodies)
    rarr = (type(rig[0]) * len(rig))(*rig)
    return cn, cni, x, barr, rarr, local, counts


def _device_run(engine, dtype, cn, cni, x, barr, rarr, local, counts, sp, dt, steps,
                pressure=None, v=None):
    n = len(x)
    td = torch.float32 if dtype == np.float32 else torch.float64
    X = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    V = (torch.from_numpy(np.ascontiguousarray(v)).cuda() if v is not None
         else torch.zeros(n, 3, dtype=td, device="cuda"))
    A = torch.zeros(n, 3, dtype=td, device="cuda")
    RHO = torch.zeros(n, dtype=td, device="cuda")
    P = (torch.from_numpy(np.ascontiguousarray(pressure)).cuda() if pressure is not None
         else torch.zeros(n, dtype=td, device="cuda"))
    ADV = torch.zeros(n, dtype=td, device="cuda")
    fluid = _capi.make_fluid(n, particle_x=X, particle_v=V, particle_a=A, particle_density=RHO,
                             particle_pressure=P, particle_density_adv=ADV)
    L = torch.from_numpy(np.ascontiguousarray(local)).cuda()
    PX = torch.zeros(len(local), 3, dtype=td, device="cuda")
    PV = torch.zeros(len(local), 3, dtype=td, device="cuda")
    PP = torch.zeros(len(local), dtype=td, device="cuda")
    pel = (_capi.PelletsF32 if dtype == np.float32 else _capi.PelletsF64)()
    pel.local_x = L.data_ptr()
    pel.num_pellets = len(local)
    for b, c in enumerate(counts):
        pel.count[b] = c
    pel.x = PX.data_ptr()
    pel.v = PV.data_ptr()
    pel.pressure = PP.data_ptr()
    fn = getattr(_capi.lib(), "al_i_step_pellets_" + _capi.suffix(dtype))
    real = _capi.real_types(dtype)[3]
    dt_c = real(dt)
    reps = []
    for _ in range(steps):
        rep = _capi.StepReport()
        _capi.check(fn(engine.handle, _capi.ptr(cn), _capi.ptr(cni), _capi.ptr(fluid),
                       _capi.ptr(barr), _capi.ptr(rarr), _capi.ptr(pel), _capi.ptr(sp),
                       _capi.ptr(dt_c), _capi.ptr(rep), None), "al_i_step_pellets")
        reps.append(rep)
    g = lambda t: t.cpu().numpy()
    return dict(x=g(X), v=g(V), density=g(RHO), pressure=g(P), a=g(A), px=g(PX), pp=g(PP),
                pv=g(PV),
                dt=float(dt_c.value), reps=reps,
                rigid=scenes.rigid_array(dtype, [rarr[b] for b in range(len(rarr))]))


def _oracle_run(dtype, cn, cni, x, barr, rarr, local, counts, sp, dt, steps, pressure=None,
                v=None):
    n = len(x)
    z = lambda *s: np.zeros(s, dtype)
    state = dict(x=np.ascontiguousarray(x).copy(),
                 v=np.ascontiguousarray(v).copy() if v is not None else z(n, 3),
                 a=z(n, 3), density=z(n), density_adv=z(n),
                 pressure=np.ascontiguousarray(pressure).copy() if pressure is not None else z(n))
    rigid = scenes.rigid_array(dtype, [rarr[b] for b in range(len(rarr))])
    dt_out, reps, px, pp = orc.run_pellets(cn, cni, barr, rigid, state, local, counts, sp, dt,
                                           steps)
    return dict(state, px=px, pp=pp, dt=dt_out, reps=reps, rigid=rigid)


def _close(a, b, rel, what):
    scale = max(np.abs(b).max(), 1e-30)
    err = np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)).max() / scale
    assert err <= rel, "%s: max error %.3e of scale %.3e (bound %.1e)" % (what, err, scale, rel)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("steps", [1, 3])
def test_pellet_step_parity(engine, dtype, steps):
    cn, cni, x, barr, rarr, local, counts = _scene(dtype)
    sp = scenes.solver_params()
    dt0 = 1e-4
    rarr_o = (type(rarr[0]) * len(rarr))(*[rarr[b] for b in range(len(rarr))])
    ref = _oracle_run(dtype, cn, cni, x, barr, rarr_o, local, counts, sp, dt0, steps)
    got = _device_run(engine, dtype, cn, cni, x, barr, rarr, local, counts, sp, dt0, steps)
    tol = TOL[(dtype, steps)]
    for r, o in zip(got["reps"], ref["reps"]):
        assert r.num_density_solve == o.num_density_solve
        assert list(r.grid_anomaly) == [0, 0, 0] == list(o.grid_anomaly)
        assert r.dt == pytest.approx(o.dt, rel=1e-5)
    assert got["reps"][0].num_density_solve >= 2
    _close(got["x"], ref["x"], tol["x"], "x")
    _close(got["v"], ref["v"], tol["v"], "v")
    _close(got["density"], ref["density"], tol["density"], "density")
    _close(got["pressure"], ref["pressure"], tol["p"], "pressure")
    _close(got["px"], ref["px"], tol["x"], "pellet x")
    _close(got["pp"], ref["pp"], tol["p"], "pellet pressure")
    _close(got["rigid"][:, :3], ref["rigid"][:, :3], tol["x"], "rigid x")
    f_ref = np.array(ref["reps"][-1].force[1])
    assert np.abs(f_ref).max() > 0
    _close(np.array(got["reps"][-1].force[1]), f_ref, tol["force"], "sphere force")
    _close(np.array(got["reps"][-1].torque[1]), np.array(ref["reps"][-1].torque[1]),
           tol["force"], "sphere torque")
    # the fluid at the walls feels the container pellets
    assert got["pp"].max() > 0


def _neighbors_brute(points, beads, h):
    d2 = ((points[:, None, :] - beads[None, :, :]) ** 2).sum(-1)
    return d2 < h * h


def test_pellet_extrapolation_shepard_at_small_scale(engine):
    dtype = np.float64
    cn, cni, x, barr, rarr, local, counts = _scene(dtype, sphere=False)
    rng = np.random.Generator(np.random.PCG64(7))
    p_in = rng.uniform(100.0, 200.0, size=len(x))
    sp = scenes.solver_params(min_density_solve=0, max_density_solve=0)
    got = _device_run(engine, dtype, cn, cni, x, barr, rarr, local, counts, sp, 1e-5, 1,
                      pressure=p_in)
    h = float(cn.kernel_radius)
    px = got["px"]
    nb = _neighbors_brute(px, x, h)
    r = np.sqrt(((px[:, None, :] - x[None]) ** 2).sum(-1))
    q = r / h
    k = float(cn.cubic_kernel_k)
    W = np.where(q <= 0.5, k * (6 * q ** 3 - 6 * q ** 2 + 1), 2 * k * (1 - q) ** 3) * nb
    ws = W.sum(1)
    has = ws > 0
    want = np.where(has, (W * p_in[None]).sum(1) / np.where(has, ws, 1), 0.0)
    assert has.sum() > 300
    np.testing.assert_allclose(got["pp"], want, rtol=1e-9, atol=1e-9)


def test_pellet_extrapolation_linear_at_large_scale(engine):
    """r = 0.5 m: the MLS plane is active; a linear pressure field (positive
    everywhere) comes back exactly at pellets surrounded by beads (a sphere
    of pellets placed inside the fluid block, off the lattice)."""
    dtype = np.float64
    kw = dict(r=0.5, lattice=(10, 10, 10), container=False, sphere_at=(9.5, 9.2, 9.6))
    cn, cni, x, barr, rarr, local, counts = _scene(dtype, **kw)
    rarr_o = (type(rarr[0]) * len(rarr))(*[rarr[b] for b in range(len(rarr))])  # pre-step pose
    a0, grad = 1000.0, np.array([30.0, -20.0, 10.0])
    p_in = a0 + x @ grad
    sp = scenes.solver_params(min_density_solve=0, max_density_solve=0, max_dt=1e-4)
    got = _device_run(engine, dtype, cn, cni, x, barr, rarr, local, counts, sp, 1e-5, 1,
                      pressure=p_in)
    h = float(cn.kernel_radius)
    px = got["px"]
    cnt = _neighbors_brute(px, x, h).sum(1)
    full = cnt >= 24
    assert full.sum() > 20
    np.testing.assert_allclose(got["pp"][full], a0 + px[full] @ grad, rtol=1e-9)
    # and the oracle agrees everywhere
    cn2, cni2, x2, barr2, _, local2, counts2 = _scene(dtype, **kw)
    ref = _oracle_run(dtype, cn2, cni2, x2, barr2, rarr_o, local2, counts2, sp, 1e-5, 1,
                      pressure=p_in)
    _close(got["pp"], ref["pp"], 1e-10, "pellet pressure")


def test_pellet_step_errors(engine):
    dtype = np.float32
    cn, cni, x, barr, rarr, local, counts = _scene(dtype)
    bad = list(counts)
    bad[0] += 1
    with pytest.raises(_capi.EngineError):
        _device_run(engine, dtype, cn, cni, x, barr, rarr, local, bad, scenes.solver_params(),
                    1e-4, 1)


def test_sampling_with_pellets(engine):
    """sample_position_density / compute_sample_velocity / _vorticity
    _with_pellets: samples see the pellets (world positions and velocities
    from a pellet step) as in the reference's *_with_pellets kernels."""
    dtype = np.float32
    cn, cni, x, barr, rarr, local, counts = _scene(dtype)
    got = _device_run(engine, dtype, cn, cni, x, barr, rarr, local, counts,
                      scenes.solver_params(), 1e-4, 1)
    r = float(cn.particle_radius)
    g = np.linspace(-5 * r, 35 * r, 21)
    sx = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3).astype(dtype)
    s = len(sx)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    X, RHO, V, SX = dev(got["x"]), dev(got["density"]), dev(got["v"]), dev(sx)
    PX, PV = dev(got["px"]), dev(got["pv"])
    outs = {k: torch.zeros((s, 3) if k in ("v", "vorticity") else (s,), device="cuda")
            for k in ("density", "position_density", "v", "vorticity")}
    req = _capi.SampleF32()
    req.sample_x = SX.data_ptr()
    req.num_samples = s
    req.particle_density = RHO.data_ptr()
    req.particle_v = V.data_ptr()
    req.sample_density = outs["density"].data_ptr()
    req.sample_position_density = outs["position_density"].data_ptr()
    req.sample_v = outs["v"].data_ptr()
    req.sample_vorticity = outs["vorticity"].data_ptr()
    req.pellet_x = PX.data_ptr()
    req.pellet_v = PV.data_ptr()
    req.num_pellets = len(local)
    _capi.check(_capi.lib().al_sample_fluid_f32(engine.handle, _capi.ptr(cn), _capi.ptr(cni),
                                                X.data_ptr(), len(x), None, _capi.ptr(req),
                                                None), "sample with pellets")
    ref, overflow = orc.sample_fluid(cn, cni, got["x"], None, sx, got["density"], got["v"],
                                     outputs=("density", "position_density", "v", "vorticity"),
                                     pellet_x=got["px"], pellet_v=got["pv"])
    assert not overflow
    for k in ("density", "position_density", "v"):
        _close(outs[k].cpu().numpy(), ref[k], 1e-5, k)
    _close(outs["vorticity"].cpu().numpy(), ref["vorticity"], 1e-4, "vorticity")
    # the pellets count: samples in the container walls have position density
    pd = outs["position_density"].cpu().numpy()
    in_wall = np.any(sx < -4 * r, axis=1)  # more than h from every particle
    assert pd[in_wall].max() > 0 and outs["density"].cpu().numpy()[in_wall].max() == 0
    # a moving pellet sphere gives samples near it the sphere's velocity
    assert np.abs(ref["v"]).max() > 0


def test_periodic_pellet_pipe_matches_oracle(engine):
    """SolverI::step<1> on the pellet branch: a pipe of pellet rings, periodic
    in y over 8 cells, fluid falling through the seam."""
    dtype = np.float32
    r = 0.01
    cn = scenes.make_const(dtype, r)
    h = float(cn.kernel_radius)
    L = 8 * h
    R, centre = 0.1, 0.15
    ys = -L / 2 + r + 2 * r * np.arange(int(round(L / (2 * r))))
    rings = []
    for k in range(3):
        rho = R + r + 2 * r * k
        m = int(round(2 * np.pi * rho / (2 * r)))
        th = 2 * np.pi * np.arange(m) / m
        ring = np.stack([rho * np.cos(th), np.zeros(m), rho * np.sin(th)], 1)
        for y in ys:
            rings.append(ring + np.array([0.0, y, 0.0]))
    local = np.concatenate(rings).astype(dtype)
    a = np.arange(centre - R + 1.5 * r, centre + R - r, 2 * r)
    fy = -L / 2 + 1e-4 + 2 * r * np.arange(int(round(L / (2 * r))))
    X, Y, Z = np.meshgrid(a, fy, a, indexing="ij")
    x = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
    x = x[np.hypot(x[:, 0] - centre, x[:, 2] - centre) < R - r].astype(dtype)
    v = np.zeros_like(x)
    v[:, 1] = -2.0
    cni = scenes.make_consti((0.0, -L / 2, 0.0), (0.3, L / 2, 0.3), h, 1)
    cni.grid_offset[1] = -4
    cni.grid_res[1] = 8
    body = _body(dtype, 0.0, (1, 1, 1), 0.0)
    barr = (type(body) * 1)(body)
    rarr = (type(scenes.rigid_state(dtype)) * 1)(scenes.rigid_state(dtype, x=(centre, 0.0, centre)))
    rarr_o = (type(rarr[0]) * 1)(rarr[0])
    sp = scenes.solver_params(wrap_y=1, wrap_length=L)
    steps = 3
    ref = _oracle_run(dtype, cn, cni, x, barr, rarr_o, local, [len(local)], sp, 1e-4, steps, v=v)
    got = _device_run(engine, dtype, cn, cni, x, barr, rarr, local, [len(local)], sp, 1e-4, steps,
                      v=v)
    for rr, o in zip(got["reps"], ref["reps"]):
        assert rr.num_density_solve == o.num_density_solve
        assert list(rr.grid_anomaly) == [0, 0, 0]
    crossed = (x[:, 1] < -L / 2 + 1e-3) & (got["x"][:, 1] > L / 2 - 3e-3)
    assert crossed.sum() > 10
    dx = got["x"].astype(np.float64) - ref["x"]
    dx[:, 1] -= L * np.round(dx[:, 1] / L)
    assert np.abs(dx).max() <= 5e-5 * 0.3
    _close(got["v"], ref["v"], 1e-2, "v")
    _close(got["density"], ref["density"], 5e-3, "density")
    _close(got["pressure"], ref["pressure"], 5e-2, "pressure")
