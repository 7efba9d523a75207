"""The reference's Python object model (Depot / Store / Pile / SolverDf /
SolverIi / SolverI, alluvion/depot.py and lib/pyalluvion.cu) over the
engine, through the pybind11 module.  A scene built the reference's way
(Depot, Pile.add with analytic distances, solver fields) must step exactly
as the same scene driven through the C ABI: same constants, grids, bodies
and parameters reach the same entry points, so positions, velocities, dt
and rigid kinematics agree bit for bit."""
import numpy as np
import pytest
import torch

from alluvion_b200 import _capi, scenes
from alluvion_b200.depot import Depot, VolumeMethod

pytestmark = pytest.mark.gpu

R = 0.01
LATTICE = (8, 12, 8)
SIZE = (0.3, 0.4, 0.3)
SPHERE = dict(x=(0.15, 0.33, 0.15), r=0.04, rho=700.0)


def _abi_scene(engine, dtype):
    x = scenes.fluid_block(LATTICE, (0.02, 0.02, 0.02), R, dtype, seed=5)
    cn = scenes.make_const(dtype, R)
    h = float(cn.kernel_radius)
    mass = SPHERE["rho"] * 4 / 3 * np.pi * SPHERE["r"] ** 3
    bodies = [dict(shape=_capi.SHAPE_BOX, params=scenes.box_params(SIZE), sign=-1.0,
                   resolution=24, use_distance_grid=False, mass=0.0,
                   x=tuple(np.asarray(SIZE) / 2)),
              dict(shape=_capi.SHAPE_SPHERE, params=[SPHERE["r"]], sign=1.0, resolution=16,
                   use_distance_grid=False, mass=mass,
                   inertia=scenes.sphere_inertia(mass, SPHERE["r"]), x=SPHERE["x"])]
    cni = scenes.make_consti(-0.5 * h * np.ones(3), np.asarray(SIZE) + 0.5 * h, h, len(bodies))
    return scenes.DeviceScene(engine, dtype, cn, cni, x, bodies), x, mass


def _depot_scene(dtype, x, abi, mass, method="df"):
    dp = Depot(dtype)
    cn, cni = dp.cn, dp.cni
    h = 4 * R
    cn.set_kernel_radius(h)
    cn.set_particle_attr(R, 1000.0 * (2 * R) ** 3, 1000.0)
    cn.viscosity = 0.01
    cn.boundary_viscosity = 0.01
    cn.dfsph_factor_epsilon = 1e-6
    cn.gravity = (0.0, -9.81, 0.0)
    cni.grid_res = list(abi.cni.grid_res)
    cni.grid_offset = list(abi.cni.grid_offset)
    cni.max_num_particles_per_cell = abi.cni.max_num_particles_per_cell
    cni.max_num_neighbors_per_particle = abi.cni.max_num_neighbors_per_particle
    dp.copy_cn()
    runner = dp.Runner()
    pile = dp.Pile(dp, runner, 0)
    pile.add(dp.BoxDistance.create(SIZE), [24, 24, 24], sign=-1, x=list(np.asarray(SIZE) / 2))
    pile.add(dp.SphereDistance.create(SPHERE["r"]), [16, 16, 16], mass=mass,
             inertia_tensor=list(scenes.sphere_inertia(mass, SPHERE["r"])), x=list(SPHERE["x"]))
    pile.set_gravity((0.0, -9.81, 0.0))
    cls = {"df": dp.SolverDf, "ii": dp.SolverIi, "i": dp.SolverI}[method]
    solver = cls(runner, pile, dp, max_num_particles=len(x) + 100)
    solver.num_particles = len(x)
    solver.particle_x.set(x)
    solver.particle_v.set_zero()
    solver.reset_solving_var()
    solver.initial_dt = 2e-4
    solver.reset_t()
    solver.max_dt = 2e-4
    solver.cfl = 0.4
    return dp, pile, solver


@pytest.mark.parametrize("method", ["df", "ii", "i"])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_depot_steps_match_the_c_abi(engine, method, dtype):
    abi, x, mass = _abi_scene(engine, dtype)
    dp, pile, solver = _depot_scene(dtype, x, abi, mass, method)
    sp = scenes.solver_params()
    dt = 2e-4
    T = np.dtype(dtype).type
    t = T(0)
    for k in range(4):
        dt, rep = abi.step(method, sp, dt)
        solver.step()
        assert solver.dt == dt
        t = T(t + T(dt))
    st = abi.state()
    n = len(x)
    gx = solver.particle_x.get()[:n]
    gv = solver.particle_v.get()[:n]
    np.testing.assert_array_equal(gx, st["x"])
    np.testing.assert_array_equal(gv, st["v"])
    np.testing.assert_array_equal(solver.particle_density.get()[:n], st["density"])
    if method == "df":
        np.testing.assert_array_equal(solver.particle_kappa.get()[:n], st["kappa"])
        assert solver.num_density_solve == rep.num_density_solve
        assert solver.num_divergence_solve == rep.num_divergence_solve
    else:
        np.testing.assert_array_equal(solver.particle_pressure.get()[:n], st["pressure"])
        assert solver.num_density_solve == rep.num_density_solve
    # the sphere's kinematics: same device integration, written back to the pile
    rig = abi.rigid[1]
    np.testing.assert_array_equal(np.asarray(pile.x[1], dtype), np.asarray(rig.x[:], dtype))
    np.testing.assert_array_equal(np.asarray(pile.v[1], dtype), np.asarray(rig.v[:], dtype))
    np.testing.assert_array_equal(np.asarray(pile.q[1], dtype), np.asarray(rig.q[:], dtype))
    assert pile.x[1][1] < SPHERE["x"][1]  # it falls
    assert solver.t == t
    assert solver.max_v2 > 0 and solver.utilized_cfl > 0


def test_variables_and_neighbors(engine):
    dtype = np.float32
    abi, x, mass = _abi_scene(engine, dtype)
    dp, pile, solver = _depot_scene(dtype, x, abi, mass)
    n = len(x)
    # Coated get / set, byte offsets, zero-copy torch views
    v = dp.create([n], 3)
    assert v.get_shape() == [n] and v.get_num_primitives_per_element() == 3
    a = np.arange(3 * n, dtype=np.float32).reshape(n, 3)
    v.set(a)
    np.testing.assert_array_equal(v.get(), a)
    t = torch.as_tensor(v, device="cuda")
    assert t.shape == (n, 3) and t.dtype == torch.float32
    t.mul_(2)
    np.testing.assert_array_equal(v.get(), 2 * a)
    v.set(np.ones((1, 3), np.float32), offset=12)
    g = v.get()
    assert (g[1] == 1).all()
    np.testing.assert_array_equal(g[0], 2 * a[0])
    np.testing.assert_array_equal(g[2:], 2 * a[2:])
    with pytest.raises(RuntimeError):
        v.set(np.ones((n + 1, 3), np.float32))
    u = dp.create(4, 1, np.uint32)
    u.set(np.array([1, 2, 3, 4], np.uint32))
    assert u.get().tolist() == [1, 2, 3, 4]
    dp.remove(u)
    assert u.get_linear_shape() == 0
    # the standalone neighbor update in the reference layout (density with
    # the boundary terms of compute_all_boundaries)
    solver.compute_all_boundaries()
    solver.update_particle_neighbors()
    assert solver.grid_anomaly.get().tolist() == [0, 0, 0]
    nbr = solver.particle_neighbors.get()
    cnt = solver.particle_num_neighbors.get()[:n]
    from oracle import binding as orc
    odens, ocount, oindex, _, flags = orc.update_particle_neighbors(abi.cn, abi.cni, x)
    np.testing.assert_array_equal(cnt, ocount)
    j = nbr[:n, :, 3].view(np.uint32)
    for i in range(0, n, 97):
        assert j[i, :cnt[i]].tolist() == oindex[i, :cnt[i]].tolist()


def test_unsupported_options_raise(engine):
    dp = Depot(np.float32)
    dp.cn.set_kernel_radius(0.04)
    dp.cn.set_particle_attr(0.01, 0.008, 1000.0)
    dp.cni.grid_res = [8, 8, 8]
    dp.cni.max_num_neighbors_per_particle = 64
    dp.cni.max_num_particles_per_cell = 64
    runner = dp.Runner()
    pile = dp.Pile(dp, runner, 0)
    with pytest.raises(RuntimeError):
        dp.SolverDf(runner, pile, dp, 100, enable_vorticity=True)
    # pellets belong to VolumeMethod.pellets piles, within max_num_pellets
    with pytest.raises(RuntimeError):
        pile.add(dp.SphereDistance.create(0.05), [4, 4, 4], pellets=np.zeros((3, 3), np.float32))
    ppile = dp.Pile(dp, runner, 0, volume_method=VolumeMethod.pellets, max_num_pellets=4)
    with pytest.raises(RuntimeError):
        ppile.add(dp.SphereDistance.create(0.05), [4, 4, 4], pellets=np.zeros((5, 3), np.float32))
    s = dp.SolverDf(runner, pile, dp, 100)
    s.num_particles = 101
    s.dt = 1e-4
    with pytest.raises(RuntimeError):
        s.step()



def _depot_consts(dp, cni_src, r=R):
    cn, cni = dp.cn, dp.cni
    cn.set_kernel_radius(4 * r)
    cn.set_particle_attr(r, 1000.0 * (2 * r) ** 3, 1000.0)
    cn.viscosity = 0.01
    cn.boundary_viscosity = 0.01
    cn.dfsph_factor_epsilon = 1e-6
    cn.gravity = (0.0, -9.81, 0.0)
    cni.grid_res = list(cni_src.grid_res)
    cni.grid_offset = list(cni_src.grid_offset)
    cni.max_num_particles_per_cell = cni_src.max_num_particles_per_cell
    cni.max_num_neighbors_per_particle = cni_src.max_num_neighbors_per_particle
    return cn, cni


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_depot_pellet_step_matches_the_c_abi(engine, dtype):
    """SolverI on a pile with VolumeMethod.pellets (a box of pellets and a
    moving, spinning sphere of pellets) steps as al_i_step_pellets does;
    the pellets' world positions and pressures land after the particles in
    particle_x / particle_pressure, as in the reference."""
    from test_gpu_pellets import _scene as pellet_scene, _device_run
    r = 0.01
    cn_abi, cni_abi, x, barr, rarr, local, counts = pellet_scene(dtype)
    sp = scenes.solver_params()
    ref = _device_run(engine, dtype, cn_abi, cni_abi, x, barr, rarr, local, counts, sp, 1e-4, 2)
    dp = Depot(dtype)
    _depot_consts(dp, cni_abi, r)
    runner = dp.Runner()
    pile = dp.Pile(dp, runner, 0, volume_method=VolumeMethod.pellets,
                   max_num_pellets=len(local))
    size = 30 * r
    c0 = counts[0]
    pile.add(dp.BoxShellDistance.create([size] * 3, 2 * r), [1, 1, 1], pellets=local[:c0],
             x=[size / 2] * 3)
    rad = 4 * r
    m = 0.2
    pile.add(dp.SphereDistance.create(rad), [1, 1, 1], pellets=local[c0:], mass=m,
             inertia_tensor=list(scenes.sphere_inertia(m, rad)),
             x=list(r * np.asarray((23.5, 8.0, 15.0))))
    v, om = pile.v, pile.omega
    v[1], om[1] = [-0.2, 0.0, 0.0], [0.0, 0.0, 1.0]
    pile.v, pile.omega = v, om
    pile.set_gravity((0.0, -9.81, 0.0))
    assert pile.num_pellets == len(local)
    solver = dp.SolverI(runner, pile, dp, max_num_particles=len(x))
    n = len(x)
    solver.num_particles = n
    solver.particle_x.set(x)
    solver.initial_dt = 1e-4
    solver.reset_t()
    solver.max_dt, solver.cfl = 2e-4, 0.4
    for _ in range(2):
        solver.step()
    gx = solver.particle_x.get()
    np.testing.assert_array_equal(gx[:n], ref["x"])
    np.testing.assert_array_equal(solver.particle_v.get()[:n], ref["v"])
    np.testing.assert_array_equal(solver.particle_pressure.get()[:n], ref["pressure"])
    np.testing.assert_array_equal(gx[n:n + len(local)], ref["px"])
    np.testing.assert_array_equal(solver.particle_pressure.get()[n:n + len(local)], ref["pp"])
    assert solver.dt == ref["dt"]
    np.testing.assert_array_equal(np.asarray(pile.x[1], dtype), ref["rigid"][1, :3])
    # the other solvers do not step pellet piles
    with pytest.raises(RuntimeError):
        dp.SolverDf(runner, pile, dp, max_num_particles=n).step()


def test_solver_pellet_matches_the_c_abi(engine):
    """SolverPellet (set_pellets, step) relaxes pellets inside a sphere as
    al_relax_pellets_f32 does: positions, displacements (particle_v) and
    densities bit for bit."""
    dtype = np.float32
    cn = scenes.make_const(dtype, 0.01)
    Rs = 0.2
    body = scenes.make_body(dtype, cn, _capi.SHAPE_SPHERE, [Rs], 8, sign=-1.0)
    cni = scenes.make_consti((-Rs - 0.05,) * 3, (Rs + 0.05,) * 3, float(cn.kernel_radius))
    m = int(np.ceil(Rs / 0.02))
    a = 0.02 * (np.arange(-m, m + 1) + 0.25)
    g = np.stack(np.meshgrid(a, a, a, indexing="ij"), -1).reshape(-1, 3)
    g = g[np.linalg.norm(g, axis=1) < Rs - 0.03]
    rng = np.random.Generator(np.random.PCG64(2))
    x = (g + rng.uniform(-0.004, 0.004, g.shape)).astype(np.float32)
    X = torch.from_numpy(x.copy()).cuda()
    DX = torch.zeros_like(X)
    RHO = torch.zeros(len(x), device="cuda")
    p = _capi.pellet_relax_params()
    for _ in range(2):
        _capi.check(_capi.lib().al_relax_pellets_f32(
            engine.handle, _capi.ptr(cn), _capi.ptr(cni), _capi.ptr(body), X.data_ptr(), len(x),
            _capi.ptr(p), 1, DX.data_ptr(), RHO.data_ptr(), None), "relax")
    dp = Depot(dtype)
    _depot_consts(dp, cni, 0.01)
    runner = dp.Runner()
    pile = dp.Pile(dp, runner, 0, volume_method=VolumeMethod.pellets, max_num_pellets=0)
    pile.add(dp.SphereDistance.create(Rs), [8, 8, 8], sign=-1)
    solver = dp.SolverPellet(runner, pile, dp, max_num_particles=len(x))
    assert (solver.cohesion, solver.adhesion, solver.cfl_factor) == (4.0, 2.0, 0.25)
    pel = dp.create(len(x), 3)
    pel.set(x)
    solver.set_pellets(pel)
    assert solver.num_particles == len(x)
    for _ in range(2):
        solver.step()
    n = len(x)
    np.testing.assert_array_equal(solver.particle_x.get()[:n], X.cpu().numpy())
    np.testing.assert_array_equal(solver.particle_v.get()[:n], DX.cpu().numpy())
    np.testing.assert_array_equal(solver.particle_density.get()[:n], RHO.cpu().numpy())


def test_variable_and_pile_files_match_the_reference_layouts(engine, tmp_path):
    """Variable.write_file / read_file and Pile.write_file / read_file /
    get_size_from_file produce the reference's byte layouts (the ones
    alluvion_b200.alu restates) and read them back; float files load into
    double variables."""
    from alluvion_b200 import alu
    dp = Depot(np.float32)
    rng = np.random.Generator(np.random.PCG64(8))
    a = rng.normal(size=(10, 3)).astype(np.float32)
    v = dp.create(10, 3)
    v.set(a)
    p_all, p_part = tmp_path / "all.alu", tmp_path / "part.alu"
    v.write_file(str(p_all))
    v.write_file(str(p_part), 4, 2)  # elements 2..5
    ref_all, ref_part = tmp_path / "ref_all.alu", tmp_path / "ref_part.alu"
    alu.write_alu(ref_all, a, 3)
    alu.write_alu(ref_part, a[2:6], 3)
    assert p_all.read_bytes() == ref_all.read_bytes()
    assert p_part.read_bytes() == ref_part.read_bytes()
    w = dp.create(10, 3)
    assert w.read_file(str(p_part)) == 4
    np.testing.assert_array_equal(w.get()[:4], a[2:6])
    d = dp.create(10, 3, np.float64)
    assert d.read_file(str(p_all)) == 10
    np.testing.assert_array_equal(d.get(), a.astype(np.float64))
    with pytest.raises(RuntimeError):
        dp.create(10, 1).read_file(str(p_all))  # primitives per element differ
    with pytest.raises(RuntimeError):
        v.write_file(str(p_all), 11)
    # pile state files
    runner = dp.Runner()
    dp.cn.set_kernel_radius(0.04)
    dp.cn.set_particle_attr(0.01, 0.008, 1000.0)
    pile = dp.Pile(dp, runner, 0)
    for k in range(3):
        pile.add(dp.SphereDistance.create(0.05), [4, 4, 4], mass=1.0,
                 x=[0.1 * k, 0.2, 0.3], q=[0.0, 0.0, 0.0, 1.0])
    vv = pile.v
    vv[1] = [1.0, 2.0, 3.0]
    pile.v = vv
    pf = tmp_path / "pile.bin"
    pile.write_file(str(pf), 2.0, 1.0, 1.0)
    rig = scenes.rigid_array(np.float32, [
        scenes.rigid_state(np.float32, x=(0.1 * k, 0.2, 0.3), v=(1.0, 2.0, 3.0) if k == 1
                           else (0, 0, 0)) for k in range(3)]).reshape(-1, 13)
    rf = tmp_path / "ref_pile.bin"
    alu.write_pile(rf, rig, x_scale=2.0)
    assert pf.read_bytes() == rf.read_bytes()
    assert dp.Pile.get_size_from_file(str(pf)) == 3
    pile.read_file(str(rf), 1, 2, 1)  # body 1 of the file into body 2
    assert pile.v[2] == [1.0, 2.0, 3.0]
    assert pile.x[2] == pytest.approx([0.2, 0.4, 0.6])


def test_sample_all_boundaries_matches_the_c_abi(engine):
    """Solver.sample_all_boundaries (solver.hpp:186-203) writes the same
    boundary terms at sample points as al_compute_particle_boundary_f32
    called with the sample positions."""
    dtype = np.float32
    abi, x, mass = _abi_scene(engine, dtype)
    dp, pile, solver = _depot_scene(dtype, x, abi, mass)
    rng = np.random.Generator(np.random.PCG64(4))
    s = 3000
    sx = rng.uniform(0.0, 0.3, size=(s, 3)).astype(np.float32)
    vx = dp.create(s, 3)
    vx.set(sx)
    nb = pile.get_size()
    vb, vk = dp.create([nb, s], 4), dp.create([nb, s], 4)
    solver.sample_all_boundaries(vx, vb, vk, s)
    sx_d = torch.from_numpy(sx).cuda()
    sb = torch.zeros(nb, s, 4, device="cuda")
    sbk = torch.zeros(nb, s, 4, device="cuda")
    _capi.check(_capi.lib().al_compute_particle_boundary_f32(
        engine.handle, _capi.ptr(abi.cn), nb, _capi.ptr(abi.bodies), _capi.ptr(abi.rigid),
        sx_d.data_ptr(), s, sb.data_ptr(), sbk.data_ptr(), None), "boundary")
    np.testing.assert_array_equal(vb.get(), sb.cpu().numpy())
    np.testing.assert_array_equal(vk.get(), sbk.cpu().numpy())
    assert np.abs(vk.get()[:, :, 3]).max() > 0
    # rows of a [nb][capacity] variable with capacity != num_samples would
    # sit at another stride than the reference's Variable<2> indexing: refused
    wb, wk = dp.create([nb, s + 10], 4), dp.create([nb, s + 10], 4)
    with pytest.raises(Exception, match="num_samples"):
        solver.sample_all_boundaries(vx, wb, wk, s)
