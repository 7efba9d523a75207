"""Sampling and post-processing on the device against the oracle's
restatements, through the C ABI:

* al_sample_fluid_f32: sample_fluid (1- and 3-component quantities),
  sample_fluid_density, sample_position_density, compute_sample_velocity and
  compute_sample_vorticity on a dam break with a moving, spinning sphere.
  Both sum neighbors in canonical order; bounds relative to each output's
  scale: 1e-5 for densities, quantities and velocities (float32, FMA
  contraction on the device), 1e-4 for vorticity (a difference of
  velocities).  Known answer: a sample placed exactly on particle s, with
  index s, misses that particle (the reference's sample list skips the
  particle whose index equals the sample's), so its position density is the
  particle's density minus rho0 V W(0).
* masks: compute_density_mask exactly; compute_boundary_mask for an
  analytic sphere and a mesh box (distance grid), rotated, against the
  oracle; compute_distance_mask_multiple against numpy except within
  rounding of the threshold.
* histogram256 (with and without mask, aligned and unaligned, ragged n,
  NaN / inf / v_max / below v_min): bit-exact against the oracle, and at
  2^27 values against a torch restatement of the quantization.
* calculate_kl_divergence within 1e-12 relative of the oracle.
"""
import ctypes

import numpy as np
import pytest
import torch

from alluvion_b200 import _capi, scenes
from oracle import binding as orc
from conftest import dev, host

pytestmark = pytest.mark.gpu


def _scene(engine):
    # a kinematic sphere just above the block (fluid to y = 0.21), moving and spinning
    sphere = dict(shape=_capi.SHAPE_SPHERE, params=[0.04], sign=1.0, resolution=16,
                  use_distance_grid=True, mass=0.0, x=(0.12, 0.255, 0.11), v=(0.3, -0.1, 0.2),
                  omega=(1.0, 2.0, -0.5))
    sc = scenes.dam_break(engine, np.float32, (10, 10, 10), 0.01, (0.3, 0.3, 0.3), [sphere],
                          seed=3, volume_resolution=16)
    sp = scenes.solver_params(integrate_rigids=0)
    for _ in range(3):
        sc.step("df", sp, 2e-4)
    return sc


def _samples(sc, rng):
    x = host(sc.x)
    lat = np.stack(np.meshgrid(*[np.linspace(-0.01, 0.31, 17)] * 3, indexing="ij"),
                   -1).reshape(-1, 3)
    near = x[:500] + rng.normal(scale=0.004, size=(500, 3))
    return np.ascontiguousarray(np.concatenate([near, lat]), np.float32)


def _boundary(engine, sc, sx_dev):
    nb = sc.num_boundaries
    s = sx_dev.shape[0]
    sb = torch.zeros(nb, s, 4, device="cuda")
    sbk = torch.zeros(nb, s, 4, device="cuda")
    _capi.check(_capi.lib().al_compute_particle_boundary_f32(
        engine.handle, _capi.ptr(sc.cn), nb, _capi.ptr(sc.bodies), _capi.ptr(sc.rigid),
        _capi.ptr(sx_dev), s, _capi.ptr(sb), _capi.ptr(sbk), None), "boundary")
    return sb, sbk


def _request(sx, rho, v, q, sb, sbk, outs):
    req = _capi.SampleF32()
    req.sample_x = sx.data_ptr()
    req.num_samples = sx.shape[0]
    req.particle_density = rho.data_ptr()
    req.particle_v = v.data_ptr()
    if q is not None:
        req.particle_quantity = q.data_ptr()
        req.quantity_dim = 1 if q.dim() == 1 else q.shape[1]
    req.sample_boundary = sb.data_ptr() if sb is not None else None
    req.sample_boundary_kernel = sbk.data_ptr() if sbk is not None else None
    for k, name in (("density", "sample_density"), ("position_density", "sample_position_density"),
                    ("quantity", "sample_quantity"), ("v", "sample_v"),
                    ("vorticity", "sample_vorticity")):
        if k in outs:
            setattr(req, name, outs[k].data_ptr())
    return req


def _close(got, ref, rel, what):
    scale = max(float(np.abs(ref).max()), 1e-12)
    err = float(np.abs(got - ref).max()) / scale
    assert err <= rel, "%s: max error %.3e of scale %.3e" % (what, err, scale)


@pytest.mark.parametrize("qdim", [1, 3])
def test_sample_fluid_matches_oracle(engine, qdim):
    rng = np.random.Generator(np.random.PCG64(11))
    sc = _scene(engine)
    sx_h = _samples(sc, rng)
    sx = dev(sx_h)
    s = len(sx_h)
    sb, sbk = _boundary(engine, sc, sx)
    q = sc.a if qdim == 3 else sc.kappa_v
    outs = {"density": torch.zeros(s, device="cuda"),
            "position_density": torch.zeros(s, device="cuda"),
            "quantity": torch.zeros((s, 3) if qdim == 3 else (s,), device="cuda"),
            "v": torch.zeros(s, 3, device="cuda"), "vorticity": torch.zeros(s, 3, device="cuda")}
    req = _request(sx, sc.density, sc.v, q, sb, sbk, outs)
    st = _capi.lib().al_sample_fluid_f32(engine.handle, _capi.ptr(sc.cn), _capi.ptr(sc.cni),
                                         _capi.ptr(sc.x), sc.n, _capi.ptr(sc.rigid),
                                         _capi.ptr(req), None)
    _capi.check(st, "al_sample_fluid_f32")
    _, _, rigid = sc.host_bodies()
    ref, overflow = orc.sample_fluid(sc.cn, sc.cni, host(sc.x), rigid, sx_h, host(sc.density),
                                     host(sc.v), host(q), host(sb), host(sbk))
    assert not overflow
    got = {k: host(t) for k, t in outs.items()}
    assert (got["density"] > 0).sum() > 500 and (got["density"] == 0).sum() > 500
    for k in ("density", "position_density", "quantity", "v"):
        _close(got[k], ref[k], 1e-5, k)
    _close(got["vorticity"], ref["vorticity"], 1e-4, "vorticity")
    # the moving sphere contributes to velocities near it
    assert np.abs(host(sbk)[1, :, 3]).max() > 0


def test_sample_fluid_without_bodies_and_empty(engine):
    rng = np.random.Generator(np.random.PCG64(12))
    sc = _scene(engine)
    sx_h = _samples(sc, rng)
    sx = dev(sx_h)
    s = len(sx_h)
    cni = _capi.ConstI.from_buffer_copy(sc.cni)
    cni.num_boundaries = 0
    outs = {"density": torch.zeros(s, device="cuda"), "v": torch.zeros(s, 3, device="cuda"),
            "vorticity": torch.zeros(s, 3, device="cuda")}
    req = _request(sx, sc.density, sc.v, None, None, None, outs)
    _capi.check(_capi.lib().al_sample_fluid_f32(engine.handle, _capi.ptr(sc.cn), _capi.ptr(cni),
                                                _capi.ptr(sc.x), sc.n, None, _capi.ptr(req),
                                                None), "al_sample_fluid_f32")
    ref, _ = orc.sample_fluid(sc.cn, cni, host(sc.x), None, sx_h, host(sc.density), host(sc.v),
                              outputs=("density", "v", "vorticity"))
    for k in ("density", "v"):
        _close(host(outs[k]), ref[k], 1e-5, k)
    _close(host(outs["vorticity"]), ref["vorticity"], 1e-4, "vorticity")
    # no samples: nothing to do; no particles: zeros
    req.num_samples = 0
    _capi.check(_capi.lib().al_sample_fluid_f32(engine.handle, _capi.ptr(sc.cn), _capi.ptr(cni),
                                                _capi.ptr(sc.x), sc.n, None, _capi.ptr(req),
                                                None), "empty samples")
    req.num_samples = s
    outs["density"].fill_(7.0)
    _capi.check(_capi.lib().al_sample_fluid_f32(engine.handle, _capi.ptr(sc.cn), _capi.ptr(cni),
                                                None, 0, None, _capi.ptr(req), None),
                "no particles")
    assert float(outs["density"].abs().max()) == 0.0
    # vorticity without velocity output is rejected
    bad = _request(sx, sc.density, sc.v, None, None, None, {"vorticity": outs["vorticity"]})
    assert _capi.lib().al_sample_fluid_f32(engine.handle, _capi.ptr(sc.cn), _capi.ptr(cni),
                                           _capi.ptr(sc.x), sc.n, None, _capi.ptr(bad),
                                           None) == _capi.AL_ERR_INVALID


def test_sample_on_particles_skips_own_index(engine):
    sc = _scene(engine)
    n = sc.n
    nb = sc.num_boundaries
    # particle densities at the current positions (self term included)
    pb = torch.zeros(nb, n, 4, device="cuda")
    pbk = torch.zeros(nb, n, 4, device="cuda")
    _capi.check(_capi.lib().al_compute_particle_boundary_f32(
        engine.handle, _capi.ptr(sc.cn), nb, _capi.ptr(sc.bodies), _capi.ptr(sc.rigid),
        _capi.ptr(sc.x), n, _capi.ptr(pb), _capi.ptr(pbk), None), "boundary")
    rho = torch.zeros(n, device="cuda")
    cnt = torch.zeros(n, dtype=torch.int32, device="cuda")
    _capi.check(_capi.lib().al_update_particle_neighbors_f32(
        engine.handle, _capi.ptr(sc.cn), _capi.ptr(sc.cni), _capi.ptr(sc.x), n, _capi.ptr(pbk),
        _capi.ptr(rho), _capi.ptr(cnt), None, None, None), "neighbors")
    # samples exactly on the particles, same indices
    pd = torch.zeros(n, device="cuda")
    req = _request(sc.x, sc.density, sc.v, None, pb, pbk, {"position_density": pd})
    _capi.check(_capi.lib().al_sample_fluid_f32(engine.handle, _capi.ptr(sc.cn), _capi.ptr(sc.cni),
                                                _capi.ptr(sc.x), n, _capi.ptr(sc.rigid),
                                                _capi.ptr(req), None), "sample")
    self_term = float(sc.cn.density0) * float(sc.cn.particle_vol) * float(sc.cn.cubic_kernel_zero)
    np.testing.assert_allclose(host(pd) + self_term, host(rho), rtol=2e-5, atol=1e-3)
    # the same points under indices shifted by half the block (so the
    # particle sharing a sample's index is far from it) include every particle
    shift = n // 2
    perm = torch.roll(sc.x, shift, 0).contiguous()
    pb2, pbk2 = _boundary(engine, sc, perm)
    pd2 = torch.zeros(n, device="cuda")
    req = _request(perm, sc.density, sc.v, None, pb2, pbk2, {"position_density": pd2})
    _capi.check(_capi.lib().al_sample_fluid_f32(engine.handle, _capi.ptr(sc.cn), _capi.ptr(sc.cni),
                                                _capi.ptr(sc.x), n, _capi.ptr(sc.rigid),
                                                _capi.ptr(req), None), "sample shifted")
    np.testing.assert_allclose(host(pd2), np.roll(host(rho), shift), rtol=2e-5, atol=1e-3)


def test_sample_fluid_periodic_y(engine):
    """make_neighbor_list<1>: a column periodic in y with period L = 8 cells;
    samples near y = +-L/2 see particles across the seam."""
    rng = np.random.Generator(np.random.PCG64(31))
    cn = scenes.make_const(np.float32, 0.01)
    h = float(cn.kernel_radius)
    L = 8 * h
    cni = scenes.make_consti((0.0, -L / 2, 0.0), (0.2, L / 2, 0.2), h,
                             max_num_neighbors_per_particle=128)
    cni.grid_offset[1] = -4
    cni.grid_res[1] = 8
    n = 1500
    x = np.stack([rng.uniform(0.02, 0.18, n), rng.uniform(-0.159, 0.159, n),
                  rng.uniform(0.02, 0.18, n)], 1).astype(np.float32)
    rho = rng.uniform(900, 1100, n).astype(np.float32)
    v = rng.normal(size=(n, 3)).astype(np.float32)
    q = rng.normal(size=n).astype(np.float32)
    sx_h = np.stack([rng.uniform(0.03, 0.17, 3000), rng.uniform(-0.159, 0.159, 3000),
                     rng.uniform(0.03, 0.17, 3000)], 1).astype(np.float32)
    sx = dev(sx_h)
    s = len(sx_h)
    xd, rd, vd, qd = dev(x), dev(rho), dev(v), dev(q)
    outs = {"density": torch.zeros(s, device="cuda"), "quantity": torch.zeros(s, device="cuda"),
            "v": torch.zeros(s, 3, device="cuda"), "vorticity": torch.zeros(s, 3, device="cuda")}
    req = _request(sx, rd, vd, qd, None, None, outs)
    req.wrap_y = 1
    req.wrap_length = L
    _capi.check(_capi.lib().al_sample_fluid_f32(engine.handle, _capi.ptr(cn), _capi.ptr(cni),
                                                _capi.ptr(xd), n, None, _capi.ptr(req), None),
                "periodic sample")
    ref, overflow = orc.sample_fluid(cn, cni, x, None, sx_h, rho, v, q,
                                     outputs=("density", "quantity", "v", "vorticity"),
                                     wrap_length=L)
    assert not overflow
    got = {k: host(t) for k, t in outs.items()}
    for k in ("density", "quantity", "v"):
        _close(got[k], ref[k], 1e-5, k)
    _close(got["vorticity"], ref["vorticity"], 1e-4, "vorticity")
    # across the seam: without wrapping, samples within h of y = +-L/2 lose density
    flat, _ = orc.sample_fluid(cn, cni, x, None, sx_h, rho, v, outputs=("density",))
    edge = np.abs(np.abs(sx_h[:, 1]) - L / 2) < 0.5 * h
    inner = np.abs(sx_h[:, 1]) < L / 2 - h
    assert np.all(got["density"][edge] > flat["density"][edge])
    np.testing.assert_allclose(got["density"][inner], flat["density"][inner], rtol=1e-6)
    # a non-positive period is rejected
    req.wrap_length = 0.0
    assert _capi.lib().al_sample_fluid_f32(engine.handle, _capi.ptr(cn), _capi.ptr(cni),
                                           _capi.ptr(xd), n, None, _capi.ptr(req),
                                           None) == _capi.AL_ERR_INVALID


def test_masks(engine):
    rng = np.random.Generator(np.random.PCG64(21))
    # density mask
    d = rng.normal(size=10001).astype(np.float32)
    d[::7] = 0.0
    m = torch.zeros(len(d), dtype=torch.int32, device="cuda")
    d_d = dev(d)
    _capi.check(_capi.lib().al_density_mask_f32(engine.handle, _capi.ptr(d_d), len(d),
                                                _capi.ptr(m), None), "density mask")
    assert np.array_equal(host(m), (d > 0).astype(np.int32))
    # distance mask, 3 buoys
    gx = rng.uniform(-1, 1, size=(20000, 3)).astype(np.float32)
    buoys = rng.uniform(-0.5, 0.5, size=(3, 3)).astype(np.float32)
    out = torch.zeros(3, len(gx), device="cuda")
    thr = np.float32(0.4)
    gx_d, buoys_d = dev(gx), dev(buoys)  # held: the launch reads them
    _capi.check(_capi.lib().al_distance_mask_multiple_f32(
        engine.handle, _capi.ptr(gx_d), len(gx), _capi.ptr(buoys_d), 3, ctypes.c_float(thr),
        _capi.ptr(out), None), "distance mask")
    diff = buoys[:, None, :] - gx[None]
    d2 = (diff[..., 0] * diff[..., 0] + diff[..., 1] * diff[..., 1]) + diff[..., 2] * diff[..., 2]
    want = (d2 <= thr * thr).astype(np.float32)
    bad = host(out) != want
    assert not np.any(bad & (np.abs(d2 - thr * thr) > 1e-6)), int(bad.sum())
    assert 0 < want.sum() < want.size


def test_boundary_mask_matches_oracle(engine):
    rng = np.random.Generator(np.random.PCG64(22))
    q = np.array([0.2, -0.4, 0.1, 0.8])
    q /= np.linalg.norm(q)
    specs = [dict(shape=_capi.SHAPE_SPHERE, params=[0.05], sign=1.0, resolution=16,
                  use_distance_grid=True, x=(0.15, 0.12, 0.14), q=tuple(q)),
             dict(shape=_capi.SHAPE_MESH, mesh=scenes.cube_mesh(0.04), resolution=20,
                  x=(0.16, 0.2, 0.15), q=tuple(q))]
    sc = scenes.dam_break(engine, np.float32, (4, 4, 4), 0.01, (0.3, 0.3, 0.3), specs, seed=0,
                          volume_resolution=12)
    hb, keep, rigid = sc.host_bodies()
    sx = rng.uniform(0.05, 0.27, size=(30000, 3)).astype(np.float32)
    for b in (1, 2):
        m0 = rng.uniform(size=len(sx)).astype(np.float32) + 0.5
        mask, sx_d = dev(m0), dev(sx)
        _capi.check(_capi.lib().al_boundary_mask_f32(
            engine.handle, ctypes.byref(sc.bodies[b]), ctypes.byref(sc.rigid[b]),
            _capi.ptr(sx_d), len(sx), ctypes.c_float(0.01), _capi.ptr(mask), None), "mask")
        rig = (type(sc.rigid[0]) * 1)(sc.rigid[b])
        ref = orc.boundary_mask(hb[b], rig, sx, 0.01, m0.copy())
        got = host(mask)
        bad = got != ref
        assert bad.sum() <= 3, (b, int(bad.sum()))
        zeroed = (ref == 0).sum()
        assert 100 < zeroed < len(sx) - 100, zeroed


SPECIALS = np.array([np.nan, np.inf, -np.inf, 1.0, 0.0, -0.25, 1.5, 0.999999, 3e9, -3e9],
                    np.float32)


@pytest.mark.parametrize("n", [0, 1, 3, 4, 5, 1000003])
@pytest.mark.parametrize("masked", [False, True])
@pytest.mark.parametrize("offset", [0, 1])
def test_histogram256_matches_oracle(engine, n, masked, offset):
    rng = np.random.Generator(np.random.PCG64(n + 7 * masked + 13 * offset))
    v = rng.normal(0.5, 0.3, size=n + offset).astype(np.float32)
    if n > 20:
        v[offset:offset + len(SPECIALS)] = SPECIALS
    mk = rng.choice(np.array([0.0, 1.0, 0.5, 1.0], np.float32), size=n + offset)
    vd, md = dev(v), dev(mk)
    hist = torch.full((256,), 12345, dtype=torch.int32, device="cuda")
    vp = vd.data_ptr() + 4 * offset
    mp = md.data_ptr() + 4 * offset if masked else None
    _capi.check(_capi.lib().al_histogram256_f32(engine.handle, vp, mp, n, ctypes.c_float(0.0),
                                                ctypes.c_float(1.0), _capi.ptr(hist), None),
                "histogram")
    ref = orc.histogram256(v[offset:], 0.0, 1.0, mk[offset:] if masked else None)
    got = host(hist).view(np.uint32)
    assert np.array_equal(got, ref), np.nonzero(got != ref)
    assert int(got.sum()) == (int((mk[offset:] == 1).sum()) if masked else n)


def test_histogram256_large_and_kl(engine):
    n = 1 << 27  # 512 MB, larger than L2
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    v = torch.randn(n, device="cuda", generator=g) * 0.2 + 0.4
    hist = torch.zeros(256, dtype=torch.int32, device="cuda")
    vmin, vmax = np.float32(-0.3), np.float32(1.1)
    _capi.check(_capi.lib().al_histogram256_f32(engine.handle, _capi.ptr(v), None, n,
                                                ctypes.c_float(vmin), ctypes.c_float(vmax),
                                                _capi.ptr(hist), None), "histogram")
    sinv = np.float32(256.0 / (float(vmax) - float(vmin)))
    t = (v - float(vmin)) * float(sinv)  # float32 sub, then mul: each rounded once
    qv = torch.where(torch.isnan(t), torch.zeros_like(t), t).floor().clamp(0, 4294967295.0)
    want = torch.bincount((qv.double().long() & 255), minlength=256)
    assert torch.equal(hist.long(), want)
    del t, qv
    # KL divergence of two histograms against the oracle
    h2 = torch.zeros(256, dtype=torch.int32, device="cuda")
    w = v[: n // 3] * 1.1
    _capi.check(_capi.lib().al_histogram256_f32(engine.handle, _capi.ptr(w), None, w.numel(),
                                                ctypes.c_float(vmin), ctypes.c_float(vmax),
                                                _capi.ptr(h2), None), "histogram 2")
    out = ctypes.c_double()
    _capi.check(_capi.lib().al_kl_divergence(engine.handle, _capi.ptr(hist), _capi.ptr(h2), n,
                                             w.numel(), ctypes.c_double(1e-3), 256,
                                             ctypes.byref(out), None), "kl")
    ref = orc.kl_divergence(host(hist).view(np.uint32), host(h2).view(np.uint32), n, w.numel(),
                            1e-3)
    assert ref > 0 and abs(out.value - ref) <= 1e-12 * abs(ref), (out.value, ref)
    # identical histograms: zero
    _capi.check(_capi.lib().al_kl_divergence(engine.handle, _capi.ptr(hist), _capi.ptr(hist), n,
                                             n, ctypes.c_double(1e-3), 256, ctypes.byref(out),
                                             None), "kl self")
    assert abs(out.value) < 1e-12
