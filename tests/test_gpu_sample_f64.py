"""Sampling and post-processing in double precision (Runner<double>'s
sample_fluid family, masks and histogram256) on the device against the
oracle's float64 restatements, through the C ABI:

* al_sample_fluid_f64 on a float64 dam break with a moving, spinning
  sphere: densities, quantity, velocity and vorticity within 1e-11 of each
  output's scale (float64; summation in the same canonical order, FMA
  contraction on the device).
* al_density_mask_f64 exactly, al_distance_mask_multiple_f64 against numpy
  away from the threshold, al_boundary_mask_f64 against the oracle.
* al_histogram256_f64 bit-exact against the oracle (with and without mask,
  16-byte aligned and unaligned, ragged n, NaN / inf / v_max), where the
  quantization forms (v - v_min) * step_inverse in double and converts it
  to float before rounding down, as quantize<double> does.
"""
import ctypes

import numpy as np
import pytest
import torch

from alluvion_b200 import _capi, scenes
from oracle import binding as orc
from conftest import dev, host

pytestmark = pytest.mark.gpu

F64 = torch.float64


def _scene(engine):
    sphere = dict(shape=_capi.SHAPE_SPHERE, params=[0.04], sign=1.0, resolution=16,
                  use_distance_grid=True, mass=0.0, x=(0.12, 0.255, 0.11), v=(0.3, -0.1, 0.2),
                  omega=(1.0, 2.0, -0.5))
    sc = scenes.dam_break(engine, np.float64, (10, 10, 10), 0.01, (0.3, 0.3, 0.3), [sphere],
                          seed=3, volume_resolution=16)
    sp = scenes.solver_params(integrate_rigids=0)
    for _ in range(3):
        sc.step("df", sp, 2e-4)
    return sc


def _close(got, ref, rel, what):
    scale = max(float(np.abs(ref).max()), 1e-300)
    err = float(np.abs(got - ref).max()) / scale
    assert err <= rel, "%s: max error %.3e of scale %.3e" % (what, err, scale)


@pytest.mark.parametrize("qdim", [1, 3])
def test_sample_fluid_f64_matches_oracle(engine, qdim):
    rng = np.random.Generator(np.random.PCG64(21))
    sc = _scene(engine)
    x = host(sc.x)
    lat = np.stack(np.meshgrid(*[np.linspace(-0.01, 0.31, 15)] * 3, indexing="ij"),
                   -1).reshape(-1, 3)
    sx_h = np.ascontiguousarray(np.concatenate([x[:400] + rng.normal(scale=0.004, size=(400, 3)),
                                                lat]), np.float64)
    sx = dev(sx_h)
    s = len(sx_h)
    nb = sc.num_boundaries
    sb = torch.zeros(nb, s, 4, dtype=F64, device="cuda")
    sbk = torch.zeros(nb, s, 4, dtype=F64, device="cuda")
    _capi.check(_capi.lib().al_compute_particle_boundary_f64(
        engine.handle, _capi.ptr(sc.cn), nb, _capi.ptr(sc.bodies), _capi.ptr(sc.rigid),
        sx.data_ptr(), s, sb.data_ptr(), sbk.data_ptr(), None), "boundary")
    q = sc.a if qdim == 3 else sc.kappa_v
    outs = {"density": torch.zeros(s, dtype=F64, device="cuda"),
            "position_density": torch.zeros(s, dtype=F64, device="cuda"),
            "quantity": torch.zeros((s, 3) if qdim == 3 else (s,), dtype=F64, device="cuda"),
            "v": torch.zeros(s, 3, dtype=F64, device="cuda"),
            "vorticity": torch.zeros(s, 3, dtype=F64, device="cuda")}
    req = _capi.SampleF64()
    req.sample_x = sx.data_ptr()
    req.num_samples = s
    req.particle_density = sc.density.data_ptr()
    req.particle_v = sc.v.data_ptr()
    req.particle_quantity = q.data_ptr()
    req.quantity_dim = qdim
    req.sample_boundary = sb.data_ptr()
    req.sample_boundary_kernel = sbk.data_ptr()
    for k, name in (("density", "sample_density"), ("position_density", "sample_position_density"),
                    ("quantity", "sample_quantity"), ("v", "sample_v"),
                    ("vorticity", "sample_vorticity")):
        setattr(req, name, outs[k].data_ptr())
    _capi.check(_capi.lib().al_sample_fluid_f64(engine.handle, _capi.ptr(sc.cn),
                                                _capi.ptr(sc.cni), sc.x.data_ptr(), sc.n,
                                                _capi.ptr(sc.rigid), _capi.ptr(req), None),
                "al_sample_fluid_f64")
    _, _, rigid = sc.host_bodies()
    ref, overflow = orc.sample_fluid(sc.cn, sc.cni, x, rigid, sx_h, host(sc.density),
                                     host(sc.v), host(q), host(sb), host(sbk))
    assert not overflow
    got = {k: host(t) for k, t in outs.items()}
    assert (got["density"] > 0).sum() > 400 and (got["density"] == 0).sum() > 400
    for k in ("density", "position_density", "quantity", "v", "vorticity"):
        _close(got[k], ref[k], 1e-11, k)


def test_masks_f64(engine):
    rng = np.random.Generator(np.random.PCG64(22))
    d = rng.normal(size=10001)
    d[::7] = 0.0
    mask = torch.zeros(len(d), dtype=torch.int32, device="cuda")
    d_d = dev(d)  # device inputs are held until the launches have read them
    _capi.check(_capi.lib().al_density_mask_f64(engine.handle, d_d.data_ptr(), len(d),
                                                mask.data_ptr(), None), "density mask")
    np.testing.assert_array_equal(host(mask), (d > 0).astype(np.int32))
    gx = rng.uniform(-1, 1, size=(20000, 3))
    buoys = rng.uniform(-0.5, 0.5, size=(3, 3))
    thr = 0.4
    m = torch.zeros(3, len(gx), dtype=F64, device="cuda")
    gx_d, buoys_d = dev(gx), dev(buoys)
    _capi.check(_capi.lib().al_distance_mask_multiple_f64(
        engine.handle, gx_d.data_ptr(), len(gx), buoys_d.data_ptr(), 3,
        ctypes.c_double(thr), m.data_ptr(), None), "distance mask")
    d2 = ((buoys[:, None, :] - gx[None, :, :]) ** 2).sum(-1)
    far = np.abs(d2 - thr * thr) > 1e-12
    np.testing.assert_array_equal(host(m)[far], (d2 <= thr * thr).astype(np.float64)[far])
    # boundary mask: a rotated analytic sphere
    cn = scenes.make_const(np.float64, 0.01)
    body = scenes.make_body(np.float64, cn, _capi.SHAPE_SPHERE, [0.1], 8)
    q = np.array([0.1, 0.3, -0.2, 0.9])
    q /= np.linalg.norm(q)
    rigid = scenes.rigid_state(np.float64, x=(0.05, -0.02, 0.01), q=tuple(q))
    sx = rng.uniform(-0.2, 0.2, size=(30000, 3))
    m0 = rng.uniform(size=len(sx)) + 0.5
    mk, sx_d = dev(m0.copy()), dev(sx)
    _capi.check(_capi.lib().al_boundary_mask_f64(
        engine.handle, _capi.ptr(body), _capi.ptr(rigid), sx_d.data_ptr(), len(sx),
        ctypes.c_double(0.02), mk.data_ptr(), None), "boundary mask")
    ref = orc.boundary_mask(body, scenes.rigid_array(np.float64, [rigid]).reshape(-1, 13), sx,
                            0.02, m0.copy())
    np.testing.assert_array_equal(host(mk), ref)
    assert 0 < (host(mk) == 0).sum() < len(sx)


@pytest.mark.parametrize("n", [0, 1, 2, 3, 1000003])
@pytest.mark.parametrize("masked", [False, True])
@pytest.mark.parametrize("offset", [0, 1])
def test_histogram256_f64_matches_oracle(engine, n, masked, offset):
    rng = np.random.Generator(np.random.PCG64(23 + n))
    v = rng.normal(0.5, 0.3, size=n + offset)
    if n > 8:
        v[offset + 1] = np.nan
        v[offset + 2] = np.inf
        v[offset + 3] = -np.inf
        v[offset + 4] = 1.0  # v_max wraps to bin 0
        v[offset + 5] = -5.0
    mk = rng.choice(np.array([0.0, 1.0, 0.5, 1.0]), size=n + offset)
    vd, md = dev(v), dev(mk)
    vp = vd.data_ptr() + 8 * offset if n else None
    mp = (md.data_ptr() + 8 * offset) if (masked and n) else None
    h = torch.zeros(256, dtype=torch.int32, device="cuda")
    _capi.check(_capi.lib().al_histogram256_f64(engine.handle, vp, mp, n, ctypes.c_double(0.0),
                                                ctypes.c_double(1.0), h.data_ptr(), None),
                "al_histogram256_f64")
    ref = orc.histogram256(v[offset:], 0.0, 1.0, mk[offset:] if masked else None)
    np.testing.assert_array_equal(host(h).view(np.uint32), ref)
    if not masked:
        assert int(host(h).view(np.uint32).sum()) == n
