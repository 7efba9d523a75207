"""The Runner metric reductions (calculate_se, calculate_se_weighted,
calculate_se_yz_masked, sum_products; runner.hpp:715-744, 4710-4800)
through the C ABI against numpy restatements of the reference's functors.

Each per-element term is formed in the arrays' real type exactly as numpy
forms it (float32 or float64, correctly rounded), so calculate_se matches
bit for bit; the sums are taken in double on both sides, in different
orders, so they agree within 1e-12 of their magnitude (float32 inputs) and
1e-13 (float64).  Ragged and empty inputs included."""
import ctypes

import numpy as np
import pytest
import torch

from alluvion_b200 import _capi
from conftest import dev, host

pytestmark = pytest.mark.gpu


def _sq(d):
    """|d|^2 summed over the last axis in order, in d's type."""
    s = d[..., 0] * d[..., 0]
    for k in range(1, d.shape[-1]):
        s = s + d[..., k] * d[..., k]
    return s


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("n,dims", [(0, 3), (1, 1), (1000, 1), (1000003, 3), (4097, 4)])
def test_metrics_match_numpy(engine, dtype, n, dims):
    rng = np.random.Generator(np.random.PCG64(n + dims))
    sfx = "f32" if dtype == np.float32 else "f64"
    lib = _capi.lib()
    v0 = rng.normal(size=(n, dims)).astype(dtype)
    v1 = rng.normal(size=(n, dims)).astype(dtype)
    w = rng.uniform(size=n).astype(dtype)
    mask = rng.choice(np.array([0.0, 1.0, 0.5], dtype), size=n)
    d0, d1, dw, dm = dev(v0), dev(v1), dev(w), dev(mask)
    se = torch.zeros(max(n, 1), dtype=d0.dtype, device="cuda")
    p = lambda t: t.data_ptr() if n else None
    _capi.check(getattr(lib, "al_calculate_se_" + sfx)(engine.handle, p(d0), p(d1), se.data_ptr(),
                                                       n, dims, None), "se")
    want_se = _sq(v0 - v1)
    np.testing.assert_array_equal(host(se)[:n], want_se)
    tol = 1e-12 if dtype == np.float32 else 1e-13
    out = ctypes.c_double()
    _capi.check(getattr(lib, "al_calculate_se_weighted_" + sfx)(
        engine.handle, p(d0), p(d1), p(dw), n, dims, ctypes.byref(out), None), "se weighted")
    ref = (w * want_se).astype(np.float64).sum()
    assert out.value == pytest.approx(ref, rel=tol, abs=1e-300)
    res = (ctypes.c_double * 4)()
    _capi.check(getattr(lib, "al_sum_products_" + sfx)(engine.handle, p(d0), p(d1), n, dims, res,
                                                       None), "sum products")
    ref = (v0 * v1).astype(np.float64).sum(axis=0)
    for k in range(dims):
        assert res[k] == pytest.approx(ref[k], rel=tol, abs=tol * max(1.0, abs(ref).max()) * 10)
    if dims == 3:
        _capi.check(getattr(lib, "al_calculate_se_yz_masked_" + sfx)(
            engine.handle, p(d0), p(d1), p(dm), n, ctypes.byref(out), None), "se yz masked")
        d = v0 - v1
        term = d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2]
        ref = np.where(mask == 1, term, 0).astype(np.float64).sum()
        assert out.value == pytest.approx(ref, rel=tol, abs=1e-300)


def test_metrics_reject_bad_dims(engine):
    out = ctypes.c_double()
    x = torch.zeros(8, device="cuda")
    assert _capi.lib().al_calculate_se_weighted_f32(engine.handle, x.data_ptr(), x.data_ptr(),
                                                    x.data_ptr(), 1, 5, ctypes.byref(out),
                                                    None) == _capi.AL_ERR_INVALID


def test_runner_statics_over_depot_variables(engine):
    """The same reductions as the reference's Runner static methods on
    Depot variables, with element offsets (runner.hpp:4710-4815)."""
    from alluvion_b200.depot import Depot
    dp = Depot(np.float32)
    rng = np.random.Generator(np.random.PCG64(3))
    n, off = 5000, 7
    a = rng.normal(size=(n + off, 3)).astype(np.float32)
    b = rng.normal(size=(n + off, 3)).astype(np.float32)
    w = rng.uniform(size=n + off).astype(np.float32)
    va, vb, vw, vse = dp.create(n + off, 3), dp.create(n + off, 3), dp.create(n + off, 1), \
        dp.create(n + off, 1)
    va.set(a)
    vb.set(b)
    vw.set(w)
    R = dp.Runner
    R.calculate_se(va, vb, vse, n, off)
    se = _sq(a - b)
    np.testing.assert_array_equal(vse.get()[off:], se[off:])
    got = R.calculate_se_weighted(va, vb, vw, n, off)
    assert got == pytest.approx(float((w[off:] * se[off:]).astype(np.float64).sum()), rel=1e-6)
    sp = R.sum_products(va, vb, n, off)
    np.testing.assert_allclose(sp, (a[off:] * b[off:]).astype(np.float64).sum(0), rtol=1e-5,
                               atol=1e-3)
    assert isinstance(R.sum_products(vw, vw, n, off), float)
    m = dp.create(n + off, 1)
    mk = rng.choice(np.array([0.0, 1.0], np.float32), size=n + off)
    m.set(mk)
    d = a - b
    ref = np.where(mk == 1, d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2], 0)[off:].astype(np.float64)
    assert R.calculate_se_yz_masked(va, vb, m, n, off) == pytest.approx(ref.sum(), rel=1e-6)
    hp, hq = dp.create(256, 1, np.uint32), dp.create(256, 1, np.uint32)
    p = rng.integers(0, 50, 256).astype(np.uint32)
    q = rng.integers(0, 50, 256).astype(np.uint32)
    hp.set(p)
    hq.set(q)
    from oracle import binding as orc
    kl = R.calculate_kl_divergence(hp, hq, int(p.sum()), int(q.sum()), 1e-3)
    assert kl == pytest.approx(orc.kl_divergence(p, q, int(p.sum()), int(q.sum()), 1e-3),
                               rel=1e-6)
    with pytest.raises(RuntimeError):
        R.calculate_se_weighted(va, vb, vw, n + off + 1, 0)
