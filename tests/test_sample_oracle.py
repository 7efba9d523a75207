"""CPU checks of the oracle's sampling and histogram restatements.

* histogram256: hand-worked known answers of the reference's quantize
  (runner.hpp:4516-4536): floor((v - v_min) * step_inverse) saturated to
  uint32 by __float2uint_rd, low byte kept -- so v_max itself wraps into
  bin 0, NaN and everything below v_min land in bin 0, +inf in bin 255;
  with a mask only entries equal to 1 count (runner.hpp:4466-4479).
* calculate_kl_divergence against a direct numpy sum.
* sample_fluid: the grid-based oracle against a brute-force loop over every
  particle (pure Python, small case), including the reference's exclusion
  of the particle whose index equals the sample's (runner.hpp:1895).
"""
import math

import numpy as np

from alluvion_b200 import scenes
from oracle import binding as orc


def test_histogram_known_answers():
    v = np.array([0.0, 0.5, 0.99, 1.0, -1.0, np.nan, 2.0, 0.25, np.inf, -np.inf, 1.0 - 2 ** -10],
                 np.float32)
    h = orc.histogram256(v, 0.0, 1.0)
    want = np.zeros(256, np.uint32)
    # 0, 1.0 (= 256 -> 0), -1, NaN, 2.0 (= 512 -> 0), -inf
    want[0] = 6
    want[128] = 1   # 0.5
    want[253] = 1   # 0.99 * 256 = 253.44
    want[64] = 1    # 0.25
    want[255] = 2   # +inf saturates to 2^32 - 1; 1 - 2^-10 -> 255.75
    assert np.array_equal(h, want), np.nonzero(h != want)
    mask = np.array([1, 0, 1, 0.5, 1, 1, 0, 1, 1, 0, 1], np.float32)
    hm = orc.histogram256(v, 0.0, 1.0, mask)
    want_m = np.zeros(256, np.uint32)
    want_m[0] = 3      # 0.0, -1.0, NaN
    want_m[253] = 1
    want_m[64] = 1
    want_m[255] = 2
    assert np.array_equal(hm, want_m), np.nonzero(hm != want_m)
    # a shifted range: step_inverse = float(256 / (4 - (-4))) = 32
    h2 = orc.histogram256(np.array([-4.0, -3.99, 0.0, 3.99], np.float32), -4.0, 4.0)
    assert h2[0] == 2 and h2[128] == 1 and h2[255] == 1


def test_kl_divergence_matches_numpy():
    rng = np.random.Generator(np.random.PCG64(3))
    p = rng.integers(0, 50, size=256).astype(np.uint32)
    q = rng.integers(0, 50, size=256).astype(np.uint32)
    p[::5] = 0
    q[::7] = 0
    n_p, n_q = int(p.sum()), int(q.sum())
    lb = 0.5
    want = sum(pi / n_p * math.log(pi / max(qi, lb) * (n_q / n_p))
               for pi, qi in zip(p.astype(float), q.astype(float)) if pi > 0)
    got = orc.kl_divergence(p, q, n_p, n_q, lb)
    assert abs(got - want) <= 1e-12 * abs(want)


def _brute_force(cn, x, rho, v, sx):
    h2 = float(cn.kernel_radius_sqr)
    h = float(cn.kernel_radius)
    k = float(cn.cubic_kernel_k)

    def w(r):
        q = r / h
        if q > 1:
            return 0.0
        if q <= 0.5:
            return k * (6 * q ** 3 - 6 * q ** 2 + 1)
        return k * 2 * (1 - q) ** 3

    dens = np.zeros(len(sx))
    vel = np.zeros((len(sx), 3))
    for s, xs in enumerate(sx):
        for j, xj in enumerate(x):
            d = xs - xj
            if j == s or float(d @ d) >= h2:
                continue
            ww = w(math.sqrt(float(d @ d)))
            dens[s] += float(cn.particle_vol) * ww
            vel[s] += float(cn.particle_mass) / rho[j] * ww * v[j]
    return dens * float(cn.density0), vel


def test_sample_oracle_against_brute_force():
    rng = np.random.Generator(np.random.PCG64(9))
    cn = scenes.make_const(np.float32, 0.01)
    cni = scenes.make_consti((0, 0, 0), (0.2, 0.2, 0.2), float(cn.kernel_radius))
    x = rng.uniform(0.02, 0.18, size=(400, 3)).astype(np.float32)
    rho = rng.uniform(900, 1100, size=400).astype(np.float32)
    v = rng.normal(size=(400, 3)).astype(np.float32)
    # the first 50 samples sit on particles 0..49 (same indices), the rest anywhere
    sx = np.concatenate([x[:50], rng.uniform(0.0, 0.2, size=(150, 3))]).astype(np.float32)
    out, overflow = orc.sample_fluid(cn, cni, x, None, sx, rho, v,
                                     outputs=("density", "v", "vorticity"))
    assert not overflow
    dens, vel = _brute_force(cn, x.astype(np.float64), rho.astype(np.float64),
                             v.astype(np.float64), sx.astype(np.float64))
    np.testing.assert_allclose(out["density"], dens, rtol=1e-5, atol=1e-3)
    np.testing.assert_allclose(out["v"], vel, rtol=1e-4, atol=1e-4 * np.abs(vel).max())
    assert np.abs(out["vorticity"]).max() > 0
    # samples on particles 0..49 with the same indices miss exactly the
    # W(0) self term of a sum over every particle
    w0 = float(cn.density0) * float(cn.particle_vol) * float(cn.cubic_kernel_zero)
    full = dens[:50] + w0
    assert np.all(out["density"][:50] < full) and np.all(out["density"][:50] > 0)
    # rolled: sample i sits on particle i - 1 (included) and particle i is left out
    rolled = np.roll(sx[:50], 1, 0)
    out2, _ = orc.sample_fluid(cn, cni, x, None, rolled, rho, v, outputs=("density",))
    dens2, _ = _brute_force(cn, x.astype(np.float64), rho.astype(np.float64),
                            v.astype(np.float64), rolled.astype(np.float64))
    np.testing.assert_allclose(out2["density"], dens2, rtol=1e-5, atol=1e-3)
