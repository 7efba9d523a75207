"""CPU checks of the learned warm-start network's oracle
(oracle/warmnet_oracle.py) before it is trusted as the checker of the
tensor-core kernels: the analytic gradient against central differences of
the float64 loss, BF16 rounding, GELU and its derivative, one Adam step."""
import numpy as np

from oracle import warmnet_oracle as wo


def _batch(seed=1, B=64):
    rng = np.random.Generator(np.random.PCG64(seed))
    xn = rng.normal(size=(B, wo.NF))
    t = rng.normal(size=(B, wo.NO))
    return xn, t


def test_parameter_count_matches_header():
    assert wo.NUM_PARAMS == 5122
    p = wo.init_params(0)
    assert p.shape == (5122,) and p.dtype == np.float32
    d = wo.unpack(p)
    assert np.all(d["b1"] == 0) and d["W2"].shape == (64, 64)


def test_gradient_matches_central_differences():
    p = wo.init_params(3).astype(np.float64)
    xn, t = _batch()
    _, g = wo.loss_and_grad(p, xn, t, quantize=False)
    rng = np.random.Generator(np.random.PCG64(7))
    # every block of the layout, a few entries each
    idx = np.concatenate([rng.integers(lo, hi, 6) for lo, hi in
                          [(0, 768), (768, 832), (832, 4928), (4928, 4992), (4992, 5120),
                           (5120, 5122)]])
    for i in idx:
        fd = wo.finite_difference(p, xn, t, int(i))
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)) + 1e-8, (i, fd, g[i])


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -3.14159, 1e-30, 0.0])
    got = wo.bf16(x)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: ties to even -> 1
    assert got[0] == 1.0 and got[1] == 1.0 and got[2] == 1.0 + 2 ** -7
    assert abs(got[3] - -3.140625) == 0
    assert np.all(np.abs(got - x) <= np.abs(x) * 2 ** -8)


def test_gelu_and_derivative():
    x = np.linspace(-6, 6, 241)
    h = 1e-6
    fd = (wo.gelu(x + h) - wo.gelu(x - h)) / (2 * h)
    np.testing.assert_allclose(wo.gelu_grad(x), fd, atol=1e-8)
    assert abs(wo.gelu(0.0)) == 0 and abs(wo.gelu(6.0) - 6.0) < 1e-6


def test_quantised_gradient_close_to_float64():
    p = wo.init_params(5).astype(np.float64)
    xn, t = _batch(2, 256)
    l64, g64 = wo.loss_and_grad(p, xn, t, quantize=False)
    lq, gq = wo.loss_and_grad(p, xn, t, quantize=True)
    assert abs(lq - l64) <= 2e-2 * l64
    assert np.linalg.norm(gq - g64) <= 5e-2 * np.linalg.norm(g64)


def test_adam_first_step_moves_by_lr():
    p = np.zeros(4)
    g = np.array([1.0, -2.0, 0.5, 0.0])
    p1, m, v = wo.adam(p, g, np.zeros(4), np.zeros(4), 1, lr=1e-3)
    np.testing.assert_allclose(p1[:3], -1e-3 * np.sign(g[:3]), rtol=1e-6)
    assert p1[3] == 0
