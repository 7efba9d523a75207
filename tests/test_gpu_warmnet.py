"""Tensor-core kernels of the learned warm start against the CPU oracle
(oracle/warmnet_oracle.py), through the C ABI.

The oracle rounds to BF16 at the same points as the kernels and computes
in float64; remaining differences come from FP32 accumulation order, the
hardware tanh approximation inside GELU (relative error ~5e-4) and the
BF16 roundings those shift across a rounding boundary.  Bound, per output
with s = max(std, mean |value|) of the oracle's outputs: max |gpu - oracle|
<= 2e-2 s, mean <= 2e-3 s.
"""
import ctypes

import numpy as np
import pytest
import torch

from alluvion_b200 import _capi
from oracle import warmnet_oracle as wo

pytestmark = pytest.mark.gpu


def _net(seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    params = wo.init_params(seed)
    d = wo.unpack(params)
    d["b1"] = rng.normal(0, 0.1, 64)
    d["b2"] = rng.normal(0, 0.1, 64)
    d["b3"] = rng.normal(0, 0.1, 2)
    params = wo.pack(d).astype(np.float32)
    shift = rng.normal(0, 1, 12).astype(np.float32)
    scale = rng.uniform(0.5, 2.0, 12).astype(np.float32)
    out_scale = np.array([2.0, 0.5], np.float32)
    return params, shift, scale, out_scale


def _forward(engine, params_dev, shift, scale, out_scale, feats):
    net = _capi.make_warm_net(params_dev, shift, scale, out_scale)
    n = feats.shape[0]
    f = torch.from_numpy(np.ascontiguousarray(feats, np.float32)).cuda()
    out = torch.zeros((max(n, 1), 2), dtype=torch.float32, device="cuda")
    st = _capi.lib().al_warm_net_forward_f32(engine.handle, ctypes.byref(net),
                                             _capi.ptr(f) if n else None, n,
                                             _capi.ptr(out), None)
    _capi.check(st, "al_warm_net_forward_f32")
    return out[:n].cpu().numpy()


@pytest.mark.parametrize("n", [1, 1000, 200_003])
def test_forward_matches_oracle(engine, n):
    params, shift, scale, out_scale = _net(11)
    pdev = torch.from_numpy(params).cuda()
    rng = np.random.Generator(np.random.PCG64(n))
    feats = (shift + rng.normal(0, 1, (n, 12)) / scale).astype(np.float32)
    got = _forward(engine, pdev, shift, scale, out_scale, feats)
    ref = wo.predict(params, feats, shift, scale, out_scale)
    err = np.abs(got - ref)
    sd = np.maximum(ref.std(0), np.abs(ref).mean(0)) + 1e-12
    assert np.all(err.max(0) <= 2e-2 * sd), (err.max(0), sd)
    assert np.all(err.mean(0) <= 2e-3 * sd), (err.mean(0), sd)


def test_forward_empty(engine):
    params, shift, scale, out_scale = _net(3)
    pdev = torch.from_numpy(params).cuda()
    got = _forward(engine, pdev, shift, scale, out_scale, np.zeros((0, 12), np.float32))
    assert got.shape == (0, 2)


def _gradient(engine, params_dev, shift, scale, out_scale, feats, targets):
    net = _capi.make_warm_net(params_dev, shift, scale, out_scale)
    n = feats.shape[0]
    f = torch.from_numpy(np.ascontiguousarray(feats, np.float32)).cuda()
    t = torch.from_numpy(np.ascontiguousarray(targets, np.float32)).cuda()
    g = torch.zeros(_capi.WARM_NUM_PARAMS, dtype=torch.float32, device="cuda")
    loss = ctypes.c_double()
    st = _capi.lib().al_warm_net_gradient_f32(engine.handle, ctypes.byref(net), _capi.ptr(f),
                                              _capi.ptr(t), n, _capi.ptr(g), ctypes.byref(loss),
                                              None)
    _capi.check(st, "al_warm_net_gradient_f32")
    return g.cpu().numpy().astype(np.float64), loss.value


BLOCKS = [("W1", 0, 768), ("b1", 768, 832), ("W2", 832, 4928), ("b2", 4928, 4992),
          ("W3", 4992, 5120), ("b3", 5120, 5122)]


@pytest.mark.parametrize("n", [100, 70_001])
def test_gradient_matches_oracle(engine, n):
    """Loss and every parameter block's gradient against the oracle's
    quantised backward pass: relative L2 error <= 2e-2 per block, loss
    <= 1e-3 relative (70,001 rows: several tiles accumulate per CTA)."""
    params, shift, scale, out_scale = _net(21)
    pdev = torch.from_numpy(params).cuda()
    rng = np.random.Generator(np.random.PCG64(n + 5))
    feats = (shift + rng.normal(0, 1, (n, 12)) / scale).astype(np.float32)
    targets = (rng.normal(0, 1, (n, 2)) * out_scale).astype(np.float32)
    g, loss = _gradient(engine, pdev, shift, scale, out_scale, feats, targets)
    xn = wo.normalise(feats, shift, scale)
    ref_loss, ref = wo.loss_and_grad(params, xn, targets / out_scale)
    assert abs(loss - ref_loss) <= 1e-3 * ref_loss, (loss, ref_loss)
    for name, lo, hi in BLOCKS:
        e = np.linalg.norm(g[lo:hi] - ref[lo:hi]) / (np.linalg.norm(ref[lo:hi]) + 1e-30)
        assert e <= 2e-2, (name, e)


def test_adam_step_matches_oracle(engine):
    rng = np.random.Generator(np.random.PCG64(4))
    p = rng.normal(size=_capi.WARM_NUM_PARAMS).astype(np.float32)
    g = rng.normal(size=_capi.WARM_NUM_PARAMS).astype(np.float32)
    m = rng.normal(0, 0.1, _capi.WARM_NUM_PARAMS).astype(np.float32)
    v = rng.uniform(0, 0.1, _capi.WARM_NUM_PARAMS).astype(np.float32)
    dev = [torch.from_numpy(a.copy()).cuda() for a in (p, g, m, v)]
    st = _capi.lib().al_warm_net_adam_f32(engine.handle, *[_capi.ptr(t) for t in dev], 7,
                                          ctypes.c_float(1e-3), None)
    _capi.check(st, "al_warm_net_adam_f32")
    torch.cuda.synchronize()
    rp, rm, rv = wo.adam(p.astype(np.float64), g.astype(np.float64), m.astype(np.float64),
                         v.astype(np.float64), 7, lr=1e-3)
    # float32 against float64: each moment is a sum of terms of size ~|g|, so
    # the bound is a few float32 ulps of those terms (|g| <~ 4: 2e-7 for m)
    np.testing.assert_allclose(dev[0].cpu().numpy(), rp, rtol=1e-5, atol=1e-7)
    np.testing.assert_allclose(dev[2].cpu().numpy(), rm, rtol=1e-5, atol=2e-7)
    np.testing.assert_allclose(dev[3].cpu().numpy(), rv, rtol=1e-5, atol=2e-8)


def test_training_reduces_loss_on_teacher_targets(engine):
    """Adam with the engine's own gradients fits a teacher network's outputs:
    the loss falls by at least 10x in 300 steps of 8,192 rows."""
    teacher, shift, scale, out_scale = _net(31)
    student = wo.init_params(32)
    rng = np.random.Generator(np.random.PCG64(33))
    n = 8192
    pdev = torch.from_numpy(student.copy()).cuda()
    m = torch.zeros_like(pdev)
    v = torch.zeros_like(pdev)
    g = torch.zeros_like(pdev)
    losses = []
    for step in range(1, 301):
        feats = (shift + rng.normal(0, 1, (n, 12)) / scale).astype(np.float32)
        targets = wo.predict(teacher, feats, shift, scale, out_scale).astype(np.float32)
        net = _capi.make_warm_net(pdev, shift, scale, out_scale)
        f = torch.from_numpy(feats).cuda()
        t = torch.from_numpy(targets).cuda()
        loss = ctypes.c_double()
        _capi.check(_capi.lib().al_warm_net_gradient_f32(
            engine.handle, ctypes.byref(net), _capi.ptr(f), _capi.ptr(t), n, _capi.ptr(g),
            ctypes.byref(loss), None), "gradient")
        _capi.check(_capi.lib().al_warm_net_adam_f32(
            engine.handle, _capi.ptr(pdev), _capi.ptr(g), _capi.ptr(m), _capi.ptr(v), step,
            ctypes.c_float(3e-3), None), "adam")
        losses.append(loss.value)
    assert np.mean(losses[-10:]) <= 0.1 * np.mean(losses[:10]), (losses[:3], losses[-3:])
