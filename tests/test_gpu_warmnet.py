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
