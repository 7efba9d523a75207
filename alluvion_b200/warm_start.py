"""Learned warm start for the DFSPH solves: data collection from the
engine's own converged steps, training with the engine's tensor-core
forward/backward kernels and Adam, and the al_warm_start handle a step
takes.  PyTorch only holds device buffers and samples batches; all network
arithmetic runs in the engine (al_warm_net_gradient_f32,
al_warm_net_adam_f32, al_warm_net_forward_f32, al_df_step_warm_f32).

No counterpart in the reference: it replaces the previous-step warm starts
of warm_start_divergence_solve_0 (runner.hpp:3230-3249) and
warm_start_pressure_solve0 (runner.hpp:3430-3449) by predictions of the
converged kappa_v and kappa, under the same gates; the solves' tolerances
still decide convergence.
"""
import ctypes

import numpy as np

from . import _capi

NF = _capi.WARM_NUM_FEATURES


def collect(scene, sp, steps, per_step, seed=0, dt=None, skip=5):
    """Runs `steps` plain DFSPH steps of `scene` and returns device tensors
    (features [M][12], targets [M][2]) of `per_step` random particles per
    step after the first `skip`: each step's features and its converged
    {kappa_v, kappa} in solve units (particle_kappa_v / dt of the step,
    particle_kappa / dt^2 of the pressure solve, i.e. after update_dt)."""
    import torch
    n = scene.n
    rng = np.random.Generator(np.random.PCG64(seed))
    feat = torch.zeros((n, NF), dtype=torch.float32, device="cuda")
    ws = _capi.WarmStart()
    ws.net = None
    ws.features_out = feat.data_ptr()
    dt = float(sp.max_dt) if dt is None else dt
    xs, ts = [], []
    for k in range(steps):
        dt_in = dt
        dt, _ = scene.step("df", sp, dt, warm=ws)
        if k < skip:
            continue
        idx = torch.from_numpy(rng.choice(n, min(per_step, n), replace=False)).cuda()
        t = torch.stack([scene.kappa_v[idx] / dt_in, scene.kappa[idx] / (dt * dt)], 1)
        xs.append(feat[idx].clone())
        ts.append(t)
    return torch.cat(xs), torch.cat(ts)


class WarmStartNet:
    """Trained network: FP32 master parameters on the device plus the input
    shift/scale and output scale of al_warm_net."""

    def __init__(self, params, shift, scale, out_scale):
        import torch
        self.params = params if hasattr(params, "data_ptr") else \
            torch.from_numpy(np.ascontiguousarray(params, np.float32)).cuda()
        self.shift = np.asarray(shift, np.float32)
        self.scale = np.asarray(scale, np.float32)
        self.out_scale = np.asarray(out_scale, np.float32)
        self._net = _capi.make_warm_net(self.params, self.shift, self.scale, self.out_scale)
        self._ws = _capi.WarmStart()
        self._ws.net = ctypes.cast(ctypes.pointer(self._net), ctypes.c_void_p).value
        self._ws.features_out = None

    def warm_start(self):
        """The al_warm_start a step takes (valid while this object lives)."""
        return self._ws

    def net(self):
        return self._net

    def predict(self, engine, features):
        """Device [n][12] features -> device [n][2] {kappa_v, kappa}."""
        import torch
        n = features.shape[0]
        out = torch.zeros((max(n, 1), 2), dtype=torch.float32, device="cuda")
        _capi.check(_capi.lib().al_warm_net_forward_f32(
            engine.handle, ctypes.byref(self._net), _capi.ptr(features) if n else None, n,
            _capi.ptr(out), None), "al_warm_net_forward_f32")
        return out[:n]

    def save(self, path):
        np.savez(path, params=self.params.cpu().numpy(), shift=self.shift, scale=self.scale,
                 out_scale=self.out_scale)

    @classmethod
    def load(cls, path):
        d = np.load(path)
        return cls(d["params"], d["shift"], d["scale"], d["out_scale"])


def normalisation(features, targets):
    """Input shift/scale (mean, 1/std) and output scale (std) of a data set."""
    x = features.double()
    t = targets.double()
    shift = x.mean(0).cpu().numpy()
    sd = x.std(0).cpu().numpy()
    scale = np.where(sd > 0, 1.0 / np.maximum(sd, 1e-30), 1.0)
    osd = t.std(0).cpu().numpy()
    return shift, scale, np.where(osd > 0, osd, 1.0)


def init_params(seed=0):
    """He-style initial weights (normal, std sqrt(2 / fan_in)), zero biases,
    in the flat layout of al_warm_net.params."""
    rng = np.random.Generator(np.random.PCG64(seed))
    h = _capi.WARM_HIDDEN
    parts = [rng.normal(0.0, np.sqrt(2.0 / NF), (h, NF)), np.zeros(h),
             rng.normal(0.0, np.sqrt(2.0 / h), (h, h)), np.zeros(h),
             rng.normal(0.0, np.sqrt(2.0 / h), (_capi.WARM_NUM_OUTPUTS, h)),
             np.zeros(_capi.WARM_NUM_OUTPUTS)]
    flat = np.concatenate([p.ravel() for p in parts]).astype(np.float32)
    assert flat.size == _capi.WARM_NUM_PARAMS
    return flat


def fit(engine, features, targets, steps=10000, batch=65536, lr=1e-3, seed=0, init=None,
        schedule=((0.6, 1.0), (0.9, 0.3), (1.0, 0.1))):
    """Adam on 0.5 * mean squared error of the normalised outputs, with the
    engine's gradient and Adam kernels, on random batches of the data set.
    schedule: (fraction of steps, lr factor) pieces.  Returns
    (WarmStartNet, per-step losses)."""
    import torch
    shift, scale, out_scale = normalisation(features, targets)
    params = init_params(seed) if init is None else np.asarray(init, np.float32)
    net = WarmStartNet(params, shift, scale, out_scale)
    p = net.params
    m = torch.zeros_like(p)
    v = torch.zeros_like(p)
    g = torch.zeros_like(p)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    n = features.shape[0]
    b = min(batch, n)
    loss = ctypes.c_double()
    losses = []
    for step in range(1, steps + 1):
        idx = torch.randint(0, n, (b,), device="cuda", generator=gen)
        x = features[idx].contiguous()
        t = targets[idx].contiguous()
        _capi.check(_capi.lib().al_warm_net_gradient_f32(
            engine.handle, ctypes.byref(net.net()), _capi.ptr(x), _capi.ptr(t), b, _capi.ptr(g),
            ctypes.byref(loss), None), "al_warm_net_gradient_f32")
        f = next(fac for frac, fac in schedule if step <= frac * steps)
        _capi.check(_capi.lib().al_warm_net_adam_f32(
            engine.handle, _capi.ptr(p), _capi.ptr(g), _capi.ptr(m), _capi.ptr(v), step,
            ctypes.c_float(lr * f), None), "al_warm_net_adam_f32")
        losses.append(loss.value)
    return net, losses
