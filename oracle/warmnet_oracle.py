"""CPU oracle of the learned warm-start network (test infrastructure only:
imported by tests/, __graft_entry__.smoke() and bench.py's CPU legs).

The network has no counterpart in the reference; it is the per-particle
MLP 12 -> 64 -> 64 -> 2 with GELU in the tanh form of Hendrycks & Gimpel
(2016), g(x) = x/2 (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))).  The engine
computes its products on the tensor cores with BF16 operands and FP32
accumulation; this restatement computes in float64 and rounds to BF16
(round to nearest even) at exactly the points where the engine does:
the normalised inputs, the weights, the hidden activations and, in the
backward pass, the output and pre-activation gradients that feed
tensor-core products (every weight and bias gradient is such a product).
`quantize=False` gives the plain float64 network, against which finite
differences pin the analytic gradient.

Parameter layout (flat float32, as include/alluvion_b200.h states):
W1[64][12], b1[64], W2[64][64], b2[64], W3[2][64], b3[2].
Loss: L = 0.5 / B * sum_{r, o} (y_ro - t_ro)^2 over a batch of B rows.
"""
import numpy as np

NF, NH, NO = 12, 64, 2
SIZES = [("W1", (NH, NF)), ("b1", (NH,)), ("W2", (NH, NH)), ("b2", (NH,)),
         ("W3", (NO, NH)), ("b3", (NO,))]
NUM_PARAMS = sum(int(np.prod(s)) for _, s in SIZES)  # 5122
C = np.sqrt(2.0 / np.pi)
A = 0.044715


def unpack(flat):
    out, o = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = np.asarray(flat[o:o + n], dtype=np.float64).reshape(shape)
        o += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], dtype=np.float64).ravel() for name, _ in SIZES])


def bf16(x):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(C * (x + A * x ** 3)))


def gelu_grad(x):
    t = np.tanh(C * (x + A * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * C * (1.0 + 3.0 * A * x * x)


def init_params(seed=0):
    """He-style initialisation (float32), biases zero."""
    rng = np.random.Generator(np.random.PCG64(seed))
    d = {}
    for name, shape in SIZES:
        if name.startswith("W"):
            d[name] = rng.normal(0.0, np.sqrt(2.0 / shape[1]), size=shape)
        else:
            d[name] = np.zeros(shape)
    return pack(d).astype(np.float32)


def normalise(features, shift, scale):
    return (np.asarray(features, np.float64) - np.asarray(shift, np.float64)) * \
        np.asarray(scale, np.float64)


def forward(params, xn, quantize=True):
    """Returns (y, cache) for normalised inputs xn [B][12]."""
    q = bf16 if quantize else (lambda v: np.asarray(v, np.float64))
    p = unpack(params)
    W1, W2, W3 = q(p["W1"]), q(p["W2"]), q(p["W3"])
    x = q(xn)
    z1 = x @ W1.T + p["b1"]
    h1 = q(gelu(z1))
    z2 = h1 @ W2.T + p["b2"]
    h2 = q(gelu(z2))
    y = h2 @ W3.T + p["b3"]
    return y, dict(x=x, z1=z1, h1=h1, z2=z2, h2=h2, W1=W1, W2=W2, W3=W3)


def predict(params, features, shift, scale, out_scale, quantize=True):
    y, _ = forward(params, normalise(features, shift, scale), quantize)
    return y * np.asarray(out_scale, np.float64)


def loss_and_grad(params, xn, targets, quantize=True):
    """L = 0.5 / B * sum (y - t)^2 and dL/dparams (flat float64)."""
    q = bf16 if quantize else (lambda v: np.asarray(v, np.float64))
    y, c = forward(params, xn, quantize)
    B = y.shape[0]
    t = np.asarray(targets, np.float64)
    loss = 0.5 / B * np.sum((y - t) ** 2)
    dy = (y - t) / B
    g = {}
    # the engine forms every weight and bias gradient as a tensor-core
    # product of BF16 operands: dy, dz2 and dz1 are rounded there
    dyq = q(dy)
    g["W3"] = dyq.T @ c["h2"]
    g["b3"] = dyq.sum(0)
    dz2 = (dy @ c["W3"]) * gelu_grad(c["z2"])
    dz2q = q(dz2)
    g["b2"] = dz2q.sum(0)
    g["W2"] = dz2q.T @ c["h1"]
    dz1 = (dz2q @ c["W2"]) * gelu_grad(c["z1"])
    dz1q = q(dz1)
    g["b1"] = dz1q.sum(0)
    g["W1"] = dz1q.T @ c["x"]
    return loss, pack(g)


def finite_difference(params, xn, targets, index, eps=1e-6):
    """Central difference of the float64 (unquantised) loss in one parameter."""
    p = np.asarray(params, np.float64).copy()
    p[index] += eps
    lp, _ = loss_and_grad(p, xn, targets, quantize=False)
    p[index] -= 2 * eps
    lm, _ = loss_and_grad(p, xn, targets, quantize=False)
    return (lp - lm) / (2 * eps)


def adam(params, grad, m, v, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update (Kingma & Ba 2015) in float64; returns new (p, m, v)."""
    m = b1 * m + (1 - b1) * grad
    v = b2 * v + (1 - b2) * grad * grad
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return params - lr * mh / (np.sqrt(vh) + eps), m, v
