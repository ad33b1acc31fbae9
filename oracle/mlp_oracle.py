"""CPU restatement of the surrogate network's forward and backward passes.

TEST INFRASTRUCTURE ONLY: the product trains and runs the network with the CUDA
kernels of libcbf.so (csrc/mlp.cu); this module is the checker their gradients
are compared with.  The surrogate has no counterpart in the reference project,
so the restatement follows the network's definition rather than a reference
file:

    4 inputs -> fixed Fourier encoding (128) -> 256 -> 256 -> 256 -> 17,
    SiLU on the hidden layers,
    output 0 = normalised LLE (loss wLle * squared error),
    outputs 1..16 = logits of the 16-way regime class (softmax cross-entropy),
    loss = batch mean of both terms.

The encoding (not trained) keeps the 4 inputs and adds, for 62 fixed
frequencies b_k (fourier_freqs), sin(2 pi p_k) and cos(2 pi p_k) of
p_k = b_k0 x1 + b_k1 x2 over the two swept-parameter inputs: a small MLP on raw
coordinates cannot resolve the fine regime structure of a bifurcation map
(it fits low frequencies first), the encoded one can.

With ``bf16=True`` the values are rounded to bfloat16 (round to nearest even)
where the kernels round them: the encoded input rows, the weights fed to the tensor
cores, the hidden activations, the output gradient and the hidden-layer
gradients that feed further products.  Biases, pre-activations, the outputs and
the bias gradients stay FP32 (here: float64), and the products accumulate at
full precision.  With ``bf16=False`` it is plain float64 backpropagation, which
the CPU tests pin against central finite differences.
"""
from __future__ import annotations

import numpy as np

K_RAW, K_FREQ, K_HID, K_OUT, K_CLS = 4, 62, 256, 17, 16
K_IN = K_RAW + 2 * K_FREQ  # first-layer inputs: 128

# flat parameter layout: W1[256x128] b1 W2[256x256] b2 W3[256x256] b3 W4[17x256] b4
_SHAPES = [("W1", (K_HID, K_IN)), ("b1", (K_HID,)), ("W2", (K_HID, K_HID)), ("b2", (K_HID,)),
           ("W3", (K_HID, K_HID)), ("b3", (K_HID,)), ("W4", (K_OUT, K_HID)), ("b4", (K_OUT,))]
NUM_PARAMS = sum(int(np.prod(s)) for _, s in _SHAPES)


def offsets():
    out, o = {}, 0
    for name, shape in _SHAPES:
        n = int(np.prod(shape))
        out[name] = (o, shape)
        o += n
    return out


def unpack(params):
    p = np.asarray(params, np.float64)
    return {k: p[o:o + int(np.prod(s))].reshape(s) for k, (o, s) in offsets().items()}


def pack(d):
    return np.concatenate([np.asarray(d[k], np.float64).ravel() for k, _ in _SHAPES])


def bf16(x):
    """Round to bfloat16, nearest even (finite inputs), returned as float64."""
    f = np.asarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32).astype(np.float64)


def fourier_freqs(seed=0x5EED):
    """The encoding's 62 x 2 frequencies (cycles per unit of the [-1, 1] axes), as
    mlp.cu builds them: per value one xorshift64 word (state seed * 0x9E3779B97F4A7C15
    + 1), b = (sum of its four low bytes - 510) / 16 -- an Irwin-Hall approximation
    of a normal distribution with standard deviation about 9, exact in float32."""
    mask = 0xFFFFFFFFFFFFFFFF
    s = (seed * 0x9E3779B97F4A7C15 + 1) & mask
    b = np.empty((K_FREQ, 2), np.float32)
    for k in range(K_FREQ):
        for j in range(2):
            s ^= (s << 13) & mask
            s ^= s >> 7
            s ^= (s << 17) & mask
            b[k, j] = np.float32((sum((s >> (8 * i)) & 255 for i in range(4)) - 510) / 16.0)
    return b


def encode(x, scale=1.0):
    """First-layer inputs of raw rows x (n, 4): the 4 values, then for each
    frequency k, sin(2 pi s p_k) and cos(2 pi s p_k), p_k = fl(fl(b_k0 x1) +
    fl(b_k1 x2)) in float32 (the kernels' operation order), s the network's
    frequency scale (a power of two: the scaling is exact); the sines and cosines
    are evaluated here in float64 and rounded to float32, the kernels' sincospif
    is within about an ulp of that."""
    x = np.asarray(x, np.float32).reshape(-1, K_RAW)
    b = fourier_freqs()
    p = (x[:, 1:2] * b[None, :, 0]) + (x[:, 2:3] * b[None, :, 1])  # float32 products and sum
    v = np.pi * ((2.0 * scale) * p.astype(np.float64))
    e = np.empty((len(x), K_IN), np.float32)
    e[:, :K_RAW] = x
    e[:, K_RAW::2] = np.sin(v).astype(np.float32)
    e[:, K_RAW + 1::2] = np.cos(v).astype(np.float32)
    return e


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward_backward(params, x, y_lle, y_cls, w_lle, bf16_round=True, scale=1.0):
    """Returns (loss, grads[NUM_PARAMS], out[n, 17]) for the batch of raw rows
    (x [n, 4], y_lle, y_cls)."""
    r = bf16 if bf16_round else (lambda a: np.asarray(a, np.float64))
    P = unpack(params)
    W = {k: r(P[k]) for k in ("W1", "W2", "W3", "W4")}
    x = r(encode(x, scale).astype(np.float64))
    n = x.shape[0]
    z1 = x @ W["W1"].T + P["b1"]
    h1 = r(_silu(z1))
    z2 = h1 @ W["W2"].T + P["b2"]
    h2 = r(_silu(z2))
    z3 = h2 @ W["W3"].T + P["b3"]
    h3 = r(_silu(z3))
    out = h3 @ W["W4"].T + P["b4"]

    y_lle = np.asarray(y_lle, np.float64)
    y_cls = np.asarray(y_cls, np.int64)
    e = out[:, 0] - y_lle
    logits = out[:, 1:]
    mx = logits.max(axis=1, keepdims=True)
    ex = np.exp(logits - mx)
    p = ex / ex.sum(axis=1, keepdims=True)
    onehot = np.zeros_like(p)
    onehot[np.arange(n), y_cls] = 1.0
    ce = -np.log(np.maximum(p[np.arange(n), y_cls], 1e-30))
    loss = float(np.mean(w_lle * e * e + ce))

    d = np.zeros_like(out)
    d[:, 0] = 2.0 * w_lle * e / n
    d[:, 1:] = (p - onehot) / n
    db = r(d)
    g = {}
    g["W4"] = db.T @ h3
    g["b4"] = d.sum(axis=0)
    dz3 = (db @ W["W4"]) * _silu_grad(z3)
    dz3b = r(dz3)
    g["W3"] = dz3b.T @ h2
    g["b3"] = dz3.sum(axis=0)
    dz2 = (dz3b @ W["W3"]) * _silu_grad(z2)
    dz2b = r(dz2)
    g["W2"] = dz2b.T @ h1
    g["b2"] = dz2.sum(axis=0)
    dz1 = (dz2b @ W["W2"]) * _silu_grad(z1)
    dz1b = r(dz1)
    g["W1"] = dz1b.T @ x
    g["b1"] = dz1.sum(axis=0)
    return loss, pack(g), out


def loss_only(params, x, y_lle, y_cls, w_lle):
    return forward_backward(params, x, y_lle, y_cls, w_lle, bf16_round=False)[0]


def init_params(seed):
    """Same initialisation as cbf_mlp_create: uniform +-sqrt(6/fan_in) weights from
    a xorshift64 stream, zero biases."""
    p = np.zeros(NUM_PARAMS, np.float64)
    st = [(seed * 0x9E3779B97F4A7C15 + 1) & 0xFFFFFFFFFFFFFFFF]

    def rnd():
        s = st[0]
        s ^= (s << 13) & 0xFFFFFFFFFFFFFFFF
        s ^= s >> 7
        s ^= (s << 17) & 0xFFFFFFFFFFFFFFFF
        st[0] = s
        return (s >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0

    off = offsets()
    for name, fan in (("W1", K_IN), ("W2", K_HID), ("W3", K_HID), ("W4", K_HID)):
        o, shape = off[name]
        bound = np.sqrt(6.0 / fan)
        cnt = int(np.prod(shape))
        p[o:o + cnt] = [np.float32(rnd() * bound) for _ in range(cnt)]
    return p


# ---------------------------------------------------------------------------
# Grid prediction (the surrogate map's prediction step), restated.

SYSTEM_FEATURE = {1: -1.0, 2: 0.0, 3: 1.0}  # Rossler, Lorenz, Chen


def grid_features(system, nPts, ranges, idxMut, values, grid_values):
    """The network's 4 FP32 inputs of grid points whose two swept parameters are
    grid_values[:, 0] and grid_values[:, 1] (doubles): the system code, each
    swept parameter mapped to [-1, 1] as ((float)p - lo) * (2 / (hi - lo)) - 1 in
    FP32, and the first unswept parameter of values[1..3] divided by 10."""
    f32 = np.float32
    lo0, lo1 = f32(ranges[0]), f32(ranges[2])
    inv0 = f32(2.0 / (ranges[1] - ranges[0])) if ranges[1] != ranges[0] else f32(0)
    inv1 = f32(2.0 / (ranges[3] - ranges[2])) if ranges[3] != ranges[2] else f32(0)
    third = 1
    while third in idxMut:
        third += 1
    t = f32(values[third] * 0.1) if third < 4 else f32(0)
    g = np.asarray(grid_values, np.float64)
    x = np.empty((len(g), K_RAW), np.float32)
    x[:, 0] = f32(SYSTEM_FEATURE[system])
    x[:, 1] = (g[:, 0].astype(np.float32) - lo0) * inv0 - f32(1)
    x[:, 2] = (g[:, 1].astype(np.float32) - lo1) * inv1 - f32(1)
    x[:, 3] = t
    return x


def predict(params, x, lle_mean, lle_std, scale=1.0):
    """Forward pass with the kernels' BF16 rounding points (exact accumulation):
    (LLE = out0 * std + mean, class = argmax of out1..16, softmax maximum,
    the raw outputs (n, 17), the gap between the two largest logits)."""
    n = len(x)
    _, _, out = forward_backward(params, x, np.zeros(n), np.zeros(n, np.int64), 1.0, bf16_round=True,
                                 scale=scale)
    logits = out[:, 1:]
    cls = logits.argmax(axis=1)
    srt = np.sort(logits, axis=1)
    margin = srt[:, -1] - srt[:, -2]
    pm = np.exp(logits - logits.max(axis=1, keepdims=True))
    conf = 1.0 / pm.sum(axis=1)
    return out[:, 0] * lle_std + lle_mean, cls, conf, out, margin
