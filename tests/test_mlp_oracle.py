"""CPU checks of the surrogate network's oracle (oracle/mlp_oracle.py).

The oracle is what the GPU gradients are compared with, so it is pinned first:
its float64 backward pass against central finite differences of its own loss,
and its bfloat16 rounding against torch's float32 -> bfloat16 conversion.
"""
import numpy as np
import pytest

import mlp_oracle as M


def _batch(rng, n):
    x = rng.uniform(-1, 1, (n, 4))
    yl = rng.normal(size=n)
    yc = rng.integers(0, 16, n)
    return x, yl, yc


def test_layout():
    off = M.offsets()
    assert M.NUM_PARAMS == 128 * 256 + 256 + 2 * (256 * 256 + 256) + 17 * 256 + 17
    assert off["b4"][0] + 17 == M.NUM_PARAMS
    p = np.arange(M.NUM_PARAMS, dtype=np.float64)
    assert np.array_equal(M.pack(M.unpack(p)), p)


def test_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.normal(size=20000).astype(np.float32) * 10.0 ** rng.integers(-8, 8, 20000),
                        np.array([0.0, -0.0, 1.0, 1.00390625, 1.005859375, 1.0078125], np.float32)])
    want = torch.from_numpy(x).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(M.bf16(x), want)


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = M.init_params(7)
    p[M.offsets()["b1"][0]:M.offsets()["b1"][0] + 256] = rng.normal(scale=0.1, size=256)
    p[M.offsets()["b4"][0]:] = rng.normal(scale=0.1, size=17)
    x, yl, yc = _batch(rng, 24)
    _, g, _ = M.forward_backward(p, x, yl, yc, 0.7, bf16_round=False)
    picks = rng.choice(M.NUM_PARAMS, 60, replace=False)
    for name in ("W1", "b1", "W4", "b4", "b3"):
        o, shape = M.offsets()[name]
        picks = np.append(picks, o + rng.integers(0, int(np.prod(shape)), 3))
    eps = 1e-6
    for i in picks:
        q = p.copy()
        q[i] += eps
        lp = M.loss_only(q, x, yl, yc, 0.7)
        q[i] -= 2 * eps
        lm = M.loss_only(q, x, yl, yc, 0.7)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_bf16_path_is_close_to_exact_path():
    """BF16 rounding perturbs the gradient by well under 5 % (relative L2)."""
    rng = np.random.default_rng(2)
    p = M.init_params(3)
    x, yl, yc = _batch(rng, 64)
    l0, g0, _ = M.forward_backward(p, x, yl, yc, 1.0, bf16_round=False)
    l1, g1, _ = M.forward_backward(p, x, yl, yc, 1.0, bf16_round=True)
    assert abs(l1 - l0) < 0.02 * abs(l0)
    assert np.linalg.norm(g1 - g0) < 0.05 * np.linalg.norm(g0)


def test_fourier_encoding():
    """The fixed encoding: 62 exact float32 frequencies with a spread of about 9
    cycles per unit, and rows of (x, sin 2 pi p_k, cos 2 pi p_k)."""
    b = M.fourier_freqs()
    assert b.shape == (62, 2) and b.dtype == np.float32
    assert np.array_equal(b * 16, np.round(b * 16)) and np.abs(b).max() <= 510 / 16
    assert 7 < b.std() < 11
    x = np.array([[1.0, 0.25, -0.5, 0.3], [-1.0, 0.0, 0.0, 0.0]], np.float32)
    e = M.encode(x)
    assert e.shape == (2, 128) and np.array_equal(e[:, :4], x)
    p = (b[:, 0] * np.float32(0.25) + b[:, 1] * np.float32(-0.5)).astype(np.float64)
    assert np.allclose(e[0, 4::2], np.sin(2 * np.pi * p), atol=1e-7)
    assert np.allclose(e[0, 5::2], np.cos(2 * np.pi * p), atol=1e-7)
    assert np.array_equal(e[1, 4::2], np.zeros(62, np.float32)) and np.array_equal(e[1, 5::2], np.ones(62, np.float32))


def test_init_is_deterministic_and_bounded():
    a, b = M.init_params(5), M.init_params(5)
    assert np.array_equal(a, b)
    W2 = M.unpack(a)["W2"]
    assert np.abs(W2).max() <= np.sqrt(6 / 256) * (1 + 1e-7) and W2.std() > 0.05
    assert not M.unpack(a)["b2"].any()
