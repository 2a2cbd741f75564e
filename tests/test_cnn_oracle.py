"""CPU checks of the network oracle (oracle/cnn_ref.py): the convolution
against a direct sum, the adjoint identity, bfloat16 rounding against
torch's, and the analytic FP64 gradient against central finite differences.
These pin the checker that the GPU gradient tests compare with."""
import math

import numpy as np
import pytest

from oracle import cnn_ref as R


def rand_params(seed, scale=0.3):
    rng = np.random.default_rng(seed)
    w = rng.normal(0, scale, size=(R.NL, R.NT, R.C, R.C)) * R.masks()[0]
    b = rng.normal(0, 0.1, size=(R.NL, R.C)) * R.masks()[1]
    return w, b


def test_conv_matches_direct_sum():
    rng = np.random.default_rng(0)
    a = rng.normal(size=(4, 5, 6, R.C))
    w = rng.normal(size=(R.NT, R.C, R.C))
    out = R.conv(a, w)
    z, y, x = 1, 4, 0
    ref = np.zeros(R.C)
    for t, (dz, dy, dx) in enumerate(R.taps()):
        ref += w[t] @ a[(z + dz) % 4, (y + dy) % 5, (x + dx) % 6]
    np.testing.assert_allclose(out[z, y, x], ref, rtol=1e-12)


def test_conv_t_is_the_adjoint():
    rng = np.random.default_rng(1)
    a = rng.normal(size=(3, 4, 5, R.C))
    g = rng.normal(size=(3, 4, 5, R.C))
    w = rng.normal(size=(R.NT, R.C, R.C))
    lhs = np.sum(R.conv(a, w) * g)
    rhs = np.sum(a * R.conv_t(g, w))
    assert lhs == pytest.approx(rhs, rel=1e-12)


def test_bf16_rounding_matches_torch():
    import torch
    rng = np.random.default_rng(2)
    x = np.concatenate([rng.normal(size=2000) * 10.0 ** rng.integers(-8, 8, size=2000),
                        [0.0, -0.0, 1.0, 1.00390625, 1.01171875, 3.0e-39]]).astype(np.float32)
    ref = torch.from_numpy(x).to(torch.bfloat16).to(torch.float64).numpy()
    np.testing.assert_array_equal(R.bf16(x), ref)


def test_gelu_definition():
    x = np.linspace(-5, 5, 101)
    # the tanh form stays within 1e-3 of the exact x * Phi(x)
    phi = 0.5 * (1 + np.array([math.erf(v / math.sqrt(2)) for v in x]))
    np.testing.assert_allclose(R.gelu(x), x * phi, rtol=0, atol=1e-3)
    u = math.sqrt(2 / math.pi) * (x + 0.044715 * x ** 3)
    np.testing.assert_allclose(R.gelu(x), x / (1 + np.exp(-2 * u)), rtol=1e-13, atol=1e-15)
    h = 1e-6
    fd = (R.gelu(x + h) - R.gelu(x - h)) / (2 * h)
    np.testing.assert_allclose(R.gelu_grad(x), fd, rtol=1e-7, atol=1e-9)


def test_exact_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    shape = (4, 5, 6)
    u = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    target = u + 0.05 * (rng.normal(size=shape) + 1j * rng.normal(size=shape))
    w, b = rand_params(4)
    s = 0.5
    loss, dw, db = R.loss_and_grad(u, target, w, b, s, emulate=False)
    picks = [(0, 13, 3, 1), (1, 0, 7, 9), (2, 26, 15, 4), (3, 5, 1, 12), (3, 22, 0, 0)]
    for (l, t, co, ci) in picks:
        h = 1e-5
        wp, wm = w.copy(), w.copy()
        wp[l, t, co, ci] += h
        wm[l, t, co, ci] -= h
        fd = (R.loss_and_grad(u, target, wp, b, s, emulate=False)[0] -
              R.loss_and_grad(u, target, wm, b, s, emulate=False)[0]) / (2 * h)
        assert dw[l, t, co, ci] == pytest.approx(fd, rel=1e-5, abs=1e-10)
    for (l, c) in [(0, 3), (2, 11), (3, 1)]:
        h = 1e-5
        bp, bm = b.copy(), b.copy()
        bp[l, c] += h
        bm[l, c] -= h
        fd = (R.loss_and_grad(u, target, w, bp, s, emulate=False)[0] -
              R.loss_and_grad(u, target, w, bm, s, emulate=False)[0]) / (2 * h)
        assert db[l, c] == pytest.approx(fd, rel=1e-5, abs=1e-10)


def test_emulated_forward_is_close_to_exact():
    rng = np.random.default_rng(5)
    shape = (4, 4, 4)
    u = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    w, b = rand_params(6)
    d_e, _ = R.forward(u, w, b, 1.0, emulate=True)
    d_x, _ = R.forward(u, w, b, 1.0, emulate=False)
    rel = np.linalg.norm(d_e - d_x) / np.linalg.norm(d_x)
    assert 1e-5 < rel < 3e-2  # bfloat16 rounding, present and bounded
