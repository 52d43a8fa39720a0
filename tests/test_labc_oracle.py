"""CPU checks of the learned-boundary pieces that need no GPU: the float64
MLP restatement in oracle/ against finite differences, BF16 rounding, and the
training-sample feature definition against a hand-computed stencil."""
import numpy as np

import mlp_oracle as M
from xfdtd_cuda_b200 import labc


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    x = rng.standard_normal((40, 8))
    y = rng.standard_normal(40)
    q = M.bf16(labc.init_weights(5))
    loss, g = M.loss_grad_rounded(x, y, q)
    idx = rng.choice(M.NP, 60, replace=False)
    for p in idx:
        e = np.zeros(M.NP)
        e[p] = 1e-6
        lp, _ = M.loss_grad_rounded(x, y, q + e)
        lm, _ = M.loss_grad_rounded(x, y, q - e)
        assert abs((lp - lm) / 2e-6 - g[p]) <= 1e-6 * (1 + abs(g[p]))


def test_bf16_rounding_is_nearest_even():
    vals = np.array([1.0, 1.00390625, 1.005859375, -3.1415926, 65504.0, 1e-30], np.float32)
    r = M.bf16(vals)
    for v, q in zip(vals, r):
        # representable in 8 mantissa bits and the nearest such value
        u = np.float32(q).view(np.uint32)
        assert (u & 0xFFFF) == 0
        assert abs(q - v) <= abs(v) * 2.0 ** -8
    assert M.bf16(np.float32(1.005859375))[()] == 1.0078125  # tie -> even


def test_feature_definition():
    rng = np.random.default_rng(1)
    planes = rng.standard_normal((5, 3, 7, 6))
    x, y = labc.features(planes, margin=1, thresh=0.0)
    # first sample: t = 1, u = 1, v = 1
    P = planes
    f = np.array([P[1, 0, 1, 1], P[1, 1, 1, 1], P[1, 2, 1, 1], P[2, 1, 1, 1], P[2, 2, 1, 1], P[0, 0, 1, 1], P[0, 1, 1, 1],
                  P[1, 1, 2, 1] + P[1, 1, 0, 1] + P[1, 1, 1, 2] + P[1, 1, 1, 0] - 4 * P[1, 1, 1, 1]])
    s = np.abs(f[:7]).max()
    assert np.allclose(x[0], f / s, rtol=1e-6)
    assert np.isclose(y[0], P[2, 0, 1, 1] / s, rtol=1e-6)
    assert x.shape == (3 * 5 * 4, 8)
