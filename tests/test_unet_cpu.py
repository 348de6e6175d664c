"""CPU checks of the learned p' preconditioner's specification (oracle/unet.py):
its backward pass is the exact gradient of its forward pass (finite
differences, BF16 rounding off), and the library, the Python mirror and the
oracle agree on the parameter layout."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import unet as U  # noqa: E402

from mach2d_b200 import unet  # noqa: E402


def test_parameter_layout_agrees():
    assert U.param_count() == unet.param_count() == 489169
    assert [(ci, co) for ci, co, _ in U.LAYERS] == list(unet.LAYERS)
    assert np.array_equal(U.init_params(3), unet.init_params(3))


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = U.init_params(1).astype(np.float64)
    p[-17:] = rng.standard_normal(17) * 0.3
    feat = rng.standard_normal((2, 11, 8, 16))
    t = rng.standard_normal((2, 8, 16))
    m = np.ones((2, 8, 16))
    m[:, :, 13:] = 0
    sc = 1.0 / m.sum()
    _, g, _ = U.loss_grad(p, feat, t, m, sc, bf16_rounding=False)
    layers = U.split(np.arange(p.size))[0]
    idx = list(rng.choice(p.size, 24, replace=False))
    idx += [int(layers[0][0][2, 4, 5]), int(layers[0][1][3]), int(layers[7][1][0]), int(layers[13][1][5]),
            p.size - 1, p.size - 5]
    for i in idx:
        e = 1e-5
        pp = p.copy()
        pp[i] += e
        lp = U.loss_grad(pp, feat, t, m, sc, False)[0]
        pp[i] -= 2 * e
        lm = U.loss_grad(pp, feat, t, m, sc, False)[0]
        fd = (lp - lm) / (2 * e)
        assert abs(fd - g[i]) <= 1e-4 * (abs(fd) + abs(g[i])) + 1e-9, i


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 1.0 + 2 ** -9])
    assert list(U.bf16(x)) == [1.0, 1.0, 1.0 + 2 ** -6, -2.5, 1.0]
