"""The learned-preconditioner oracle (oracle/unet.py) checked on its own: gradients against
central differences, BF16 rounding, the transposed convolution as the adjoint, and the parameter
layout the library exports.  No GPU."""
import numpy as np

from oracle import unet
from paracfd_b200 import learned_parameter_count


def test_library_parameter_count_matches_oracle():
    assert learned_parameter_count() == unet.param_count() == 179728


def test_bf16_rounding_is_round_to_nearest_even():
    assert unet.bf16(1.0) == 1.0
    assert unet.bf16(1.0 + 2.0 ** -8) == 1.0                 # tie -> even
    assert unet.bf16(1.0 + 3 * 2.0 ** -8) == 1.0 + 2.0 ** -6  # tie -> even (up)
    assert unet.bf16(1.0 + 2.0 ** -8 + 2.0 ** -12) == 1.0 + 2.0 ** -7
    assert unet.bf16(-3.0) == -3.0


def test_conv_transpose_is_the_adjoint():
    rng = np.random.default_rng(1)
    for n, cin, cout in ((8, 16, 16), (4, 32, 64), (2, 64, 32)):
        x = rng.standard_normal((2, n, n, n, cin))
        g = rng.standard_normal((2, n, n, n, cout))
        w = rng.standard_normal((27, cout, cin))
        lhs = (unet.conv(x, w) * g).sum()
        rhs = (x * unet.conv_transpose(g, w)).sum()
        assert abs(lhs - rhs) <= 1e-10 * abs(lhs)
        gw = unet.conv_weight_grad(g, x)
        assert abs((gw * w).sum() - lhs) <= 1e-10 * abs(lhs)


def test_oracle_gradients_match_central_differences():
    rng = np.random.default_rng(0)
    p = unet.init_params(1)
    B = 2
    r = rng.standard_normal((B, 512))
    dinv = np.abs(rng.standard_normal((B, 512))) + 0.5
    mask = (rng.random((B, 512)) > 0.1).astype(float)
    x, _ = unet.prepare(r, dinv, mask)
    t = rng.standard_normal((B, 512)) * 0.1
    _, g = unet.loss_and_grads(p, x, t, mask, rounding=False)
    checked = 0
    for name, shape in unet.param_shapes():
        flat = np.abs(g[name]).ravel()
        for idx in np.argsort(flat)[-2:]:
            idx = np.unravel_index(idx, shape)
            e = 1e-6
            q = {k: v.copy() for k, v in p.items()}
            q[name][idx] += e
            lp, _ = unet.loss_and_grads(q, x, t, mask, rounding=False)
            q[name][idx] -= 2 * e
            lm, _ = unet.loss_and_grads(q, x, t, mask, rounding=False)
            fd = (lp - lm) / (2 * e)
            assert abs(fd - g[name][idx]) <= 1e-5 * max(abs(fd), 1e-3), (name, idx, fd, g[name][idx])
            checked += 1
    assert checked == 2 * len(unet.param_shapes())


def test_forward_is_positively_homogeneous_through_the_brick_scale():
    rng = np.random.default_rng(4)
    p = unet.init_params(2)
    r = rng.standard_normal((1, 512))
    dinv = np.ones((1, 512))
    mask = np.ones((1, 512))
    x1, s1 = unet.prepare(r, dinv, mask)
    x2, s2 = unet.prepare(5.0 * r, dinv, mask)
    z1, _ = unet.forward(p, x1, rounding=False)
    z2, _ = unet.forward(p, x2, rounding=False)
    assert np.allclose(s2 * z2, 5.0 * s1 * z1)
