"""CPU checks of the surrogate oracle: its analytic gradients against FP64
finite differences, conv identities, and the exact mean-mass projection."""
import numpy as np

from oracle import surrogate_oracle as so


def test_bf16_rounding_is_nearest_even():
    # bf16 keeps 7 explicit mantissa bits: the spacing just above 1.0 is 2^-7
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -8 + 2 ** -12, -2.5, 3.14159], dtype=np.float32)
    r = so.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                          # tie -> even (down)
    assert r[2] == np.float32(1.0 + 2 ** -6)    # tie -> even (up)
    assert r[3] == np.float32(1.0 + 2 ** -7)    # above the tie -> up
    assert r[4] == -2.5
    assert r[5] == np.float32(3.140625)


def test_conv_dgrad_is_adjoint_of_conv():
    rng = np.random.default_rng(0)
    x = rng.normal(size=(2, 7, 9, 5))
    w = rng.normal(size=(4, 3, 3, 5))
    dy = rng.normal(size=(2, 7, 9, 4))
    lhs = (so.conv3x3(x, w) * dy).sum()
    assert abs(lhs - (x * so.conv3x3_dgrad(dy, w)).sum()) < 1e-9 * abs(lhs)
    assert abs(lhs - (w * so.conv3x3_wgrad(x, dy)).sum()) < 1e-9 * abs(lhs)


def test_gradients_match_finite_differences():
    # float64 "bf16" bypass: check the calculus, not the rounding
    rng = np.random.default_rng(1)
    params = [p.astype(np.float64) for p in so.init_params(3)]
    params[6] = params[6] * 10
    c = 0.5 + 0.2 * rng.standard_normal((2, 6, 5))
    orig = so.bf16
    so.bf16 = lambda a: np.asarray(a, dtype=np.float64)
    try:
        o, cache = so.forward(params, c, 0.5, 4.0)
        t = rng.standard_normal(o.shape)
        L, do = so.mse_loss_and_grad(o, t)
        grads = so.backward(params, cache, do)
        eps = 1e-6
        for pi in (0, 1, 2, 3, 5, 6, 7):
            p = params[pi]
            for idx in [tuple(rng.integers(0, s) for s in p.shape) for _ in range(4)]:
                old = p[idx]
                p[idx] = old + eps
                Lp = so.mse_loss_and_grad(so.forward(params, c, 0.5, 4.0)[0], t)[0]
                p[idx] = old - eps
                Lm = so.mse_loss_and_grad(so.forward(params, c, 0.5, 4.0)[0], t)[0]
                p[idx] = old
                fd = (Lp - Lm) / (2 * eps)
                assert abs(fd - grads[pi][idx]) <= 1e-6 + 1e-5 * abs(fd), (pi, idx, fd, grads[pi][idx])
    finally:
        so.bf16 = orig


def test_step_projection_conserves_mass_exactly():
    rng = np.random.default_rng(2)
    params = so.init_params(0)
    params[7] = params[7] + 0.3  # bias that would add mass without the projection
    c = rng.uniform(0.3, 0.7, size=(16, 16))
    cn = so.step(params, c, 0.5, 4.0, 0.01)
    assert abs(cn.mean() - c.mean()) <= 1e-15
