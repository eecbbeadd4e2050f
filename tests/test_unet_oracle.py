"""The U-Net oracle checks itself: analytic gradients against central finite
differences, and the layer helpers against their definitions."""
import numpy as np

import unet_oracle as uo


def test_param_count():
    _, n = uo.offsets()
    assert n == 104337


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    _, n = uo.offsets()
    p = rng.normal(0, 0.2, n)
    r = rng.normal(0, 1, (1, 8, 8, 8))
    t = rng.normal(0, 1, (1, 8, 8, 8))
    loss, g = uo.loss_grad(p, r, t)
    off, _ = uo.offsets()
    picks = [off[l] + k for l in range(13) for k in (0, 7)] + [off[l + 1] - 1 for l in range(13)] + [n - 1, n - 5]
    h = 1e-6
    for i in picks:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (uo.loss_grad(pp, r, t)[0] - uo.loss_grad(pm, r, t)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_pool_up_adjoint():
    rng = np.random.default_rng(1)
    x = rng.normal(size=(2, 4, 6, 8, 3))
    y = rng.normal(size=(2, 2, 3, 4, 3))
    assert np.isclose((uo.pool(x) * y).sum(), (x * uo.pool_bwd(y)).sum())
    assert np.isclose((uo.up(y) * x).sum(), (y * uo.up_bwd(x)).sum())


def test_bf16_round():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5e-3], np.float32)
    r = uo.bf16_round(v)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == np.float32(1.0 + 2 ** -7)
