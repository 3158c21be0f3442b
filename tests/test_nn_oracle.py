"""The CPU oracle of the surrogate's operations against finite differences
(FP64), so that it can serve as the reference for the GPU kernels."""

import numpy as np

from oracle import nn_ref


def _fd(f, x, idx, h=1e-6):
    xp = x.copy()
    xm = x.copy()
    xp[idx] += h
    xm[idx] -= h
    return (f(xp) - f(xm)) / (2 * h)


def test_conv_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    x = rng.standard_normal((2, 4, 6, 4, 3))
    w = rng.standard_normal((5, 27, 3))
    b = rng.standard_normal(5)
    gz = rng.standard_normal((2, 4, 6, 4, 5))
    dx, dw, db = nn_ref.conv_bwd(x, w, gz, 3)

    def loss_x(xx):
        return float((nn_ref.conv_fwd(xx, w, b, 3) * gz).sum())

    def loss_w(ww):
        return float((nn_ref.conv_fwd(x, ww, b, 3) * gz).sum())

    for idx in [(0, 0, 0, 0, 0), (1, 3, 5, 3, 2), (0, 2, 1, 3, 1)]:
        assert abs(_fd(loss_x, x, idx) - dx[idx]) < 1e-6
    for idx in [(0, 0, 0), (4, 26, 2), (2, 13, 1)]:
        assert abs(_fd(loss_w, w, idx) - dw[idx]) < 1e-6
    assert np.allclose(db, gz.reshape(-1, 5).sum(0))


def test_unet_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    params = {}
    for name, ci, co, k, act in nn_ref.LAYERS:
        params[name] = (rng.standard_normal((co, k ** 3, ci)) * (1.0 / np.sqrt(k ** 3 * ci)),
                        rng.standard_normal(co) * 0.1)
    x = rng.standard_normal((1, 8, 8, 8, 16))
    tgt = rng.standard_normal((1, 8, 8, 8, 16))
    slope = 0.1

    def loss_of(pp):
        out, _ = nn_ref.unet_forward(pp, x, slope)
        return float(((out - tgt) ** 2).sum())

    out, cache = nn_ref.unet_forward(params, x, slope)
    grads = nn_ref.unet_backward(params, cache, 2 * (out - tgt), slope)
    for name, idx in [("e1", (3, 13, 2)), ("e4", (100, 5, 17)), ("d3", (7, 20, 300)), ("d1", (1, 26, 70)),
                      ("out", (2, 0, 5))]:
        w, b = params[name]

        def f(ww, name=name):
            pp = dict(params)
            pp[name] = (ww, params[name][1])
            return loss_of(pp)

        fd = _fd(f, w, idx, 1e-5)
        an = grads[name][0][idx]
        assert abs(fd - an) <= 1e-5 * max(1.0, abs(an)), (name, fd, an)
