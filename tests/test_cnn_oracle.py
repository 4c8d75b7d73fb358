"""CPU tests of the closure network's numpy oracle: analytic gradient against central finite
differences (this pins the oracle that checks the CUDA kernels)."""
import numpy as np

from oracle import cnn_oracle as CO


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    layers, ch = 3, 4
    n = sum(co * ci * 9 + co for ci, co in CO.layer_shapes(layers, ch))
    p = rng.standard_normal(n) * 0.3
    x = rng.standard_normal((2, 3, 8, 6))
    t = rng.standard_normal((2, 1, 8, 6))
    loss, g = CO.loss_grad(p, layers, ch, x, t)
    for i in rng.choice(n, 25, replace=False):
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (CO.loss_grad(pp, layers, ch, x, t)[0] - CO.loss_grad(pm, layers, ch, x, t)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_oracle_conv_is_periodic():
    rng = np.random.default_rng(1)
    x = rng.standard_normal((1, 3, 5, 7))
    w = rng.standard_normal((2, 3, 3, 3))
    b = np.zeros(2)
    y = CO.conv3x3(x, w, b)
    ys = CO.conv3x3(np.roll(x, (2, 3), axis=(2, 3)), w, b)
    np.testing.assert_allclose(np.roll(y, (2, 3), axis=(2, 3)), ys, atol=1e-12)
