"""The learned-smoother oracle checked against finite differences, and the Gaussian random
field checked for its covariance (host only)."""
import numpy as np

import cnn_oracle as co
from grico_b200.grf import GaussianRandomField


def _net(seed=0, chans=(2, 4, 3, 1)):
    rng = np.random.default_rng(seed)
    return co.Net([(rng.standard_normal((chans[k + 1], chans[k], 27)) * 0.3, rng.standard_normal(chans[k + 1]) * 0.1)
                   for k in range(len(chans) - 1)])


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(1)
    net = _net()
    x = rng.standard_normal((2, 2, 5, 4, 3))
    t = rng.standard_normal((2, 1, 5, 4, 3))
    loss, grads = net.gradients(x, t)
    for layer in range(3):
        for j in rng.choice(net.layers[layer][0].size, 4, replace=False):
            w = net.layers[layer][0]
            idx = np.unravel_index(j, w.shape)
            h = 1e-6
            w[idx] += h
            lp = co.mse(net.forward(x)[-1], t)[0]
            w[idx] -= 2 * h
            lm = co.mse(net.forward(x)[-1], t)[0]
            w[idx] += h
            assert abs((lp - lm) / (2 * h) - grads[layer][0][idx]) <= 1e-6 * max(1.0, abs(grads[layer][0][idx]))


def test_conv_oracle_is_a_correlation_with_zero_padding():
    x = np.zeros((1, 1, 3, 3, 3))
    x[0, 0, 1, 1, 1] = 1.0
    w = np.zeros((1, 1, 27))
    w[0, 0, 0] = 2.0          # tap (kx, ky, kz) = (0, 0, 0) reads x[v + (-1, -1, -1)]
    y = co.conv3d(x, w)
    assert y[0, 0, 2, 2, 2] == 2.0 and np.count_nonzero(y) == 1


def test_gaussian_random_field_covariance():
    vals = []
    for seed in range(4):
        g = GaussianRandomField(seed, corr_length=0.05, variance=2.0)
        vals.append(g.values)
    v = np.stack(vals)
    assert abs(v.var() - 2.0) < 0.15
    lag = 4   # one correlation length at 4 points per length
    corr = np.mean(v * np.roll(v, lag, axis=1)) / v.var()
    assert abs(corr - np.exp(-0.5)) < 0.05
