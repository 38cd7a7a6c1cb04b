"""The learned preconditioner's CPU oracle checked against itself: its analytic gradients against
finite differences (float64, no BF16 rounding), and the adjoint pairs it is built from."""
import numpy as np
import pytest

from oracle import unet_oracle as U


def test_adjoint_pairs():
    rng = np.random.default_rng(3)
    x = rng.standard_normal((3, 5, 4, 6))
    w = rng.standard_normal((27, 7, 6))
    y = rng.standard_normal((3, 5, 4, 7))
    assert np.isclose(np.sum(U.conv(x, w) * y), np.sum(x * U.conv_t(y, w)))
    c = rng.standard_normal(U.coarser((3, 5, 4)) + (2,))
    f = rng.standard_normal((3, 5, 4, 2))
    assert np.isclose(np.sum(U.up(c, (3, 5, 4)) * f), np.sum(c * U.up_adjoint(f, c.shape[:3])))
    assert np.isclose(np.sum(U.pool(f) * c), np.sum(f * U.pool_adjoint(c, (3, 5, 4))))


@pytest.mark.parametrize("levels", [2, 3, 5])
def test_gradients_match_finite_differences(levels):
    rng = np.random.default_rng(5)
    flat = U.init_params(1, levels).astype(np.float64)
    shape = (3, 5, 4) if levels <= 3 else (3, 9, 11)
    x = rng.standard_normal(shape + (U.CIO,))
    dy = rng.standard_normal(shape + (U.CIO,))
    net = U.Net(flat, use_bf16=False, levels=levels)
    net.forward(x)
    gw, gb = net.backward(dy)
    grad = U.join_params(gw, gb)

    def loss(p):
        return float(np.sum(U.Net(p, use_bf16=False, levels=levels).forward(x) * dy))

    # probe entries of every layer (weights and biases)
    probes = []
    off = 0
    for cin, cout, _ in U.layers(levels):
        nw = 27 * cin * cout
        probes += [off + int(rng.integers(nw)), off + nw + int(rng.integers(cout))]
        off += nw + cout
    h = 1e-6
    for k in probes:
        e = np.zeros_like(flat)
        e[k] = h
        fd = (loss(flat + e) - loss(flat - e)) / (2 * h)
        assert abs(fd - grad[k]) <= 1e-6 * max(1.0, abs(fd)), (k, fd, grad[k])
