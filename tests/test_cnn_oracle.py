"""CPU checks of the warm-start network's FP64 oracle (finite differences,
adjoint identity) and of the parameter layout the C ABI documents."""
import numpy as np

from oracle import cnn_oracle as O


def test_oracle_gradient_matches_finite_differences():
    blocks = 1
    p = O.init_params(blocks, 3)
    rng = np.random.default_rng(1)
    x = rng.uniform(0, 1, (3, 4, 5))
    xc = x + rng.normal(0, 0.1, x.shape)
    w = rng.uniform(0.5, 1, x.shape)
    loss, g, _ = O.loss_and_grad(p, x, xc, blocks, s_in=2.0, s_out=3.0, w=w)
    idx = np.concatenate([rng.choice(p.size, 30, replace=False), [0, 5, O.TAPS * O.C + 3, p.size - 1]])
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (O.loss_and_grad(pp, x, xc, blocks, 2.0, 3.0, w)[0] - O.loss_and_grad(pm, x, xc, blocks, 2.0, 3.0, w)[0])
        fd /= 2 * h
        assert abs(fd - g[i]) <= 1e-4 * abs(fd) + 1e-9, (i, fd, g[i])


def test_parameter_layout():
    for b in (0, 1, 4):
        n = O.num_params(b)
        d = O.unpack(np.arange(n, dtype=np.float64), b)
        assert d["W_in"].shape == (27, 32) and len(d["W"]) == 2 * b
        assert d["b_out"][0] == n - 1
        assert np.array_equal(O.pack(d), np.arange(n))
    assert O.num_params(4) == 223201


def test_conv_is_adjoint_of_data_gradient():
    rng = np.random.default_rng(0)
    a = rng.normal(size=(3, 5, 4, 32))
    g = rng.normal(size=(3, 5, 4, 32))
    W = rng.normal(size=(27, 32, 32))
    lhs = np.sum(O.conv(a, W) * g)
    rhs = np.sum(a * O.conv_data_grad(g, W))
    assert abs(lhs - rhs) <= 1e-9 * abs(lhs)
