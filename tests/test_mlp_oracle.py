"""CPU checks of the surrogate MLP's oracle: its backward pass against finite differences."""
import numpy as np

from oracle import mlp_oracle as mo


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5e-3], np.float32)
    r = mo.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0  # tie -> even
    assert r[2] == np.float32(1.0 + 2 ** -6)  # tie -> even (up)
    assert r[3] == 1.0
    assert abs(r[4] - x[4]) <= 2 ** -9 * abs(x[4])


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = mo.init_params(1).astype(np.float64)
    f = rng.uniform(-1, 1, (48, 7))
    t = rng.normal(0, 0.1, (48, 5))
    _, g = mo.loss_and_grad(p, f, t, bf16_round=False)
    idx = [mo.OFF_W0 + 3, mo.OFF_W0 + 16 * 5 + 7, mo.OFF_W1 + 100, mo.OFF_W2 + 5000, mo.OFF_W3 + 77,
           mo.OFF_B1 + 3, mo.OFF_B2 + 50, mo.OFF_B3 + 127, mo.OFF_W4 + 2 * 128 + 9, mo.OFF_B4 + 4]
    for i in idx:
        e = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += e
        pm[i] -= e
        fd = (mo.loss_and_grad(pp, f, t, bf16_round=False)[0] - mo.loss_and_grad(pm, f, t, bf16_round=False)[0]) / (2 * e)
        assert abs(fd - g[i]) <= 1e-6 * abs(g[i]) + 1e-9, (i, fd, g[i])
    # padded entries have zero gradient
    assert np.all(g[mo.OFF_W4 + 5 * 128:mo.OFF_B4] == 0) and np.all(g[mo.OFF_B4 + 5:] == 0)
    W0g = g[mo.OFF_W0:mo.OFF_W1].reshape(128, 16)
    assert np.all(W0g[:, 8:] == 0)
