"""Host-side logic of the surrogate (no GPU): the learning-rate schedule splits the steps and scales
the rate as listed, and the state normalisation round-trips."""
import numpy as np

from netflux_b200 import surrogate as sur


class _FakeMLP:
    def __init__(self):
        self.calls = []

    def train(self, steps, batch, lr, seed=0, n_report=20):
        self.calls.append((steps, batch, lr, seed, n_report))
        return {"loss": np.full(n_report, lr), "ms": float(steps)}


def test_lr_schedule_splits_steps_and_scales_rate():
    f = _FakeMLP()
    r = sur.MLP.train_schedule(f, 1001, batch=512, lr=1e-3, seed=5, n_report=20)
    steps = [c[0] for c in f.calls]
    assert sum(steps) == 1001 and steps[:3] == [500, 200, 150]
    lrs = [c[2] for c in f.calls]
    assert np.allclose(lrs, [1e-3 * m for _, m in sur.LR_SCHEDULE])
    assert all(c[1] == 512 and c[3] == 5 for c in f.calls)
    assert r["ms"] == 1001.0 and len(r["loss"]) == sum(c[4] for c in f.calls)


def test_lr_schedule_skips_empty_pieces():
    f = _FakeMLP()
    sur.MLP.train_schedule(f, 3, lr=1.0, schedule=((0.5, 1.0), (0.0, 0.5), (0.5, 0.1)))
    assert [(c[0], c[2]) for c in f.calls] == [(2, 1.0), (1, 0.1)]


def test_state_normalisation_round_trips():
    fs = (1.2, 150.0, 10.0, 0.0, 1.0e5)
    rng = np.random.default_rng(0)
    rho = fs[0] * (1 + 0.1 * rng.standard_normal(100))
    u = fs[1] + 10 * rng.standard_normal(100)
    p = fs[4] * (1 + 0.1 * rng.standard_normal(100))
    U = np.column_stack([rho, rho * u, rho * fs[2], np.zeros(100), p / 0.4 + 0.5 * rho * (u * u + fs[2] ** 2)])
    back = sur.denormalise_state(sur.normalise_state(U, fs), fs)
    V = np.hypot(fs[1], fs[2])
    scale = np.array([fs[0], fs[0] * V, fs[0] * V, fs[0] * V, fs[4] / 0.4 + 0.5 * fs[0] * V * V])
    assert np.max(np.abs(back - U) / scale) < 1e-6  # float32 normalised values
