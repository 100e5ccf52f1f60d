"""Surrogate MLP on the GPU: the tcgen05 GEMM, forward pass and gradients against the CPU oracle
(BF16 rounding emulated), and training."""
import numpy as np
import pytest

from helpers import gpu_available  # noqa: F401
from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu


def bits(x: np.ndarray) -> np.ndarray:
    return (mo.bf16(x).view(np.uint32) >> 16).astype(np.uint16)


@pytest.mark.parametrize("N,K", [(128, 128), (16, 16), (144, 64), (256, 32)])
def test_tcgen05_gemm_matches_cpu(N, K):
    from netflux_b200 import surrogate as sur
    rng = np.random.default_rng(N * 1000 + K)
    A = mo.bf16(rng.normal(size=(128, K)).astype(np.float32))
    B = mo.bf16(rng.normal(size=(N, K)).astype(np.float32))
    D = sur.gemm_selftest(bits(A), bits(B))
    ref = A.astype(np.float64) @ B.astype(np.float64).T
    assert np.max(np.abs(D - ref)) <= 1e-5 * np.max(np.abs(ref)) * np.sqrt(K)


def test_mlp_forward_matches_oracle():
    from netflux_b200 import surrogate as sur
    m = sur.MLP(seed=3)
    p = m.get_params()
    rng = np.random.default_rng(1)
    f = rng.uniform(-1, 1, (1000, 7)).astype(np.float32)
    y, _ = m.predict(f)
    yo, _ = mo.forward(p, f)
    err = np.abs(y - yo)
    print("forward: max", err.max(), "mean", err.mean(), "scale", np.abs(yo).max())
    assert err.max() <= 2e-2 * np.abs(yo).max()
    assert err.mean() <= 2e-3 * np.abs(yo).max()


def test_mlp_gradients_match_oracle():
    from netflux_b200 import surrogate as sur
    m = sur.MLP(seed=5)
    p = m.get_params()
    rng = np.random.default_rng(2)
    n = 777  # not a multiple of the 128-row tiles or the 64-row chunks
    f = rng.uniform(-1, 1, (n, 7)).astype(np.float32)
    t = rng.normal(0, 0.2, (n, 5)).astype(np.float32)
    loss, g = m.gradients(f, t)
    lo, go = mo.loss_and_grad(p, f, t)
    print("loss", loss, lo)
    assert abs(loss - lo) <= 1e-3 * lo
    blocks = {"W0": (mo.OFF_W0, mo.OFF_W1), "W1": (mo.OFF_W1, mo.OFF_W2), "W2": (mo.OFF_W2, mo.OFF_W3),
              "W3": (mo.OFF_W3, mo.OFF_B1), "b": (mo.OFF_B1, mo.OFF_W4), "W4": (mo.OFF_W4, mo.OFF_B4),
              "b4": (mo.OFF_B4, mo.N_PARAM)}
    for name, (a, b) in blocks.items():
        ga, gb = g[a:b].astype(np.float64), go[a:b]
        rel = np.linalg.norm(ga - gb) / max(np.linalg.norm(gb), 1e-30)
        cos = ga @ gb / max(np.linalg.norm(ga) * np.linalg.norm(gb), 1e-30)
        print(name, "rel L2", rel, "cos", cos)
        assert rel <= 3e-2 and cos >= 0.999, name


def test_mlp_training_fits_a_smooth_field():
    from netflux_b200 import surrogate as sur
    rng = np.random.default_rng(4)
    f = rng.uniform(-1, 1, (50000, 7)).astype(np.float32)
    t = np.column_stack([0.1 * np.sin(2 * f[:, 0]) * f[:, 4], 0.05 * f[:, 1] * f[:, 5], 0.02 * np.cos(f[:, 2]),
                         0.03 * f[:, 3] ** 2, 0.1 * np.tanh(f[:, 0] + f[:, 6])]).astype(np.float32)
    m = sur.MLP(seed=7)
    m.set_data(f, t)
    r0 = m.train(1, batch=4096, lr=1e-3, n_report=1)
    r = m.train(600, batch=4096, lr=1e-3, n_report=6)
    print("loss", r0["loss"], r["loss"], "ms", r["ms"])
    assert r["loss"][-1] <= 0.05 * r0["loss"][0]


def test_warm_start_gains_over_free_stream_start():
    """Train on batched steady solutions of small channels, then warm-start a held-out (Mach, h):
    it reaches the same absolute residual in fewer steps and lands on the plain solve's state."""
    from netflux_b200 import sweep as SW
    from netflux_b200 import surrogate as sur
    from netflux_b200 import meshgen as mg
    cases = SW.sample_cases(8, 11, 12, 16, (0.35, 0.55), (0.05, 0.1))
    res = SW.run_batched(cases, "mixed", 1e-6, 100000, 50)
    assert all(c["converged"] for c in res["per_case"])
    F, T = SW.training_data(res, cases)
    mlp = sur.MLP(seed=1)
    mlp.set_data(F, T)
    tr = mlp.train(3000, 16384, 1e-3, seed=1, n_report=3)
    c = {"nx": 14, "mach": 0.45, "h": 0.08}
    mesh = SW.case_mesh(c)
    fs = mg.bump_freestream(c["mach"])
    plain = sur.solve_plain(mesh, fs, 1e-6, "mixed", 100000, 50)
    warm = sur.solve_warm(mesh, fs, mlp, c["mach"], c["h"], 1e-6, "mixed", 100000, 50)
    d = np.linalg.norm(warm["U"] - plain["U"]) / np.linalg.norm(plain["U"])
    d0 = np.linalg.norm(warm["U_warm"] - plain["U"]) / np.linalg.norm(plain["U"])
    print("train loss", tr["loss"], "plain steps", plain["steps"], "warm steps", warm["steps"],
          "warm start L2", d0, "final L2", d, "fallback", warm["fallback"])
    assert plain["converged"] and warm["converged"] and warm["fallback"] is None
    assert warm["res_final"] <= 1e-6 * plain["res_fs"]
    assert warm["steps"] < plain["steps"]
    assert d <= 1e-6  # the warm-started solve lands within 1e-6 relative L2 of the plain one


def test_wall_distance_matches_brute_force():
    from netflux_b200 import _lib as L
    rng = np.random.default_rng(3)
    pts = rng.uniform(0, 3, (5000, 3)).astype(np.float32)
    wall = rng.uniform(0, 3, (3001, 3)).astype(np.float32)
    out = np.empty(5000, np.float32)
    assert L.load().nf_wall_distance(L.fptr(pts), 5000, L.fptr(wall), 3001, L.fptr(out)) == L.NF_OK
    ref = np.sqrt(((pts[:, None, :].astype(np.float64) - wall[None, :, :]) ** 2).sum(-1).min(1))
    assert np.max(np.abs(out - ref)) <= 1e-5 * np.max(ref)
