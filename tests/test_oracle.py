"""The CPU oracle is pinned against the reference's own outputs (CPU only).

The golden fixtures were produced by the NetFlux reference compiled from its
own sources (tests/golden/make_golden.py); the C restatement must reproduce
them bit for bit. Where the reference build exists (this container), it is
also run live on a freshly seeded case.
"""
import numpy as np
import pytest

from helpers import CASES, golden, mesh, rel_linf, tet_mesh
from netflux_b200 import meshgen as mg
from oracle import pyoracle as po


def _run(g, n_steps, **kw):
    m = mesh(g)
    pats = m.patches()
    return po.run_oracle(m.export(), pats, [g["freestream"]] * len(pats), g["U0"], n_steps, **kw)


@pytest.mark.parametrize("case", CASES)
def test_oracle_rk3_bitwise(case):
    g = golden(case)
    o = _run(g, 1)
    assert np.array_equal(o["dt"], g["dt1"])
    assert np.array_equal(o["U"], g["U1"])


@pytest.mark.parametrize("case", CASES)
def test_oracle_100_steps_bitwise(case):
    g = golden(case)
    o = _run(g, 100, fields=False)
    assert np.array_equal(o["dt"], g["dt100"])
    assert np.array_equal(o["U"], g["U100"])


@pytest.mark.parametrize("case", CASES)
def test_oracle_stage_intermediates_bitwise(case):
    g = golden(case)
    o = _run(g, 1, time_scheme=0)
    assert np.array_equal(o["U"], g["euler_U"])
    assert np.array_equal(o["V"], g["euler_V"])          # incl. ghost cells
    assert np.array_equal(o["grad"], g["euler_grad"])
    assert np.array_equal(o["limiter"], g["euler_limiter"])
    assert np.array_equal(o["R"], g["euler_R"])


@pytest.mark.parametrize("case", CASES)
def test_oracle_first_order_bitwise(case):
    g = golden(case)
    o = _run(g, 3, spatial_order=0, limiter=0)
    assert np.array_equal(o["dt"], g["first_dt3"])
    assert np.array_equal(o["U"], g["first_U3"])


def test_limiter_range_and_geometry_kats():
    for case in CASES:
        g = golden(case)
        lim = g["euler_limiter"]
        assert lim.min() >= 0.0 and lim.max() <= 1.0          # Numerics.hpp:238-249
        nc = g["dS"].shape[0]
        # sum of S_out over the faces of every interior cell vanishes (closed cells)
        acc = np.zeros((nc, 3))
        ij = g["face_ij"].astype(np.int64)
        np.add.at(acc, ij[:, 0], g["S"])
        inner = ij[:, 1] < nc
        np.add.at(acc, ij[inner, 1], -g["S"][inner])
        assert np.abs(acc).max() < 1e-14
        assert np.all(g["vol"][:nc] > 0)


def test_freestream_preservation():
    """A uniform state with rho = 1 stays uniform on a far-field box (KAT1)."""
    g = golden("cube4")
    m = mesh(g)
    pats = m.patches()
    fs = (1.0, 0.5, 0.1, -0.2, 1.0 / 1.4)
    U0 = mg.uniform_state(m.n_cells, fs)
    o = po.run_oracle(m.export(), pats, [fs] * len(pats), U0, 5)
    assert rel_linf(o["U"], U0) < 1e-13


def test_slip_box_conserves_mass_and_energy():
    """Closed slip-wall box: total mass and energy change only by round-off (KAT2)."""
    g = golden("slipbox5")
    U100, U0 = g["U100"], g["U0"]
    vol = g["vol"][: U0.shape[0]]
    for k in (0, 4):
        m0 = np.sum(U0[:, k] * vol)
        m1 = np.sum(U100[:, k] * vol)
        assert abs(m1 - m0) / abs(m0) < 1e-13


@pytest.mark.skipif(not po.reference_available(), reason="reference build not present")
def test_reference_live_matches_oracle(tmp_path):
    """Run the compiled reference on a new seed and compare with the oracle."""
    m = mg.sod_mesh(24, 3, 3, jitter=0.05, seed=99)
    U0 = mg.sod_initial_state(m)
    fs = mg.SOD_LEFT
    mg.write_case(str(tmp_path / "case"), m, fs, U0=U0)
    ref = po.run_reference(str(tmp_path / "case"), 7, geometry=True)
    from netflux_b200 import solver as S
    mm = S.Mesh.from_su2(str(tmp_path / "case" / "mesh.su2"), {n: mg.BC_CODES[t] for n, t in m.patch_types.items()})
    pats = mm.patches()
    o = po.run_oracle(mm.export(), pats, [fs] * len(pats), U0, 7)
    assert np.array_equal(o["U"], ref["U"])
    assert np.array_equal(o["dt"], ref["dt"])


@pytest.mark.skipif(not po.reference_available("nf_ref"), reason="reference build not present")
def test_reference_with_debug_dump_agrees(tmp_path):
    """The as-shipped reference (per-stage debug dump on) computes the same state."""
    g = golden("cube4")
    m = tet_mesh(g)
    mg.write_case(str(tmp_path / "case"), m, tuple(g["freestream"]), U0=g["U0"])
    a = po.run_reference(str(tmp_path / "case"), 1, variant="nf_ref")
    assert np.array_equal(a["U"], g["U1"])


def test_reference_free_stream_start_leaves_solution_old_zero(tmp_path):
    """NetFlux's own free-stream start writes only `solution` (SolverData.cpp:50-58), so its first
    TVD-RK3 step combines with a zero solution_old (Solver.cpp:127-132). The oracle reproduces the
    reference program bit for bit with U_old_first = 0, and differs from it without."""
    if not po.reference_available():
        pytest.skip("compiled reference not built")
    from netflux_b200 import solver as S
    m = mg.bump_mesh(8, 4, 4, h=0.1)
    fs = mg.bump_freestream(0.5)
    case = str(tmp_path / "case")
    mg.write_case(case, m, fs)  # no U0.bin: the reference initialises itself
    ref = po.run_reference(case, 3)
    mm = S.Mesh.from_tet_mesh(m)
    pats = mm.patches()
    U0 = mg.uniform_state(mm.n_cells, fs)
    o = po.run_oracle(mm.export(), pats, [fs] * len(pats), U0, 3, U_old_first=np.zeros_like(U0), fields=False)
    assert np.array_equal(o["U"], ref["U"])
    o2 = po.run_oracle(mm.export(), pats, [fs] * len(pats), U0, 3, fields=False)
    assert not np.allclose(o2["U"], ref["U"])
