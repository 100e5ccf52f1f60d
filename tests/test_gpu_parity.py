"""Parity of the CUDA path with the reference (golden fixtures) and the oracle.

Tolerances are relative L-infinity errors per conserved variable, max over
cells |a - b| / max |b| (the momentum components measured against the
momentum magnitude max ||rho u||, see helpers.rel_linf):
  * reference-order FP64: 1e-14 (bit-exact except pow() in far-field ghosts)
  * FP64: 1e-12 after 1 TVD-RK3 step, 1e-9 after 100 steps
  * mixed FP32 face work / FP64 state: 1e-5 after 1 step
"""
import numpy as np
import pytest

from helpers import CASES, config_for, golden, mesh, rel_l2, rel_linf
from netflux_b200 import _lib as L
from netflux_b200 import meshgen as mg
from netflux_b200 import solver as S
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

TOL_REF = 1e-14
TOL_FP64_1 = 1e-12
TOL_FP64_100 = 1e-9
TOL_MIXED_1 = 1e-5


def run(g, precision, n_steps, time_scheme="TVD_RK3", spatial_order="Second", limiter="Barth", keep=False,
        use_advance=False, **kw):
    cfg = config_for(time_scheme=time_scheme, spatial_order=spatial_order, limiter=limiter, precision=precision,
                     freestream=tuple(g["freestream"]), **kw)
    m = mesh(g)
    s = S.EulerSolver(cfg, m, U0=g["U0"], keep_stage_fields=keep)
    dts = []
    if use_advance:
        s.advance(n_steps)
    else:
        for _ in range(n_steps):
            s.calc_timestep(cfg)
            dts.append(cfg.get_delta_time())
            s.step(cfg)
    U = s.get_solver_data().get_solution()
    return s, U, np.array(dts)


@pytest.mark.parametrize("case", CASES)
def test_ref_order_one_step(case):
    g = golden(case)
    _, U, dts = run(g, "fp64_ref", 1)
    assert rel_linf(dts, g["dt1"]) <= TOL_REF
    assert rel_linf(U, g["U1"]) <= TOL_REF


def test_ref_order_bitwise_without_far_field():
    """No pow() on the path (slip walls only): the GPU reproduces the reference bit for bit."""
    g = golden("slipbox5")
    _, U, dts = run(g, "fp64_ref", 1)
    assert np.array_equal(dts, g["dt1"])
    assert np.array_equal(U, g["U1"])
    _, U, dts = run(g, "fp64_ref", 100)
    assert np.array_equal(U, g["U100"])


@pytest.mark.parametrize("case", CASES)
def test_ref_order_stage_intermediates(case):
    g = golden(case)
    s, U, _ = run(g, "fp64_ref", 1, time_scheme="ExplicitEuler", keep=True)
    d = s.get_solver_data()
    nc = U.shape[0]
    assert rel_linf(d.get_primvars(), g["euler_V"][:nc]) <= TOL_REF
    assert rel_linf(d.get_primvars_gradient(), g["euler_grad"]) <= 1e-12
    assert np.abs(d.get_primvars_limiter() - g["euler_limiter"]).max() <= 1e-12
    assert rel_linf(d.get_flux_balance(), g["euler_R"]) <= 1e-12
    assert rel_linf(U, g["euler_U"]) <= TOL_REF


@pytest.mark.parametrize("case", CASES)
def test_fp64_one_and_hundred_steps(case):
    g = golden(case)
    _, U1, _ = run(g, "fp64", 1)
    assert rel_linf(U1, g["U1"]) <= TOL_FP64_1
    _, U100, _ = run(g, "fp64", 100, use_advance=True)
    assert rel_linf(U100, g["U100"]) <= TOL_FP64_100


@pytest.mark.parametrize("case", CASES)
def test_ref_order_hundred_steps(case):
    g = golden(case)
    _, U, _ = run(g, "fp64_ref", 100, use_advance=True)
    assert rel_linf(U, g["U100"]) <= 1e-12


@pytest.mark.parametrize("precision", ["mixed", "mixed32"])
@pytest.mark.parametrize("case", CASES)
def test_mixed_one_step(case, precision):
    g = golden(case)
    _, U, _ = run(g, precision, 1)
    print(case, precision, "one step: Linf", rel_linf(U, g["U1"]), "L2", rel_l2(U, g["U1"]))
    err = rel_linf(U, g["U1"])
    assert err <= TOL_MIXED_1, err


@pytest.mark.parametrize("precision", ["mixed", "mixed32"])
@pytest.mark.parametrize("case", CASES)
def test_mixed_forms_explicit_euler_and_first_order(case, precision):
    """The mixed forms on the other schemes: one explicit-Euler step (the time step from the
    timestep kernel every step) and three first-order steps, against the compiled reference."""
    g = golden(case)
    _, U, _ = run(g, precision, 1, time_scheme="ExplicitEuler")
    e1 = rel_linf(U, g["euler_U"])
    _, U, _ = run(g, precision, 3, spatial_order="First", limiter="NONE")
    e3 = rel_linf(U, g["first_U3"])
    print(case, precision, "explicit Euler 1 step:", e1, "first order 3 steps:", e3)
    assert e1 <= TOL_MIXED_1 and e3 <= TOL_MIXED_1


@pytest.mark.parametrize("case", CASES)
def test_mixed32_hundred_steps(case):
    """The mixed form with FP32 copies over 100 steps of the compiled reference's run: its error
    grows with the FP32 rounding of the primitives it gathers (stated, bounded loosely)."""
    g = golden(case)
    _, U, _ = run(g, "mixed32", 100, use_advance=True)
    print(case, "mixed32 100 steps: Linf", rel_linf(U, g["U100"]), "L2", rel_l2(U, g["U100"]))
    assert rel_linf(U, g["U100"]) <= 1e-3


@pytest.mark.parametrize("case", CASES)
def test_first_order(case):
    g = golden(case)
    _, U, dts = run(g, "fp64_ref", 3, spatial_order="First", limiter="NONE")
    assert rel_linf(dts, g["first_dt3"]) <= TOL_REF
    assert rel_linf(U, g["first_U3"]) <= TOL_REF


def test_advance_graph_equals_step_loop():
    g = golden("cube4")
    _, a, _ = run(g, "fp64", 7)
    _, b, _ = run(g, "fp64", 7, use_advance=True)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("precision", ["fp64", "mixed", "mixed32"])
def test_tuning_changes_nothing(precision):
    """Tuned launch shapes compute the same bits and leave the state untouched."""
    g = golden("bump12")
    cfg = config_for(precision=precision, freestream=tuple(g["freestream"]))
    a = S.EulerSolver(cfg, mesh(g), U0=g["U0"])
    a.advance(3)
    b = S.EulerSolver(cfg, mesh(g), U0=g["U0"])
    b.advance(1)
    before = b.get_solver_data().get_solution()
    shapes = b.tune()
    assert np.array_equal(b.get_solver_data().get_solution(), before)
    assert shapes["flux"]["block"] in (64, 128)
    b.advance(2)
    assert np.array_equal(a.get_solver_data().get_solution(), b.get_solver_data().get_solution())


@pytest.mark.parametrize("precision", ["fp64", "mixed", "mixed32"])
def test_every_launch_variant_computes_the_same_bits(precision):
    """Every block size and variant the tuner may pick (pipelined loads, register caps) gives the same state."""
    g = golden("bump12")
    cfg = config_for(precision=precision, freestream=tuple(g["freestream"]))
    out = {}
    n_grad, n_flux = S.LAUNCH_VARIANTS[precision]
    for block in (64, 128):
        for gv in range(n_grad):
            for fv in range(n_flux) if gv == 0 else (0,):
                s = S.EulerSolver(cfg, mesh(g), U0=g["U0"])
                s.set_launch_shapes(gradient=(block, gv), flux=(block, fv))
                s.advance(3)
                out[(block, gv, fv)] = s.get_solver_data().get_solution()
                s.close()
    # separate shapes for the two kernels, fixed through nf_set_launch_shapes
    s = S.EulerSolver(cfg, mesh(g), U0=g["U0"])
    s.set_launch_shapes(gradient=(64, n_grad - 1), flux=(128, n_flux - 1))
    s.advance(3)
    out["mixed shapes"] = s.get_solver_data().get_solution()
    with pytest.raises(L.NetFluxError):
        s.set_launch_shapes(gradient=(64, n_grad), flux=(64, 0))
    with pytest.raises(L.NetFluxError):
        s.set_launch_shapes(gradient=(64, 0), flux=(64, n_flux))
    with pytest.raises(L.NetFluxError):
        s.set_launch_shapes(gradient=(64, 0), flux=(200, 0))
    s.close()
    ref = out[(128, 0, 0)]
    for k, U in out.items():
        assert np.array_equal(U, ref), k


def test_deterministic_repeat():
    g = golden("sod40")
    _, a, _ = run(g, "fp64", 20, use_advance=True)
    _, b, _ = run(g, "fp64", 20, use_advance=True)
    assert np.array_equal(a, b)


def _oracle(g, n, **kw):
    m = mesh(g)
    pats = m.patches()
    return po.run_oracle(m.export(), pats, [g["freestream"]] * len(pats), g["U0"], n, **kw)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-14), ("mixed", 1e-6), ("mixed32", 1e-5)])
def test_fused_time_step_matches_oracle(precision, tol):
    """From the second step on the time step is computed inside the step: FP64 by the last stage's
    gradient kernel (the last stage input's primitives, projected areas from the normals in
    registers), the mixed forms by the stage-2 flux kernel from the FP64 primitives of its result
    (the same state). Each step's dt agrees with the oracle's calc_timestep: FP64 to a few ulp, the
    mixed forms to their state's own error."""
    g = golden("bump12")
    _, U, dts = run(g, precision, 20)
    o = _oracle(g, 20, fields=False)
    err = np.abs(dts - o["dt"]) / o["dt"]
    print(precision, "fused dt vs oracle: max rel", err.max())
    assert err.max() <= tol
    assert rel_linf(U, o["U"]) <= (1e-12 if precision == "fp64" else 1e-4)


def test_local_time_stepping_matches_oracle():
    g = golden("bump12")
    _, U, _ = run(g, "fp64_ref", 10, local_time_stepping=True)
    o = _oracle(g, 10, local_time_stepping=True, fields=False)
    assert rel_linf(U, o["U"]) <= 1e-13


def test_limiter_ratchet_bitwise_without_far_field():
    """Limiter ratchet from step 10 (extension), through single steps and graph replays: with no pow()
    on the path the reference-order form keeps exactly the oracle's limiter values."""
    g = golden("slipbox5")
    s, _, _ = run(g, "fp64_ref", 0, limiter_ratchet_step=10)
    cfg = s.config
    s.advance(7)
    for _ in range(5):  # the ratchet starts inside this loop
        s.calc_timestep(cfg)
        s.step(cfg)
    s.advance(28)
    o = _oracle(g, 40, limiter_ratchet_step=10, fields=False)
    live = _oracle(g, 40, fields=False)
    U = s.get_solver_data().get_solution()
    assert np.array_equal(U, o["U"])
    assert not np.array_equal(live["U"], o["U"])  # the ratchet changed the result


@pytest.mark.parametrize("precision,tol_l2", [("fp64_ref", 1e-9), ("fp64", 1e-6), ("mixed", 3e-4)])
def test_limiter_ratchet_matches_oracle(precision, tol_l2):
    """Ratchet on the bump with far field: round-off (pow() in the far-field ghosts, the fast forms'
    arithmetic) picks different limiter values in near-uniform cells, where the Barth ratio is
    noise, and the ratchet keeps them, so agreement is stated in relative L2."""
    g = golden("bump12")
    s, _, _ = run(g, precision, 0, local_time_stepping=True, limiter_ratchet_step=20)
    s.advance(60)
    o = _oracle(g, 60, local_time_stepping=True, limiter_ratchet_step=20, fields=False)
    live = _oracle(g, 60, local_time_stepping=True, fields=False)
    U = s.get_solver_data().get_solution()
    print(precision, "ratchet vs oracle: L2", rel_l2(U, o["U"]), "Linf", rel_linf(U, o["U"]),
          "| live vs ratchet oracle: L2", rel_l2(live["U"], o["U"]))
    assert rel_l2(U, o["U"]) <= tol_l2
    assert rel_l2(live["U"], o["U"]) > 10 * tol_l2


@pytest.mark.parametrize("precision,tol", [("fp64_ref", 1e-13), ("fp64", 1e-12)])
def test_set_state_old_reproduces_the_reference_free_stream_start(precision, tol):
    """U^n of the first RK3 step set apart from the state (zero, as NetFlux's own free-stream start
    leaves solution_old), through graph replays and through single steps."""
    g = golden("bump12")
    zero = np.zeros_like(g["U0"])
    o = _oracle(g, 10, U_old_first=zero, fields=False)
    s, _, _ = run(g, precision, 0)
    s.set_state_old(zero)
    s.advance(10)
    assert rel_linf(s.get_solver_data().get_solution(), o["U"]) <= tol
    s2, U2, _ = run(g, precision, 0)
    s2.set_state_old(zero)
    cfg = s2.config
    for _ in range(10):
        s2.calc_timestep(cfg)
        s2.step(cfg)
    assert rel_linf(s2.get_solver_data().get_solution(), o["U"]) <= tol


def test_t_end_clipping_matches_oracle():
    g = golden("sod40")
    t_end = 0.9 * 5 * float(g["dt1"][0])
    s, U, _ = run(g, "fp64_ref", 0, t_end=t_end)
    time = s.advance(8)
    o = _oracle(g, 8, t_end=t_end, fields=False)
    assert abs(time - t_end) <= 1e-15 * t_end
    assert rel_linf(U, g["U0"]) == 0.0  # the state before advancing
    assert rel_linf(s.get_solver_data().get_solution(), o["U"]) <= 1e-13


def test_residual_norms_match_oracle():
    g = golden("cube4")
    s, _, _ = run(g, "fp64", 3)
    res = s.residual()
    o = _oracle(g, 3, fields=False)
    assert np.allclose(res[0], o["res"][-1], rtol=1e-12, atol=0)


def test_batched_equals_individual_runs():
    """Cases concatenated into one mesh advance exactly as they do alone (local dt)."""
    gs = [golden("cube4"), golden("bump12")]
    cfgs = [config_for(precision="fp64", local_time_stepping=True, freestream=tuple(g["freestream"])) for g in gs]
    singles = []
    for g, cfg in zip(gs, cfgs):
        s = S.EulerSolver(cfg, mesh(g), U0=g["U0"])
        s.advance(5)
        singles.append(s.get_solver_data().get_solution())
    ms = [mesh(g) for g in gs]
    batch = S.Mesh.concat(ms)
    states = [list(g["freestream"]) for g, m in zip(gs, ms) for _ in m.patches()]
    sb = S.EulerSolver(cfgs[0], batch, U0=np.concatenate([g["U0"] for g in gs]), patch_states=states)
    sb.advance(5)
    Ub = sb.get_solver_data().get_solution()
    off = batch.case_offsets()
    for k, U in enumerate(singles):
        assert np.array_equal(Ub[off[k]:off[k + 1]], U)
    r = sb.residual()
    assert r.shape == (2, 2) and np.all(r[:, 0] > 0)


def test_nonphysical_state_is_reported():
    """A negative pressure injected on the host surfaces as an error status, not a fault."""
    g = golden("cube4")
    U0 = g["U0"].copy()
    U0[17, 4] = -1.0  # negative total energy -> negative pressure
    cfg = config_for(precision="fp64", freestream=tuple(g["freestream"]))
    s = S.EulerSolver(cfg, mesh(g), U0=U0)
    with pytest.raises((L.NetFluxError, RuntimeError)):
        s.calc_timestep(cfg)
        s.step(cfg)
        s.synchronize()


def test_residual_max_norm_keeps_nan():
    """A NaN in the state makes both residual norms NaN: the max norm does not drop it."""
    g = golden("cube4")
    U0 = g["U0"].copy()
    U0[17, 1] = np.nan
    cfg = config_for(precision="fp64", freestream=tuple(g["freestream"]))
    s = S.EulerSolver(cfg, mesh(g), U0=U0)
    s.calc_timestep(cfg)
    s.step(cfg)
    r = s.residual()
    assert np.isnan(r[0, 0]) and np.isnan(r[0, 1]), r
    s.close()


def test_sod_tube_against_oracle_and_mixed_error():
    """Sod tube with the limiter active at the shock: FP64 and mixed vs the oracle."""
    m = mg.sod_mesh(100, 4, 4, jitter=0.05, seed=5)
    U0 = mg.sod_initial_state(m)
    mm = S.Mesh.from_tet_mesh(m)
    pats = mm.patches()
    n = 60
    o = po.run_oracle(mm.export(), pats, [mg.SOD_LEFT] * len(pats), U0, n, fields=False)
    out = {}
    for prec in ("fp64", "mixed"):
        cfg = config_for(precision=prec, freestream=mg.SOD_LEFT)
        s = S.EulerSolver(cfg, mm, U0=U0)
        s.advance(n)
        out[prec] = s.get_solver_data().get_solution()
    assert rel_linf(out["fp64"], o["U"]) <= TOL_FP64_100
    print("sod mixed: Linf", rel_linf(out["mixed"], o["U"]), "L2", rel_l2(out["mixed"], o["U"]))
    assert rel_linf(out["mixed"], o["U"]) <= 1e-3
    assert rel_l2(out["mixed"], o["U"]) <= 1e-4


def _bump_case(nx, h, mach):
    m = mg.bump_mesh(nx, nx // 2, nx // 2, h=h)
    fs = mg.bump_freestream(mach)
    return m, fs


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-6), ("mixed", 1e-6)])
def test_steady_solve_reaches_tolerance(precision, tol):
    """Unlimited second order converges: the oracle drops the residual below 1e-6 within ~5000 steps."""
    m, fs = _bump_case(12, 0.1, 0.5)
    mm = S.Mesh.from_tet_mesh(m)
    cfg = config_for(precision=precision, limiter="NONE", local_time_stepping=True, freestream=fs)
    s = S.EulerSolver(cfg, mm, U0=mg.uniform_state(mm.n_cells, fs))
    out = s.solve_steady(tol=tol, max_steps=20000, check_every=25)
    assert out["converged"][0], out
    assert out["res"][0] <= tol * out["res0"][0]
    assert out["steps"][0] % 25 == 1  # checked every 25 steps after the first


def test_steady_barth_plateau_matches_oracle():
    """With the Barth limiter the reference's residual stalls near a 2.5e-3 drop (limiter chatter):
    the driver reports the case as not converged, at the oracle's plateau."""
    m, fs = _bump_case(12, 0.1, 0.5)
    mm = S.Mesh.from_tet_mesh(m)
    n = 2001
    pats = mm.patches()
    o = po.run_oracle(mm.export(), pats, [fs] * len(pats), mg.uniform_state(mm.n_cells, fs), n,
                      local_time_stepping=True, fields=False)
    cfg = config_for(precision="fp64", local_time_stepping=True, freestream=fs)
    s = S.EulerSolver(cfg, mm, U0=mg.uniform_state(mm.n_cells, fs))
    out = s.solve_steady(tol=1e-4, max_steps=n, check_every=25)
    assert not out["converged"][0]
    assert out["steps"][0] == n
    assert abs(out["res0"][0] / o["res"][0, 0] - 1.0) <= 1e-12
    drop, drop_o = out["res"][0] / out["res0"][0], o["res"][n - 1, 0] / o["res"][0, 0]
    assert 1e-3 <= drop_o <= 1e-2
    assert 0.5 <= drop / drop_o <= 2.0


def test_steady_barth_with_ratchet_reaches_1e6_like_oracle():
    """Barth limiter with the ratchet started at a 1e-2 drop converges to a 1e-6 drop; the converged
    state is the oracle's run with the ratchet started at the same step."""
    m, fs = _bump_case(12, 0.1, 0.5)
    mm = S.Mesh.from_tet_mesh(m)
    U0 = mg.uniform_state(mm.n_cells, fs)
    every = 25
    cfg = config_for(precision="fp64", local_time_stepping=True, freestream=fs, limiter_ratchet_drop=1e-2)
    s = S.EulerSolver(cfg, mm, U0=U0)
    out = s.solve_steady(tol=1e-6, max_steps=20000, check_every=every)
    assert out["converged"][0], out
    n = int(out["steps"][0])
    pats = mm.patches()
    live = po.run_oracle(mm.export(), pats, [fs] * len(pats), U0, n, local_time_stepping=True, fields=False)
    r = live["res"][:, 0]
    checks = np.arange(1 + every, n + 1, every)  # residual checks after that many steps
    k = int(checks[np.argmax(r[checks - 1] <= 1e-2 * r[0])])
    o = po.run_oracle(mm.export(), pats, [fs] * len(pats), U0, n, local_time_stepping=True,
                      limiter_ratchet_step=k, fields=False)
    assert o["res"][n - 1, 0] <= 1e-6 * o["res"][0, 0] < o["res"][n - 1 - every, 0]  # same convergence step
    U = s.get_solver_data().get_solution()
    print("steady ratchet vs oracle: L2", rel_l2(U, o["U"]), "Linf", rel_linf(U, o["U"]))
    assert rel_l2(U, o["U"]) <= 1e-7


def test_steady_mixed_lands_on_the_fp64_state():
    """Mixed and FP64 steady solves (1e-6 drop) reach the same state to FP32-level accuracy."""
    m, fs = _bump_case(12, 0.1, 0.5)
    mm = S.Mesh.from_tet_mesh(m)
    U0 = mg.uniform_state(mm.n_cells, fs)
    res = {}
    for prec in ("fp64", "mixed"):
        cfg = config_for(precision=prec, limiter="NONE", local_time_stepping=True, freestream=fs)
        s = S.EulerSolver(cfg, mm, U0=U0)
        out = s.solve_steady(tol=1e-6, max_steps=20000, check_every=25)
        assert out["converged"][0], (prec, out)
        res[prec] = s.get_solver_data().get_solution()
    print("steady mixed vs fp64: L2", rel_l2(res["mixed"], res["fp64"]), "Linf", rel_linf(res["mixed"], res["fp64"]))
    assert rel_l2(res["mixed"], res["fp64"]) <= 1e-5


def test_steady_residual_of_the_two_mixed_forms():
    """The difference form reaches a 1e-6 density-residual drop like FP64; the form with FP32 copies
    of the primitives rounds every gathered value at |V| 2^-24, and its residual stalls above that
    (the reached drop is printed; it must still fall by three decades)."""
    m, fs = _bump_case(12, 0.1, 0.5)
    mm = S.Mesh.from_tet_mesh(m)
    U0 = mg.uniform_state(mm.n_cells, fs)
    out = {}
    for prec in ("mixed", "mixed32"):
        cfg = config_for(precision=prec, limiter="NONE", local_time_stepping=True, freestream=fs)
        s = S.EulerSolver(cfg, mm, U0=U0)
        out[prec] = s.solve_steady(tol=1e-6, max_steps=20000, check_every=25)
        s.close()
        r = out[prec]
        print(prec, "steady: converged", bool(r["converged"][0]), "steps", int(r["steps"][0]),
              "drop", float(r["res"][0] / r["res0"][0]))
    assert out["mixed"]["converged"][0]
    assert out["mixed32"]["res"][0] <= 1e-3 * out["mixed32"]["res0"][0]


def test_batched_steady_freezes_converged_cases_exactly():
    """Each case of a batch stops where it would alone; frozen cases do not move."""
    cases = [_bump_case(10, 0.05, 0.4), _bump_case(12, 0.12, 0.6)]
    meshes = [S.Mesh.from_tet_mesh(m) for m, _ in cases]
    singles = []
    for (m, fs), mm in zip(cases, meshes):
        cfg = config_for(precision="fp64", local_time_stepping=True, freestream=fs)
        s = S.EulerSolver(cfg, mm, U0=mg.uniform_state(mm.n_cells, fs))
        out = s.solve_steady(tol=1e-3, max_steps=20000, check_every=20)
        singles.append((out, s.get_solver_data().get_solution()))
    batch = S.Mesh.concat(meshes)
    states = [list(fs) for (m, fs), mm in zip(cases, meshes) for _ in mm.patches()]
    U0 = np.concatenate([mg.uniform_state(mm.n_cells, fs) for (m, fs), mm in zip(cases, meshes)])
    cfg = config_for(precision="fp64", local_time_stepping=True, freestream=cases[0][1])
    sb = S.EulerSolver(cfg, batch, U0=U0, patch_states=states)
    out = sb.solve_steady(tol=1e-3, max_steps=20000, check_every=20)
    Ub = sb.get_solver_data().get_solution()
    off = batch.case_offsets()
    for k, (o, U) in enumerate(singles):
        assert out["steps"][k] == o["steps"][0]
        assert np.array_equal(Ub[off[k]:off[k + 1]], U)


def test_fast_reciprocal_and_rsqrt_within_two_ulp():
    """The fast FP64 form's 1/x and 1/sqrt(x) (FP32 estimate + two Newton-Raphson steps) against
    correctly rounded values, over 12 decades either side of 1."""
    rng = np.random.default_rng(7)
    x = 10.0 ** rng.uniform(-12, 12, 200000)
    r = np.empty_like(x)
    q = np.empty_like(x)
    assert L.load().nf_fastmath_selftest(L.dptr(x), x.size, L.dptr(r), L.dptr(q)) == L.NF_OK
    ulp = lambda v: np.spacing(np.abs(v))
    e_rcp = np.abs(r - 1.0 / x) / ulp(1.0 / x)
    e_rsq = np.abs(q - 1.0 / np.sqrt(x)) / ulp(1.0 / np.sqrt(x))
    print("max ulp: rcp", e_rcp.max(), "rsqrt", e_rsq.max())
    assert e_rcp.max() <= 2 and e_rsq.max() <= 2
