"""Parity at the full sizes of the workloads, against the oracle (or the compiled reference):
  * unit cube, 20^3 hexes x 6 tets (48,000 cells), Gaussian density bump, far field all round,
    TVD-RK3 at CFL 0.8: against the compiled reference (or the oracle where it is not built),
    FP64 <= 1e-12 after 1 step and <= 1e-9 after 100 steps;
  * Sod tube, 400 x 8 x 8 hexes x 6 tets (153,600 cells), slip sides, far-field ends, to t = 0.2
    (about 1,200 steps): FP64 and mixed against the oracle run to the same time;
  * the bump channel, 128 x 64 x 64 hexes x 6 tets (3,145,728 cells, the bench workload): one
    TVD-RK3 step with local time stepping and the Barth limiter against the oracle, from the bench's
    free-stream state and from a perturbed state; plus size-independent properties (repeatability,
    launch shapes). The 100-step comparison at this size takes the oracle about 7 minutes and runs
    when NETFLUX_LONG_PARITY=1;
  * seeded cases of the batched sweep (bump channels of random Mach and bump height), 50 steps.
Errors are relative L-infinity with the momentum components scaled by max |rho u| (helpers.rel_linf);
every test also prints each conserved variable's own relative L-infinity and L2 (helpers.per_variable).
The oracle runs in a background thread (the ctypes call releases the interpreter lock) while the GPU
runs, so a test takes about as long as the oracle alone."""
import os
import tempfile
import threading

import numpy as np
import pytest

from helpers import format_per_variable, per_variable, rel_l2, rel_linf
from netflux_b200 import meshgen as mg
from netflux_b200 import solver as S
from netflux_b200 import sweep as SW
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

CUBE_FS = (1.0, 0.5, 0.0, 0.0, 1.0 / 1.4)
TOL_FP64_1 = 1e-12
TOL_FP64_100 = 1e-9
TOL_MIXED_1 = 1e-5


class Background:
    """Run fn(*args, **kw) in a thread; .result() joins it and re-raises its exception."""

    def __init__(self, fn, *args, **kw):
        self._out, self._err = None, None

        def body():
            try:
                self._out = fn(*args, **kw)
            except BaseException as e:  # noqa: BLE001 - re-raised in result()
                self._err = e

        self._t = threading.Thread(target=body, daemon=True)
        self._t.start()

    def result(self):
        self._t.join()
        if self._err is not None:
            raise self._err
        return self._out


def _cube():
    m = mg.cube_mesh(20, jitter=0.1, seed=1234)
    return m, mg.cube_initial_state(m)


def _gpu(mesh, U0, precision, n, freestream, patch_states=None, **kw):
    cfg = S.Config(precision=precision, CFL=0.8, density_fs=freestream[0], velocity_fs=list(freestream[1:4]),
                   pressure_fs=freestream[4], **kw)
    s = S.EulerSolver(cfg, mesh, U0=U0, patch_states=patch_states)
    s.advance(n)
    U = s.get_solver_data().get_solution()
    s.close()
    return U


def _report(label, errs):
    for prec, e in errs.items():
        print(f"{label} {prec}: rel Linf (momentum as one vector) {rel_linf(*e):.2e}; per variable: "
              f"{format_per_variable(per_variable(*e))}")


def test_config1_cube_48k_cells():
    m, U0 = _cube()
    with tempfile.TemporaryDirectory() as d:
        mg.write_case(d, m, CUBE_FS, U0)
        mesh = S.Mesh.from_su2(os.path.join(d, "mesh.su2"), {"farfield": mg.BC_CODES["FarField"]})
        assert mesh.n_cells == 48000
        if po.reference_available():
            ref1 = po.run_reference(d, 1)["U"]
            ref100 = po.run_reference(d, 100)["U"]
            kind = "compiled reference"
        else:
            pats = mesh.patches()
            ref1 = po.run_oracle(mesh.export(), pats, [CUBE_FS] * len(pats), U0, 1, fields=False)["U"]
            ref100 = po.run_oracle(mesh.export(), pats, [CUBE_FS] * len(pats), U0, 100, fields=False)["U"]
            kind = "oracle"
    pairs = {}
    for prec in ("fp64_ref", "fp64", "mixed"):
        pairs[prec] = ((_gpu(mesh, U0, prec, 1, CUBE_FS), ref1), (_gpu(mesh, U0, prec, 100, CUBE_FS), ref100))
    _report(f"config 1 vs {kind}, 1 step,", {p: v[0] for p, v in pairs.items()})
    _report(f"config 1 vs {kind}, 100 steps,", {p: v[1] for p, v in pairs.items()})
    errs = {p: (rel_linf(*v[0]), rel_linf(*v[1])) for p, v in pairs.items()}
    assert errs["fp64_ref"][0] <= 1e-14 and errs["fp64_ref"][1] <= 1e-12
    assert errs["fp64"][0] <= TOL_FP64_1 and errs["fp64"][1] <= TOL_FP64_100
    assert errs["mixed"][0] <= TOL_MIXED_1


def test_config2_sod_153k_cells_to_t_0_2_against_oracle():
    """Each far-field end holds its own state (per-patch free stream) with the isentropic ghost density
    (farfield_density_fix; the reference's inverted form is exact only for rho_fs = 1, and with one
    free stream the right end drives a chaotic inflow). The oracle runs the same number of steps as
    the GPU needs to reach t = 0.2 (the last dt clipped at t_end)."""
    m = mg.sod_mesh(400, 8, 8, jitter=0.05, seed=4321)
    U0 = mg.sod_initial_state(m)
    mesh = S.Mesh.from_tet_mesh(m)
    assert mesh.n_cells == 153600
    pats = mesh.patches()
    states = [mg.SOD_RIGHT if p["name"] == "right" else mg.SOD_LEFT for p in pats]

    def config(prec):
        return S.Config(precision=prec, CFL=0.8, t_end=0.2, density_fs=1.0, velocity_fs=[0, 0, 0], pressure_fs=1.0,
                        farfield_density_fix=True)

    # steps to reach t = 0.2 (the reference-order form; every form computes the same dt history to
    # round-off, and the count is fixed for all of them)
    s = S.EulerSolver(config("fp64_ref"), mesh, U0=U0, patch_states=states)
    n_end, t = 0, 0.0
    while t < 0.2:
        t = s.advance(1)
        n_end += 1
        assert n_end < 5000
    s.close()
    oracle = Background(po.run_oracle, mesh.export(), pats, states, U0, n_end, t_end=0.2, fields=False,
                        farfield_density_fix=True)
    out = {}
    for prec in ("fp64_ref", "fp64", "mixed"):
        s = S.EulerSolver(config(prec), mesh, U0=U0, patch_states=states)
        t = s.advance(n_end)
        assert abs(t - 0.2) <= 1e-15, (prec, t)
        out[prec] = s.get_solver_data().get_solution()
        s.close()
    o = oracle.result()
    assert abs(o["time"] - 0.2) <= 1e-15
    _report(f"config 2 Sod at t=0.2 ({n_end} steps) vs oracle,", {p: (U, o["U"]) for p, U in out.items()})
    e = {p: (rel_linf(U, o["U"]), rel_l2(U, o["U"])) for p, U in out.items()}
    print("rho range", out["fp64"][:, 0].min(), out["fp64"][:, 0].max())
    assert e["fp64_ref"][0] <= 1e-11
    assert e["fp64"][0] <= TOL_FP64_100
    assert e["mixed"][0] <= 1e-3 and e["mixed"][1] <= 1e-5


def _bump3m():
    m = mg.bump_mesh(128, 64, 64, h=0.1)
    fs = mg.bump_freestream(0.5)
    mesh = S.Mesh.from_tet_mesh(m)
    assert mesh.n_cells == 3145728
    return m, fs, mesh


def _perturbed(m, fs, n):
    c = m.centroids()
    V = np.broadcast_to(np.asarray(fs, np.float64), (n, 5)).copy()
    bump = 0.02 * np.sin(2 * np.pi * c[:, 0] / 3.0) * np.sin(np.pi * c[:, 1]) * np.sin(np.pi * c[:, 2])
    V[:, 0] *= 1.0 + bump
    V[:, 4] *= 1.0 + 0.5 * bump
    return mg.prim_to_cons(V)


def test_config3_bump_3m_cells_one_step_against_oracle():
    """The benched workload: 3,145,728 tets, Mach 0.5, slip walls and far field, Barth limiter, local
    time stepping at CFL 0.8, one TVD-RK3 step, from the bench's own free-stream state and from a
    smoothly perturbed one (every cell's limiter and flux active)."""
    m, fs, mesh = _bump3m()
    pats = mesh.patches()
    grid = mesh.export()
    starts = {"free stream (bench state)": mg.uniform_state(mesh.n_cells, fs),
              "perturbed": _perturbed(m, fs, mesh.n_cells)}
    for label, U0 in starts.items():
        oracle = Background(po.run_oracle, grid, pats, [fs] * len(pats), U0, 1, local_time_stepping=True,
                            fields=False)
        out = {p: _gpu(mesh, U0, p, 1, fs, local_time_stepping=True) for p in ("fp64", "mixed", "mixed32")}
        o = oracle.result()["U"]
        _report(f"config 3 ({label}), 1 step vs oracle,", {p: (U, o) for p, U in out.items()})
        print("  max change of the step", rel_linf(o, U0))
        assert rel_linf(o, U0) > 1e-8  # the step changed the state
        assert rel_linf(out["fp64"], o) <= TOL_FP64_1, label
        assert rel_linf(out["mixed"], o) <= TOL_MIXED_1, label
        assert rel_linf(out["mixed32"], o) <= TOL_MIXED_1, label


@pytest.mark.skipif(os.environ.get("NETFLUX_LONG_PARITY") != "1",
                    reason="100 oracle steps at 3.1M tets take about 7 minutes (NETFLUX_LONG_PARITY=1)")
def test_config3_bump_3m_cells_hundred_steps_against_oracle():
    m, fs, mesh = _bump3m()
    pats = mesh.patches()
    U0 = _perturbed(m, fs, mesh.n_cells)
    oracle = Background(po.run_oracle, mesh.export(), pats, [fs] * len(pats), U0, 100, local_time_stepping=True,
                        fields=False)
    out = {p: _gpu(mesh, U0, p, 100, fs, local_time_stepping=True) for p in ("fp64", "mixed")}
    o = oracle.result()["U"]
    _report("config 3 (perturbed), 100 steps vs oracle,", {p: (U, o) for p, U in out.items()})
    assert rel_linf(out["fp64"], o) <= TOL_FP64_100
    assert rel_linf(out["mixed"], o) <= 1e-3


def test_config3_bump_3m_cells_properties():
    """Size-independent properties at the bench size: a second run repeats every bit, and the tuned
    launch shapes change no bit."""
    m, fs, mesh = _bump3m()
    U0 = _perturbed(m, fs, mesh.n_cells)
    a = _gpu(mesh, U0, "fp64", 1, fs, local_time_stepping=True)
    b = _gpu(mesh, U0, "fp64", 1, fs, local_time_stepping=True)
    assert np.array_equal(a, b)
    cfg = S.Config(precision="fp64", CFL=0.8, density_fs=fs[0], velocity_fs=list(fs[1:4]), pressure_fs=fs[4],
                   local_time_stepping=True)
    s = S.EulerSolver(cfg, mesh, U0=U0)
    s.tune()
    s.set_state(U0)
    s.advance(1)
    assert np.array_equal(s.get_solver_data().get_solution(), a)
    s.close()


def test_config4_sweep_cases_against_oracle():
    """Seeded cases of the batched sweep's distribution (Mach in [0.3, 0.8], bump height in
    [0.05, 0.15]) at small resolutions, batched in one mesh, Barth limiter, local time stepping,
    50 steps from the free stream: every case against the oracle run on its own mesh."""
    cases = SW.sample_cases(3, 2024, 24, 40)
    meshes = [SW.case_mesh(c) for c in cases]
    fss = [mg.bump_freestream(c["mach"]) for c in cases]
    batch = S.Mesh.concat(meshes)
    states = [list(fs) for fs, mm in zip(fss, meshes) for _ in mm.patches()]
    U0s = [mg.uniform_state(mm.n_cells, fs) for fs, mm in zip(fss, meshes)]
    n = 50
    oracles = [Background(po.run_oracle, mm.export(), mm.patches(), [fs] * len(mm.patches()), U0, n,
                          local_time_stepping=True, fields=False) for mm, fs, U0 in zip(meshes, fss, U0s)]
    out = {}
    for prec in ("fp64", "mixed"):
        cfg = S.Config(precision=prec, CFL=0.8, local_time_stepping=True, density_fs=fss[0][0],
                       velocity_fs=list(fss[0][1:4]), pressure_fs=fss[0][4])
        s = S.EulerSolver(cfg, batch, U0=np.concatenate(U0s), patch_states=states)
        s.advance(n)
        out[prec] = s.get_solver_data().get_solution()
        s.close()
    off = batch.case_offsets()
    for k, (c, orc) in enumerate(zip(cases, oracles)):
        o = orc.result()["U"]
        pair = {p: (U[off[k]:off[k + 1]], o) for p, U in out.items()}
        _report(f"config 4 case nx={c['nx']} M={c['mach']:.3f} h={c['h']:.3f}, {n} steps vs oracle,", pair)
        assert rel_linf(*pair["fp64"]) <= TOL_FP64_100, c
        assert rel_linf(*pair["mixed"]) <= 1e-4, c
