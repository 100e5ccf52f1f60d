"""Parity at the full sizes of the workloads:
  * unit cube, 20^3 hexes x 6 tets (48,000 cells), Gaussian density bump, far field all round,
    TVD-RK3 at CFL 0.8: against the compiled reference (or the oracle where it is not built),
    FP64 <= 1e-12 after 1 step and <= 1e-9 after 100 steps;
  * Sod tube, 400 x 8 x 8 hexes x 6 tets (153,600 cells), slip sides, far-field ends, to t = 0.2:
    FP64 and mixed against the reference-order form, itself pinned to the oracle at this size;
  * the bump channel, 128 x 64 x 64 hexes x 6 tets (3,145,728 cells), by size-independent
    properties (repeatability, launch shapes, mixed against FP64).
Errors are relative L-infinity with the momentum components scaled by max |rho u| (helpers.rel_linf)."""
import os
import tempfile

import numpy as np
import pytest

from helpers import rel_l2, rel_linf
from netflux_b200 import meshgen as mg
from netflux_b200 import solver as S
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

CUBE_FS = (1.0, 0.5, 0.0, 0.0, 1.0 / 1.4)


def _cube():
    m = mg.cube_mesh(20, jitter=0.1, seed=1234)
    return m, mg.cube_initial_state(m)


def _gpu(mesh, U0, precision, n, freestream, **kw):
    cfg = S.Config(precision=precision, CFL=0.8, density_fs=freestream[0], velocity_fs=list(freestream[1:4]),
                   pressure_fs=freestream[4], **kw)
    s = S.EulerSolver(cfg, mesh, U0=U0)
    s.advance(n)
    return s.get_solver_data().get_solution()


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
    errs = {}
    for prec in ("fp64_ref", "fp64", "mixed"):
        errs[prec] = (rel_linf(_gpu(mesh, U0, prec, 1, CUBE_FS), ref1),
                      rel_linf(_gpu(mesh, U0, prec, 100, CUBE_FS), ref100))
    print("config 1 vs", kind, {k: ("%.2e" % a, "%.2e" % b) for k, (a, b) in errs.items()})
    assert errs["fp64_ref"][0] <= 1e-14 and errs["fp64_ref"][1] <= 1e-12
    assert errs["fp64"][0] <= 1e-12 and errs["fp64"][1] <= 1e-9
    assert errs["mixed"][0] <= 1e-5


def test_config2_sod_153k_cells_to_t_0_2():
    """Each far-field end holds its own state (per-patch free stream) with the isentropic ghost density
    (farfield_density_fix; the reference's inverted form is exact only for rho_fs = 1, and with one
    free stream the right end drives a chaotic inflow). About 1,200 steps reach t = 0.2, too long for
    the oracle in a test; the reference-order form is pinned to the oracle over the first 100 steps at
    this size and is the yardstick for the FP64 and mixed forms at t = 0.2."""
    m = mg.sod_mesh(400, 8, 8, jitter=0.05, seed=4321)
    U0 = mg.sod_initial_state(m)
    mesh = S.Mesh.from_tet_mesh(m)
    assert mesh.n_cells == 153600
    pats = mesh.patches()
    states = [mg.SOD_RIGHT if p["name"] == "right" else mg.SOD_LEFT for p in pats]
    o = po.run_oracle(mesh.export(), pats, states, U0, 100, t_end=0.2, fields=False, farfield_density_fix=True)

    def run(prec, n):
        cfg = S.Config(precision=prec, CFL=0.8, t_end=0.2, density_fs=1.0, velocity_fs=[0, 0, 0], pressure_fs=1.0,
                       farfield_density_fix=True)
        s = S.EulerSolver(cfg, mesh, U0=U0, patch_states=states)
        t = s.advance(n)
        return s.get_solver_data().get_solution(), t

    U100, _ = run("fp64_ref", 100)
    pin = rel_linf(U100, o["U"])
    out, times = {}, {}
    for prec in ("fp64_ref", "fp64", "mixed"):
        out[prec], times[prec] = run(prec, 1500)  # steps past t = 0.2 have dt = 0
    assert all(abs(t - 0.2) <= 1e-15 for t in times.values())
    e = {p: (rel_linf(out[p], out["fp64_ref"]), rel_l2(out[p], out["fp64_ref"])) for p in ("fp64", "mixed")}
    print("config 2 Sod: reference order vs oracle after 100 steps %.2e;" % pin, "at t=0.2 vs reference order:",
          {k: ("Linf %.2e" % a, "L2 %.2e" % b) for k, (a, b) in e.items()},
          "rho range", out["fp64"][:, 0].min(), out["fp64"][:, 0].max())
    assert pin <= 1e-13
    assert e["fp64"][0] <= 1e-9
    assert e["mixed"][0] <= 1e-3 and e["mixed"][1] <= 1e-5


def test_config3_bump_3m_cells_properties():
    """The 3,145,728-tet channel (the bench workload), one TVD-RK3 step with local time stepping from
    a smoothly perturbed free stream. It is too large for the oracle, so it is checked by properties
    that do not depend on size: a second run repeats every bit, the tuned launch shapes change no
    bit, and the mixed form stays within its 1e-5 bar of FP64."""
    m = mg.bump_mesh(128, 64, 64, h=0.1)
    fs = mg.bump_freestream(0.5)
    mesh = S.Mesh.from_tet_mesh(m)
    assert mesh.n_cells == 3145728
    c = m.centroids()
    V = np.broadcast_to(np.asarray(fs, np.float64), (mesh.n_cells, 5)).copy()
    bump = 0.02 * np.sin(2 * np.pi * c[:, 0] / 3.0) * np.sin(np.pi * c[:, 1]) * np.sin(np.pi * c[:, 2])
    V[:, 0] *= 1.0 + bump
    V[:, 4] *= 1.0 + 0.5 * bump
    U0 = mg.prim_to_cons(V)
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
    mixed = _gpu(mesh, U0, "mixed", 1, fs, local_time_stepping=True)
    err = rel_linf(mixed, a)
    print("config 3, mixed vs FP64 after 1 step: %.2e; max change of the step %.2e"
          % (err, rel_linf(a, U0)))
    assert err <= 1e-5
    assert rel_linf(a, U0) > 1e-6  # the step did change the state
