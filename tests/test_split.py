"""One mesh as 2 and 3 parts on the GPU (split.SplitSolver over nf_split_*): the halo primitives
written into each receiving part by a kernel that reads the owner's buffer before every stage, the
parts' streams ordered by events, the global dt the minimum over parts reduced on the device. The
owned cells step as the undivided mesh does; without the exchange they do not."""
import time

import numpy as np
import pytest

from helpers import config_for, rel_linf
from netflux_b200 import meshgen as mg
from netflux_b200 import solver as S
from netflux_b200 import split as SP

pytestmark = pytest.mark.gpu


def _case():
    m = mg.bump_mesh(12, 6, 6, h=0.1)
    fs = mg.bump_freestream(0.5)
    c = m.centroids()
    V = np.broadcast_to(np.asarray(fs, np.float64), (m.n_cells, 5)).copy()
    bump = 0.05 * np.sin(2 * np.pi * c[:, 0] / 3.0) * np.sin(np.pi * c[:, 1]) * np.sin(np.pi * c[:, 2])
    V[:, 0] *= 1.0 + bump
    V[:, 4] *= 1.0 + 0.5 * bump
    return m, fs, mg.prim_to_cons(V)


@pytest.mark.parametrize("precision,lts", [("fp64", True), ("fp64", False), ("mixed", True)])
def test_split_mesh_steps_as_the_undivided_mesh(precision, lts):
    m, fs, U0 = _case()
    cfg = config_for(precision=precision, freestream=fs, local_time_stepping=lts)
    whole = S.EulerSolver(cfg, S.Mesh.from_tet_mesh(m), U0=U0)
    whole.advance(6)
    ref = whole.get_solver_data().get_solution()
    whole.close()
    for n_parts in (2, 3):
        sp = SP.SplitSolver(cfg, m, U0, n_parts)
        sp.advance(6)
        U = sp.get_solution()
        sp.close()
        err = rel_linf(U, ref)
        print(precision, "local dt" if lts else "global dt", n_parts, "parts: rel Linf", err,
              "bitwise" if np.array_equal(U, ref) else "")
        assert err <= 1e-13
    sp = SP.SplitSolver(cfg, m, U0, 2, exchange=False)
    sp.advance(6)
    assert rel_linf(sp.get_solution(), ref) > 1e-6
    sp.close()


def test_split_at_size_queues_without_host_waits():
    """A 48x24x24-hex channel (82,944 tets) as 4 parts on one GPU for 30 steps: the owned cells equal
    the undivided mesh's, and the device time per step is printed beside the undivided one's."""
    m = mg.bump_mesh(48, 24, 24, h=0.1)
    fs = mg.bump_freestream(0.5)
    U0 = mg.prim_to_cons(np.broadcast_to(np.asarray(fs, np.float64), (m.n_cells, 5)).copy())
    cfg = config_for(precision="fp64", freestream=fs, local_time_stepping=True)
    whole = S.EulerSolver(cfg, S.Mesh.from_tet_mesh(m), U0=U0)
    whole.advance(2)
    whole.synchronize()
    t0 = time.perf_counter()
    whole.advance(30)
    whole.synchronize()
    t_whole = (time.perf_counter() - t0) / 30
    ref = whole.get_solver_data().get_solution()
    sp = SP.SplitSolver(cfg, m, U0, 4, devices=[0, 0, 0, 0])
    sp.advance(2)
    sp.synchronize()
    t0 = time.perf_counter()
    sp.advance(30)
    sp.synchronize()
    t_split = (time.perf_counter() - t0) / 30
    U = sp.get_solution()
    err = rel_linf(U, ref)
    print(f"82,944 tets: undivided {1e3 * t_whole:.3f} ms/step, 4 parts {1e3 * t_split:.3f} ms/step, "
          f"{sp.n_halo_values // 5} halo cells a stage, rel Linf {err:.3g}")
    sp.close()
    whole.close()
    assert err <= 1e-13


def test_split_refuses_mismatched_parts():
    m = mg.bump_mesh(6, 3, 3, h=0.1)
    fs = mg.bump_freestream(0.5)
    U0 = mg.prim_to_cons(np.broadcast_to(np.asarray(fs, np.float64), (m.n_cells, 5)).copy())
    a = S.EulerSolver(config_for(precision="fp64", freestream=fs), S.Mesh.from_tet_mesh(m), U0=U0)
    b = S.EulerSolver(config_for(precision="mixed", freestream=fs), S.Mesh.from_tet_mesh(m), U0=U0)
    import ctypes as C
    from netflux_b200 import _lib as L
    lib = L.load()
    h = lib.nf_split_create((C.c_void_p * 2)(a._h, b._h), 2)
    assert not h and "differ" in lib.nf_split_last_error(None).decode()
    h = lib.nf_split_create((C.c_void_p * 2)(a._h, a._h), 2)
    assert not h and "twice" in lib.nf_split_last_error(None).decode()
    h = lib.nf_split_create((C.c_void_p * 1)(a._h), 1)
    bad = np.array([0, m.n_cells + 5], np.int64)
    assert lib.nf_split_link(h, 0, 0, L.i64ptr(bad), L.i64ptr(bad), 2) == L.NF_ERR_ARG
    lib.nf_split_destroy(h)
    a.close()
    b.close()


def test_split_of_the_benched_channel_in_two_parts():
    """The 3,145,728-tet bench channel (128x64x64 hexes, Mach 0.5, local time stepping, FP64) as 2
    parts on one GPU for 10 steps: the owned cells equal the undivided mesh's, and the device time
    per step of the split is printed beside the undivided one's (the halo and the per-stage event
    ordering are the difference)."""
    m = mg.bump_mesh(128, 64, 64, h=0.1)
    fs = mg.bump_freestream(0.5)
    U0 = mg.prim_to_cons(np.broadcast_to(np.asarray(fs, np.float64), (m.n_cells, 5)).copy())
    cfg = config_for(precision="fp64", freestream=fs, local_time_stepping=True)
    whole = S.EulerSolver(cfg, S.Mesh.from_tet_mesh(m), U0=U0)
    whole.advance(2)
    t0 = time.perf_counter()
    whole.advance(10)
    t_whole = (time.perf_counter() - t0) / 10
    ref = whole.get_solver_data().get_solution()
    whole.close()
    sp = SP.SplitSolver(cfg, m, U0, 2, devices=[0, 0])
    sp.advance(2)
    sp.synchronize()
    t0 = time.perf_counter()
    sp.advance(10)
    sp.synchronize()
    t_split = (time.perf_counter() - t0) / 10
    U = sp.get_solution()
    n_cells = sum(len(p["cells"]) for p in sp.parts)
    sp.close()
    err = rel_linf(U, ref)
    print(f"3,145,728 tets: undivided {1e3 * t_whole:.3f} ms/step, 2 parts {1e3 * t_split:.3f} ms/step "
          f"({n_cells:,} cells with the halo), rel Linf {err:.3g}")
    assert err <= 1e-13
