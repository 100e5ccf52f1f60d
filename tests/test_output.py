"""The VTK writer against NetFlux's own program (CPU): for the state the oracle computes, the file
output.write_vtk_ascii writes equals, character for character, the file the reference program
writes at the same time step."""
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from netflux_b200 import meshgen as mg
from netflux_b200 import output as O
from netflux_b200 import solver as S
from oracle import pyoracle as po

HERE = os.path.dirname(os.path.abspath(__file__))
REF_EXE = os.path.join(HERE, "..", "oracle", "_ref", "netflux")


def _run_reference_program(case):
    work = tempfile.mkdtemp()
    try:
        r = subprocess.run([REF_EXE, case + "/"], cwd=work, capture_output=True, text=True, timeout=600)
    finally:
        shutil.rmtree(work, ignore_errors=True)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]


@pytest.mark.parametrize("kind", ["bump", "sod"])
def test_vtk_text_equals_reference_program(tmp_path, kind):
    if not os.access(REF_EXE, os.X_OK):
        pytest.skip("reference program not built (make -C oracle)")
    if kind == "bump":
        m, fs = mg.bump_mesh(6, 3, 3, h=0.1), mg.bump_freestream(0.5)
    else:  # jittered nodes: coordinates with all their digits
        m, fs = mg.sod_mesh(12, 2, 2, jitter=0.05, seed=5), mg.SOD_LEFT
    n, stride = 4, 2
    case = str(tmp_path / "case")
    mg.write_case(case, m, fs, n_timesteps=n, write_stride=stride)  # the program's free-stream start
    os.makedirs(os.path.join(case, "output"), exist_ok=True)
    _run_reference_program(case)
    mm = S.Mesh.from_tet_mesh(m)
    pats = mm.patches()
    U0 = mg.uniform_state(mm.n_cells, fs)
    for k in range(0, n + 1, stride):
        # the program's free-stream start leaves solution_old zero for the first step
        U = U0 if k == 0 else po.run_oracle(mm.export(), pats, [fs] * len(pats), U0, k,
                                            U_old_first=np.zeros_like(U0), fields=False)["U"]
        mine = str(tmp_path / f"mine{k}.vtk")
        O.write_vtk_ascii(mine, m.nodes, m.reader_tets(), U)
        ref = O.vtk_filename(os.path.join(case, "output") + "/", k)
        assert open(mine).read() == open(ref).read(), k


def test_vtk_rejects_wrong_state_shape(tmp_path):
    m = mg.bump_mesh(2, 1, 1, h=0.1)
    with pytest.raises(ValueError):
        O.write_vtk_ascii(str(tmp_path / "x.vtk"), m.nodes, m.reader_tets(), np.zeros((m.n_cells + 1, 5)))


def test_restart_file_round_trips(tmp_path):
    rng = np.random.default_rng(1)
    U = rng.random((37, 5))
    path = str(tmp_path / "r.npz")
    O.save_restart(path, U, timestep=12, time=0.25)
    r = O.load_restart(path)
    assert np.array_equal(r["U"], U) and r["timestep"] == 12 and r["time"] == 0.25
    with pytest.raises(ValueError):
        O.save_restart(path, U[:, :4], 0)


def test_restart_file_records_and_checks_its_mesh(tmp_path):
    from netflux_b200 import solver as S
    a = S.Mesh.from_tet_mesh(mg.bump_mesh(4, 2, 2, h=0.1))
    b = S.Mesh.from_tet_mesh(mg.bump_mesh(4, 2, 2, h=0.05))  # same size, other geometry
    U = np.random.default_rng(2).random((a.n_cells, 5))
    path = str(tmp_path / "r.npz")
    O.save_restart(path, U, timestep=3, time=0.5, mesh=a)
    r = O.load_restart(path, mesh=a)
    assert np.array_equal(r["U"], U) and r["mesh_sha256"] == O.mesh_fingerprint(a)
    assert r["case_offsets"].tolist() == [0, a.n_cells]
    with pytest.raises(ValueError, match="different mesh"):
        O.load_restart(path, mesh=b)
    c = S.Mesh.from_tet_mesh(mg.bump_mesh(6, 2, 2, h=0.1))
    with pytest.raises(ValueError, match="size"):
        O.load_restart(path, mesh=c)
    with pytest.raises(ValueError):
        O.save_restart(path, U[:-1], 0, mesh=a)
