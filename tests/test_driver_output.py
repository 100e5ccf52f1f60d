"""The Python Driver's output against NetFlux's own program (CPU): the SU2 reader round-trips the
writer's files, and a Driver run over the oracle (standing in for the GPU solver) writes the same
n=<k>.vtk files, character for character, as the reference program on the same case directory."""
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from netflux_b200 import meshgen as mg
from netflux_b200 import solver as S
from oracle import pyoracle as po

HERE = os.path.dirname(os.path.abspath(__file__))
REF_EXE = os.path.join(HERE, "..", "oracle", "_ref", "netflux")


@pytest.mark.parametrize("kind", ["bump", "sod"])
def test_su2_reader_round_trips(tmp_path, kind):
    m = mg.bump_mesh(6, 3, 3, h=0.1) if kind == "bump" else mg.sod_mesh(10, 2, 2, jitter=0.05, seed=3)
    path = str(tmp_path / "mesh.su2")
    mg.write_su2(path, m)
    r = mg.read_su2(path, m.patch_types)
    assert np.array_equal(r.nodes, m.nodes) and np.array_equal(r.tets, m.tets)
    assert [n for n, _ in r.markers] == [n for n, _ in m.markers]
    assert all(np.array_equal(a, b) for (_, a), (_, b) in zip(r.markers, m.markers))


def test_su2_reader_rejects_other_elements(tmp_path):
    path = str(tmp_path / "bad.su2")
    with open(path, "w") as f:
        f.write("NDIME= 3\nNELEM= 1\n12 0 1 2 3 4 5 6 7\nNPOIN= 0\nNMARK= 0\n")
    with pytest.raises(ValueError):
        mg.read_su2(path, {})


class _OracleSolver:
    """The reference program's trajectory from its free-stream start (solution_old zero), by the
    oracle: the state after k steps is recomputed from the start, so the stale-primitive time step
    of the reference carries over exactly."""

    def __init__(self, mesh, fs):
        self.grid, self.pats, self.fs = mesh.export(), mesh.patches(), fs
        self.U0 = mg.uniform_state(mesh.n_cells, fs)
        self.k = 0

    def calc_timestep(self, cfg):
        cfg.set_delta_time(0.0)

    def step(self, cfg):
        self.k += 1

    def get_solver_data(self):
        return self

    def get_solution(self):
        if self.k == 0:
            return self.U0
        return po.run_oracle(self.grid, self.pats, [self.fs] * len(self.pats), self.U0, self.k,
                             U_old_first=np.zeros_like(self.U0), fields=False)["U"]

    def synchronize(self):
        pass


def test_driver_writes_the_reference_programs_files(tmp_path):
    if not os.access(REF_EXE, os.X_OK):
        pytest.skip("reference program not built (make -C oracle)")
    m, fs = mg.bump_mesh(6, 3, 3, h=0.1), mg.bump_freestream(0.5)
    ref_case, our_case = str(tmp_path / "ref"), str(tmp_path / "ours")
    for c in (ref_case, our_case):
        mg.write_case(c, m, fs, n_timesteps=5, write_stride=2)
    os.makedirs(os.path.join(ref_case, "output"))
    work = tempfile.mkdtemp()
    try:
        r = subprocess.run([REF_EXE, ref_case + "/"], cwd=work, capture_output=True, text=True, timeout=600)
    finally:
        shutil.rmtree(work, ignore_errors=True)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]

    os.makedirs(os.path.join(our_case, "output"))
    open(os.path.join(our_case, "output", "stale.vtk"), "w").close()  # emptied like Output's constructor
    cfg = S.Config(our_case)
    mesh = S.Mesh.from_su2(cfg.get_mesh_filename_path(), cfg.patch_bc)
    d = S.Driver(cfg, write_output=True, solver=_OracleSolver(mesh, fs))
    d.solve()
    assert cfg.get_timestep() == 5
    ours = sorted(os.listdir(os.path.join(our_case, "output")))
    theirs = sorted(os.listdir(os.path.join(ref_case, "output")))
    assert ours == theirs == ["n=0.vtk", "n=2.vtk", "n=4.vtk"]
    for name in ours:
        a = open(os.path.join(our_case, "output", name)).read()
        b = open(os.path.join(ref_case, "output", name)).read()
        assert a == b, name
