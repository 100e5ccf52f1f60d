"""The drop-in: NetFlux's own program (Driver, Output, grid reader, config parser, compiled from the
reference sources) relinked with netflux_b200/dropin/Solver.cpp in place of src/Solver.cpp, so that
calc_timestep and step run on the GPU. Its VTK output must match the unmodified reference program's
on the same case (the files print 6 significant digits)."""
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from netflux_b200 import meshgen as mg

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(HERE, "..", "oracle", "_ref")


def _vtk_cell_data(path):
    """density, velocity (3) and pressure per cell from a NetFlux VTK file."""
    lines = open(path).read().split("\n")
    i = next(k for k, l in enumerate(lines) if l.startswith("CELL_DATA"))
    n = int(lines[i].split()[1])
    out = {}
    k = i + 1
    while k < len(lines):
        l = lines[k]
        if l.startswith("SCALARS"):
            name = l.split()[1]
            out[name] = np.array([float(x) for x in lines[k + 2:k + 2 + n]])
            k += 2 + n
        elif l.startswith("VECTORS"):
            name = l.split()[1]
            out[name] = np.array([[float(x) for x in r.split()] for r in lines[k + 1:k + 1 + n]])
            k += 1 + n
        else:
            k += 1
    return out


def _run(exe, case, env=None):
    work = tempfile.mkdtemp()
    try:  # the reference appends its stage dump to ./debug_log.txt
        r = subprocess.run([exe, case + "/"], cwd=work, capture_output=True, text=True, timeout=600, env=env)
    finally:
        shutil.rmtree(work, ignore_errors=True)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r


@pytest.mark.parametrize("precision", ["fp64", "fp64_ref"])
def test_dropin_program_matches_reference_program(precision):
    ref_exe, dropin_exe = os.path.join(REF, "netflux"), os.path.join(REF, "netflux_dropin")
    if not (os.access(ref_exe, os.X_OK) and os.access(dropin_exe, os.X_OK)):
        pytest.skip("reference program or drop-in not built (make -C oracle)")
    m = mg.bump_mesh(12, 6, 6, h=0.1)
    fs = mg.bump_freestream(0.5)
    n = 20
    with tempfile.TemporaryDirectory() as d:
        cases = {}
        for name in ("ref", "dropin"):
            c = os.path.join(d, name)
            mg.write_case(c, m, fs, n_timesteps=n, write_stride=10)
            os.makedirs(os.path.join(c, "output"), exist_ok=True)
            cases[name] = c
        _run(ref_exe, cases["ref"])
        env = dict(os.environ, NETFLUX_B200_PRECISION=precision)
        _run(dropin_exe, cases["dropin"], env)
        for k in (0, 10, 20):
            a = _vtk_cell_data(os.path.join(cases["ref"], "output", f"n={k}.vtk"))
            b = _vtk_cell_data(os.path.join(cases["dropin"], "output", f"n={k}.vtk"))
            assert set(a) == set(b) and len(a) >= 3
            for f in a:
                scale = np.max(np.abs(a[f]))
                err = np.max(np.abs(a[f] - b[f])) / scale
                assert err <= 2e-6, (k, f, err)
