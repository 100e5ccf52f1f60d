"""The NF_DEBUG build (make -C netflux_b200/csrc debug, loaded with NETFLUX_B200_DEBUG=1): its kernels
check every mesh index they read (an index out of range is reported as NF_ERR_MESH and redirected
in bounds). On valid meshes it reports nothing and computes the release build's bits, in every
arithmetic form. The debug library runs in a child process (one library per process)."""
import os
import subprocess
import sys

import numpy as np
import pytest

from helpers import config_for, golden, mesh
from netflux_b200 import solver as S

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, {root!r}); sys.path.insert(0, {tests!r})
from helpers import config_for, golden, mesh
from netflux_b200 import _lib as L, solver as S
assert L.LIB_PATH.endswith("libnetflux_b200_debug.so"), L.LIB_PATH
out = {{}}
for case in ("bump12", "wallbox5"):
    g = golden(case)
    for prec in ("fp64_ref", "fp64", "mixed"):
        for lts in (False, True):
            cfg = config_for(precision=prec, freestream=tuple(g["freestream"]), local_time_stepping=lts)
            s = S.EulerSolver(cfg, mesh(g), U0=g["U0"])
            s.advance(4)
            s.synchronize()
            np.save({tmp!r} + "/%s_%s_%d.npy" % (case, prec, lts), s.get_solver_data().get_solution())
            s.close()
print("debug ok")
"""


def test_debug_build_reports_nothing_and_matches_release(tmp_path):
    lib = os.path.join(ROOT, "netflux_b200", "lib", "libnetflux_b200_debug.so")
    if not os.path.exists(lib):
        pytest.fail("NF_DEBUG library not built (make -C netflux_b200/csrc debug)")
    code = CHILD.format(root=ROOT, tests=os.path.join(ROOT, "tests"), tmp=str(tmp_path))
    r = subprocess.run([sys.executable, "-c", code], env=dict(os.environ, NETFLUX_B200_DEBUG="1"),
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "debug ok" in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]
    for case in ("bump12", "wallbox5"):
        g = golden(case)
        for prec in ("fp64_ref", "fp64", "mixed"):
            for lts in (False, True):
                cfg = config_for(precision=prec, freestream=tuple(g["freestream"]), local_time_stepping=lts)
                s = S.EulerSolver(cfg, mesh(g), U0=g["U0"])
                s.advance(4)
                U = s.get_solver_data().get_solution()
                s.close()
                assert np.array_equal(U, np.load(tmp_path / ("%s_%s_%d.npy" % (case, prec, lts)))), (case, prec, lts)
