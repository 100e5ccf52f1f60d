"""One mesh as 2 and 3 parts on the GPU (split.SplitSolver): the halo primitives exchanged through
device buffers before every stage, the global dt the minimum over parts. The owned cells step as
the undivided mesh does; without the exchange they do not."""
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


class _NoExchange(SP.SplitSolver):
    def exchange(self):
        pass


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
    sp = _NoExchange(cfg, m, U0, 2)
    sp.advance(6)
    assert rel_linf(sp.get_solution(), ref) > 1e-6
    sp.close()
