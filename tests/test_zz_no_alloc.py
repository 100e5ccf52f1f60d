"""The allocation-free residual-norm entry point against the solver's own.

nf_residual_norms_noalloc exists for callers that cannot allocate device
memory when they need the reduction (under a fixed memory pool, in real-time
loops that must not block on the allocator); its partial sums live in a fixed array
inside the library. This file is collected last so a failure here cannot hide
any other test, and it passes both on its own and after the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import config_for
from netflux_b200 import _lib as L
from netflux_b200 import meshgen as mg
from netflux_b200 import solver as S

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # the FP64 tolerance of the parity tests


def _call(values_dev, out_dev, stream):
    lib = L.load()
    return lib.nf_residual_norms_noalloc(C.c_void_p(values_dev.data_ptr()), values_dev.numel(),
                                         C.c_void_p(out_dev.data_ptr()), C.c_void_p(stream))


def test_residual_norms_noalloc_matches_solver_twice():
    import torch

    # 48k cells: several 16384-value blocks, so the fixed partials array is used
    m = mg.cube_mesh(20, jitter=0.1, seed=1234)
    fs = (1.0, 0.5, 0.0, 0.0, 1.0 / 1.4)
    mesh = S.Mesh.from_tet_mesh(m)
    vol = mesh.export()["vol"][: mesh.n_cells]
    cfg = config_for(time_scheme="ExplicitEuler", precision="fp64", freestream=fs)
    s = S.EulerSolver(cfg, mesh, U0=mg.cube_initial_state(m), keep_stage_fields=True)
    stream = torch.cuda.current_stream().cuda_stream
    out = torch.full((2,), -1.0, dtype=torch.float64, device="cuda")
    for call in range(2):  # two calls in a row; the second reuses the scratch
        s.calc_timestep(cfg)
        s.step(cfg)
        expected = s.residual()[0]  # existing entry point (nf_get_residual)
        R = s.get_solver_data().get_flux_balance()
        r = torch.tensor(R[:, 0] / vol, dtype=torch.float64, device="cuda")
        assert _call(r, out, stream) == L.NF_OK, L.last_error(None)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.allclose(got, expected, rtol=RTOL, atol=0.0), (call, got, expected)
    s.close()


def test_residual_norms_noalloc_rejects_oversize_and_handles_empty():
    import torch

    stream = torch.cuda.current_stream().cuda_stream
    out = torch.full((2,), -1.0, dtype=torch.float64, device="cuda")
    lib = L.load()
    rc = lib.nf_residual_norms_noalloc(C.c_void_p(out.data_ptr()), 134217729, C.c_void_p(out.data_ptr()),
                                       C.c_void_p(stream))
    assert rc == L.NF_ERR_ARG
    assert "capacity" in L.last_error(None)
    empty = torch.empty(0, dtype=torch.float64, device="cuda")
    assert _call(empty, out, stream) == L.NF_OK
    torch.cuda.synchronize()
    assert out.cpu().numpy().tolist() == [0.0, 0.0]


def test_residual_norms_noalloc_keeps_nan():
    """A NaN anywhere in the values shows in both norms (a non-finite residual must not vanish from
    the max norm), in the first block and in a later one."""
    import torch

    stream = torch.cuda.current_stream().cuda_stream
    out = torch.full((2,), -1.0, dtype=torch.float64, device="cuda")
    for pos in (5, 40000):
        v = torch.linspace(-1.0, 1.0, 50000, dtype=torch.float64, device="cuda")
        v[pos] = float("nan")
        assert _call(v, out, stream) == L.NF_OK, L.last_error(None)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.isnan(got[0]) and np.isnan(got[1]), (pos, got)
