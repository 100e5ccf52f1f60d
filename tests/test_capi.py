"""The C-ABI library loads and exports every symbol its header declares;
host-side option handling (CPU only, no compute calls)."""
import ctypes as C
import os
import re

import pytest

from helpers import gpu_available
from netflux_b200 import _lib as L
from netflux_b200 import meshgen as mg
from netflux_b200 import solver as S

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "netflux_b200.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(nf_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = L.load()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(L.EXPORTED)


def test_mesh_size_limit_of_one_solver():
    """The largest mesh one solver takes (32-bit offsets into the 20 face-state rows): 107,374,080
    cells; one more is refused with a message, as nf_create refuses it."""
    lib = L.load()
    k_max = (2 ** 31 - 1) // 20 // 64 * 64 - 64
    assert k_max == 107374080
    assert 20 * ((k_max + 63) // 64 * 64) < 2 ** 31
    assert lib.nf_check_mesh_size(k_max, 2 * k_max) == L.NF_OK
    assert lib.nf_check_mesh_size(k_max + 1, 2 * k_max) == L.NF_ERR_MESH
    assert "at most 107374080" in L.last_error(None)
    assert lib.nf_check_mesh_size(1, 0) == L.NF_OK
    assert lib.nf_check_mesh_size(0, 0) == L.NF_ERR_MESH
    assert lib.nf_check_mesh_size(1000, 2 ** 30) == L.NF_ERR_MESH


def test_params_default():
    p = L.NfParams()
    L.load().nf_params_default(C.byref(p))
    assert p.time_scheme == L.NF_TVD_RK3 and p.spatial_order == L.NF_SECOND_ORDER
    assert p.limiter == L.NF_LIMITER_BARTH and p.precision == L.NF_PREC_FP64
    assert p.cfl == 0.8 and tuple(p.freestream) == (1.225, 0.0, 0.0, 0.0, 101325.0)


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU error path")
def test_create_without_gpu_fails_loudly():
    m = S.Mesh.from_tet_mesh(mg.cube_mesh(2))
    cfg = S.Config(time_scheme="TVD_RK3")
    with pytest.raises(L.NetFluxError, match="nf_create"):
        S.EulerSolver(cfg, m)


def test_config_from_input_yml(tmp_path):
    m = mg.sod_mesh(4, 2, 2)
    mg.write_case(str(tmp_path), m, mg.SOD_LEFT, n_timesteps=7, time_scheme="ExplicitEuler", cfl=0.5)
    cfg = S.Config(str(tmp_path))
    assert cfg.get_n_timesteps() == 7 and cfg.get_CFL() == 0.5
    assert cfg.get_time_scheme() == L.NF_EXPLICIT_EULER
    assert cfg.patch_bc == {"left": 2, "right": 2, "sides": 1}
    assert cfg.get_primvars_inf() == mg.SOD_LEFT
    cfg.set_delta_time(0.25)
    assert cfg.get_delta_time() == 0.25


def test_config_errors(tmp_path):
    (tmp_path / "input.yml").write_text("solver: Euler\nn_timesteps: 1\nCFL: 0.5\ntime_scheme: TVD_RK3\n"
                                        "spatial_order: Second\ninviscid_flux_scheme: Rusanov\n"
                                        "initial_cond: Freestream\n")
    with pytest.raises(RuntimeError, match="patches"):
        S.Config(str(tmp_path))
    (tmp_path / "input.yml").write_text("solver: Euler\nn_timesteps: 1\nCFL: 0.5\ntime_scheme: TVD_RK3\n"
                                        "spatial_order: Second\ninviscid_flux_scheme: HLLC\n"
                                        "initial_cond: Freestream\npatches:\n  - a: SlipWall\n")
    with pytest.raises(RuntimeError, match="Rusanov"):
        S.Config(str(tmp_path))
