"""Host mesh builder: bitwise agreement with the reference's face grid and
error behaviour of the SU2 reader (CPU only)."""
import os

import numpy as np
import pytest

from helpers import CASES, golden, mesh, tet_mesh
from netflux_b200 import _lib as L
from netflux_b200 import meshgen as mg
from netflux_b200 import solver as S


@pytest.mark.parametrize("case", CASES)
def test_face_grid_matches_reference_bitwise(case):
    g = golden(case)
    e = mesh(g).export()
    assert np.array_equal(e["face_ij"], g["face_ij"])
    for k in ("S", "ri", "rj", "vol", "centroid", "dS"):
        assert np.array_equal(e[k], g[k]), k


@pytest.mark.parametrize("case", CASES)
def test_patches_match_reference(case):
    g = golden(case)
    pats = mesh(g).patches()
    assert len(pats) == g["patches"].shape[0]
    for p, (t, first, n) in zip(pats, g["patches"]):
        assert (p["type"], p["first_face"], p["n_faces"]) == (t, first, n)


def test_su2_round_trip(tmp_path):
    g = golden("sod40")
    tm = tet_mesh(g)
    mg.write_su2(str(tmp_path / "mesh.su2"), tm)
    bc = {n: mg.BC_CODES[t] for n, t in tm.patch_types.items()}
    a = S.Mesh.from_su2(str(tmp_path / "mesh.su2"), bc).export()
    b = mesh(g).export()
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def test_hilbert_renumbering_is_local():
    m = S.Mesh.from_tet_mesh(mg.cube_mesh(12, seed=3))
    p = m.permutation()
    assert np.array_equal(np.sort(p), np.arange(m.n_cells))
    ij = m.export()["face_ij"].astype(np.int64)
    inner = ij[:, 1] < m.n_cells
    d_sfc = np.abs(p[ij[inner, 0]] - p[ij[inner, 1]])
    rng = np.random.default_rng(0).permutation(m.n_cells)
    d_rand = np.abs(rng[ij[inner, 0]] - rng[ij[inner, 1]])
    assert np.median(d_sfc) * 20 < np.median(d_rand)


def _su2(tmp_path, text):
    p = tmp_path / "mesh.su2"
    p.write_text(text)
    return str(p)


ONE_TET = """NDIME= 3
NELEM= 1
10 0 2 1 3
NPOIN= 4
0.0 0.0 0.0
1.0 0.0 0.0
0.0 1.0 0.0
0.0 0.0 1.0
NMARK= 1
MARKER_TAG= wall
MARKER_ELEMS= 4
5 0 1 2
5 0 1 3
5 0 2 3
5 1 2 3
"""


def test_single_tet_reads(tmp_path):
    m = S.Mesh.from_su2(_su2(tmp_path, ONE_TET), {"wall": L.NF_BC_SLIP_WALL})
    assert (m.n_cells, m.n_faces, m.n_interior_faces) == (1, 4, 0)
    e = m.export()
    assert abs(e["vol"][0] - 1.0 / 6.0) < 1e-16


def test_marker_not_in_patch_list(tmp_path):
    with pytest.raises(L.NetFluxError, match="not named in input file"):
        S.Mesh.from_su2(_su2(tmp_path, ONE_TET), {"other": 1})


def test_marker_triangle_without_tet_face(tmp_path):
    bad = ONE_TET.replace("5 1 2 3\n", "5 1 2 0\n").replace("5 0 1 2\n", "5 0 1 2\n")
    bad = ONE_TET.replace("MARKER_ELEMS= 4", "MARKER_ELEMS= 5") + "5 0 1 2\n"
    with pytest.raises(L.NetFluxError):
        S.Mesh.from_su2(_su2(tmp_path, bad), {"wall": 1})


def test_non_tet_element_rejected(tmp_path):
    hexa = ONE_TET.replace("10 0 2 1 3", "12 0 1 2 3 0 1 2 3")
    with pytest.raises(L.NetFluxError, match="only tetrahedral"):
        S.Mesh.from_su2(_su2(tmp_path, hexa), {"wall": 1})


def test_missing_file_and_bad_header(tmp_path):
    with pytest.raises(L.NetFluxError, match="Couldn't open"):
        S.Mesh.from_su2(str(tmp_path / "nope.su2"), {"wall": 1})
    with pytest.raises(L.NetFluxError, match="NDIME"):
        S.Mesh.from_su2(_su2(tmp_path, ONE_TET.replace("NDIME=", "NDIM=")), {"wall": 1})


def test_uncovered_boundary_faces_are_counted(tmp_path):
    partial = ONE_TET.replace("MARKER_ELEMS= 4", "MARKER_ELEMS= 3").replace("5 1 2 3\n", "")
    m = S.Mesh.from_su2(_su2(tmp_path, partial), {"wall": 1})
    assert m.info.n_uncovered_boundary_faces == 1
    assert m.n_faces == 3


def test_concat_offsets_and_patches():
    a = S.Mesh.from_tet_mesh(mg.cube_mesh(3, seed=1))
    b = S.Mesh.from_tet_mesh(mg.sod_mesh(6, 2, 2))
    c = S.Mesh.concat([a, b])
    assert c.n_cells == a.n_cells + b.n_cells
    assert list(c.case_offsets()) == [0, a.n_cells, a.n_cells + b.n_cells]
    assert [p["case"] for p in c.patches()] == [0] * len(a.patches()) + [1] * len(b.patches())
    assert c.n_faces == a.n_faces + b.n_faces


def test_parallel_build_equals_serial_build(monkeypatch):
    """The builder's threaded sorts and loops (meshes above 65,536 face records) give the mesh the
    one-thread build gives, bit for bit."""
    m = mg.bump_mesh(40, 20, 20, h=0.1)  # 96,000 tets: every parallel path runs
    out = []
    for threads in ("1", "7"):
        monkeypatch.setenv("NETFLUX_B200_HOST_THREADS", threads)
        mm = S.Mesh.from_tet_mesh(m)
        out.append((mm.export(), mm.permutation(), mm.patches()))
    (a, pa, qa), (b, pb, qb) = out
    assert set(a) == set(b)
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(pa, pb) and qa == qb
