"""The device mesh builder (nf_mesh_from_arrays_device) against the host builder: the same grid
bit for bit -- face pairs and order, normals, areas, centroid vectors, volumes, centroids, ghost
centroids, projected areas, patches, the Hilbert permutation -- and the same step on it; the same
error text for invalid input (every check runs before the access it guards)."""
import time

import numpy as np
import pytest

from helpers import CASES, config_for, golden, tet_mesh
from netflux_b200 import _lib as L
from netflux_b200 import meshgen as mg
from netflux_b200 import solver as S

pytestmark = pytest.mark.gpu


def _same_grid(a: S.Mesh, b: S.Mesh):
    ea, eb = a.export(), b.export()
    for k in ea:
        assert np.array_equal(ea[k], eb[k]), k
    assert np.array_equal(a.permutation(), b.permutation())
    assert a.patches() == b.patches()
    for f in ("n_nodes", "n_interior_cells", "n_ghost_cells", "n_interior_faces", "n_total_faces",
              "n_uncovered_boundary_faces", "n_cases"):
        assert getattr(a.info, f) == getattr(b.info, f), f


@pytest.mark.parametrize("case", CASES)
def test_device_builder_matches_host_builder_on_goldens(case):
    g = golden(case)
    m = tet_mesh(g)
    host, dev = S.Mesh.from_tet_mesh(m), S.Mesh.from_tet_mesh(m, device=0)
    _same_grid(host, dev)
    # and the reference's own face grid (the golden fixture written by the compiled reference)
    e = dev.export()
    assert np.array_equal(e["face_ij"], g["face_ij"]) and np.array_equal(e["S"], g["S"])
    # the same step on either grid (the node-based layout comes from the tets and face nodes)
    cfg = config_for(precision="fp64", freestream=tuple(g["freestream"]))
    U = []
    for mesh in (host, dev):
        s = S.EulerSolver(cfg, mesh, U0=g["U0"])
        s.advance(3)
        U.append(s.get_solver_data().get_solution())
        s.close()
    assert np.array_equal(U[0], U[1])


def test_device_builder_at_full_size_and_with_uncovered_faces():
    for m in (mg.cube_mesh(20, jitter=0.1, seed=1234), mg.bump_mesh(128, 64, 64, h=0.1)):
        t0 = time.perf_counter()
        host = S.Mesh.from_tet_mesh(m)
        t1 = time.perf_counter()
        dev = S.Mesh.from_tet_mesh(m, device=0)
        t2 = time.perf_counter()
        print(f"{m.n_cells} tets: host build {t1 - t0:.3f} s, device build {t2 - t1:.3f} s")
        _same_grid(host, dev)
    # a marker listing only part of the boundary: the rest is dropped, as NetFlux drops it
    m = mg.box_tet_mesh(4, 3, 3, jitter=0.1, seed=8)
    name, tris = m.markers[0]
    part = mg.TetMesh(nodes=m.nodes, tets=m.tets, markers=[(name, tris[: len(tris) // 2])],
                      patch_types=m.patch_types)
    host, dev = S.Mesh.from_tet_mesh(part), S.Mesh.from_tet_mesh(part, device=0)
    assert host.info.n_uncovered_boundary_faces > 0
    _same_grid(host, dev)
    # batched meshes from device-built parts
    a = S.Mesh.concat([S.Mesh.from_tet_mesh(mg.bump_mesh(6, 3, 3, h=0.1), device=0),
                       S.Mesh.from_tet_mesh(mg.cube_mesh(3), device=0)])
    b = S.Mesh.concat([S.Mesh.from_tet_mesh(mg.bump_mesh(6, 3, 3, h=0.1)), S.Mesh.from_tet_mesh(mg.cube_mesh(3))])
    _same_grid(a, b)


def _error(m: mg.TetMesh, device) -> str:
    with pytest.raises(L.NetFluxError) as e:
        S.Mesh.from_tet_mesh(m, device=device)
    return str(e.value)


def test_device_builder_reports_the_host_builders_errors():
    m = mg.box_tet_mesh(3, 3, 3, jitter=0.1, seed=9)
    tets = np.asarray(m.tets, np.int64)
    name, tris = m.markers[0]
    tris = np.asarray(tris, np.int64)
    bad = []
    t = tets.copy()
    t[5, 2] = m.nodes.shape[0] + 3  # a missing node
    bad.append(mg.TetMesh(nodes=m.nodes, tets=t, markers=m.markers, patch_types=m.patch_types))
    t = tets.copy()
    t[7, 3] = t[7, 0]  # a degenerate tet
    bad.append(mg.TetMesh(nodes=m.nodes, tets=t, markers=m.markers, patch_types=m.patch_types))
    x = tris.copy()
    x[4] = [tets[13, 0], tets[13, 1], tets[40, 3]]  # a triangle that is no face
    bad.append(mg.TetMesh(nodes=m.nodes, tets=tets, markers=[(name, x)], patch_types=m.patch_types))
    x = np.concatenate([tris, tris[2:3]])  # a face listed twice
    bad.append(mg.TetMesh(nodes=m.nodes, tets=tets, markers=[(name, x)], patch_types=m.patch_types))
    x = tris.copy()
    x[1, 0] = -1  # a marker node that does not exist
    bad.append(mg.TetMesh(nodes=m.nodes, tets=tets, markers=[(name, x)], patch_types=m.patch_types))
    for b in bad:
        host, dev = _error(b, None), _error(b, 0)
        assert host == dev, (host, dev)
