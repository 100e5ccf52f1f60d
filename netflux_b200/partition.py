"""Decomposition of one tetrahedral mesh across ranks (host side).

The cells are split into contiguous ranges of a space-filling-curve order
(the library's Hilbert renumbering, ``Mesh.permutation()``), so each part is
compact and its surface small. Each part is extended by ``layers`` layers of
neighbouring cells (its halo). Its local mesh lists the owned cells, then the
halo cells layer by layer, each group in global order, with the boundary
markers of those cells; the faces where the halo is cut off are left
unlisted, which NetFlux drops (FV_Grid.cpp:79-85), or listed under a marker
of their own (``cut_marker``, a far field by default). They touch only the
outermost halo layer, whose results are never used; as a far field they keep
those cells' throwaway updates physical (with the ghost at the free stream, a
uniform flow crosses them undisturbed), so a solver's validity checks stay
quiet there.

Why two layers per stage: the flux balance of an owned cell reads its
neighbours' face states, which need the neighbours' gradients and limiters,
which need the neighbours' neighbours. So with the halo primitives exchanged
before every stage, 2 layers make the stage exact for the owned cells; with
2·s layers, s stages run between exchanges (6 layers: one exchange per
TVD-RK3 step), trading redundant halo work for fewer exchanges.

``exchange_plan`` lists, for every ordered pair of parts, which owned cells of
one part fill which halo cells of the other. The same lists drive an
exchange over gloo on the CPU and over NCCL between GPUs.
"""
from typing import Dict, List, Optional

import numpy as np

from .meshgen import FAR_FIELD, TetMesh

# the face opposite vertex q of a tetrahedron: the other three vertices
_FACE_VERTS = np.array([[1, 2, 3], [0, 2, 3], [0, 1, 3], [0, 1, 2]])


def _face_keys(tets: np.ndarray) -> np.ndarray:
    """Sorted vertex triples of every tet face, [n_cells * 4][3] (cell-major)."""
    f = np.sort(tets[:, _FACE_VERTS], axis=2)
    return f.reshape(-1, 3)


def cell_neighbours(tets: np.ndarray) -> np.ndarray:
    """[n_cells][4]: the cell across the face opposite vertex q, or -1 on the boundary."""
    tets = np.asarray(tets, dtype=np.int64)
    n = tets.shape[0]
    keys = _face_keys(tets)
    order = np.lexsort((keys[:, 2], keys[:, 1], keys[:, 0]))
    k = keys[order]
    same = np.all(k[1:] == k[:-1], axis=1)
    nb = np.full(4 * n, -1, np.int64)
    i = np.nonzero(same)[0]
    a, b = order[i], order[i + 1]
    nb[a] = b // 4
    nb[b] = a // 4
    return nb.reshape(n, 4)


def partition(mesh: TetMesh, sfc_rank: np.ndarray, n_parts: int, layers: int = 2,
              cut_marker: Optional[str] = None, cut_type: str = FAR_FIELD) -> List[Dict[str, np.ndarray]]:
    """Split the cells into ``n_parts`` contiguous ranges of ``sfc_rank`` (each cell's position along
    the curve) and add ``layers`` halo layers to each. Every part holds ``cells`` (global ids, owned
    first, then the halo by layer), ``n_owned``, ``layer`` (0 for owned cells, else the halo layer)
    and ``mesh`` (its local TetMesh, cells in the order of ``cells``). With ``cut_marker``, each
    part mesh lists the faces where its halo is cut off under a marker of that name and boundary
    type ``cut_type``."""
    n = mesh.n_cells
    if not 1 <= n_parts <= max(n, 1):
        raise ValueError("n_parts must be between 1 and the number of cells")
    if layers < 0:
        raise ValueError("layers must be >= 0")
    nb = cell_neighbours(mesh.tets)
    by_curve = np.argsort(np.asarray(sfc_rank), kind="stable")
    owner = np.empty(n, np.int64)
    bounds = np.linspace(0, n, n_parts + 1).round().astype(np.int64)
    for p in range(n_parts):
        owner[by_curve[bounds[p]:bounds[p + 1]]] = p
    parts = []
    for p in range(n_parts):
        level = np.full(n, -1, np.int64)
        owned = np.nonzero(owner == p)[0]
        level[owned] = 0
        front = owned
        groups = [owned]
        for lay in range(1, layers + 1):
            cand = nb[front].ravel()
            cand = np.unique(cand[cand >= 0])
            new = cand[level[cand] < 0]
            level[new] = lay
            groups.append(new)
            front = new
        cells = np.concatenate(groups)
        extra = None
        if cut_marker is not None:
            # faces of the part's cells whose neighbour cell is outside the part
            nbc = nb[cells]
            ci, q = np.nonzero((nbc >= 0) & (level[np.maximum(nbc, 0)] < 0))
            tets = np.asarray(mesh.tets, dtype=np.int64)
            extra = [(cut_marker, tets[cells[ci][:, None], _FACE_VERTS[q]], cut_type)]
        parts.append({"cells": cells, "n_owned": int(owned.size), "layer": level[cells],
                      "owner": owner[cells], "mesh": sub_mesh(mesh, cells, extra)})
    return parts


def sub_mesh(mesh: TetMesh, cells: np.ndarray, extra_markers=None) -> TetMesh:
    """The TetMesh of the given cells (in that order): the nodes they use, renumbered in ascending
    global order, and each marker's triangles that are faces of these cells; ``extra_markers``
    ((name, triangles in global node ids, boundary type) triples) are appended."""
    cells = np.asarray(cells, dtype=np.int64)
    tets = np.asarray(mesh.tets, dtype=np.int64)[cells]
    used = np.unique(tets)
    new_id = np.full(mesh.nodes.shape[0], -1, np.int64)
    new_id[used] = np.arange(used.size)
    faces = _face_keys(tets)
    order = np.lexsort((faces[:, 2], faces[:, 1], faces[:, 0]))
    fk = faces[order]
    markers = []
    for name, tris in mesh.markers:
        tris = np.asarray(tris, dtype=np.int64)
        if tris.shape[0] == 0:
            markers.append((name, tris.reshape(0, 3)))
            continue
        tk = np.sort(tris, axis=1)
        # a triangle is kept when its sorted triple is a face of one of the cells
        pos = _search_rows(fk, tk)
        keep = pos >= 0
        markers.append((name, new_id[tris[keep]]))
    patch_types = dict(mesh.patch_types)
    for name, tris, btype in extra_markers or []:
        markers.append((name, new_id[np.asarray(tris, dtype=np.int64).reshape(-1, 3)]))
        patch_types[name] = btype
    return TetMesh(nodes=np.asarray(mesh.nodes)[used], tets=new_id[tets], markers=markers,
                   patch_types=patch_types)


def _search_rows(sorted_rows: np.ndarray, rows: np.ndarray) -> np.ndarray:
    """Index of each row of ``rows`` in the lexicographically sorted ``sorted_rows`` (its first
    occurrence), or -1. Rows are merged and compared column by column, never packed into one
    integer key, so any int64 values work (node ids of meshes of any size)."""
    sorted_rows = np.asarray(sorted_rows, dtype=np.int64)
    rows = np.asarray(rows, dtype=np.int64)
    n, m = sorted_rows.shape[0], rows.shape[0]
    res = np.full(m, -1, np.int64)
    if n == 0 or m == 0:
        return res
    allr = np.concatenate([sorted_rows, rows])
    tag = np.concatenate([np.zeros(n, np.int64), np.ones(m, np.int64)])
    # stable: within a run of equal rows the sorted rows come first, in their own order
    order = np.lexsort((tag,) + tuple(allr[:, k] for k in range(allr.shape[1] - 1, -1, -1)))
    r = allr[order]
    starts = np.ones(n + m, bool)
    starts[1:] = np.any(r[1:] != r[:-1], axis=1)
    first = order[np.maximum.accumulate(np.where(starts, np.arange(n + m), 0))]  # first row of each run
    hit = (order >= n) & (first < n)
    res[order[hit] - n] = first[hit]
    return res


def exchange_plan(parts: List[Dict[str, np.ndarray]]) -> Dict[int, Dict[int, Dict[str, np.ndarray]]]:
    """plan[p][q] = {"send": local indices of p's owned cells that q needs, "recv": local indices of
    q's halo cells they fill}, both in the same order. Only pairs that exchange something appear."""
    local_of = []
    for part in parts:
        m = {}
        owned = part["cells"][:part["n_owned"]]
        m.update(zip(owned.tolist(), range(owned.size)))
        local_of.append(m)
    plan: Dict[int, Dict[int, Dict[str, np.ndarray]]] = {p: {} for p in range(len(parts))}
    for q, part in enumerate(parts):
        halo = np.arange(part["n_owned"], part["cells"].size)
        if halo.size == 0:
            continue
        owners = part["owner"][halo]
        for p in np.unique(owners).tolist():
            h = halo[owners == p]
            send = np.array([local_of[p][g] for g in part["cells"][h].tolist()], np.int64)
            plan[p][q] = {"send": send, "recv": h.astype(np.int64)}
    return plan


def exchange(plan, fields: List[np.ndarray]) -> None:
    """Apply the plan in place on per-part arrays (one process holding every part)."""
    for p, dests in plan.items():
        for q, lists in dests.items():
            fields[q][lists["recv"]] = fields[p][lists["send"]]
