"""Decomposition of one mesh across ranks (netflux_b200/partition.py), checked on the CPU with the
oracle standing in for each rank's solver: with the halo exchanged as planned, the owned cells of
every part evolve as the same cells of the undivided mesh (to round-off: each part sums its faces in
its own order). Two halo layers carry one stage between exchanges (explicit Euler steps, or TVD-RK3
stages through the oracle's stage entry points), six carry a TVD-RK3 step."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from netflux_b200 import meshgen as mg
from netflux_b200 import partition as P
from netflux_b200 import solver as S
from oracle import pyoracle as po

RUN = dict(local_time_stepping=True, dt_from_current_state=True, fields=False)


def _case():
    m = mg.bump_mesh(8, 4, 4, h=0.1)
    fs = mg.bump_freestream(0.5)
    mm = S.Mesh.from_tet_mesh(m)
    U0 = mg.uniform_state(mm.n_cells, fs)
    # a non-uniform start so that gradients and limiters are exercised from the first stage
    rng = np.random.default_rng(2)
    U0 = U0 * (1.0 + 0.02 * rng.standard_normal(U0.shape))
    return m, fs, mm, U0


def _global(mm, fs, U0, n_steps, time_scheme):
    pats = mm.patches()
    return po.run_oracle(mm.export(), pats, [fs] * len(pats), U0, n_steps, time_scheme=time_scheme, **RUN)["U"]


def _rel_linf(a, b):
    return float(np.max(np.abs(a - b) / np.max(np.abs(b), axis=0)))


def test_neighbours_and_halo_layers():
    m, _, mm, _ = _case()
    nb = P.cell_neighbours(m.tets)
    n_interior = int((nb >= 0).sum()) // 2
    assert n_interior + m.n_boundary_faces == mm.export()["face_ij"].shape[0]
    rows, cols = np.nonzero(nb >= 0)
    assert np.all(nb[nb[rows, cols]] .max(axis=1) >= 0)  # every neighbour has neighbours back
    assert all(rows[i] in nb[nb[rows[i], cols[i]]] for i in range(0, rows.size, 17))
    parts = P.partition(m, mm.permutation(), 3, layers=2)
    owned = np.concatenate([p["cells"][:p["n_owned"]] for p in parts])
    assert np.array_equal(np.sort(owned), np.arange(m.n_cells))
    for p in parts:
        level = {c: l for c, l in zip(p["cells"].tolist(), p["layer"].tolist())}
        for c, l in level.items():
            if l < 2:  # every neighbour of an owned or first-layer cell is in the part
                assert all(n < 0 or n in level for n in nb[c])
        assert np.all(np.diff(p["layer"]) >= 0)


@pytest.mark.parametrize("time_scheme,layers,steps_between", [(0, 2, 1), (0, 6, 3), (1, 6, 1)])
def test_parts_with_exchange_match_the_undivided_mesh(time_scheme, layers, steps_between):
    m, fs, mm, U0 = _case()
    n_steps = 6 if time_scheme == 0 else 3
    ref = _global(mm, fs, U0, n_steps, time_scheme)
    parts = P.partition(m, mm.permutation(), 3, layers=layers)
    plan = P.exchange_plan(parts)
    meshes = [S.Mesh.from_tet_mesh(p["mesh"]) for p in parts]
    U = [U0[p["cells"]].copy() for p in parts]
    done = 0
    while done < n_steps:
        k = min(steps_between, n_steps - done)
        for i, mesh in enumerate(meshes):
            pats = mesh.patches()
            U[i] = po.run_oracle(mesh.export(), pats, [fs] * len(pats), U[i], k, time_scheme=time_scheme,
                                 **RUN)["U"]
        P.exchange(plan, U)
        done += k
    out = np.empty_like(U0)
    for p, u in zip(parts, U):
        out[p["cells"][:p["n_owned"]]] = u[:p["n_owned"]]
    assert _rel_linf(out, ref) <= 1e-12


@pytest.mark.parametrize("global_dt", [False, True])
@pytest.mark.parametrize("cut_marker", [None, "halo_cut"])
def test_rk3_with_two_layers_and_an_exchange_per_stage(global_dt, cut_marker):
    """The production plan: 2 halo layers, the halo states exchanged after every TVD-RK3 stage, and
    with a global time step the minimum taken over the owned cells of all parts (an all-reduce).
    The cut faces dropped or listed as a far field: the owned cells step the same either way."""
    m, fs, mm, U0 = _case()
    pats = mm.patches()
    ref = po.run_oracle(mm.export(), pats, [fs] * len(pats), U0, 3, time_scheme=1,
                        local_time_stepping=not global_dt, dt_from_current_state=True, fields=False)["U"]
    parts = P.partition(m, mm.permutation(), 3, layers=2, cut_marker=cut_marker)
    plan = P.exchange_plan(parts)
    so = []
    for p in parts:
        mesh = S.Mesh.from_tet_mesh(p["mesh"])
        pp = mesh.patches()
        so.append(po.StageOracle(mesh.export(), pp, [fs] * len(pp), time_scheme=1, local_time_stepping=True))
    U = [U0[p["cells"]].copy() for p in parts]
    for _ in range(3):
        dts = [o.timestep(u) for o, u in zip(so, U)]
        dt_g = min(float(np.min(dtl[:p["n_owned"]])) for (_, dtl), p in zip(dts, parts))
        Un = [u.copy() for u in U]
        for stage in range(3):
            U = [o.stage(u, un, stage, dt_g, None) if global_dt else o.stage(u, un, stage, 0.0, dtl)
                 for o, u, un, (_, dtl) in zip(so, U, Un, dts)]
            P.exchange(plan, U)
    out = np.empty_like(U0)
    for p, u in zip(parts, U):
        out[p["cells"][:p["n_owned"]]] = u[:p["n_owned"]]
    assert _rel_linf(out, ref) <= 1e-12


def test_cut_marker_lists_exactly_the_cut_faces():
    """With cut_marker every face between a part's cells and the rest of the mesh is listed under
    that marker (a far field by default), once, and every such face belongs to an outermost-layer
    cell."""
    m = mg.bump_mesh(8, 4, 4, h=0.1)
    nb = P.cell_neighbours(m.tets)
    for layers in (1, 2):
        for p in P.partition(m, np.arange(m.n_cells), 3, layers=layers, cut_marker="cut",
                             cut_type=mg.SLIP_WALL if layers == 1 else mg.FAR_FIELD):
            pm = p["mesh"]
            assert pm.patch_types["cut"] == (mg.SLIP_WALL if layers == 1 else mg.FAR_FIELD)
            inside = np.zeros(m.n_cells, bool)
            inside[p["cells"]] = True
            nbc = nb[p["cells"]]
            ci, q = np.nonzero((nbc >= 0) & ~inside[np.maximum(nbc, 0)])
            assert np.all(p["layer"][ci] == layers)
            cut = np.sort(dict(pm.markers)["cut"], axis=1)
            local = np.sort(np.asarray(pm.tets)[ci[:, None], P._FACE_VERTS[q]], axis=1)
            assert cut.shape == local.shape
            assert np.array_equal(cut[np.lexsort(cut.T[::-1])], local[np.lexsort(local.T[::-1])])


def test_too_few_layers_is_not_exact():
    """The check has teeth: one layer per stage leaves the owned cells at the part edges wrong."""
    m, fs, mm, U0 = _case()
    ref = _global(mm, fs, U0, 2, 0)
    parts = P.partition(m, mm.permutation(), 3, layers=1)
    plan = P.exchange_plan(parts)
    U = [U0[p["cells"]].copy() for p in parts]
    for _ in range(2):
        for i, p in enumerate(parts):
            mesh = S.Mesh.from_tet_mesh(p["mesh"])
            pats = mesh.patches()
            U[i] = po.run_oracle(mesh.export(), pats, [fs] * len(pats), U[i], 1, time_scheme=0, **RUN)["U"]
        P.exchange(plan, U)
    out = np.empty_like(U0)
    for p, u in zip(parts, U):
        out[p["cells"][:p["n_owned"]]] = u[:p["n_owned"]]
    assert _rel_linf(out, ref) > 1e-8


def _rank(rank, world, port, out):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        m, fs, mm, U0 = _case()
        parts = P.partition(m, mm.permutation(), world, layers=2)
        plan = P.exchange_plan(parts)
        me = parts[rank]
        mesh = S.Mesh.from_tet_mesh(me["mesh"])
        pats = mesh.patches()
        U = U0[me["cells"]].copy()
        for _ in range(4):
            U = po.run_oracle(mesh.export(), pats, [fs] * len(pats), U, 1, time_scheme=0, **RUN)["U"]
            reqs, bufs = [], []
            for q, lists in plan[rank].items():
                reqs.append(dist.isend(torch.from_numpy(np.ascontiguousarray(U[lists["send"]])), q))
            for p in range(world):
                if rank in plan[p]:
                    buf = torch.empty((plan[p][rank]["recv"].size, 5), dtype=torch.float64)
                    reqs.append(dist.irecv(buf, p))
                    bufs.append((plan[p][rank]["recv"], buf))
            for r in reqs:
                r.wait()
            for idx, buf in bufs:
                U[idx] = buf.numpy()
        gathered = [None] * world
        dist.all_gather_object(gathered, (me["cells"][:me["n_owned"]], U[:me["n_owned"]]))
        if rank == 0:
            full = np.empty_like(U0)
            for cells, u in gathered:
                full[cells] = u
            out["err"] = _rel_linf(full, _global(mm, fs, U0, 4, 0))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_exchange_halos():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
    assert out["err"] <= 1e-12


def test_partition_edge_cases():
    m, _, mm, _ = _case()
    one = P.partition(m, mm.permutation(), 1, layers=2)
    assert one[0]["n_owned"] == m.n_cells and one[0]["cells"].size == m.n_cells  # no halo
    assert P.exchange_plan(one) == {0: {}}
    bare = P.partition(m, mm.permutation(), 4, layers=0)
    assert all(p["cells"].size == p["n_owned"] for p in bare)
    assert sum(p["n_owned"] for p in bare) == m.n_cells
    with pytest.raises(ValueError):
        P.partition(m, mm.permutation(), 0)
    with pytest.raises(ValueError):
        P.partition(m, mm.permutation(), 2, layers=-1)


def test_search_rows_matches_brute_force_for_large_ids():
    """Rows are matched column by column: ids far above 2^21 (where three ids no longer pack into
    one int64) still find their rows, first occurrence first."""
    rng = np.random.default_rng(5)
    base = np.array([2 ** 40, 2 ** 39, 2 ** 41], np.int64)
    rows = base + rng.integers(0, 4, (300, 3))
    srt = rows[np.lexsort((rows[:, 2], rows[:, 1], rows[:, 0]))]
    queries = np.concatenate([rows[:50], base + rng.integers(3, 6, (50, 3))])
    got = P._search_rows(srt, queries)
    for q, g in zip(queries, got):
        eq = np.nonzero(np.all(srt == q, axis=1))[0]
        assert g == (eq[0] if eq.size else -1)
    assert P._search_rows(srt[:0], queries).tolist() == [-1] * len(queries)
    assert P._search_rows(srt, queries[:0]).size == 0


def test_sub_mesh_with_node_ids_above_2_21_keeps_every_marker():
    """The same mesh with 3,000,000 unused nodes in front of its own: the part meshes keep the same
    boundary triangles (an int64 key of three packed ids would overflow here and drop them)."""
    m = mg.box_tet_mesh(4, 3, 3, jitter=0.1, seed=3)
    off = 3_000_000
    nodes = np.zeros((off + m.nodes.shape[0], 3))
    nodes[off:] = m.nodes
    big = mg.TetMesh(nodes=nodes, tets=np.asarray(m.tets, np.int64) + off,
                     markers=[(n, np.asarray(t, np.int64) + off) for n, t in m.markers],
                     patch_types=dict(m.patch_types))
    cells = np.arange(0, m.n_cells, 3)
    a, b = P.sub_mesh(m, cells), P.sub_mesh(big, cells)
    assert np.array_equal(a.tets, b.tets)
    assert sum(t.shape[0] for _, t in a.markers) > 0
    for (na, ta), (nb_, tb) in zip(a.markers, b.markers):
        assert na == nb_ and np.array_equal(ta, tb)
