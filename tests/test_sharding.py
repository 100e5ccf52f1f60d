"""Case sharding of the batched sweep across ranks: the split and the gather, with world_size 2 gloo
ranks on CPU (the solve is replaced by a stand-in that records which cases a rank ran)."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from netflux_b200 import sweep as SW


def test_partition_is_complete_and_balanced():
    cases = SW.sample_cases(64, 0, 16, 40)
    parts = SW.partition_cases(cases, 4)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(64))
    loads = [sum(SW.case_work(cases[i]) for i in p) for p in parts]
    assert max(loads) <= 1.15 * min(loads)


def _fake_run(cases, **kw):
    return {"per_case": [dict(c, cells=int(1.5 * c["nx"] ** 3), steps=100 + c["nx"], converged=True,
                              rank=int(os.environ["RANK"])) for c in cases]}


def _worker(rank, world, port, cases, out):
    os.environ["RANK"] = str(rank)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)

    def gather(items):
        res = [None] * world
        dist.all_gather_object(res, items)
        return res
    merged, _, mine = SW.run_sharded(cases, rank, world, gather, run=_fake_run)
    out[rank] = (merged, mine)
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_shard_and_gather():
    cases = SW.sample_cases(10, 3, 16, 40)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(2, port, cases, out), nprocs=2, join=True)
    m0, mine0 = out[0]
    m1, mine1 = out[1]
    assert sorted(mine0 + mine1) == list(range(10)) and not set(mine0) & set(mine1)
    assert m0 == m1  # every rank holds every record
    for i, r in enumerate(m0):
        assert r["nx"] == cases[i]["nx"] and r["steps"] == 100 + cases[i]["nx"]
        assert r["rank"] == (0 if i in mine0 else 1)


def test_threaded_case_meshes_equal_serial_ones():
    cases = SW.sample_cases(6, 5, 8, 14)
    serial = SW.build_case_meshes(cases, threads=1)
    threaded = SW.build_case_meshes(cases, threads=4)
    for a, b in zip(serial, threaded):
        ea, eb = a.export(), b.export()
        assert a.n_cells == b.n_cells and all(np.array_equal(ea[k], eb[k]) for k in ea)
        assert np.array_equal(a.permutation(), b.permutation())
