"""Batched bump-channel sweep and the surrogate warm-start study.

    python -m netflux_b200.sweep --cases 64 --nx 16 40 --eval-pairs 16 --eval-nx 40 --out DIR
    torchrun --nproc-per-node N -m netflux_b200.sweep ...   (cases sharded over N GPUs)

1. Sweep: `cases` bump channels (seeded hex resolution nx, ny = nz = nx / 2,
   inflow Mach and bump height) are concatenated into one device mesh with
   per-case offsets and far-field states, and advanced together (one launch
   per kernel per stage, the step as CUDA graph replays) with local time
   stepping until every case's density residual has dropped by `tol`;
   converged cases are frozen while the others continue.
2. The converged fields become the surrogate's training set (features: cell
   centroid, wall distance, Mach, bump height, lower-wall height; targets:
   conserved variables normalised by the free stream), and the MLP is trained
   with Adam.
3. Held-out (Mach, h) pairs are solved from the free stream and from the
   surrogate's warm start (with the free-stream fallback) to the same
   absolute residual; steps, device time and the relative L2 difference of
   the final states are recorded.
"""
import argparse
import json
import os
import time
from typing import Dict, List

import numpy as np

from . import meshgen as mg
from . import _lib as L
from . import solver as S
from . import surrogate as sur


def sample_cases(n: int, seed: int, nx_lo: int, nx_hi: int, mach=(0.3, 0.8), h=(0.05, 0.15)) -> List[Dict]:
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nx = int(rng.integers(nx_lo, nx_hi + 1))
        nx += nx % 2  # ny = nz = nx / 2
        out.append({"nx": nx, "mach": float(rng.uniform(*mach)), "h": float(rng.uniform(*h))})
    return out


def case_mesh(c: Dict) -> S.Mesh:
    return S.Mesh.from_tet_mesh(mg.bump_mesh(c["nx"], c["nx"] // 2, c["nx"] // 2, h=c["h"]))


def case_work(c: Dict) -> float:
    """Estimated cost of one case: cells (1.5 nx^3) times steps to converge (about nx^1.6)."""
    return 1.5 * c["nx"] ** 3 * c["nx"] ** 1.6


def partition_cases(cases: List[Dict], world: int) -> List[List[int]]:
    """Whole cases per rank, longest first onto the least-loaded rank."""
    order = sorted(range(len(cases)), key=lambda i: -case_work(cases[i]))
    load = [0.0] * world
    parts: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = int(np.argmin(load))
        parts[r].append(i)
        load[r] += case_work(cases[i])
    return [sorted(p) for p in parts]


def run_sharded(cases: List[Dict], rank: int, world: int, gather, run=None, **kw):
    """This rank's share of the cases as one batched solve; the per-case records
    of every rank gathered (gather: list of this rank's items -> list over ranks).
    There is no collective on the data path: cases are independent."""
    run = run or run_batched
    parts = partition_cases(cases, world)
    mine = [cases[i] for i in parts[rank]]
    res = run(mine, **kw) if mine else {"per_case": []}
    gathered = gather(list(zip(parts[rank], res["per_case"])))
    merged = [None] * len(cases)
    for recs in gathered:
        for i, r in recs:
            merged[i] = r
    return merged, res, parts[rank]


def build_case_meshes(cases: List[Dict], threads: int = 0) -> List[S.Mesh]:
    """The cases' meshes, built on host threads (the mesh generator and the library's builder
    release the interpreter for most of their work); the list is in case order and each mesh is
    the one a serial build gives. The host's cores are split between the builds: with w builds at
    once each builder uses at most cores / w threads of its own (nf_set_host_threads)."""
    from concurrent.futures import ThreadPoolExecutor
    cores = os.cpu_count() or 1
    n = threads or min(16, cores)
    if n <= 1 or len(cases) <= 1:
        return [case_mesh(c) for c in cases]
    workers = min(n, len(cases))
    lib = L.load()
    lib.nf_set_host_threads(max(1, cores // workers))
    try:
        with ThreadPoolExecutor(max_workers=workers) as ex:
            return list(ex.map(case_mesh, cases))
    finally:
        lib.nf_set_host_threads(0)


def run_batched(cases: List[Dict], precision: str = "mixed", tol: float = 1e-6, max_steps: int = 400000,
                check_every: int = 100, device: int = -1, limiter: str = "none") -> Dict:
    t0 = time.perf_counter()
    meshes = build_case_meshes(cases)
    fss = [mg.bump_freestream(c["mach"]) for c in cases]
    batch = S.Mesh.concat(meshes)
    t_mesh = time.perf_counter() - t0
    states = [list(fs) for fs, m in zip(fss, meshes) for _ in m.patches()]
    U0 = np.concatenate([mg.uniform_state(m.n_cells, fs) for fs, m in zip(fss, meshes)])
    s = S.EulerSolver(sur.steady_config(fss[0], precision, limiter), batch, U0=U0, patch_states=states,
                      device=device)
    s.tune()
    out = s.solve_steady(tol, max_steps, check_every)
    U = s.get_solver_data().get_solution()
    s.close()
    off = batch.case_offsets()
    per_case = []
    work = 0.0
    for k, c in enumerate(cases):
        n = int(off[k + 1] - off[k])
        steps = int(out["steps"][k])
        work += 3.0 * n * steps
        per_case.append(dict(c, cells=n, steps=steps, converged=bool(out["converged"][k]),
                             ms=float(out["ms"][k]), res0=float(out["res0"][k]), res=float(out["res"][k])))
    total_ms = float(np.max(out["ms"]))
    return {"per_case": per_case, "cells": int(batch.n_cells), "total_ms": total_ms, "mesh_s": t_mesh,
            "mcell_stages_per_s": work / (total_ms * 1e-3) / 1e6, "U": U, "meshes": meshes, "offsets": off}


def training_data(res: Dict, cases: List[Dict]):
    F, T = [], []
    for k, (c, m) in enumerate(zip(cases, res["meshes"])):
        U = res["U"][res["offsets"][k]:res["offsets"][k + 1]]
        F.append(sur.case_features(m, c["mach"], c["h"]))
        T.append(sur.normalise_state(U, mg.bump_freestream(c["mach"])))
    return np.concatenate(F), np.concatenate(T)


def evaluate(mlp: sur.MLP, pairs: List[Dict], nx: int, precision: str, tol: float, max_steps: int,
             limiter: str = "none", check_every: int = 100) -> List[Dict]:
    rows = []
    for p in pairs:
        c = dict(p, nx=nx)
        mesh = case_mesh(c)
        fs = mg.bump_freestream(c["mach"])
        plain = sur.solve_plain(mesh, fs, tol, precision, max_steps, check_every, limiter=limiter)
        warm = sur.solve_warm(mesh, fs, mlp, c["mach"], c["h"], tol, precision, max_steps, check_every,
                              limiter=limiter)
        d = float(np.linalg.norm(warm["U"] - plain["U"]) / np.linalg.norm(plain["U"]))
        d0 = float(np.linalg.norm(warm["U_warm"] - plain["U"]) / np.linalg.norm(plain["U"]))
        rows.append({"mach": c["mach"], "h": c["h"], "cells": mesh.n_cells,
                     "plain": {k: v for k, v in plain.items() if k != "U"},
                     "warm": {k: v for k, v in warm.items() if k not in ("U", "U_warm")},
                     "final_rel_l2": d, "warm_start_rel_l2": d0,
                     "time_ratio": (warm["ms"] + 1e3 * warm["prep_s"]) / plain["ms"] if plain["ms"] > 0 else None,
                     "step_ratio": warm["steps"] / plain["steps"] if plain["steps"] > 0 else None})
        print(json.dumps({k: v for k, v in rows[-1].items()}, default=float), flush=True)
    return rows


def headline(mlp: sur.MLP, tol: float, max_steps: int, limiter: str = "none") -> Dict:
    """Time to a `tol` residual drop on the 3,145,728-tet channel (128 x 64 x 64 hexes, Mach 0.5,
    h = 0.1): FP64 and mixed from the free stream, mixed from the surrogate's warm start, all to
    the same absolute residual."""
    c = {"nx": 128, "mach": 0.5, "h": 0.1}
    mesh = S.Mesh.from_tet_mesh(mg.bump_mesh(128, 64, 64, h=0.1))
    fs = mg.bump_freestream(0.5)
    out = {"cells": mesh.n_cells, "limiter": limiter}
    for prec in ("fp64", "mixed"):
        r = sur.solve_plain(mesh, fs, tol, prec, max_steps, check_every=500, limiter=limiter)
        out["plain_" + prec] = {k: v for k, v in r.items() if k != "U"}
        if prec == "mixed":
            U_plain = r["U"]
        print(json.dumps({prec: out["plain_" + prec]}, default=float), flush=True)
    w = sur.solve_warm(mesh, fs, mlp, c["mach"], c["h"], tol, "mixed", max_steps, check_every=500, limiter=limiter)
    out["warm_mixed"] = {k: v for k, v in w.items() if k not in ("U", "U_warm")}
    out["warm_final_rel_l2"] = float(np.linalg.norm(w["U"] - U_plain) / np.linalg.norm(U_plain))
    out["warm_start_rel_l2"] = float(np.linalg.norm(w["U_warm"] - U_plain) / np.linalg.norm(U_plain))
    t64 = out["plain_fp64"]["ms"]
    out["time_ratio_mixed_vs_fp64"] = out["plain_mixed"]["ms"] / t64
    out["time_ratio_warm_mixed_vs_fp64"] = (w["ms"] + 1e3 * w["prep_s"]) / t64
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--cases", type=int, default=64)
    ap.add_argument("--nx", type=int, nargs=2, default=[16, 40])
    # the unlimited scheme diverges where the flow over the bump turns
    # transonic (about M + 2 h > 0.8); the default range stays below that
    ap.add_argument("--mach", type=float, nargs=2, default=[0.3, 0.55])
    ap.add_argument("--h", type=float, nargs=2, default=[0.05, 0.11])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--precision", default="mixed")
    ap.add_argument("--tol", type=float, default=1e-6)
    ap.add_argument("--max-steps", type=int, default=400000)
    ap.add_argument("--train-steps", type=int, default=20000)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--lr-schedule", choices=["step", "constant"], default="step",
                    help="step: lr, lr/3.3, lr/10, lr/33 over 50/20/15/15 %% of the steps")
    ap.add_argument("--fine-cases", type=int, default=0,
                    help="additional seeded cases at --fine-nx (closer to the resolution of the 3.1M-tet case)")
    ap.add_argument("--fine-nx", type=int, default=96)
    ap.add_argument("--eval-pairs", type=int, default=16)
    ap.add_argument("--eval-nx", type=int, default=40)
    ap.add_argument("--limiter", choices=sorted(sur.STEADY_LIMITERS), default="none",
                    help="none: the unlimited scheme; barth-ratchet: the reference's Barth limiter, ratcheted "
                         "once a case's residual has dropped 1e-2 (needed where the flow turns transonic)")
    ap.add_argument("--eval-check-every", type=int, default=100)
    ap.add_argument("--eval-skip", type=int, default=0,
                    help="leave out the first pairs of the held-out list (evaluated in an earlier run)")
    ap.add_argument("--load-mlp", default="", help="start from these parameters (.npy) instead of training")
    ap.add_argument("--skip-sweep", action="store_true", help="with --load-mlp: no sweep, no training")
    ap.add_argument("--out", required=True)
    ap.add_argument("--save-data", default="", help="write the training set (features, targets) to this .npz")
    ap.add_argument("--headline", action="store_true",
                    help="also solve the 128x64x64 channel (Mach 0.5, h 0.1) to the tolerance: FP64 and mixed "
                         "from the free stream, mixed from the surrogate's warm start")
    a = ap.parse_args(argv)
    os.makedirs(a.out, exist_ok=True)
    summary = {"args": vars(a)}

    cases = sample_cases(a.cases, a.seed, a.nx[0], a.nx[1], a.mach, a.h)
    if a.fine_cases:
        cases += sample_cases(a.fine_cases, a.seed + 7, a.fine_nx, a.fine_nx, a.mach, a.h)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        # one process per GPU; cases are sharded whole, the only exchange is
        # the final gather of records and training arrays (gloo, host side)
        import datetime

        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=3600))

        def gather(items):
            out = [None] * world
            dist.all_gather_object(out, items)
            return out
        local = int(os.environ.get("LOCAL_RANK", rank))
        merged, res, mine = run_sharded(cases, rank, world, gather, precision=a.precision, tol=a.tol,
                                        max_steps=a.max_steps, device=local)
        sub = [cases[i] for i in mine]
        FT = training_data(res, sub) if sub else (np.zeros((0, 7), np.float32), np.zeros((0, 5), np.float32))
        parts = gather([FT])
        times = gather([res.get("total_ms", 0.0)])
        if rank != 0:
            dist.barrier()
            dist.destroy_process_group()
            return
        F = np.concatenate([p[0][0] for p in parts])
        T = np.concatenate([p[0][1] for p in parts])
        work = sum(3.0 * r["cells"] * r["steps"] for r in merged)
        total_ms = max(t[0] for t in times)
        summary["sweep"] = {"per_case": merged, "cells": int(sum(r["cells"] for r in merged)), "ranks": world,
                            "total_ms": total_ms, "mcell_stages_per_s": work / (total_ms * 1e-3) / 1e6}
    elif a.skip_sweep:
        F = T = None
    else:
        res = run_batched(cases, a.precision, a.tol, a.max_steps, limiter=a.limiter)
        summary["sweep"] = {k: v for k, v in res.items() if k not in ("U", "meshes", "offsets")}
        F, T = training_data(res, cases)
        del res
    if a.skip_sweep:
        if not a.load_mlp:
            raise SystemExit("--skip-sweep needs --load-mlp")
        mlp = sur.MLP(seed=a.seed)
        mlp.set_params(np.load(a.load_mlp))
        return finish(a, summary, mlp, world)
    sw = summary["sweep"]
    print(json.dumps({"sweep_cells": sw["cells"], "total_ms": sw["total_ms"],
                      "mcell_stages_per_s": sw["mcell_stages_per_s"],
                      "converged": sum(c["converged"] for c in sw["per_case"])}), flush=True)
    if a.save_data:
        np.savez_compressed(a.save_data, features=F, targets=T, cases=json.dumps(cases))

    mlp = sur.MLP(seed=a.seed)
    mlp.set_data(F, T)
    if a.lr_schedule == "step":
        tr = mlp.train_schedule(a.train_steps, a.batch, a.lr, seed=a.seed, n_report=20)
    else:
        tr = mlp.train(a.train_steps, a.batch, a.lr, seed=a.seed, n_report=20)
    summary["training"] = {"samples": int(F.shape[0]), "steps": a.train_steps, "batch": a.batch, "lr": a.lr,
                           "lr_schedule": a.lr_schedule,
                           "ms": tr["ms"], "loss": tr["loss"].tolist()}
    np.save(os.path.join(a.out, "mlp_params.npy"), mlp.get_params())
    print(json.dumps({"train_ms": tr["ms"], "loss_first": float(tr["loss"][0]), "loss_last": float(tr["loss"][-1])}),
          flush=True)
    return finish(a, summary, mlp, world)


def finish(a, summary: Dict, mlp: sur.MLP, world: int):
    """Warm-start evaluation on held-out pairs, the optional headline, the summary file."""
    rng = np.random.default_rng(a.seed + 1)
    pairs = [{"mach": float(rng.uniform(*a.mach)), "h": float(rng.uniform(*a.h))} for _ in range(a.eval_pairs)]
    pairs = pairs[a.eval_skip:]
    rows = evaluate(mlp, pairs, a.eval_nx, a.precision, a.tol, a.max_steps, a.limiter, a.eval_check_every)
    summary["eval"] = rows
    ok = [r for r in rows if r["time_ratio"] is not None]
    summary["eval_summary"] = {
        "median_time_ratio": float(np.median([r["time_ratio"] for r in ok])) if ok else None,
        "median_step_ratio": float(np.median([r["step_ratio"] for r in ok])) if ok else None,
        "max_final_rel_l2": float(max(r["final_rel_l2"] for r in rows)) if rows else None,
        "fallbacks": sum(1 for r in rows if r["warm"]["fallback"])}
    if a.headline:
        summary["headline"] = headline(mlp, a.tol, a.max_steps, a.limiter)
        print(json.dumps(summary["headline"], default=float), flush=True)
    with open(os.path.join(a.out, "summary.json"), "w") as f:
        json.dump(summary, f, indent=1, default=float)
    print(json.dumps(summary["eval_summary"]), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
