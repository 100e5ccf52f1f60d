"""Benchmark of the explicit second-order Euler step (TVD-RK3) on B200.

Workload (default): the steady bump channel, [0,3]x[0,1]^2 with a
0.1*sin^2 bump, 128x64x64 hexes x 6 = 3,145,728 tets, Mach 0.5 free stream,
local time stepping at CFL 0.8, FP64. One bench step = one TVD-RK3 step
(3 cell-stages per cell). Synthetic mesh generated in-process; every working
array is far larger than the 126 MB L2, so no flush is needed between steps.
The smaller cube and Sod cases fit the L2 and are reported as L2-warm
figures (config.l2 says which).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--case bump|cube|sod] [--precision fp64|mixed|mixed32|fp64_ref]

Prints one JSON line on rank 0. ``value`` is Mcell-RK-stages/s with the state
resident in HBM (CUDA events on the solver's stream, max over ranks);
``e2e`` is the same metric through the public API with the state copied
host->device and back every step; ``roofline`` is the dominant kernel's
algorithmic HBM bytes per launch over its event-timed duration against the
measured copy bandwidth; ``cpu_baseline`` is the NetFlux reference compiled
from its sources, timed on this host's cores on a bounded sample.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-RK-stages/s"
HBM_FALLBACK_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--case", default="bump", choices=["bump", "cube", "sod"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed", "mixed32", "fp64_ref"])
    ap.add_argument("--scale", type=int, default=1, help="divide the hex counts (quick runs)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=50)
    ap.add_argument("--steady", action="store_true",
                    help="also time a local-time-stepping solve of the benched channel to a 1e-6 density-residual "
                         "drop (minutes)")
    ap.add_argument("--no-steady-quick", action="store_true",
                    help="skip the quick time-to-solution study on a 24x12x12 channel")
    ap.add_argument("--no-mixed-forms", action="store_true",
                    help="skip timing the two mixed forms beside the FP64 step (FP64 runs only)")
    ap.add_argument("--steady-max", type=int, default=60000)
    ap.add_argument("--steady-limiter", choices=["none", "barth-ratchet"], default="none")
    ap.add_argument("--block", type=int, default=0, help="fix the block size (no tuning)")
    ap.add_argument("--variant", type=int, default=0, help="with --block: fast-kernel variant")
    ap.add_argument("--shapes", type=int, nargs=4, default=None, metavar=("GB", "GV", "FB", "FV"),
                    help="fix the gradient and flux kernels' (block, variant) separately (no tuning)")
    return ap.parse_args()


def l2_note(stage_bytes: float) -> str:
    """How the timed steps meet the L2: one stage's algorithmic bytes against the 126 MB L2."""
    mb = stage_bytes / 1e6
    if mb > 126.0:
        return f"working set {mb:.0f} MB per stage > 126 MB L2 (no flush needed)"
    return (f"working set {mb:.0f} MB per stage fits the 126 MB L2; steps run back to back, so this is an "
            "L2-warm figure (not flushed)")


def case_mesh(name: str, scale: int):
    from netflux_b200 import meshgen as mg
    if name == "bump":
        m = mg.bump_mesh(128 // scale, 64 // scale, 64 // scale, h=0.1)
        fs = mg.bump_freestream(0.5)
        return m, fs, mg.uniform_state(m.n_cells, fs), True, "bump channel 128x64x64 hexes, 6 tets each"
    if name == "cube":
        m = mg.cube_mesh(20 // scale, jitter=0.1, seed=1234)
        fs = (1.0, 0.5, 0.0, 0.0, 1.0 / 1.4)
        return m, fs, mg.cube_initial_state(m), False, "unit cube 20^3 hexes, 6 tets each, Gaussian density bump"
    m = mg.sod_mesh(400 // scale, 8, 8, jitter=0.05, seed=4321)
    return m, mg.SOD_LEFT, mg.sod_initial_state(m), False, "Sod tube 400x8x8 hexes, 6 tets each"


def case_mesh_desc(name: str) -> str:
    return {"bump": "bump channel 128x64x64 hexes, 6 tets each",
            "cube": "unit cube 20^3 hexes, 6 tets each, Gaussian density bump",
            "sod": "Sod tube 400x8x8 hexes, 6 tets each"}[name]


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                sm.append(float(f[1]))
                mx.append(float(f[2]))
                for n, v in zip(names, f[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        except Exception:
            pass
        finally:
            try:
                os.remove(self.path)
            except Exception:
                pass
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def algorithmic_bytes(n_cells: int, n_faces: int, n_boundary: int, n_nodes: int, precision: str,
                      local_dt: bool):
    """Compulsory HBM bytes of one launch of each stage kernel (every datum the
    kernel must read or write, once; neighbours' values are other cells' own
    values and are not counted again), averaged over the three stages.

    FP64 (gradient_node / flux_node), per cell:
      gradient: V (40), 4 vertex ids (16), 4 neighbour ids (16), face code (4),
        vol (8), writes 4 face states (160); per node 32 (xyz + pad); per
        boundary face one ghost state (40); the last stage also writes the
        next step's dt (8 with local time stepping; its projected areas come
        from the normals in registers): a third of that on average.
      flux: 4 own face states (160), 4 neighbour face ids (16), face code (4),
        4 vertex ids (16), U (40), U^n (40 at stages 2 and 3: 2/3 on average),
        vol (8), local dt (8 with local time stepping), writes U and V (80) and
        R_rho/vol at the first stage (8, 1/3 on average); per node 32; per
        boundary face one boundary flux (40).
    Mixed (gradient_delta / flux_delta, FP32 differences to FP64 state):
      gradient: V (40), ids (32), code (4), vol (8), writes 4 FP32 increments
        (80); per node 16; per boundary face an FP64 ghost (40).
      flux: own V (40), own increments (80), neighbour face ids (16), code (4),
        vertex ids (16), U, U^n, vol, dt, writes U, V and R_rho as above; per
        node 16; per boundary face an FP32 flux difference (20); stage 2 also
        reads dS (24) and writes the next step's dt (8 with local time
        stepping): a third of that on average.
    Mixed with FP32 copies (the FP32 node kernels, NF_PREC_MIXED32):
      gradient: FP32 V (20), ids (32), code (4), vol (8), writes 4 FP32 face
        states (80); per node 16; per boundary face an FP32 ghost (20).
      flux: 4 own FP32 face states (80), neighbour face ids (16), code (4),
        vertex ids (16), U, U^n, vol, dt, writes U (40), the FP32 V (20) and
        R_rho (no FP64 V: the stage-2 flux kernel computes the next dt from its
        FP64 result); per node 16; per boundary face an FP32 flux (20); the
        next step's dt as in the difference form.
    """
    lts = 8 if local_dt else 0
    upd = 40 + 40 * 2 / 3 + 8 + lts + 80 + 8 / 3  # U, U^n, vol, dt, U and V out, R_rho
    if precision == "mixed":
        grad = n_cells * (40 + 16 + 16 + 4 + 8 + 80) + n_nodes * 16 + n_boundary * 40
        flux = n_cells * (40 + 80 + 16 + 4 + 16 + upd + (24 + lts) / 3) + n_nodes * 16 + n_boundary * 20
    elif precision == "mixed32":
        upd32 = 40 + 40 * 2 / 3 + 8 + lts + 40 + 20 + 8 / 3 + (24 + lts) / 3
        grad = n_cells * (20 + 16 + 16 + 4 + 8 + 80) + n_nodes * 16 + n_boundary * 20
        flux = n_cells * (80 + 16 + 4 + 16 + upd32) + n_nodes * 16 + n_boundary * 20
    else:
        grad = n_cells * (40 + 16 + 16 + 4 + 8 + 160 + lts / 3) + n_nodes * 32 + n_boundary * 40
        flux = n_cells * (160 + 16 + 4 + 16 + upd) + n_nodes * 32 + n_boundary * 40
    return {"flux": flux, "gradient": grad}


# DRAM bytes per cell of one launch (dram__bytes_read.sum + dram__bytes_write.sum), captured
# with ncu on the full 3,145,728-tet bump channel with the tuned launch shapes, averaged over the
# three stages of a step like the event-timed launch durations (FP64: gradient 64/7, flux 64/9,
# stages 755.3 / 749.8 / 780.6 and 1108.6 / 1221.7 / 1227.9 MB; mixed: gradient 64/7, flux
# 128/8, stages 506.9 / 500.9 / 500.7 and 989.5 / 1208.8 / 1104.6 MB); the bump workload's
# `roofline.traffic` is this times its cells, other workloads report null.
MEASURED_DRAM_BYTES_PER_CELL = {
    ("fp64", "gradient"): 761.9e6 / 3145728, ("fp64", "flux"): 1186.1e6 / 3145728,
    ("mixed", "gradient"): 502.8e6 / 3145728, ("mixed", "flux"): 1101.0e6 / 3145728,
}


def model_bytes_per_cell_stage(n_cells: int, n_faces: int) -> float:
    """The per-cell-stage byte model of the step's compulsory traffic (FP64):
    N_c*[3*(40 U read + 40 U write + 8 vol + 240 limited-gradient write+read)
    + 2*40 U^n read + 24 dS] + N_f*3*80, divided by 3*N_c."""
    step = n_cells * (3 * (40 + 40 + 8 + 240) + 2 * 40 + 24) + n_faces * 3 * 80
    return step / (3.0 * n_cells)


# host memory one reference process holds per cell (2.36 GB at 3,145,728 tets), with a margin
REF_BYTES_PER_CELL = 1000.0


def host_processes(n_cells: int) -> int:
    """Independent reference processes to run at once: one per host core, at most as many as the
    available host memory holds."""
    n = os.cpu_count() or 1
    try:
        with open("/proc/meminfo") as f:
            avail = next(int(l.split()[1]) * 1024 for l in f if l.startswith("MemAvailable:"))
        n = max(1, min(n, int(0.8 * avail // (REF_BYTES_PER_CELL * n_cells))))
    except Exception:
        pass
    return n


def cpu_reference_baseline(n_steps: int = 3, case: str = "bump", scale: int = 1, procs: int = 0):
    """Time the compiled reference on a bounded sample of a workload: the case's
    full mesh (scale 1), n_steps TVD-RK3 steps per single-threaded process, the
    solve timed inside each process (mesh reading and building excluded)."""
    from netflux_b200 import meshgen as mg
    from oracle import pyoracle as po  # CPU baseline leg only
    variant = "nf_ref_nodump"
    if not po.reference_available(variant):
        return None
    m, fs, U0, _, desc = case_mesh(case, scale)
    nproc = procs or host_processes(m.n_cells)
    with tempfile.TemporaryDirectory() as tmp:
        case_dir = os.path.join(tmp, "case")
        mg.write_case(case_dir, m, fs, U0=U0)
        exe = os.path.join(po.REF_DIR, variant)

        def run_many(k):
            outs, ps = [], []
            for i in range(k):
                od = os.path.join(tmp, f"o{i}")
                os.makedirs(od, exist_ok=True)
                outs.append(od)
                ps.append(subprocess.Popen([exe, case_dir, od, "--steps", str(n_steps), "--quiet"], cwd=tmp,
                                           stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL))
            for p in ps:
                p.wait()
            secs = []
            for od in outs:
                for line in open(os.path.join(od, "meta.txt")):
                    if line.startswith("seconds"):
                        secs.append(float(line.split()[1]))
            return secs

        one = run_many(1)[0]
        many = run_many(nproc) if nproc > 1 else [one]
    cs = m.n_cells * 3 * n_steps
    return {
        "single_core": cs / one / 1e6,
        "all_cores": cs * len(many) / max(many) / 1e6,
        "cores": nproc,
        "sample": f"{desc} ({m.n_cells} tets{', hex counts / %d' % scale if scale > 1 else ', the full mesh'}), "
                  f"{n_steps} TVD-RK3 steps per process, reference compiled from its sources (debug dump "
                  f"linked out), {nproc} independent single-threaded processes, solve time only",
        "same_config": scale == 1,
    }


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import pyoracle as po  # reference arm: the reference's own CPU code
    if not po.reference_available("nf_ref_nodump"):
        print(json.dumps({"impl": "reference", "unavailable": "reference build (oracle/_ref) missing"}))
        return
    # every step of every process is one TVD-RK3 step of the full workload; the sample is bounded
    # to 3 steps per process at the 3.1M-tet channel (about 10 s of solving each)
    n_steps = max(1, min(args.steps, 3 if args.case == "bump" and args.scale == 1 else args.steps))
    res = cpu_reference_baseline(n_steps=n_steps, case=args.case, scale=args.scale)
    val = res["all_cores"]
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(val, 3), "unit": "Mcell-stages/s",
        "n_gpus": 0, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": case_mesh_desc(args.case), "sample": res["sample"],
                   "same_config": res["same_config"]},
        "cpu_baseline": {"value": round(val, 3), "unit": "Mcell-stages/s", "cores": res["cores"],
                         "kind": "reference", "sample": res["sample"],
                         "single_core": round(res["single_core"], 4), "same_config": res["same_config"]},
        "e2e": {"value": round(val, 3), "unit": "Mcell-stages/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def host_link(nbytes: int, reps: int = 5):
    """Pinned host <-> device copy rates (GB/s) for one transfer of nbytes: host to device alone,
    device to host alone, and both at once on two streams (the total of both directions), each over
    reps back-to-back copies timed with CUDA events on the copying streams."""
    import torch
    n = nbytes // 8
    h_in = torch.empty(n, dtype=torch.float64, pin_memory=True)
    h_out = torch.empty(n, dtype=torch.float64, pin_memory=True)
    d_a = torch.empty(n, dtype=torch.float64, device="cuda")
    d_b = torch.empty(n, dtype=torch.float64, device="cuda")
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()

    def run(h2d: bool, d2h: bool) -> float:
        torch.cuda.synchronize()
        start = torch.cuda.Event(enable_timing=True)
        start.record()
        ends = []
        for on, st, fn in ((h2d, s1, lambda: d_a.copy_(h_in, non_blocking=True)),
                           (d2h, s2, lambda: h_out.copy_(d_b, non_blocking=True))):
            if not on:
                continue
            st.wait_event(start)
            with torch.cuda.stream(st):
                for _ in range(reps):
                    fn()
                e = torch.cuda.Event(enable_timing=True)
                e.record()
            ends.append(e)
        torch.cuda.synchronize()
        return max(start.elapsed_time(e) for e in ends) / 1e3

    run(True, True)  # warm
    t_in, t_out, t_both = run(True, False), run(False, True), run(True, True)
    return {"bytes": int(nbytes), "h2d_gbs": round(reps * nbytes / t_in / 1e9, 2),
            "d2h_gbs": round(reps * nbytes / t_out / 1e9, 2),
            "both_total_gbs": round(2 * reps * nbytes / t_both / 1e9, 2)}


def mixed_forms(mesh, cfg_kw: dict, U0, steps: int, warmup: int, fp64_ms: float, device: int) -> dict:
    """The two mixed forms on the benched mesh and state, each tuned and timed like the FP64 step
    (CUDA events around `steps` graph-replayed steps), with each step's time against the FP64 one
    measured in the same run: the mixed-precision speed-up the FP64 line is compared with."""
    from netflux_b200 import _lib as L
    from netflux_b200 import solver as S
    lib = L.load()
    out = {}
    for prec in ("mixed", "mixed32"):
        cfg = S.Config(precision=prec, **cfg_kw)
        s = S.EulerSolver(cfg, mesh, U0=U0, device=device)
        s.advance(max(warmup, 3) - 2)
        shapes = s.tune()
        s.advance(2)
        ms = C.c_double()
        kms = (C.c_double * L.NF_KERNEL_COUNT)()
        kl = (C.c_int64 * L.NF_KERNEL_COUNT)()
        rc = lib.nf_time_steps(s._h, steps, 0, C.byref(ms), kms, kl)
        if rc != 0:
            raise RuntimeError(L.last_error(s._h))
        s.close()
        step_ms = ms.value / steps
        out[prec] = {"value": round(mesh.n_cells * 3 / (step_ms * 1e-3) / 1e6, 3), "ms_per_step": round(step_ms, 5),
                     "speedup_vs_fp64": round(fp64_ms / step_ms, 4), "launch_shapes": shapes}
    return out


def steady_quick(device: int):
    """Time to a 1e-6 density-residual drop on a small channel (24 x 12 x 12 hexes, 20,736 tets,
    Mach 0.5, h = 0.1, unlimited scheme, local time stepping at CFL 0.8), measured in this run:
    FP64 and mixed from the free stream, and mixed from the surrogate's warm start, the network
    trained in this run (3,000 Adam steps) on 8 converged channels of 16..22 hexes in x that do not
    include the evaluated one. All three solves stop at the same absolute residual (1e-6 of the
    free-stream start's first residual); times are device times of the solves (the warm start's
    includes its preparation)."""
    from netflux_b200 import meshgen as mg
    from netflux_b200 import surrogate as sur
    from netflux_b200 import sweep as SW
    t0 = time.perf_counter()
    cases = SW.sample_cases(8, 3, 16, 22, (0.35, 0.65), (0.05, 0.12))
    res = SW.run_batched(cases, "mixed", 1e-6, 100000, 50, device=device)
    F, T = SW.training_data(res, cases)
    mlp = sur.MLP(seed=1)
    mlp.set_data(F, T)
    tr = mlp.train_schedule(3000, 16384, 1e-3, seed=1, n_report=3)
    c = {"nx": 24, "mach": 0.5, "h": 0.1}
    mesh = SW.case_mesh(c)
    fs = mg.bump_freestream(c["mach"])
    out = {"workload": "bump channel 24x12x12 hexes, 6 tets each (20,736 tets), Mach 0.5, h 0.1, limiter none",
           "tol": 1e-6, "training": {"cases": len(cases), "samples": int(F.shape[0]), "steps": 3000,
                                     "loss": float(tr["loss"][-1]), "ms": round(float(tr["ms"]), 1)}}
    plain = {}
    for prec in ("fp64", "mixed"):
        r = sur.solve_plain(mesh, fs, 1e-6, prec, 200000, 50)
        plain[prec] = r
        out["plain_" + prec] = {"steps": r["steps"], "ms": round(r["ms"], 2), "converged": r["converged"]}
    w = sur.solve_warm(mesh, fs, mlp, c["mach"], c["h"], 1e-6, "mixed", 200000, 50)
    ms_w = w["ms"] + 1e3 * w["prep_s"]
    out["warm_mixed"] = {"steps": w["steps"], "ms": round(ms_w, 2), "converged": w["converged"],
                         "fallback": w["fallback"]}
    out["time_ratio_mixed_vs_fp64"] = round(plain["mixed"]["ms"] / plain["fp64"]["ms"], 4)
    out["time_ratio_warm_mixed_vs_fp64"] = round(ms_w / plain["fp64"]["ms"], 4)
    out["warm_final_rel_l2_vs_plain_mixed"] = float(np.linalg.norm(w["U"] - plain["mixed"]["U"]) /
                                                    np.linalg.norm(plain["mixed"]["U"]))
    out["wall_s"] = round(time.perf_counter() - t0, 1)
    mlp.close()
    return out


def main():
    args = parse()
    if args.impl == "reference":
        run_reference_arm(args)
        return
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from netflux_b200 import _lib as L
    from netflux_b200 import solver as S

    m, fs, U0, lts, desc = case_mesh(args.case, args.scale)
    t0 = time.perf_counter()
    mesh = S.Mesh.from_tet_mesh(m)
    t_mesh = time.perf_counter() - t0
    cfg = S.Config(precision=args.precision, CFL=0.8, local_time_stepping=lts, density_fs=fs[0],
                   velocity_fs=list(fs[1:4]), pressure_fs=fs[4])
    solver = S.EulerSolver(cfg, mesh, U0=U0, block_size=args.block, variant=args.variant, device=local)
    lib = L.load()
    N = mesh.n_cells

    # warm-up, launch-shape tuning, then the CUDA graph of the step
    ms = C.c_double()
    if args.shapes:  # fixed before the warm-up, so every launch has these shapes
        solver.set_launch_shapes(gradient=args.shapes[:2], flux=args.shapes[2:])
    solver.advance(max(args.warmup, 3) - 2)
    if args.shapes:
        tuned = {"gradient": {"block": args.shapes[0], "variant": args.shapes[1]},
                 "flux": {"block": args.shapes[2], "variant": args.shapes[3]}, "fixed": True}
    else:
        tuned = solver.tune() if args.block == 0 else None
    solver.advance(2)  # the last two warm-up steps capture and replay the step graph the timing replays
    kms = (C.c_double * L.NF_KERNEL_COUNT)()
    kl = (C.c_int64 * L.NF_KERNEL_COUNT)()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        rc = lib.nf_time_steps(solver._h, args.steps, 0, C.byref(ms), kms, kl)
    if rc != 0:
        raise RuntimeError(L.last_error(solver._h))
    torch.cuda.synchronize()
    dev_ms = ms.value
    if dist:
        t = torch.tensor([dev_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev_ms = float(t.item())
        dist.barrier()
    value = world * N * 3 * args.steps / (dev_ms / 1e3) / 1e6

    # per-kernel event timing (separate run, same kernels, no graph)
    rc = lib.nf_time_steps(solver._h, max(args.steps // 2, 2), 1, C.byref(ms), kms, kl)
    if rc != 0:
        raise RuntimeError(L.last_error(solver._h))
    kern = {name: (kms[i] / max(kl[i], 1), int(kl[i])) for i, name in
            ((L.NF_KERNEL_TIMESTEP, "timestep"), (L.NF_KERNEL_GRADIENT, "gradient"), (L.NF_KERNEL_FLUX, "flux"),
             (L.NF_KERNEL_OTHER, "other"))}
    nb = mesh.n_ghost
    ab = algorithmic_bytes(N, mesh.n_faces, nb, int(mesh.info.n_nodes), args.precision, lts)
    hbm, hbm_kind = measured_peaks()
    dom = max(("flux", "gradient"), key=lambda k: kern[k][0] * kern[k][1])
    ach = ab[dom] / (kern[dom][0] * 1e-3) / 1e9
    per_cell = MEASURED_DRAM_BYTES_PER_CELL.get((args.precision, dom)) if args.case == "bump" else None
    traffic = int(per_cell * N) if per_cell else None
    roof = {"bound": "hbm", "kernel": dom, "achieved": round(ach, 1), "peak": hbm, "unit": "GB/s",
            "frac": round(ach / hbm, 4), "peak_kind": hbm_kind, "traffic": traffic,
            "algorithmic_bytes_per_launch": int(ab[dom]), "avg_launch_ms": round(kern[dom][0], 5),
            "per_kernel_ms": {k: round(v[0], 5) for k, v in kern.items()}}
    model = model_bytes_per_cell_stage(N, mesh.n_faces)
    step_gbs = model * N * 3 * args.steps / (dev_ms / 1e3) / 1e9

    # end to end through the public API: host state in, step, host state out
    e2e = None
    if not args.no_e2e:
        pinned = torch.empty((N, 5), dtype=torch.float64, pin_memory=True).numpy()
        pinned[:] = solver.get_solver_data().get_solution()
        n_e = max(1, args.e2e_steps)
        outs = [torch.empty((N, 5), dtype=torch.float64, pin_memory=True).numpy() for _ in range(2)]
        ins = [pinned, torch.empty((N, 5), dtype=torch.float64, pin_memory=True).numpy()]
        ins[1][:] = pinned

        def loop_sync():  # each state goes in and comes back before the next step starts
            for _ in range(n_e):
                solver.set_state(pinned)
                solver.calc_timestep(cfg)
                solver.step(cfg)
                rc = lib.nf_get_state(solver._h, L.dptr(pinned), N)
                if rc != 0:
                    raise RuntimeError(L.last_error(solver._h))

        def loop_streamed():  # independent states: the next upload and this result's copy overlap the step
            solver.upload_begin(ins[0])
            for i in range(n_e):
                solver.upload_commit()
                if i + 1 < n_e:
                    solver.upload_begin(ins[(i + 1) % 2])
                solver.calc_timestep(cfg)
                solver.step(cfg)
                solver.snapshot_begin(outs[i % 2])
            solver.snapshot_wait()
            solver.upload_wait()

        def timed(loop):
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            loop()
            wall = time.perf_counter() - t1
            if dist:
                t = torch.tensor([wall], device="cuda", dtype=torch.float64)
                dist.all_reduce(t, op=dist.ReduceOp.MAX)
                wall = float(t.item())
            return world * N * 3 * n_e / wall / 1e6

        loop_sync()  # untimed: first use of these host buffers and of the non-graph step path
        loop_streamed()
        v_sync = timed(loop_sync)
        v_stream = timed(loop_streamed)
        link = host_link(N * 5 * 8)
        # the copies' bound: each step moves one state in and one out, at the measured rate of
        # both directions at once (or one direction alone, whichever bounds it more)
        per_step_s = max(2 * N * 5 * 8 / (link["both_total_gbs"] * 1e9), N * 5 * 8 / (link["h2d_gbs"] * 1e9),
                         N * 5 * 8 / (link["d2h_gbs"] * 1e9))
        link["bound_value"] = round(N * 3 / per_step_s / 1e6, 3)
        link["frac"] = round(v_stream / link["bound_value"], 4)
        e2e = {"value": round(v_stream, 3), "unit": "Mcell-stages/s",
               "h2d_bytes_per_step": int(N * 5 * 8), "d2h_bytes_per_step": int(N * 5 * 8 + 8),
               "steps": n_e, "sync_value": round(v_sync, 3), "host_link": link,
               "path": "per step, over the C ABI: upload_commit of a state copied from pinned memory, "
                       "calc_timestep, step, snapshot_begin into pinned memory; the next state's upload "
                       "and this result's copy run on side streams during the step, and the clock stops "
                       "when the last copy has landed. sync_value: set_state, calc_timestep, step and a "
                       "blocking get_state per step"}

    steady = None
    if args.steady:
        # The reference's live Barth limiter stalls the residual near a 5e-3 drop
        # on this channel; the subsonic flow needs no limiter, so the steady
        # solve uses limiter NONE by default (a reference option), or Barth
        # with the limiter ratchet started at a 1e-2 drop.
        lim = {"none": dict(limiter="NONE"),
               "barth-ratchet": dict(limiter="Barth", limiter_ratchet_drop=1e-2)}[args.steady_limiter]
        scfg = S.Config(precision=args.precision, CFL=0.8, local_time_stepping=True, density_fs=fs[0],
                        velocity_fs=list(fs[1:4]), pressure_fs=fs[4], **lim)
        solver.close()
        solver = S.EulerSolver(scfg, mesh, U0=U0, device=local)
        solver.tune()
        out = solver.solve_steady(tol=1e-6, max_steps=args.steady_max, check_every=100)
        steady = {"tol": 1e-6, "limiter": args.steady_limiter, "converged": bool(out["converged"][0]),
                  "steps": int(abs(out["steps"][0])),
                  "ms": round(float(out["ms"][0]), 2), "res0": float(out["res0"][0]),
                  "res_final": float(out["res"][0]),
                  "drop": float(out["res"][0] / out["res0"][0]) if out["res0"][0] > 0 else None}

    mixed = None
    if rank == 0 and world == 1 and args.precision == "fp64" and not args.no_mixed_forms:
        mixed = mixed_forms(mesh, dict(CFL=0.8, local_time_stepping=lts, density_fs=fs[0], velocity_fs=list(fs[1:4]),
                                       pressure_fs=fs[4]), U0, args.steps, args.warmup, dev_ms / args.steps, local)

    quick = None
    if rank == 0 and world == 1 and not args.no_steady_quick:
        quick = steady_quick(local)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the same workload and mesh
        res = cpu_reference_baseline(case=args.case, scale=args.scale)
        if res is not None:
            cpu = {"value": round(res["all_cores"], 4), "unit": "Mcell-stages/s", "cores": res["cores"],
                   "kind": "reference", "sample": res["sample"], "single_core": round(res["single_core"], 4),
                   "same_config": res["same_config"]}

    if rank == 0:
        kernels_per_step = sum(kl) / max(args.steps // 2, 2)
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "Mcell-stages/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dev_ms / args.steps, 5),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"fp64": "f64", "fp64_ref": "f64", "mixed": "f32+f64", "mixed32": "f32+f64"}[args.precision],
            "data": "synthetic",
            "config": {"workload": desc, "cells": N, "faces": mesh.n_faces, "time_scheme": "TVD_RK3",
                       "local_time_stepping": lts, "cfl": 0.8, "precision": args.precision,
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": l2_note(model * N), "mesh_build_s": round(t_mesh, 2),
                       "launch_shapes": tuned},
            "roofline": roof,
            "step_roofline": {"model_bytes_per_cell_stage": round(model, 1), "achieved": round(step_gbs, 1),
                              "peak": hbm, "unit": "GB/s", "frac": round(step_gbs / hbm, 4)},
            "clocks": clocks.summary(),
            "e2e": e2e,
            "gpu_launches": int(round(kernels_per_step * args.steps)),
            "cpu_baseline": cpu,
        }
        if mixed is not None:
            line["mixed_forms"] = mixed
        if quick is not None:
            line["steady_quick"] = quick
        if steady is not None:
            line["steady"] = steady
        print(json.dumps(line))
    solver.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
