"""Generate the golden fixtures in this directory from the NetFlux reference.

Run in a checkout that has the reference tree and its build (``make -C
oracle``): every fixture is produced by oracle/_ref/nf_ref_nodump, the
reference solver compiled from its own unmodified sources, on small seeded
meshes from netflux_b200.meshgen. Machines without the reference tree read
these files instead.

    python tests/golden/make_golden.py [case ...]   # all cases when none is named

Each ``<case>.npz`` holds the mesh (nodes, tets as written, markers), the
initial state, the free stream, and the reference's outputs:
  U1 / dt1                   after 1 TVD-RK3 step
  U100 / dt100               after 100 TVD-RK3 steps (smaller cases)
  euler_{V,grad,limiter,R}   intermediates of one explicit-Euler step
  geometry (face_ij, S, ri, rj, vol, centroid, dS, patches)
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from netflux_b200 import meshgen as mg  # noqa: E402
from oracle import pyoracle as po  # noqa: E402

CASES = {
    # unit-cube Gaussian density bump, all far field (the 48k-tet case shape, 4^3 hexes)
    "cube4": dict(mesh=lambda: mg.cube_mesh(4, jitter=0.1, seed=11),
                  fs=(1.0, 0.5, 0.0, 0.0, 1.0 / 1.4), U0=mg.cube_initial_state, steps100=True),
    # slip-wall Sod tube (far-field ends), 40x4x4 hexes
    "sod40": dict(mesh=lambda: mg.sod_mesh(40, 4, 4, jitter=0.05, seed=12),
                  fs=mg.SOD_LEFT, U0=mg.sod_initial_state, steps100=True),
    # bump channel at Mach 0.5, 12x6x6 hexes, started from the free stream
    "bump12": dict(mesh=lambda: mg.bump_mesh(12, 6, 6, h=0.1),
                   fs=mg.bump_freestream(0.5), U0=None, steps100=True),
    # closed slip-wall box (no far field: no pow(), conservation holds)
    "slipbox5": dict(mesh=lambda: mg.box_tet_mesh(5, 5, 5, jitter=0.1, seed=13,
                                                  side_patches={s: "walls" for s in
                                                                ("imin", "imax", "jmin", "jmax", "kmin", "kmax")},
                                                  patch_types={"walls": mg.SLIP_WALL}),
                     fs=(1.0, 0.3, -0.2, 0.1, 1.0), U0=mg.cube_initial_state, steps100=True),
    # box with every boundary type: no-slip walls (BC_NoSlipWall, Numerics.cpp:59-66) at z = 0 and 1,
    # slip walls at y = 0 and 1, far field at x = 0 and 1
    "wallbox5": dict(mesh=lambda: mg.box_tet_mesh(5, 5, 5, jitter=0.1, seed=14,
                                                  side_patches={"imin": "farfield", "imax": "farfield",
                                                                "jmin": "slip", "jmax": "slip",
                                                                "kmin": "noslip", "kmax": "noslip"},
                                                  patch_types={"farfield": mg.FAR_FIELD, "slip": mg.SLIP_WALL,
                                                               "noslip": mg.NO_SLIP_WALL}),
                     fs=(1.0, 0.4, 0.1, -0.2, 1.0 / 1.4), U0=mg.cube_initial_state, steps100=True),
}


def marker_arrays(m: mg.TetMesh):
    names = np.array([n for n, _ in m.markers])
    types = np.array([mg.BC_CODES[m.patch_types[n]] for n, _ in m.markers], np.int32)
    offs = np.zeros(len(m.markers) + 1, np.int64)
    for i, (_, t) in enumerate(m.markers):
        offs[i + 1] = offs[i] + t.shape[0]
    tris = np.concatenate([t for _, t in m.markers], axis=0).astype(np.int64)
    return names, types, offs, tris


def make(name: str, spec: dict, tmp: str) -> None:
    m = spec["mesh"]()
    fs = spec["fs"]
    U0 = spec["U0"](m) if spec["U0"] is not None else mg.uniform_state(m.n_cells, fs)
    out = {}
    names, types, offs, tris = marker_arrays(m)
    out.update(nodes=m.nodes, tets=m.tets.astype(np.int64), marker_names=names, marker_types=types,
               marker_offsets=offs, marker_tris=tris, U0=U0, freestream=np.asarray(fs, np.float64))
    # one RK3 step (+ geometry), then 100 steps
    case = os.path.join(tmp, name + "_rk3")
    mg.write_case(case, m, fs, U0=U0, time_scheme="TVD_RK3")
    r1 = po.run_reference(case, 1, geometry=True)
    out.update(U1=r1["U"], dt1=r1["dt"])
    for k in ("face_ij", "S", "ri", "rj", "vol", "centroid", "dS", "patches"):
        out[k] = r1[k]
    if spec.get("steps100"):
        r100 = po.run_reference(case, 100)
        out.update(U100=r100["U"], dt100=r100["dt"])
    # one explicit-Euler step: the intermediates of its only stage
    case = os.path.join(tmp, name + "_euler")
    mg.write_case(case, m, fs, U0=U0, time_scheme="ExplicitEuler")
    re = po.run_reference(case, 1)
    out.update(euler_U=re["U"], euler_dt=re["dt"], euler_V=re["V"], euler_grad=re["grad"],
               euler_limiter=re["limiter"], euler_R=re["R"])
    # first order, no limiter
    case = os.path.join(tmp, name + "_first")
    mg.write_case(case, m, fs, U0=U0, time_scheme="TVD_RK3", spatial_order="First")
    rf = po.run_reference(case, 3)
    out.update(first_U3=rf["U"], first_dt3=rf["dt"])
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, m.n_cells, "cells,", out["face_ij"].shape[0], "faces")


def main() -> None:
    if not po.reference_available():
        raise SystemExit("oracle/_ref/nf_ref_nodump is not built (make -C oracle with the reference tree present)")
    names = sys.argv[1:] or list(CASES)
    unknown = [n for n in names if n not in CASES]
    if unknown:
        raise SystemExit(f"unknown case(s) {unknown}; known: {list(CASES)}")
    with tempfile.TemporaryDirectory() as tmp:
        for name in names:
            make(name, CASES[name], tmp)


if __name__ == "__main__":
    main()
