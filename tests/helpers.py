"""Helpers shared by the test modules."""
from __future__ import annotations

import os
from functools import lru_cache
from typing import Dict

import numpy as np

from netflux_b200 import meshgen as mg
from netflux_b200 import solver as S

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ("cube4", "sod40", "bump12", "slipbox5", "wallbox5")


@lru_cache(maxsize=None)
def golden(name: str) -> Dict[str, np.ndarray]:
    with np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


def tet_mesh(g) -> mg.TetMesh:
    names = [str(n) for n in g["marker_names"]]
    offs = g["marker_offsets"]
    markers = [(n, g["marker_tris"][offs[i]:offs[i + 1]]) for i, n in enumerate(names)]
    inv = {v: k for k, v in mg.BC_CODES.items()}
    types = {n: inv[int(t)] for n, t in zip(names, g["marker_types"])}
    return mg.TetMesh(nodes=g["nodes"], tets=g["tets"], markers=markers, patch_types=types)


def mesh(g) -> S.Mesh:
    return S.Mesh.from_tet_mesh(tet_mesh(g))


def rel_linf(a: np.ndarray, b: np.ndarray) -> float:
    """Relative L-infinity error, the worst over the conserved variables.

    For each variable: max over cells |a - b| divided by that variable's scale
    max |b|. The three momentum components share one scale, the largest
    momentum magnitude max ||rho u||: momentum is one vector variable, and a
    component that is zero up to round-off (the cross-flow momentum of a
    channel, the transverse momentum of a 1-D tube) has no scale of its own.
    Arrays that are not [N][5] states use a per-column scale.
    """
    a = np.asarray(a).reshape(b.shape[0], -1)
    b = np.asarray(b).reshape(b.shape[0], -1)
    scale = np.abs(b).max(axis=0)
    if b.shape[1] == 5:
        scale[1:4] = np.sqrt((b[:, 1:4] ** 2).sum(axis=1)).max()
    scale = np.maximum(scale, 1e-300)
    return float((np.abs(a - b).max(axis=0) / scale).max())


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


VARIABLES = ("rho", "rho_u", "rho_v", "rho_w", "E")


def per_variable(a: np.ndarray, b: np.ndarray) -> Dict[str, Dict[str, float]]:
    """Errors of each conserved variable on its own: relative L-infinity
    max|a_k - b_k| / max|b_k| and relative L2 ||a_k - b_k|| / ||b_k||, plus the
    absolute L-infinity. Unlike rel_linf, every momentum component is measured
    against its own scale, so a component that is nearly zero everywhere shows
    a large relative figure for round-off-sized absolute differences."""
    a = np.asarray(a).reshape(b.shape[0], -1)
    b = np.asarray(b).reshape(b.shape[0], -1)
    out = {}
    for k, name in enumerate(VARIABLES[: b.shape[1]]):
        d = a[:, k] - b[:, k]
        out[name] = {"rel_linf": float(np.abs(d).max() / max(np.abs(b[:, k]).max(), 1e-300)),
                     "rel_l2": float(np.linalg.norm(d) / max(np.linalg.norm(b[:, k]), 1e-300)),
                     "abs_linf": float(np.abs(d).max()),
                     "scale": float(np.abs(b[:, k]).max())}
    return out


def format_per_variable(errs: Dict[str, Dict[str, float]]) -> str:
    return "; ".join(f"{n}: Linf {e['rel_linf']:.2e} L2 {e['rel_l2']:.2e} (abs {e['abs_linf']:.1e}, "
                     f"scale {e['scale']:.1e})" for n, e in errs.items())


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def config_for(time_scheme="TVD_RK3", spatial_order="Second", limiter="Barth", precision="fp64", cfl=0.8,
               freestream=(1.0, 0.0, 0.0, 0.0, 1.0), **kw) -> S.Config:
    return S.Config(time_scheme=time_scheme, spatial_order=spatial_order, limiter=limiter, precision=precision,
                    CFL=cfl, density_fs=freestream[0], velocity_fs=list(freestream[1:4]),
                    pressure_fs=freestream[4], **kw)
