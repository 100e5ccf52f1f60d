"""Python access to the CPU checkers — ORACLE-ONLY TEST INFRASTRUCTURE.

Imported only by tests/, ``__graft_entry__.smoke()`` and bench.py's CPU
baseline leg, to check or time the product; never by the product itself.

* ``run_oracle``: the C restatement (oracle/nf_oracle.c, built into
  oracle/lib/libnf_oracle.so) on a face-based grid exported from a mesh.
* ``run_reference``: the NetFlux reference compiled from its own sources
  (oracle/_ref/nf_ref_nodump or nf_ref) on a case directory.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile
from typing import Dict, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "lib", "libnf_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")


class _Mesh(C.Structure):
    _fields_ = [("n_cells", C.c_int64), ("n_faces", C.c_int64), ("n_interior_faces", C.c_int64),
                ("face_ij", C.POINTER(C.c_uint32)), ("S", C.POINTER(C.c_double)), ("ri", C.POINTER(C.c_double)),
                ("rj", C.POINTER(C.c_double)), ("vol", C.POINTER(C.c_double)), ("dS", C.POINTER(C.c_double)),
                ("n_patches", C.c_int), ("patch_type", C.POINTER(C.c_int)), ("patch_first", C.POINTER(C.c_int64)),
                ("patch_n", C.POINTER(C.c_int64)), ("patch_fs", C.POINTER(C.c_double))]


class _Params(C.Structure):
    _fields_ = [("time_scheme", C.c_int), ("spatial_order", C.c_int), ("limiter", C.c_int),
                ("local_time_stepping", C.c_int), ("dt_from_current_state", C.c_int),
                ("cfl", C.c_double), ("t_end", C.c_double), ("limiter_ratchet_step", C.c_int64),
                ("farfield_density_fix", C.c_int), ("U_old_first", C.POINTER(C.c_double))]


_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_LIB):
            raise ImportError(f"{ORACLE_LIB} missing: run `make -C oracle`")
        _lib = C.CDLL(ORACLE_LIB)
        _lib.nfo_run.restype = C.c_int
        _lib.nfo_run.argtypes = [C.POINTER(_Mesh), C.POINTER(_Params), C.POINTER(C.c_double), C.c_int64] + \
            [C.POINTER(C.c_double)] * 7
        _lib.nfo_timestep_of.restype = C.c_int
        _lib.nfo_timestep_of.argtypes = [C.POINTER(_Mesh), C.POINTER(_Params), C.POINTER(C.c_double),
                                         C.POINTER(C.c_double), C.POINTER(C.c_double)]
        _lib.nfo_stage.restype = C.c_int
        _lib.nfo_stage.argtypes = [C.POINTER(_Mesh), C.POINTER(_Params), C.POINTER(C.c_double),
                                   C.POINTER(C.c_double), C.c_int, C.c_double, C.POINTER(C.c_double)]
    return _lib


def _dp(a: Optional[np.ndarray]):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


def run_oracle(grid: Dict[str, np.ndarray], patches: Sequence[dict], patch_fs: Sequence[Sequence[float]],
               U0: np.ndarray, n_steps: int, time_scheme: int = 1, spatial_order: int = 1, limiter: int = 1,
               cfl: float = 0.8, local_time_stepping: bool = False, dt_from_current_state: bool = False,
               t_end: float = 0.0, n_interior_faces: Optional[int] = None, fields: bool = True,
               limiter_ratchet_step: int = 0, farfield_density_fix: bool = False,
               U_old_first: Optional[np.ndarray] = None) -> Dict[str, np.ndarray]:
    """Run the C restatement; ``grid`` is Mesh.export() (reference order).

    ``limiter_ratchet_step`` > 0 (extension): from that step on every stage's Barth
    limiter is the minimum of its live value and the value kept so far."""
    lib = _load()
    F = grid["face_ij"].shape[0]
    NC = grid["dS"].shape[0]
    NG = grid["vol"].shape[0] - NC
    nif = F - NG if n_interior_faces is None else n_interior_faces
    keep = {k: np.ascontiguousarray(grid[k]) for k in ("face_ij", "S", "ri", "rj", "vol", "dS")}
    ptype = np.array([p["type"] for p in patches], np.int32)
    pfirst = np.array([p["first_face"] for p in patches], np.int64)
    pn = np.array([p["n_faces"] for p in patches], np.int64)
    pfs = np.ascontiguousarray(np.asarray(patch_fs, np.float64).reshape(len(patches), 5))
    m = _Mesh(NC, F, nif, keep["face_ij"].ctypes.data_as(C.POINTER(C.c_uint32)), _dp(keep["S"]), _dp(keep["ri"]),
              _dp(keep["rj"]), _dp(keep["vol"]), _dp(keep["dS"]), len(patches),
              ptype.ctypes.data_as(C.POINTER(C.c_int)), pfirst.ctypes.data_as(C.POINTER(C.c_int64)),
              pn.ctypes.data_as(C.POINTER(C.c_int64)), _dp(pfs))
    U_old = np.ascontiguousarray(U_old_first, np.float64) if U_old_first is not None else None  # kept alive
    p = _Params(time_scheme, spatial_order, limiter, int(local_time_stepping), int(dt_from_current_state), cfl, t_end,
                int(limiter_ratchet_step), int(farfield_density_fix), _dp(U_old))
    U = np.ascontiguousarray(U0, dtype=np.float64).copy()
    out = {"dt": np.zeros(max(n_steps, 1)), "res": np.zeros((max(n_steps, 1), 2)), "time": np.zeros(1)}
    if fields:
        out.update(V=np.zeros((NC + NG, 5)), grad=np.zeros((NC, 15)), limiter=np.zeros((NC, 5)), R=np.zeros((NC, 5)))
    rc = lib.nfo_run(C.byref(m), C.byref(p), _dp(U), n_steps, _dp(out["dt"]), _dp(out.get("V")),
                     _dp(out.get("grad")), _dp(out.get("limiter")), _dp(out.get("R")), _dp(out["res"]),
                     _dp(out["time"]))
    if rc != 0:
        raise RuntimeError(f"oracle failed with code {rc}")
    out["U"] = U
    out["dt"] = out["dt"][:n_steps]
    out["res"] = out["res"][:n_steps]
    out["time"] = float(out["time"][0])
    return out


class StageOracle:
    """Single stages of the C restatement on one grid (extension for tests that split a step across
    ranks and exchange halo states between stages): ``timestep`` is calc_timestep from the current
    state's primitives, ``stage`` one explicit-Euler / TVD-RK3 stage with a given dt."""

    def __init__(self, grid: Dict[str, np.ndarray], patches: Sequence[dict], patch_fs: Sequence[Sequence[float]],
                 time_scheme: int = 1, spatial_order: int = 1, limiter: int = 1, cfl: float = 0.8,
                 local_time_stepping: bool = False):
        self._lib = _load()
        F = grid["face_ij"].shape[0]
        self.NC = grid["dS"].shape[0]
        NG = grid["vol"].shape[0] - self.NC
        self._keep = {k: np.ascontiguousarray(grid[k]) for k in ("face_ij", "S", "ri", "rj", "vol", "dS")}
        self._ptype = np.array([p["type"] for p in patches], np.int32)
        self._pfirst = np.array([p["first_face"] for p in patches], np.int64)
        self._pn = np.array([p["n_faces"] for p in patches], np.int64)
        self._pfs = np.ascontiguousarray(np.asarray(patch_fs, np.float64).reshape(len(patches), 5))
        k = self._keep
        self._m = _Mesh(self.NC, F, F - NG, k["face_ij"].ctypes.data_as(C.POINTER(C.c_uint32)), _dp(k["S"]),
                        _dp(k["ri"]), _dp(k["rj"]), _dp(k["vol"]), _dp(k["dS"]), len(patches),
                        self._ptype.ctypes.data_as(C.POINTER(C.c_int)),
                        self._pfirst.ctypes.data_as(C.POINTER(C.c_int64)),
                        self._pn.ctypes.data_as(C.POINTER(C.c_int64)), _dp(self._pfs))
        self.lts = bool(local_time_stepping)
        self._p = _Params(time_scheme, spatial_order, limiter, int(local_time_stepping), 1, cfl, 0.0, 0, 0, None)

    def timestep(self, U: np.ndarray):
        """(global dt, per-cell dt or None) from the primitives of U."""
        U = np.ascontiguousarray(U, np.float64)
        dt = C.c_double()
        dtl = np.empty(self.NC) if self.lts else None
        rc = self._lib.nfo_timestep_of(C.byref(self._m), C.byref(self._p), _dp(U), C.byref(dt), _dp(dtl))
        if rc != 0:
            raise RuntimeError(f"oracle timestep failed with code {rc}")
        return dt.value, dtl

    def stage(self, U: np.ndarray, Un: np.ndarray, stage: int, dt: float, dtl: Optional[np.ndarray]) -> np.ndarray:
        out = np.ascontiguousarray(U, np.float64).copy()
        Un = np.ascontiguousarray(Un, np.float64)
        dtl = np.ascontiguousarray(dtl, np.float64) if dtl is not None else None
        rc = self._lib.nfo_stage(C.byref(self._m), C.byref(self._p), _dp(out), _dp(Un), int(stage), float(dt),
                                 _dp(dtl))
        if rc != 0:
            raise RuntimeError(f"oracle stage failed with code {rc}")
        return out


def reference_available(variant: str = "nf_ref_nodump") -> bool:
    return os.access(os.path.join(REF_DIR, variant), os.X_OK)


def run_reference(case_dir: str, n_steps: int, geometry: bool = False, variant: str = "nf_ref_nodump",
                  timeout: float = 3600.0) -> Dict[str, np.ndarray]:
    """Run the compiled reference on a case directory and read its dumps."""
    exe = os.path.join(REF_DIR, variant)
    if not os.access(exe, os.X_OK):
        raise FileNotFoundError(f"{exe} not built (make -C oracle)")
    with tempfile.TemporaryDirectory() as tmp:
        out_dir = os.path.join(tmp, "out")
        os.makedirs(out_dir)
        args = [exe, os.path.abspath(case_dir), out_dir, "--steps", str(n_steps), "--quiet"]
        if geometry:
            args.append("--geometry")
        subprocess.run(args, check=True, cwd=tmp, timeout=timeout)
        meta = {}
        with open(os.path.join(out_dir, "meta.txt")) as f:
            for line in f:
                k, v = line.split()
                meta[k] = float(v)
        NC, NT = int(meta["n_interior_cells"]), int(meta["n_total_cells"])
        res = {"meta": meta, "U": np.fromfile(os.path.join(out_dir, "U.f64")).reshape(NC, 5),
               "dt": np.fromfile(os.path.join(out_dir, "dt.f64"))}
        for name, shape in (("V", (NT, 5)), ("R", (NC, 5)), ("grad", (NC, 15)), ("limiter", (NC, 5))):
            path = os.path.join(out_dir, name + ".f64")
            if os.path.exists(path):
                res[name] = np.fromfile(path).reshape(shape)
        if geometry:
            res["face_ij"] = np.fromfile(os.path.join(out_dir, "face_ij.u32"), np.uint32).reshape(-1, 2)
            for k in ("S", "ri", "rj"):
                res[k] = np.fromfile(os.path.join(out_dir, f"face_{k}.f64")).reshape(-1, 3)
            res["vol"] = np.fromfile(os.path.join(out_dir, "cell_vol.f64"))
            res["centroid"] = np.fromfile(os.path.join(out_dir, "cell_centroid.f64")).reshape(-1, 3)
            res["dS"] = np.fromfile(os.path.join(out_dir, "cell_dS.f64")).reshape(-1, 3)[:NC]
            res["patches"] = np.fromfile(os.path.join(out_dir, "patches.u32"), np.uint32).reshape(-1, 3)
        return res
