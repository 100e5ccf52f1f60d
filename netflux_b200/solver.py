"""Host-side mirror of NetFlux's solver interface over the C ABI.

Same names and meaning as the reference's C++ classes for the step path:

* ``Config`` — the options of ``input.yml`` the step reads (Config.hpp:8-175,
  ConfigParser.cpp:38-131), plus the time bookkeeping Driver uses
  (get/set_delta_time, get/set_time, get/set_timestep).
* ``Mesh`` — PrimalGrid + FV_Grid: the face-based grid built once on the host
  from an SU2 file or arrays (PrimalGrid.cpp:140-244, FV_Grid.cpp:21-205).
* ``EulerSolver`` — ``calc_timestep(config)`` writes dt into the config and
  raises ``RuntimeError("Invalid dt calculated ...")`` like Solver.cpp:267-268;
  ``step(config)`` advances one step (Solver.cpp:34-52);
  ``get_solver_data()`` returns a ``SolverData`` view whose getters download
  the device fields in the reference's AoS layout.
* ``Driver`` — Driver::solve's loop (Driver.cpp:24-61) without VTK output.

Every call goes to the CUDA library; nothing here computes the step.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, Optional, Sequence

import numpy as np

from . import _lib as L
from .meshgen import BC_CODES, TetMesh

BOUNDARY_TYPES = {"NoSlipWall": L.NF_BC_NO_SLIP_WALL, "SlipWall": L.NF_BC_SLIP_WALL, "FarField": L.NF_BC_FAR_FIELD}
TIME_SCHEMES = {"ExplicitEuler": L.NF_EXPLICIT_EULER, "TVD_RK3": L.NF_TVD_RK3}
SPATIAL_ORDERS = {"First": L.NF_FIRST_ORDER, "Second": L.NF_SECOND_ORDER}
LIMITERS = {"NONE": L.NF_LIMITER_NONE, "Barth": L.NF_LIMITER_BARTH}
PRECISIONS = {"fp64_ref": L.NF_PREC_FP64_REF, "fp64": L.NF_PREC_FP64, "mixed": L.NF_PREC_MIXED,
              "mixed32": L.NF_PREC_MIXED32}
STANDARD_AIR = (1.225, 0.0, 0.0, 0.0, 101325.0)  # Utilities.hpp:100-107
# launch variants of the gradient and flux kernels each arithmetic form offers (the tuner's candidates)
LAUNCH_VARIANTS = {"fp64_ref": (10, 10), "fp64": (10, 10), "mixed": (10, 10), "mixed32": (10, 10)}


def _check(rc: int, handle=None) -> None:
    if rc != L.NF_OK:
        raise L.NetFluxError(rc, L.last_error(handle))


class Config:
    """Options of the step, as NetFlux's Config holds them.

    Build from a sim directory (parses ``<dir>/input.yml``) or from keywords.
    """

    def __init__(self, sim_dir: Optional[str] = None, **kw):
        opts: Dict[str, object] = {}
        if sim_dir is not None:
            import yaml
            with open(os.path.join(sim_dir, "input.yml")) as f:
                opts = yaml.safe_load(f) or {}
            self.sim_dir = sim_dir if sim_dir.endswith("/") else sim_dir + "/"
        else:
            self.sim_dir = ""
        opts.update(kw)
        for key in ("solver", "time_scheme", "inviscid_flux_scheme", "spatial_order", "initial_cond",
                    "n_timesteps", "CFL"):
            if key not in opts and not (key == "solver" and sim_dir is None):
                if sim_dir is not None:
                    raise RuntimeError(f'"{key}" not specified in the configuration file')
        if opts.get("solver", "Euler") != "Euler":
            raise RuntimeError("Error: Illegal solver type specified")
        self.time_scheme = TIME_SCHEMES[opts.get("time_scheme", "TVD_RK3")]
        if opts.get("inviscid_flux_scheme", "Rusanov") != "Rusanov":
            raise RuntimeError("only the Rusanov flux is implemented")
        self.spatial_order = SPATIAL_ORDERS[opts.get("spatial_order", "Second")]
        self.limiter = LIMITERS[opts.get("limiter", "Barth")] if self.spatial_order == L.NF_SECOND_ORDER else 0
        if self.spatial_order == L.NF_SECOND_ORDER and opts.get("grad_scheme", "GreenGauss") != "GreenGauss":
            raise RuntimeError("Illegal value for grad_scheme")
        vel = opts.get("velocity_fs", [0.0, 0.0, 0.0])
        self.primvars_inf = (float(opts.get("density_fs", STANDARD_AIR[0])), float(vel[0]), float(vel[1]),
                             float(vel[2]), float(opts.get("pressure_fs", STANDARD_AIR[4])))
        self.n_timesteps = int(opts.get("n_timesteps", 1))
        self.CFL = float(opts.get("CFL", 0.8))
        self.write_stride = int(opts.get("write_stride", 1))
        self.check_physical_validity_ = bool(opts.get("check_physical_validity", False))
        patches = opts.get("patches")
        self.patch_bc: Dict[str, int] = {}
        if patches is not None:
            for entry in patches:
                ((name, t),) = entry.items()
                if name in self.patch_bc:
                    raise RuntimeError(f'Duplicate patch name "{name}" specified in config file')
                if t not in BOUNDARY_TYPES:
                    raise RuntimeError(f"Illegal value '{t}' specified for setting 'patches: {name}'")
                self.patch_bc[name] = BOUNDARY_TYPES[t]
        elif sim_dir is not None:
            raise RuntimeError('"patches" option needs to be included in the config file')
        # extensions (not in the reference's input.yml)
        self.precision = PRECISIONS[opts.get("precision", "fp64")]
        self.local_time_stepping = bool(opts.get("local_time_stepping", False))
        self.t_end = float(opts.get("t_end", 0.0))
        self.patch_farfield: Dict[str, Sequence[float]] = dict(opts.get("patch_farfield", {}))
        # limiter ratchet: from this step on / once a case's residual drop reaches this value
        self.limiter_ratchet_step = int(opts.get("limiter_ratchet_step", 0))
        self.limiter_ratchet_drop = float(opts.get("limiter_ratchet_drop", 0.0))
        # physical far-field ghost density (the reference's is exact only for rho_fs = 1)
        self.farfield_density_fix = bool(opts.get("farfield_density_fix", False))
        self.delta_time = 0.0
        self.time = 0.0
        self.timestep = 0

    # Config.hpp getters/setters used on the step path
    def get_CFL(self) -> float: return self.CFL
    def get_delta_time(self) -> float: return self.delta_time
    def set_delta_time(self, v: float) -> None: self.delta_time = float(v)
    def get_time(self) -> float: return self.time
    def set_time(self, v: float) -> None: self.time = float(v)
    def get_timestep(self) -> int: return self.timestep
    def set_timestep(self, v: int) -> None: self.timestep = int(v)
    def get_n_timesteps(self) -> int: return self.n_timesteps
    def get_primvars_inf(self): return self.primvars_inf
    def get_time_scheme(self) -> int: return self.time_scheme
    def get_spatial_order(self) -> int: return self.spatial_order
    def get_limiter(self) -> int: return self.limiter
    def get_mesh_filename_path(self) -> str: return self.sim_dir + "mesh.su2"


class Mesh:
    """PrimalGrid + FV_Grid on the host, ready to upload."""

    def __init__(self, handle):
        if not handle:
            raise L.NetFluxError(L.NF_ERR_MESH, L.last_error(None))
        self._h = handle
        info = L.NfMeshInfo()
        _check(L.load().nf_mesh_get_info(self._h, C.byref(info)))
        self.info = info
        self.n_cells = int(info.n_interior_cells)
        self.n_faces = int(info.n_total_faces)
        self.n_interior_faces = int(info.n_interior_faces)
        self.n_ghost = int(info.n_ghost_cells)
        self.n_cases = int(info.n_cases)

    @classmethod
    def from_su2(cls, path: str, patch_bc: Dict[str, int]) -> "Mesh":
        names = list(patch_bc)
        arr_n = (C.c_char_p * len(names))(*[n.encode() for n in names])
        arr_t = (C.c_int * len(names))(*[int(patch_bc[n]) for n in names])
        return cls(L.load().nf_mesh_from_su2(path.encode(), len(names), arr_n, arr_t))

    @classmethod
    def from_tet_mesh(cls, m: TetMesh, device: Optional[int] = None) -> "Mesh":
        """Build the grid from a TetMesh on the host, or with ``device`` (a CUDA device ordinal, -1 the
        current one) on the GPU; both give the same grid bit for bit."""
        nodes = np.ascontiguousarray(m.nodes, dtype=np.float64)
        tets = np.ascontiguousarray(m.tets, dtype=np.int64)
        names = [n for n, _ in m.markers]
        types = [BC_CODES[m.patch_types[n]] for n in names]
        offs = np.zeros(len(names) + 1, np.int64)
        for i, (_, t) in enumerate(m.markers):
            offs[i + 1] = offs[i] + t.shape[0]
        tris = np.ascontiguousarray(np.concatenate([t for _, t in m.markers], axis=0) if names
                                    else np.zeros((0, 3)), dtype=np.int64)
        arr_n = (C.c_char_p * len(names))(*[n.encode() for n in names])
        arr_t = (C.c_int * len(names))(*types)
        args = (nodes.shape[0], L.dptr(nodes), tets.shape[0], L.i64ptr(tets), len(names), arr_n, arr_t,
                L.i64ptr(offs), L.i64ptr(tris))
        if device is None:
            return cls(L.load().nf_mesh_from_arrays(*args))
        return cls(L.load().nf_mesh_from_arrays_device(*args, int(device)))

    @classmethod
    def concat(cls, meshes: Sequence["Mesh"]) -> "Mesh":
        arr = (C.c_void_p * len(meshes))(*[m._h for m in meshes])
        return cls(L.load().nf_mesh_concat(len(meshes), arr))

    def patches(self):
        out = []
        lib = L.load()
        for p in range(int(self.info.n_patches)):
            t, cs = C.c_int(), C.c_int()
            ff, nfc = C.c_int64(), C.c_int64()
            buf = C.create_string_buffer(256)
            _check(lib.nf_mesh_get_patch(self._h, p, C.byref(t), C.byref(ff), C.byref(nfc), C.byref(cs), buf, 256))
            out.append({"type": t.value, "first_face": ff.value, "n_faces": nfc.value, "case": cs.value,
                        "name": buf.value.decode()})
        return out

    def export(self) -> Dict[str, np.ndarray]:
        """The face-based grid in the reference's order (FV_Grid accessors)."""
        F, NT, N = self.n_faces, self.n_cells + self.n_ghost, self.n_cells
        out = {"face_ij": np.empty((F, 2), np.uint32), "S": np.empty((F, 3)), "ri": np.empty((F, 3)),
               "rj": np.empty((F, 3)), "vol": np.empty(NT), "centroid": np.empty((NT, 3)), "dS": np.empty((N, 3))}
        _check(L.load().nf_mesh_export(self._h, L.u32ptr(out["face_ij"]), L.dptr(out["S"]), L.dptr(out["ri"]),
                                       L.dptr(out["rj"]), L.dptr(out["vol"]), L.dptr(out["centroid"]),
                                       L.dptr(out["dS"])))
        return out

    def permutation(self) -> np.ndarray:
        p = np.empty(self.n_cells, np.int64)
        _check(L.load().nf_mesh_get_permutation(self._h, L.i64ptr(p)))
        return p

    def case_offsets(self) -> np.ndarray:
        o = np.empty(self.n_cases + 1, np.int64)
        _check(L.load().nf_mesh_get_case_offsets(self._h, L.i64ptr(o)))
        return o

    def close(self):
        if self._h:
            L.load().nf_mesh_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def make_params(config: Config, mesh: Mesh, keep_stage_fields: bool = False,
                patch_states: Optional[Sequence[Sequence[float]]] = None,
                block_size: int = 0, variant: int = 0, device: int = -1) -> "tuple[L.NfParams, object]":
    """nf_params for ``config`` on ``mesh`` (the patch array is returned too, to keep it alive)."""
    p = L.NfParams()
    L.load().nf_params_default(C.byref(p))
    p.time_scheme = config.time_scheme
    p.spatial_order = config.spatial_order
    p.limiter = config.limiter
    p.flux_scheme = L.NF_FLUX_RUSANOV
    p.precision = config.precision
    p.local_time_stepping = int(config.local_time_stepping)
    p.keep_stage_fields = int(keep_stage_fields)
    p.cfl = config.CFL
    p.t_end = config.t_end
    p.block_size = int(block_size)
    p.kernel_variant = int(variant)
    p.limiter_ratchet_step = config.limiter_ratchet_step
    p.limiter_ratchet_drop = config.limiter_ratchet_drop
    p.farfield_density_fix = int(config.farfield_density_fix)
    p.device = int(device)
    for k in range(5):
        p.freestream[k] = config.primvars_inf[k]
    arr = None
    pats = mesh.patches()
    if patch_states is not None or config.patch_farfield or config.patch_bc:
        arr = (L.NfPatchBC * len(pats))()
        for i, pt in enumerate(pats):
            arr[i].type = config.patch_bc.get(pt["name"], pt["type"])
            st = None
            if patch_states is not None:
                st = patch_states[i]
            elif pt["name"] in config.patch_farfield:
                st = config.patch_farfield[pt["name"]]
            st = config.primvars_inf if st is None else st
            for k in range(5):
                arr[i].farfield[k] = float(st[k])
        p.patches = C.cast(arr, C.POINTER(L.NfPatchBC))
        p.n_patches = len(pats)
    return p, arr


class SolverData:
    """The reference's SolverData getters, downloading device fields on demand."""

    def __init__(self, solver: "EulerSolver"):
        self._s = solver

    def _field(self, which: int, comps: int) -> np.ndarray:
        n = self._s.n_cells
        out = np.empty((n, comps))
        _check(L.load().nf_get_field(self._s._h, which, L.dptr(out), out.size), self._s._h)
        return out

    def get_solution(self) -> np.ndarray: return self._field(L.NF_FIELD_SOLUTION, 5)
    def get_primvars(self) -> np.ndarray: return self._field(L.NF_FIELD_PRIMVARS, 5)
    def get_primvars_gradient(self) -> np.ndarray: return self._field(L.NF_FIELD_GRADIENT, 15)
    def get_primvars_limiter(self) -> np.ndarray: return self._field(L.NF_FIELD_LIMITER, 5)
    def get_flux_balance(self) -> np.ndarray: return self._field(L.NF_FIELD_FLUX_BALANCE, 5)
    def get_local_dt(self) -> np.ndarray: return self._field(L.NF_FIELD_LOCAL_DT, 1)[:, 0]


class EulerSolver:
    """EulerSolver(config, grid): the device solver for one (possibly batched) mesh."""

    def __init__(self, config: Config, mesh: Mesh, U0: Optional[np.ndarray] = None,
                 keep_stage_fields: bool = False, patch_states=None, block_size: int = 0, variant: int = 0,
                 device: int = -1):
        self.mesh = mesh
        self.config = config
        self.n_cells = mesh.n_cells
        params, self._patch_arr = make_params(config, mesh, keep_stage_fields, patch_states, block_size, variant,
                                              device)
        self._h = L.load().nf_create(mesh._h, C.byref(params))
        if not self._h:
            raise L.NetFluxError(L.NF_ERR_ARG, L.last_error(None))
        if U0 is None:
            # SolverData.cpp:50-58: freestream initial state
            from .meshgen import uniform_state
            U0 = uniform_state(self.n_cells, config.primvars_inf)
        self.set_state(U0)

    def set_state(self, U: np.ndarray) -> None:
        U = np.ascontiguousarray(U, dtype=np.float64)
        if U.shape != (self.n_cells, 5):
            raise ValueError("state must have shape (n_cells, 5)")
        _check(L.load().nf_set_state(self._h, L.dptr(U), self.n_cells), self._h)

    def set_state_old(self, U_old: np.ndarray) -> None:
        """U^n of the next RK3 step (the reference's solution_old); see nf_set_state_old."""
        U_old = np.ascontiguousarray(U_old, dtype=np.float64)
        if U_old.shape != (self.n_cells, 5):
            raise ValueError("state must have shape (n_cells, 5)")
        _check(L.load().nf_set_state_old(self._h, L.dptr(U_old), self.n_cells), self._h)

    def calc_timestep(self, config: Config) -> None:
        dt = C.c_double()
        rc = L.load().nf_calc_timestep(self._h, C.byref(dt))
        if rc == L.NF_ERR_DT:
            raise RuntimeError(f"Invalid dt calculated (dt = {dt.value:f})")
        _check(rc, self._h)
        config.set_delta_time(dt.value)

    def set_timestep(self, dt: float) -> None:
        _check(L.load().nf_set_timestep(self._h, float(dt)), self._h)

    def step(self, config: Optional[Config] = None) -> None:
        _check(L.load().nf_step(self._h), self._h)

    def advance(self, n_steps: int) -> float:
        t = C.c_double()
        _check(L.load().nf_advance(self._h, int(n_steps), C.byref(t)), self._h)
        return t.value

    def tune(self):
        """Time the gradient/flux launch shapes on the current state and keep the fastest."""
        cfg = (C.c_int * 4)()
        _check(L.load().nf_tune(self._h, cfg), self._h)
        return {"gradient": {"block": cfg[0], "variant": cfg[1]}, "flux": {"block": cfg[2], "variant": cfg[3]}}

    def set_launch_shapes(self, gradient=(64, 0), flux=(64, 0)):
        """Fix the gradient/flux launch shapes, each (block, variant) as tune() reports them."""
        cfg = (C.c_int * 4)(int(gradient[0]), int(gradient[1]), int(flux[0]), int(flux[1]))
        _check(L.load().nf_set_launch_shapes(self._h, cfg), self._h)

    def solve_steady(self, tol: float = 1e-6, max_steps: int = 100000, check_every: int = 50) -> dict:
        """Local-time-stepping steady solve to a relative density-residual drop of ``tol`` (per case)."""
        nc = self.mesh.n_cases
        steps = np.zeros(nc, np.int64)
        r0, r1, ms = np.zeros(nc), np.zeros(nc), np.zeros(nc)
        _check(L.load().nf_solve_steady(self._h, float(tol), int(max_steps), int(check_every), L.i64ptr(steps),
                                         L.dptr(r0), L.dptr(r1), L.dptr(ms)), self._h)
        # the library returns -(steps run) for a case that did not reach tol
        return {"steps": np.abs(steps), "converged": steps > 0, "res0": r0, "res": r1, "ms": ms}

    def solve_steady_to(self, res_target, max_steps: int = 100000, check_every: int = 50) -> dict:
        """Steady solve to an absolute density residual per case (see nf_solve_steady_to)."""
        nc = self.mesh.n_cases
        tgt = np.ascontiguousarray(np.broadcast_to(np.asarray(res_target, np.float64), (nc,)))
        steps = np.zeros(nc, np.int64)
        r0, r1, ms = np.zeros(nc), np.zeros(nc), np.zeros(nc)
        _check(L.load().nf_solve_steady_to(self._h, L.dptr(tgt), int(max_steps), int(check_every), L.i64ptr(steps),
                                            L.dptr(r0), L.dptr(r1), L.dptr(ms)), self._h)
        return {"steps": np.abs(steps), "converged": steps > 0, "res0": r0, "res": r1, "ms": ms}

    def synchronize(self) -> None:
        _check(L.load().nf_synchronize(self._h), self._h)

    def residual(self) -> np.ndarray:
        out = np.empty((self.mesh.n_cases, 2))
        _check(L.load().nf_get_residual(self._h, L.dptr(out), self.mesh.n_cases), self._h)
        return out

    def get_solver_data(self) -> SolverData:
        return SolverData(self)

    def snapshot_begin(self, out: np.ndarray) -> None:
        """Start copying the state (reference cell order) into ``out`` while later steps run;
        ``out`` is a C-contiguous float64 [n_cells][5] array (pinned memory, e.g. a pinned torch
        tensor's .numpy(), makes the copy asynchronous) and must not be read before snapshot_wait()."""
        if out.dtype != np.float64 or out.shape != (self.n_cells, 5) or not out.flags.c_contiguous:
            raise ValueError("snapshot buffer must be a C-contiguous float64 array of shape (n_cells, 5)")
        _check(L.load().nf_snapshot_begin(self._h, L.dptr(out), self.n_cells), self._h)
        self._snap = out  # kept alive while the copy runs

    def snapshot_wait(self) -> Optional[np.ndarray]:
        """Wait for the snapshot in flight and return its array (None when there was none)."""
        _check(L.load().nf_snapshot_wait(self._h), self._h)
        out, self._snap = getattr(self, "_snap", None), None
        return out

    def upload_begin(self, U: np.ndarray) -> None:
        """Start copying the state ``U`` (C-contiguous float64 [n_cells][5], reference order) to the
        device while queued work runs; ``U`` must not change before upload_wait()."""
        if U.dtype != np.float64 or U.shape != (self.n_cells, 5) or not U.flags.c_contiguous:
            raise ValueError("upload buffer must be a C-contiguous float64 array of shape (n_cells, 5)")
        _check(L.load().nf_upload_begin(self._h, L.dptr(U), self.n_cells), self._h)
        self._up = (getattr(self, "_up", None) or [])[-1:] + [U]  # kept alive while copies may run

    def upload_commit(self) -> None:
        """Make the uploaded state the solver's state (as set_state does), queued on the device
        after its copy; returns without waiting for the copy."""
        _check(L.load().nf_upload_commit(self._h), self._h)

    def upload_wait(self) -> None:
        """Wait until the last upload's copy has landed (its host buffer may change afterwards)."""
        _check(L.load().nf_upload_wait(self._h), self._h)
        self._up = None

    def close(self):
        if getattr(self, "_h", None):
            L.load().nf_destroy(self._h)  # waits for a snapshot or upload in flight
            self._h = None
        self._snap = None
        self._up = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Driver:
    """Driver::solve (Driver.cpp:24-61) for one solver: calc_timestep and step until n_timesteps.

    With ``write_output`` it also writes what NetFlux's Output writes: the VTK file of the state at
    step 0 and at every ``write_stride``-th step (Output::write_vtk_ascii, Output.cpp:17-45) into
    ``<sim_dir>/output/``, which it first empties as Output's constructor does (Output.cpp:3-14).

    Without ``U0`` it starts as NetFlux's program does: the free stream in ``solution`` and
    ``solution_old`` left at zero (SolverData.cpp:50-58), which the first TVD-RK3 step combines with
    (Solver.cpp:127-132). ``solver`` and ``tet_mesh`` may be given instead of being built from the
    configuration's SU2 file."""

    def __init__(self, config: Config, U0: Optional[np.ndarray] = None, write_output: bool = False,
                 solver=None, tet_mesh=None):
        from . import meshgen as mg
        self.config = config
        self.write_output = write_output
        if tet_mesh is None and write_output:
            types = {name: next(t for t, c in mg.BC_CODES.items() if c == code)
                     for name, code in config.patch_bc.items()}
            tet_mesh = mg.read_su2(config.get_mesh_filename_path(), types)
        self.tet_mesh = tet_mesh
        if solver is None:
            self.mesh = Mesh.from_su2(config.get_mesh_filename_path(), config.patch_bc)
            solver = EulerSolver(config, self.mesh, U0)
            if U0 is None:
                solver.set_state_old(np.zeros((self.mesh.n_cells, 5)))
        self.solver = solver
        if write_output:
            import shutil
            out = self.output_dir()
            if os.path.exists(out):
                shutil.rmtree(out)
            os.makedirs(out)

    def output_dir(self) -> str:
        return self.config.sim_dir + "output/"  # Config::get_output_dir (Config.hpp:106)

    def _write(self) -> None:
        cfg = self.config
        if not self.write_output or cfg.get_timestep() % cfg.write_stride != 0:
            return
        from . import output
        U = self.solver.get_solver_data().get_solution()
        output.write_vtk_ascii(output.vtk_filename(self.output_dir(), cfg.get_timestep()), self.tet_mesh.nodes,
                               self.tet_mesh.reader_tets(), U)

    def solve(self) -> None:
        cfg = self.config
        cfg.set_timestep(0)
        cfg.set_time(0.0)
        self._write()
        while True:
            self.solver.calc_timestep(cfg)
            self.solver.step(cfg)
            cfg.set_timestep(cfg.get_timestep() + 1)
            cfg.set_time(cfg.get_time() + cfg.get_delta_time())
            self._write()
            if cfg.get_timestep() >= cfg.get_n_timesteps():
                break
        self.solver.synchronize()
