"""One mesh solved as parts on the GPU, with a halo exchange before every stage.

The cells are split along the Hilbert curve with two halo layers
(partition.partition) and every part runs on its own EulerSolver, on one
device or one device per part. The library steps the parts together
(nf_split_*): before every stage each halo cell takes its owner's primitives
and conserved stage input, written by a kernel on the receiving part's stream
that reads the owner's buffers (on the same GPU, or on a peer GPU over
NVLink), with the parts' streams ordered by events, so the host waits on
nothing inside a step.
The time step is each part's local dt (local time stepping) or, for a global
dt, the minimum over the parts, reduced on the device into every part: a
part's minimum covers its owned and halo cells, whose primitives are the
owners' after the exchange, so the minimum over parts is the undivided mesh's.
With two layers and an exchange per stage the owned cells step exactly as in
the undivided mesh (see partition.py).

The reference's MPI decomposition is a commented-out sketch
(src/parallelization/Decomposition.cpp:3-51, README.md:10 lists it as future
work); this is the device-side exchange for the Hilbert-range decomposition.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence

import numpy as np

from . import _lib as L
from . import partition as P
from . import solver as S
from .meshgen import TetMesh


CUT_MARKER = "halo_cut"


class SplitSolver:
    """``n_parts`` EulerSolvers over the Hilbert-range parts of ``mesh`` (devices[k] for part k, all on
    the current device by default). ``U0`` is the initial state in the mesh's cell order.
    ``exchange=False`` leaves the halos unexchanged (each part then steps on its own)."""

    def __init__(self, config: S.Config, mesh: TetMesh, U0: np.ndarray, n_parts: int, layers: int = 2,
                 devices: Optional[Sequence[int]] = None, patch_states=None, exchange: bool = True):
        if layers < 2:
            raise ValueError("an exchange per stage needs two halo layers")
        self.config = config
        whole = S.Mesh.from_tet_mesh(mesh)
        rank = whole.permutation()  # each cell's position along the Hilbert curve
        whole.close()
        self.n_cells = mesh.n_cells
        # the cut faces of each part as a far field at the free stream: the outermost halo cells'
        # updates (overwritten by the exchange) stay physical, so the parts' validity checks report
        # only real failures
        self.parts = P.partition(mesh, rank, n_parts, layers, cut_marker=CUT_MARKER)
        self.plan = P.exchange_plan(self.parts)
        if devices is None:
            import torch
            devices = [torch.cuda.current_device()] * n_parts
        self.devices = list(devices)
        if len(self.devices) != n_parts:
            raise ValueError("one device per part")
        U0 = np.ascontiguousarray(U0, np.float64)
        self.meshes: List[S.Mesh] = []
        self.solvers: List[S.EulerSolver] = []
        for k, part in enumerate(self.parts):
            m = S.Mesh.from_tet_mesh(part["mesh"])
            self.meshes.append(m)
            states = None if patch_states is None else [patch_states.get(pp["name"]) for pp in m.patches()]
            self.solvers.append(S.EulerSolver(config, m, U0=U0[part["cells"]], patch_states=states,
                                              device=self.devices[k]))
        lib = L.load()
        handles = (C.c_void_p * n_parts)(*[s._h for s in self.solvers])
        self._h = lib.nf_split_create(handles, n_parts)
        if not self._h:
            raise L.NetFluxError(L.NF_ERR_ARG, lib.nf_split_last_error(None).decode())
        self.n_halo_values = 0
        if exchange:
            # the plan in each part's device numbering
            perm = [m.permutation() for m in self.meshes]
            for p, dests in self.plan.items():
                for q, lists in dests.items():
                    a = np.ascontiguousarray(perm[p][lists["send"]], np.int64)
                    b = np.ascontiguousarray(perm[q][lists["recv"]], np.int64)
                    self._check(lib.nf_split_link(self._h, p, q, L.i64ptr(a), L.i64ptr(b), a.size))
                    self.n_halo_values += 5 * a.size

    def _check(self, rc: int) -> None:
        if rc != L.NF_OK:
            raise L.NetFluxError(rc, L.load().nf_split_last_error(self._h).decode())

    def step(self) -> None:
        """calc_timestep, then every stage after a halo exchange (queued on the devices)."""
        self.advance(1)

    def advance(self, n_steps: int) -> None:
        self._check(L.load().nf_split_advance(self._h, n_steps))

    def synchronize(self) -> None:
        """Wait for every part; raises on the first part whose status reports a failure."""
        self._check(L.load().nf_split_synchronize(self._h))

    def get_solution(self) -> np.ndarray:
        """The owned cells' states, in the mesh's cell order."""
        self.synchronize()
        U = np.empty((self.n_cells, 5))
        for part, s in zip(self.parts, self.solvers):
            Up = s.get_solver_data().get_solution()
            n = part["n_owned"]
            U[part["cells"][:n]] = Up[:n]
        return U

    def close(self) -> None:
        if getattr(self, "_h", None):
            L.load().nf_split_destroy(self._h)
            self._h = None
        for s in self.solvers:
            s.close()
        for m in self.meshes:
            m.close()
        self.solvers, self.meshes = [], []
