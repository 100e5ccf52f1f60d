"""One mesh solved as parts on the GPU, with a halo exchange before every stage.

The cells are split along the Hilbert curve with two halo layers
(partition.partition) and every part runs on its own EulerSolver, on one
device or one device per part. Before every stage the primitives of each
part's halo cells are replaced by those of the cells' owners: the owner
gathers them on its device (nf_halo_pack), the buffer is copied to the
receiving part's device (a peer copy when the devices differ) and scattered
there (nf_halo_unpack). With two layers and an exchange per stage the owned
cells step exactly as in the undivided mesh (see partition.py). The time step
is each part's local dt (local time stepping) or, for a global dt, the
minimum over the parts, set on every part: a part's minimum covers its owned
and halo cells, whose primitives are the owners' after the exchange, so the
minimum over parts is the undivided mesh's.

The reference's MPI decomposition is a commented-out sketch
(src/parallelization/Decomposition.cpp:3-51, README.md:10 lists it as future
work); this is the device-side exchange for the Hilbert-range decomposition.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import _lib as L
from . import partition as P
from . import solver as S
from .meshgen import TetMesh


def _check(rc: int, handle) -> None:
    if rc != L.NF_OK:
        raise L.NetFluxError(rc, L.last_error(handle))


class SplitSolver:
    """``n_parts`` EulerSolvers over the Hilbert-range parts of ``mesh`` (devices[k] for part k, all on
    the current device by default). ``U0`` is the initial state in the mesh's cell order."""

    def __init__(self, config: S.Config, mesh: TetMesh, U0: np.ndarray, n_parts: int, layers: int = 2,
                 devices: Optional[Sequence[int]] = None, patch_states=None):
        import torch
        self.torch = torch
        self.config = config
        if layers < 2:
            raise ValueError("an exchange per stage needs two halo layers")
        whole = S.Mesh.from_tet_mesh(mesh)
        rank = whole.permutation()  # each cell's position along the Hilbert curve
        whole.close()
        self.n_cells = mesh.n_cells
        self.parts = P.partition(mesh, rank, n_parts, layers)
        self.plan = P.exchange_plan(self.parts)
        self.devices = list(devices) if devices is not None else [torch.cuda.current_device()] * n_parts
        if len(self.devices) != n_parts:
            raise ValueError("one device per part")
        U0 = np.ascontiguousarray(U0, np.float64)
        self.meshes: List[S.Mesh] = []
        self.solvers: List[S.EulerSolver] = []
        for k, part in enumerate(self.parts):
            m = S.Mesh.from_tet_mesh(part["mesh"])
            self.meshes.append(m)
            states = None if patch_states is None else [patch_states[pp["name"]] for pp in m.patches()]
            self.solvers.append(S.EulerSolver(config, m, U0=U0[part["cells"]], patch_states=states,
                                              device=self.devices[k]))
        # per (sender, receiver): device cell lists on both sides and a buffer on each device
        self.links = []
        for p, dests in self.plan.items():
            dev_p = self.meshes[p].permutation()
            for q, lists in dests.items():
                dev_q = self.meshes[q].permutation()
                n = int(lists["send"].size)
                dp, dq = f"cuda:{self.devices[p]}", f"cuda:{self.devices[q]}"
                self.links.append({
                    "p": p, "q": q, "n": n,
                    "send": torch.tensor(dev_p[lists["send"]], dtype=torch.int64, device=dp),
                    "recv": torch.tensor(dev_q[lists["recv"]], dtype=torch.int64, device=dq),
                    "buf_p": torch.empty((5, n), dtype=torch.float64, device=dp),
                    "buf_q": torch.empty((5, n), dtype=torch.float64, device=dq)})
        self.n_stages = 3 if config.get_time_scheme() == L.NF_TVD_RK3 else 1

    def exchange(self) -> None:
        """Every halo cell takes its owner's primitives (those the next stage reads)."""
        lib = L.load()
        for ln in self.links:
            sp, sq = self.solvers[ln["p"]], self.solvers[ln["q"]]
            _check(lib.nf_halo_pack(sp._h, C.c_void_p(ln["send"].data_ptr()), ln["n"],
                                    C.c_void_p(ln["buf_p"].data_ptr())), sp._h)
            ln["buf_q"].copy_(ln["buf_p"])  # device to device (peer copy across devices)
            self.torch.cuda.synchronize(ln["buf_q"].device)
            _check(lib.nf_halo_unpack(sq._h, C.c_void_p(ln["recv"].data_ptr()), ln["n"],
                                      C.c_void_p(ln["buf_q"].data_ptr())), sq._h)

    def calc_timestep(self) -> float:
        """Each part's time step; with a global dt their minimum, set on every part."""
        dts = []
        for s in self.solvers:
            s.calc_timestep(self.config)
            dts.append(self.config.get_delta_time())
        dt = min(dts)
        if not self.config.local_time_stepping:
            for s in self.solvers:
                s.set_timestep(dt)
        self.config.set_delta_time(dt)
        return dt

    def step(self) -> None:
        """calc_timestep, then every stage after a halo exchange."""
        lib = L.load()
        self.calc_timestep()
        for stage in range(self.n_stages):
            self.exchange()
            for s in self.solvers:
                _check(lib.nf_stage(s._h, stage), s._h)

    def advance(self, n_steps: int) -> None:
        for _ in range(n_steps):
            self.step()

    def get_solution(self) -> np.ndarray:
        """The owned cells' states, in the mesh's cell order."""
        U = np.empty((self.n_cells, 5))
        for part, s in zip(self.parts, self.solvers):
            Up = s.get_solver_data().get_solution()
            n = part["n_owned"]
            U[part["cells"][:n]] = Up[:n]
        return U

    def close(self) -> None:
        for s in self.solvers:
            s.close()
        for m in self.meshes:
            m.close()
        self.solvers, self.meshes, self.links = [], [], []
