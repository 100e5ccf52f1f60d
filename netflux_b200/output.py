"""Solution output for the Python side of the library.

``write_vtk_ascii`` writes the legacy ASCII VTK file that NetFlux's ``Output``
writes every ``write_stride`` steps (Output.cpp:17-110, file name
``n=<timestep>.vtk``, Config.hpp:108):

- the grid: ``POINTS`` in file order, ``CELLS`` with each tetrahedron's
  vertices in the reader's order (vertices 1 and 2 of the SU2 element swapped,
  GeometryUtilities.cpp:443-466), ``CELL_TYPES`` 10;
- per cell, ``density``, ``velocity`` (ρu/ρ, ρv/ρ, ρw/ρ) and ``pressure``
  ((γ−1)(E − 0.5/ρ·|ρu|²), SolverData.hpp:194-201, in that operation order).

Every number is printed as a C++ stream prints a double at its default
precision (``%g``, 6 significant digits), so the text equals the reference
program's for the same state.

``EulerSolver.snapshot_begin`` pairs with it: it starts a copy of the state
into host memory on a side stream while the solver keeps stepping, and
``snapshot_wait`` returns it, so output need not stall the step loop.
``save_restart`` / ``load_restart`` keep a state with its step count and time.
"""
from typing import Optional

import numpy as np

GAMMA_MINUS_ONE = 0.4
VTK_TETRA = 10


def vtk_filename(output_dir: str, timestep: int) -> str:
    """The reference's name for the file of a time step (Config.hpp:108)."""
    return output_dir + "n=" + str(int(timestep)) + ".vtk"


def _g(a: np.ndarray) -> list:
    return ["%g" % x for x in np.asarray(a, dtype=np.float64).ravel()]


def write_vtk_ascii(path: str, nodes: np.ndarray, reader_tets: np.ndarray, U: np.ndarray,
                    scalar_name: str = "double", gamma_minus_one: float = GAMMA_MINUS_ONE) -> None:
    """Write the grid and the cell fields of the conserved state ``U`` [n_cells][5] (reference cell
    order). ``reader_tets`` holds each cell's vertices in the reader's order
    (``TetMesh.reader_tets()``)."""
    nodes = np.asarray(nodes, dtype=np.float64)
    t = np.asarray(reader_tets, dtype=np.int64)
    U = np.asarray(U, dtype=np.float64)
    n_nodes, n_cells = nodes.shape[0], t.shape[0]
    if U.shape != (n_cells, 5):
        raise ValueError("state must have shape (n_cells, 5)")
    rho, m1, m2, m3, E = (U[:, k] for k in range(5))
    p = gamma_minus_one * (E - 0.5 / rho * ((m1 * m1 + m2 * m2) + m3 * m3))
    out = ["# vtk DataFile Version 3.0\nNetFlux\nASCII\n\nDATASET UNSTRUCTURED_GRID\n\n",
           f"POINTS {n_nodes} {scalar_name}\n"]
    xyz = _g(nodes[:, :3])
    out.extend(f"{xyz[3 * i]} {xyz[3 * i + 1]} {xyz[3 * i + 2]}\n" for i in range(n_nodes))
    out.append(f"\nCELLS {n_cells} {n_cells + 4 * n_cells}\n")
    out.extend("4 " + "".join(f"{v} " for v in row) + "\n" for row in t.tolist())
    out.append(f"\nCELL_TYPES {n_cells}\n")
    out.append(f"{VTK_TETRA}\n" * n_cells)
    out.append(f"\nCELL_DATA {n_cells}\n")
    out.append(f"\nSCALARS density {scalar_name} 1\nLOOKUP_TABLE default\n")
    out.extend(s + "\n" for s in _g(rho))
    out.append(f"\nVECTORS velocity {scalar_name}\n")
    vel = _g(np.column_stack([m1 / rho, m2 / rho, m3 / rho]))
    out.extend(f"{vel[3 * i]} {vel[3 * i + 1]} {vel[3 * i + 2]}\n" for i in range(n_cells))
    out.append(f"\nSCALARS pressure {scalar_name} 1\nLOOKUP_TABLE default\n")
    out.extend(s + "\n" for s in _g(p))
    with open(path, "w") as f:
        f.write("".join(out))


def mesh_fingerprint(mesh) -> str:
    """SHA-256 of a Mesh's face grid in the reference's order (face cell pairs, face normals and cell
    volumes) and its case offsets: two meshes with the same fingerprint give the same step."""
    import hashlib
    g = mesh.export()
    h = hashlib.sha256()
    for k in ("face_ij", "S", "vol"):
        h.update(np.ascontiguousarray(g[k]).tobytes())
    h.update(np.ascontiguousarray(mesh.case_offsets(), np.int64).tobytes())
    return h.hexdigest()


def save_restart(path: str, U: np.ndarray, timestep: int, time: float = 0.0, mesh=None) -> None:
    """A restart file: the conserved state [n_cells][5] (reference cell order), the step count and
    the simulated time; with ``mesh`` (a solver.Mesh) also its fingerprint and case offsets, which
    load_restart checks. Restoring it with set_state is exact in U; the first time step after it is
    computed from the restored state's primitives, where an uninterrupted run uses the last stage
    input's (NetFlux's calc_timestep reads the primitives of the last stage), so the two runs
    differ from there at the size of one step's change in dt."""
    U = np.ascontiguousarray(U, dtype=np.float64)
    if U.ndim != 2 or U.shape[1] != 5:
        raise ValueError("state must have shape (n_cells, 5)")
    extra = {}
    if mesh is not None:
        if mesh.n_cells != U.shape[0]:
            raise ValueError("state size does not match the mesh")
        extra = {"mesh_sha256": np.array(mesh_fingerprint(mesh)),
                 "case_offsets": np.ascontiguousarray(mesh.case_offsets(), np.int64)}
    with open(path, "wb") as f:
        np.savez(f, U=U, timestep=np.int64(timestep), time=np.float64(time), format=np.int64(2), **extra)


def load_restart(path: str, mesh=None) -> dict:
    """Read a restart file; with ``mesh`` the file must have been written for that mesh (same
    fingerprint and case offsets, when the file records them) or ValueError is raised."""
    with np.load(path, allow_pickle=False) as z:
        if int(z["format"]) not in (1, 2):
            raise ValueError("unknown restart format")
        out = {"U": z["U"].copy(), "timestep": int(z["timestep"]), "time": float(z["time"])}
        if "mesh_sha256" in z.files:
            out["mesh_sha256"] = str(z["mesh_sha256"])
            out["case_offsets"] = z["case_offsets"].copy()
    if mesh is not None:
        if out["U"].shape[0] != mesh.n_cells:
            raise ValueError("restart file was written for a mesh of another size")
        if "mesh_sha256" in out and out["mesh_sha256"] != mesh_fingerprint(mesh):
            raise ValueError("restart file was written for a different mesh")
    return out


def write_solver_vtk(path: str, mesh, solver, U: Optional[np.ndarray] = None) -> None:
    """Write a solver's current state (or ``U``) on the TetMesh it was built from."""
    if U is None:
        U = solver.get_solver_data().get_solution()
    write_vtk_ascii(path, mesh.nodes, mesh.reader_tets(), U)
