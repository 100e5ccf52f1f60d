"""Synthetic tetrahedral meshes and case directories for the NetFlux Euler step.

Every workload here is generated, not downloaded: a structured nx*ny*nz hex grid
is cut into 6 tetrahedra per hex (a conforming split around the main diagonal
of each hex), optionally jittered and mapped, and written as an SU2 file in the
exact dialect the NetFlux reader accepts:

* ``NDIME= 3`` / ``NELEM= n`` / ``NPOIN= n`` / ``NMARK= n`` / ``MARKER_TAG= x`` /
  ``MARKER_ELEMS= n`` with a space after each ``=`` (PrimalGrid.cpp:158-219
  reads the tag and the integer as two tokens).
* Point lines hold exactly ``x y z`` with no trailing point index, because the
  reader does not skip to the end of a point line (PrimalGrid.cpp:195-200).
* Tets are written so that the reader's 1<->2 node swap
  (GeometryUtilities.cpp:452-455) leaves them with a positive signed volume
  (GeometryUtilities.cpp:307).
* Every boundary triangle belongs to exactly one marker (FV_Grid.cpp:93-115
  drops uncovered faces silently).

Coordinates are written with 17 significant digits so the text round-trips to
the identical doubles.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

GAMMA = 1.4

# Boundary types by the names NetFlux's input.yml uses (Utilities.hpp:76-80).
SLIP_WALL = "SlipWall"
NO_SLIP_WALL = "NoSlipWall"
FAR_FIELD = "FarField"
BC_CODES = {NO_SLIP_WALL: 0, SLIP_WALL: 1, FAR_FIELD: 2}


@dataclasses.dataclass
class TetMesh:
    """A tetrahedral mesh in the order it is written to the SU2 file.

    ``tets`` holds node ids as written (before the reader's 1<->2 swap);
    ``markers`` is a list of (name, (K,3) triangle node ids) in file order;
    ``patch_types`` maps each marker name to its boundary type string.
    """

    nodes: np.ndarray
    tets: np.ndarray
    markers: List[Tuple[str, np.ndarray]]
    patch_types: Dict[str, str]
    shape: Tuple[int, int, int] = (0, 0, 0)

    @property
    def n_cells(self) -> int:
        return int(self.tets.shape[0])

    @property
    def n_boundary_faces(self) -> int:
        return int(sum(t.shape[0] for _, t in self.markers))

    def reader_tets(self) -> np.ndarray:
        """Tets in the node order NetFlux uses after reading (nodes 1 and 2 swapped)."""
        return self.tets[:, [0, 2, 1, 3]]

    def centroids(self) -> np.ndarray:
        """Cell centroids with the reference's summation order.

        tetrahedron_calc_centroid (GeometryUtilities.cpp:313-316) computes
        1/4 * (n0 + n1 + n2 + n3) on the post-swap node order.
        """
        t = self.reader_tets()
        n = self.nodes
        return 0.25 * (((n[t[:, 0]] + n[t[:, 1]]) + n[t[:, 2]]) + n[t[:, 3]])


# The six tets of the conforming split of the unit hex: each walks from corner
# (0,0,0) to corner (1,1,1) along the axes in one of the 6 orders.
_PERMS = ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0))


def _hex_split_tets(nx: int, ny: int, nz: int) -> Tuple[np.ndarray, np.ndarray]:
    """Node ids of the 6*nx*ny*nz tets and the logical (i,j,k) of every node.

    Node (i,j,k) has id i + (nx+1)*(j + (ny+1)*k). Tets are ordered hex by hex
    (i fastest), six per hex.
    """
    sx, sy = nx + 1, (nx + 1) * (ny + 1)
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    base = (i + sx * j + sy * k).transpose(2, 1, 0).reshape(-1)  # i fastest
    step = (1, sx, sy)
    tets = np.empty((base.size, 6, 4), dtype=np.int64)
    for p, perm in enumerate(_PERMS):
        a = base
        b = a + step[perm[0]]
        c = b + step[perm[1]]
        d = base + 1 + sx + sy
        tets[:, p, 0], tets[:, p, 1], tets[:, p, 2], tets[:, p, 3] = a, b, c, d
    tets = tets.reshape(-1, 4)
    ni, nj, nk = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    logical = np.stack([ni.transpose(2, 1, 0).reshape(-1), nj.transpose(2, 1, 0).reshape(-1),
                        nk.transpose(2, 1, 0).reshape(-1)], axis=1)
    return tets, logical


def _orient_for_reader(nodes: np.ndarray, tets: np.ndarray) -> np.ndarray:
    """Return tets whose signed volume is positive after the reader's 1<->2 swap."""
    a, b, c, d = (nodes[tets[:, q]] for q in range(4))
    det = np.einsum("ij,ij->i", np.cross(b - a, c - a), d - a)
    if np.any(det == 0.0):
        raise ValueError("degenerate tetrahedron in generated mesh")
    out = tets.copy()
    pos = det > 0.0  # written order must be negatively oriented
    out[pos, 1], out[pos, 2] = tets[pos, 2], tets[pos, 1]
    return out


_TET_FACES = ((0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3))


def _boundary_triangles(tets: np.ndarray, logical: np.ndarray, dims: Sequence[int]) -> Dict[str, np.ndarray]:
    """Boundary triangles of the hex-split mesh grouped by box side.

    Keys: 'imin','imax','jmin','jmax','kmin','kmax'. Triangles keep the tet's
    local face node order and appear in tet order.
    """
    out: Dict[str, List[np.ndarray]] = {s: [] for s in ("imin", "imax", "jmin", "jmax", "kmin", "kmax")}
    names = (("imin", "imax"), ("jmin", "jmax"), ("kmin", "kmax"))
    faces = np.stack([tets[:, list(f)] for f in _TET_FACES], axis=1)  # (N,4,3)
    flat = faces.reshape(-1, 3)
    for ax in range(3):
        lg = logical[flat, ax]  # (F,3)
        for side, val in ((0, 0), (1, dims[ax])):
            on = np.all(lg == val, axis=1)
            out[names[ax][side]].append(flat[on])
    return {k: np.concatenate(v, axis=0) if v else np.zeros((0, 3), np.int64) for k, v in out.items()}


def box_tet_mesh(nx: int, ny: int, nz: int,
                 lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0),
                 jitter: float = 0.0, seed: int = 0,
                 side_patches: Optional[Dict[str, str]] = None,
                 patch_types: Optional[Dict[str, str]] = None,
                 y_wall=None) -> TetMesh:
    """Hex-split tet mesh of a box.

    ``jitter`` moves every interior node by U(-jitter, jitter) times the grid
    spacing in each direction (numpy PCG64 with ``seed``). ``side_patches``
    maps the six box sides to marker names (several sides may share one
    name). ``y_wall(x)`` maps nodes vertically: y = yw(x) + (hi_y - yw(x)) * eta.
    """
    tets, logical = _hex_split_tets(nx, ny, nz)
    dims = (nx, ny, nz)
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    h = (hi - lo) / np.asarray(dims, np.float64)
    nodes = lo + logical.astype(np.float64) * h
    # exact end coordinates (avoid lo + n*h rounding on the far faces)
    for ax in range(3):
        nodes[logical[:, ax] == dims[ax], ax] = hi[ax]
    if jitter > 0.0:
        rng = np.random.Generator(np.random.PCG64(seed))
        interior = np.all((logical > 0) & (logical < np.asarray(dims)), axis=1)
        disp = rng.uniform(-jitter, jitter, size=(int(interior.sum()), 3)) * h
        nodes[interior] += disp
    if y_wall is not None:
        eta = logical[:, 1].astype(np.float64) / ny
        yw = y_wall(nodes[:, 0])
        nodes[:, 1] = yw + (hi[1] - yw) * eta
        nodes[logical[:, 1] == ny, 1] = hi[1]
    tets = _orient_for_reader(nodes, tets)
    sides = _boundary_triangles(tets, logical, dims)
    if side_patches is None:
        side_patches = {s: "farfield" for s in sides}
    markers: List[Tuple[str, np.ndarray]] = []
    order: List[str] = []
    for s in ("imin", "imax", "jmin", "jmax", "kmin", "kmax"):
        name = side_patches[s]
        if name not in order:
            order.append(name)
    for name in order:
        tris = [sides[s] for s in ("imin", "imax", "jmin", "jmax", "kmin", "kmax") if side_patches[s] == name]
        markers.append((name, np.concatenate(tris, axis=0)))
    if patch_types is None:
        patch_types = {name: FAR_FIELD for name in order}
    return TetMesh(nodes=nodes, tets=tets, markers=markers, patch_types=dict(patch_types), shape=(nx, ny, nz))


# ---------------------------------------------------------------------------
# The benchmark cases (unit cube bump, Sod tube, bump channel)
# ---------------------------------------------------------------------------

def cube_mesh(n: int = 20, jitter: float = 0.1, seed: int = 1234) -> TetMesh:
    """Unit cube, n^3 hexes * 6 tets, interior jitter, one farfield marker."""
    return box_tet_mesh(n, n, n, jitter=jitter, seed=seed,
                        side_patches={s: "farfield" for s in ("imin", "imax", "jmin", "jmax", "kmin", "kmax")},
                        patch_types={"farfield": FAR_FIELD})


def cube_initial_state(mesh: TetMesh, amp: float = 0.1, sigma: float = 0.1,
                       u=(0.5, 0.0, 0.0), p: float = 1.0 / GAMMA) -> np.ndarray:
    """rho = 1 + amp*exp(-|x-c|^2/(2 sigma^2)), p = 1/gamma, u = (0.5,0,0) at cell centroids."""
    c = mesh.centroids()
    r2 = np.sum((c - 0.5) ** 2, axis=1)
    rho = 1.0 + amp * np.exp(-r2 / (2.0 * sigma * sigma))
    V = np.empty((mesh.n_cells, 5))
    V[:, 0] = rho
    V[:, 1:4] = np.asarray(u, np.float64)
    V[:, 4] = p
    return prim_to_cons(V)


def sod_mesh(nx: int = 400, ny: int = 8, nz: int = 8, jitter: float = 0.05, seed: int = 4321) -> TetMesh:
    """Channel [0,1]x[0,0.1]x[0,0.1]; slip side walls, farfield ends."""
    return box_tet_mesh(nx, ny, nz, hi=(1.0, 0.1, 0.1), jitter=jitter, seed=seed,
                        side_patches={"imin": "left", "imax": "right", "jmin": "sides",
                                      "jmax": "sides", "kmin": "sides", "kmax": "sides"},
                        patch_types={"left": FAR_FIELD, "right": FAR_FIELD, "sides": SLIP_WALL})


SOD_LEFT = (1.0, 0.0, 0.0, 0.0, 1.0)
SOD_RIGHT = (0.125, 0.0, 0.0, 0.0, 0.1)


def sod_initial_state(mesh: TetMesh, x0: float = 0.5) -> np.ndarray:
    c = mesh.centroids()
    V = np.where((c[:, 0] < x0)[:, None], np.asarray(SOD_LEFT), np.asarray(SOD_RIGHT))
    return prim_to_cons(V)


def bump_wall(h: float):
    """Lower wall y = h*sin^2(pi*(x-1)) on 1<=x<=2, zero elsewhere."""
    def yw(x):
        s = np.sin(np.pi * (x - 1.0))
        return np.where((x >= 1.0) & (x <= 2.0), h * s * s, 0.0)
    return yw


def bump_mesh(nx: int = 128, ny: int = 64, nz: int = 64, h: float = 0.1) -> TetMesh:
    """Bump channel [0,3]x[0,1]x[0,1]: slip bump/upper/sides, farfield inflow/outflow."""
    return box_tet_mesh(nx, ny, nz, hi=(3.0, 1.0, 1.0), y_wall=bump_wall(h),
                        side_patches={"imin": "inflow", "imax": "outflow", "jmin": "bump",
                                      "jmax": "upper", "kmin": "sides", "kmax": "sides"},
                        patch_types={"inflow": FAR_FIELD, "outflow": FAR_FIELD, "bump": SLIP_WALL,
                                     "upper": SLIP_WALL, "sides": SLIP_WALL})


def bump_freestream(mach: float = 0.5, rho: float = 1.0, p: float = 1.0 / GAMMA) -> Tuple[float, ...]:
    c = math.sqrt(GAMMA * p / rho)
    return (rho, mach * c, 0.0, 0.0, p)


def uniform_state(n_cells: int, V) -> np.ndarray:
    return prim_to_cons(np.broadcast_to(np.asarray(V, np.float64), (n_cells, 5)).copy())


def prim_to_cons(V: np.ndarray) -> np.ndarray:
    """EulerEqs::prim_to_cons (SolverData.hpp:165-177) with its expression order."""
    g1 = GAMMA - 1.0
    g1i = 1.0 / g1
    U = np.empty_like(V)
    U[:, 0] = V[:, 0]
    U[:, 1] = V[:, 0] * V[:, 1]
    U[:, 2] = V[:, 0] * V[:, 2]
    U[:, 3] = V[:, 0] * V[:, 3]
    U[:, 4] = g1i * V[:, 4] + (0.5 * V[:, 0]) * ((V[:, 1] * V[:, 1] + V[:, 2] * V[:, 2]) + V[:, 3] * V[:, 3])
    return U


# ---------------------------------------------------------------------------
# SU2 and input.yml writers
# ---------------------------------------------------------------------------

def _fmt_rows(arr: np.ndarray, prefix: str = "", float_rows: bool = False) -> str:
    if float_rows:
        return "\n".join(" ".join(repr(float(v)) for v in row) for row in arr.tolist())
    lines = [prefix + " ".join(str(v) for v in row) for row in arr.tolist()]
    return "\n".join(lines)


def write_su2(path: str, mesh: TetMesh) -> None:
    """Write ``mesh`` as SU2 text that NetFlux's reader accepts unchanged."""
    with open(path, "w") as f:
        f.write("NDIME= 3\n")
        f.write(f"NELEM= {mesh.n_cells}\n")
        if mesh.n_cells:
            f.write(_fmt_rows(mesh.tets, prefix="10 "))
            f.write("\n")
        f.write(f"NPOIN= {mesh.nodes.shape[0]}\n")
        f.write(_fmt_rows(mesh.nodes, float_rows=True))
        f.write("\n")
        f.write(f"NMARK= {len(mesh.markers)}\n")
        for name, tris in mesh.markers:
            f.write(f"MARKER_TAG= {name}\n")
            f.write(f"MARKER_ELEMS= {tris.shape[0]}\n")
            if tris.shape[0]:
                f.write(_fmt_rows(tris, prefix="5 "))
                f.write("\n")


def read_su2(path: str, patch_types: Dict[str, str]) -> TetMesh:
    """Read an SU2 tetrahedral mesh as NetFlux's reader does (PrimalGrid.cpp:140-244): element lines
    are "10 n0 n1 n2 n3" with anything after the nodes ignored, node coordinates are read as a
    stream of three numbers per node, and marker elements are "5 n0 n1 n2" triangles. Only
    tetrahedra are accepted (other volume elements are rejected, as in this library's builder).
    ``patch_types`` maps every marker name to its boundary type ("FarField", "SlipWall",
    "NoSlipWall"); the TetMesh keeps the file's node order of every element."""
    with open(path) as f:
        lines = f.read().split("\n")
    pos = 0

    def next_line():
        nonlocal pos
        while pos < len(lines) and not lines[pos].strip():
            pos += 1
        if pos >= len(lines):
            raise ValueError("unexpected end of the mesh file")
        pos += 1
        return lines[pos - 1].split()

    def keyword(want):
        tok = next_line()
        if len(tok) < 2 or tok[0] != want:
            raise ValueError(f"symbol '{tok[0] if tok else ''}' parsed instead of correct symbol '{want}'")
        return tok[1]

    if int(keyword("NDIME=")) != 3:
        raise ValueError("only three dimensions (NDIME= 3) are accepted")
    n_elem = int(keyword("NELEM="))
    tets = np.empty((n_elem, 4), np.int64)
    for i in range(n_elem):
        tok = next_line()
        if int(tok[0]) != 10:
            raise ValueError(f"element {i}: only tetrahedra (10) are supported, got {tok[0]}")
        tets[i] = [int(t) for t in tok[1:5]]
    n_nodes = int(keyword("NPOIN="))
    vals: List[float] = []
    while len(vals) < 3 * n_nodes:  # a stream of numbers, three per node
        vals.extend(float(t) for t in next_line())
    nodes = np.array(vals[:3 * n_nodes], np.float64).reshape(n_nodes, 3)
    markers = []
    for _ in range(int(keyword("NMARK="))):
        name = keyword("MARKER_TAG=")
        k = int(keyword("MARKER_ELEMS="))
        tris = np.empty((k, 3), np.int64)
        for i in range(k):
            tok = next_line()
            if int(tok[0]) != 5:
                raise ValueError(f"marker '{name}' element {i}: only triangles (5) are supported")
            tris[i] = [int(t) for t in tok[1:4]]
        if name not in patch_types:
            raise ValueError(f"marker '{name}' has no boundary type")
        markers.append((name, tris))
    return TetMesh(nodes=nodes, tets=tets, markers=markers, patch_types=dict(patch_types))


def input_yml_text(patch_types: Dict[str, str], freestream, cfl: float = 0.8,
                   n_timesteps: int = 1, time_scheme: str = "TVD_RK3",
                   spatial_order: str = "Second", limiter: str = "Barth",
                   write_stride: int = 1000000) -> str:
    """An input.yml in the subset ConfigParser.cpp:38-131 reads."""
    rho, u, v, w, p = (float(x) for x in freestream)
    lines = [
        "solver: Euler",
        f"n_timesteps: {int(n_timesteps)}",
        f"CFL: {repr(float(cfl))}",
        f"time_scheme: {time_scheme}",
        f"spatial_order: {spatial_order}",
        "grad_scheme: GreenGauss",
        "inviscid_flux_scheme: Rusanov",
        f"limiter: {limiter}",
        "initial_cond: Freestream",
        f"write_stride: {int(write_stride)}",
        f"density_fs: {repr(rho)}",
        f"velocity_fs: [{repr(u)}, {repr(v)}, {repr(w)}]",
        f"pressure_fs: {repr(p)}",
        "patches:",
    ]
    for name, t in patch_types.items():
        lines.append(f"  - {name}: {t}")
    return "\n".join(lines) + "\n"


def write_case(case_dir: str, mesh: TetMesh, freestream, U0: Optional[np.ndarray] = None, **yml) -> None:
    """Write ``mesh.su2``, ``input.yml`` and (optionally) ``U0.bin`` into ``case_dir``."""
    os.makedirs(case_dir, exist_ok=True)
    write_su2(os.path.join(case_dir, "mesh.su2"), mesh)
    with open(os.path.join(case_dir, "input.yml"), "w") as f:
        f.write(input_yml_text(mesh.patch_types, freestream, **yml))
    if U0 is not None:
        np.ascontiguousarray(U0, dtype="<f8").tofile(os.path.join(case_dir, "U0.bin"))
