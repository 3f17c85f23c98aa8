"""Lattice meshes in the reference's per-rank files, and non-box geometries.

The solver reads processor<pid>/lattice/{points, ghosts, neighbours,
boundary, vtkCells, recvGhosts, sendGhosts} (src/IO/readLatticeMesh.c:15-330),
files that latticeMeshPartition writes with writeLatticeMesh
(src/IO/writeLatticeMesh.c:25-200):

  points      nlocal, then one "x y z" line per local node
  ghosts      nghosts, then one "x y z" line per ghost node
  neighbours  "nlocal D Q", then one line of Q neighbour indices per local
              node (pull source x - c_k, -1 = none)
  boundary    nbd, then per patch: name, count, one node index per line
  vtkCells    ncells cellType, then the cells' node indices
  recvGhosts / sendGhosts   worldSize, then per rank: rank, count, indices

``read_lattice_mesh`` parses them (whitespace-separated, as fscanf does);
``write_lattice_mesh`` writes the same layout (the reference's printf
formats), so meshes made here run on the reference and the reverse.
``mesh_case`` turns a single-rank mesh (worldSize 1, no ghosts: the one
device domain of this path) into a case for :class:`Lattice`; any such mesh
runs on the operator path.  ``channel_with_cylinder`` builds a non-box
geometry: a channel with a solid disc removed, its wall nodes as patches.
"""
import os
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import abi
from .cases import VEL, Case


@dataclass
class LatticeMesh:
    lattice: int
    points: np.ndarray          # [nlocal + nghosts][3] int
    nb: np.ndarray              # [nlocal][Q] int32
    patch_names: List[str]
    patches: List[np.ndarray]   # uint32 node indices per patch
    nlocal: int
    nghosts: int = 0
    vtk_cells: Optional[np.ndarray] = None  # [ncells][cellType] int, or None
    recv_ghosts: List[np.ndarray] = field(default_factory=list)  # per rank
    send_ghosts: List[np.ndarray] = field(default_factory=list)  # per rank

    @property
    def Q(self):
        return abi.Q_OF[self.lattice]


def _ints(path):
    with open(path) as fp:
        return fp.read().split()


def read_lattice_mesh(root=".", pid=0):
    """processor<pid>/lattice/* under root -> LatticeMesh (readLatticeMesh.c)."""
    d = os.path.join(root, f"processor{pid}", "lattice")
    t = _ints(os.path.join(d, "points"))
    nlocal = int(t[0])
    pts = np.array(t[1:1 + 3 * nlocal], dtype=np.int64).reshape(nlocal, 3)
    gpath = os.path.join(d, "ghosts")
    nghosts = 0
    gpts = np.zeros((0, 3), dtype=np.int64)
    if os.path.exists(gpath):
        t = _ints(gpath)
        nghosts = int(t[0])
        gpts = np.array(t[1:1 + 3 * nghosts], dtype=np.int64).reshape(nghosts, 3)
    t = _ints(os.path.join(d, "neighbours"))
    n_nb, _dim, Q = int(t[0]), int(t[1]), int(t[2])
    if n_nb != nlocal:
        raise ValueError(f"neighbours lists {n_nb} nodes, points {nlocal}")
    if Q not in (9, 15):
        raise ValueError(f"unknown lattice with Q = {Q}")
    nb = np.array(t[3:3 + nlocal * Q], dtype=np.int64).reshape(nlocal, Q)
    t = _ints(os.path.join(d, "boundary"))
    nbd, i = int(t[0]), 1
    names, patches = [], []
    for _ in range(nbd):
        names.append(t[i])
        cnt = int(t[i + 1])
        patches.append(np.array(t[i + 2:i + 2 + cnt], dtype=np.uint32))
        i += 2 + cnt
    cells = None
    cpath = os.path.join(d, "vtkCells")
    if os.path.exists(cpath):
        t = _ints(cpath)
        nc, ct = int(t[0]), int(t[1])
        cells = np.array(t[2:2 + nc * ct], dtype=np.int64).reshape(nc, ct)

    def ghosts(name):
        p = os.path.join(d, name)
        if not os.path.exists(p):
            return []
        t = _ints(p)
        ws, i, out = int(t[0]), 1, []
        for _ in range(ws):
            cnt = int(t[i + 1])
            out.append(np.array(t[i + 2:i + 2 + cnt], dtype=np.uint32))
            i += 2 + cnt
        return out

    return LatticeMesh(abi.D2Q9 if Q == 9 else abi.D3Q15, np.vstack([pts, gpts]).astype(np.int32),
                       nb.astype(np.int32), names, patches, nlocal, nghosts, cells, ghosts("recvGhosts"),
                       ghosts("sendGhosts"))


def write_lattice_mesh(mesh, root=".", pid=0):
    """LatticeMesh -> processor<pid>/lattice/* in writeLatticeMesh's layout."""
    d = os.path.join(root, f"processor{pid}", "lattice")
    os.makedirs(d, exist_ok=True)
    P = np.asarray(mesh.points)
    with open(os.path.join(d, "points"), "w") as fp:
        fp.write(f"{mesh.nlocal}\n")
        fp.writelines(f"{x} {y} {z}\n" for x, y, z in P[:mesh.nlocal].tolist())
    with open(os.path.join(d, "ghosts"), "w") as fp:
        fp.write(f"{mesh.nghosts}\n")
        fp.writelines(f"{x} {y} {z}\n" for x, y, z in P[mesh.nlocal:mesh.nlocal + mesh.nghosts].tolist())
    Q = mesh.Q
    with open(os.path.join(d, "neighbours"), "w") as fp:
        fp.write(f"{mesh.nlocal} {2 if Q == 9 else 3} {Q}\n")
        fp.writelines("".join(f"{v} " for v in row) + "\n" for row in np.asarray(mesh.nb).tolist())
    ws = max(1, len(mesh.recv_ghosts))
    for name, lists in (("recvGhosts", mesh.recv_ghosts), ("sendGhosts", mesh.send_ghosts)):
        with open(os.path.join(d, name), "w") as fp:
            fp.write(f"{ws}\n\n")
            for r in range(ws):
                lst = lists[r] if r < len(lists) else np.zeros(0, dtype=np.uint32)
                fp.write(f"{r}\n{len(lst)}\n")
                fp.writelines(f"{v}\n" for v in np.asarray(lst).tolist())
                fp.write("\n")
    with open(os.path.join(d, "boundary"), "w") as fp:
        fp.write(f"{len(mesh.patches)}\n\n")
        for nm, p in zip(mesh.patch_names, mesh.patches):
            fp.write(f"{nm}\n{len(p)}\n")
            fp.writelines(f"{v}\n" for v in np.asarray(p).tolist())
            fp.write("\n")
    cells = mesh.vtk_cells if mesh.vtk_cells is not None else np.zeros((0, 4 if Q == 9 else 8), dtype=np.int64)
    with open(os.path.join(d, "vtkCells"), "w") as fp:
        fp.write(f"{len(cells)} {cells.shape[1]}\n")
        fp.writelines("".join(f"{v} " for v in row) + "\n" for row in np.asarray(cells).tolist())


def mesh_case(mesh, name, eos, f, g, rho, U, T, meta=None):
    """A single-rank mesh and its fields -> Case (bounding-box dims, no axis
    marked periodic: the neighbour table says where it wraps)."""
    if mesh.nghosts or len(mesh.recv_ghosts) > 1:
        raise ValueError("the device lattice is one domain: a mesh with ghost nodes or several ranks "
                         "must be re-partitioned for one rank first")
    pts = np.asarray(mesh.points[:mesh.nlocal])
    d = 3 if mesh.lattice == abi.D3Q15 else 2
    dims = tuple(int(pts[:, j].max() - pts[:, j].min() + 1) for j in range(d))
    return Case(name, mesh.lattice, dims, (False,) * d, np.asarray(mesh.nb, dtype=np.int32),
                pts.astype(np.int32), list(mesh.patches), list(mesh.patch_names), eos, f, g,
                np.asarray(rho, dtype=np.float64), np.asarray(U, dtype=np.float64),
                np.asarray(T, dtype=np.float64), meta=dict(meta or {}))


def channel_with_cylinder(nx, ny, cx, cy, radius, periodic_x=True):
    """D2Q9 channel of nx x ny nodes with the solid disc |x - c| < radius
    removed.  Walls at y = 0 and y = ny - 1; x wraps when periodic_x.
    Patches: "bottom", "top" (channel walls) and "cylinder" (fluid nodes with
    a removed neighbour), in that order, like the boundary files of a
    partitioned SALOME mesh.  Node order: x fastest over the fluid nodes."""
    vel = VEL[abi.D2Q9]
    yy, xx = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    solid = (xx - cx) ** 2 + (yy - cy) ** 2 < radius ** 2
    fluid = ~solid
    index = -np.ones((ny, nx), dtype=np.int64)
    index[fluid] = np.arange(int(fluid.sum()))
    fy, fx = np.nonzero(fluid)
    n = fy.size
    nb = np.empty((n, 9), dtype=np.int32)
    for k, c in enumerate(vel):
        sx, sy = fx - c[0], fy - c[1]
        ok = (sy >= 0) & (sy < ny)
        if periodic_x:
            sx = sx % nx
        else:
            ok &= (sx >= 0) & (sx < nx)
        src = np.full(n, -1, dtype=np.int64)
        src[ok] = index[sy[ok], sx[ok]]
        nb[:, k] = src
    points = np.stack([fx, fy, np.zeros(n, dtype=np.int64)], axis=1).astype(np.int32)
    bottom = np.nonzero(fy == 0)[0].astype(np.uint32)
    top = np.nonzero(fy == ny - 1)[0].astype(np.uint32)
    walls = (fy == 0) | (fy == ny - 1)
    near = ((nb == -1).any(axis=1)) & ~walls
    cyl = np.nonzero(near)[0].astype(np.uint32)
    return LatticeMesh(abi.D2Q9, points, nb, ["bottom", "top", "cylinder"], [bottom, top, cyl], n)
