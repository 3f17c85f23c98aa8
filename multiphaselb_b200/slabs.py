"""Slab decomposition of a box lattice over several handles (one per rank or
device), with the reference's ghost-node exchange.

The reference runs each MPI rank on its part of the mesh plus ghost nodes
and exchanges them inside the time step (multiPhasePP.c:163-240):
sendPdfField / recvPdfField after each field's boundaries, syncScalarField
of the heat source and syncVectorField of the interaction force.  Here a box
(cases.box_mesh layout, x fastest) is cut into slabs along its slowest axis
(y in 2D, z in 3D); each slab's lattice holds its own planes plus one ghost
plane on each cut (wrapping on a periodic axis), and a step runs the
reference's operators on every slab with the ghost planes refreshed from
their owners at the same points:

    collision f                                    -> ghost f (surface tension on only)
    lbstream f, updateBoundaries f                 -> ghost f
    collision g, lbstream g, updateBoundaries g   -> ghost g
    macroDensity
    heatSource                                     -> ghost S
    macroTemperature
    interForce                                     -> ghost Fi, Ft
    macroVelocity

Ghost nodes have no neighbours and lie on no boundary patch, as in the
reference's partitioned meshes (latticeMeshPartition.c:564-590, 679-725):
they do not stream, and whatever a ghost node computes is overwritten by an
exchange before an owned node reads it.  The surface-tension collision needs
neighbours, so with it on the reference collides the local nodes only and
syncs the post-collision PDFs to the ghosts (liMRTCollision.c:33-37,126-131;
xuMRTCollision.c:32-36,108-113); so does this runner.  The gathered owned
nodes are then bit-identical to the single-domain run, with one exception
that the reference has too: a fixedT / fixedU / fixedRandomT wall that
crosses a cut extrapolates from the ghost's PDF, which has not streamed when
the boundaries run (the exchange follows them), where the single domain
reads the streamed value (tests/test_slabs.py).  fixedRandomT seeds rand()
with the rank; slab r runs as rank rank0 + r.

Between device handles (LatticeHandle) the exchange moves only the ghost
planes, device to device (mplb_gpu_copy_nodes: one strided copy per field
and plane, peer to peer when the slabs sit on different GPUs, ordered on the
handles' streams without a host synchronisation).  Any other handle with the
operator interface (a CPU checker in the tests) is exchanged through host
copies of its fields: download, copy the ghost planes, upload.
"""
from dataclasses import dataclass
from typing import Callable, List

import numpy as np

from . import abi
from .cases import Case

FIELDS = ("rho", "U", "T", "Fi", "Ft", "S", "f", "g")


@dataclass
class Slab:
    rank: int
    planes: List[int]        # global plane index of every local plane, in local order
    own_lo: int              # local index of the first owned plane
    own_hi: int              # one past the last owned plane (local index)
    case: Case
    gidx: np.ndarray         # global node of every local node


def _box_geometry(case):
    d3 = case.lattice == abi.D3Q15
    dims = tuple(case.dims)
    nplanes = dims[2] if d3 else dims[1]
    plane = int(np.prod(dims[:-1]))
    periodic = bool(case.periodic[-1])
    return nplanes, plane, periodic


def split(case: Case, ranks: int, rank0: int = 0) -> List[Slab]:
    """Cut a box case into `ranks` slabs along its slowest axis; slab r runs
    as rank rank0 + r (the pid that seeds fixedRandomT)."""
    nplanes, P, periodic = _box_geometry(case)
    if ranks < 2:
        raise ValueError("a split needs at least two slabs")
    if nplanes < 2 * ranks:
        raise ValueError(f"{nplanes} planes cannot give {ranks} slabs of at least two planes")
    cuts = [round(r * nplanes / ranks) for r in range(ranks + 1)]
    slabs = []
    for r in range(ranks):
        a, b = cuts[r], cuts[r + 1]
        lo = a - 1 if a > 0 else (nplanes - 1 if periodic else None)
        hi = b if b < nplanes else (0 if periodic else None)
        planes = ([lo] if lo is not None else []) + list(range(a, b)) + ([hi] if hi is not None else [])
        own_lo = 1 if lo is not None else 0
        own_hi = own_lo + (b - a)
        where = {p: j for j, p in enumerate(planes)}
        gidx = np.concatenate([p * P + np.arange(P) for p in planes]).astype(np.int64)
        # neighbour table: the global source mapped into the slab, -1 outside it
        gnb = np.asarray(case.nb, dtype=np.int64)[gidx]
        src_plane = np.where(gnb >= 0, gnb // P, -1)
        lut = np.full(nplanes, -1, dtype=np.int64)
        for p, j in where.items():
            lut[p] = j
        lj = np.where(gnb >= 0, lut[np.maximum(src_plane, 0)], -1)
        nb = np.where(lj >= 0, lj * P + gnb % P, -1).astype(np.int32)
        # ghost nodes get no neighbours, as in the reference's partition
        # (latticeMeshPartition.c:564-590 fills nb for local nodes only)
        nb[:own_lo * P] = -1
        nb[own_hi * P:] = -1
        # owned part of every patch, in patch order
        owned = np.zeros(case.n, dtype=bool)
        owned[a * P:b * P] = True
        local_of = np.full(case.n, -1, dtype=np.int64)
        local_of[gidx[own_lo * P:own_hi * P]] = np.arange(own_lo * P, own_hi * P)
        patches = [local_of[np.asarray(p, dtype=np.int64)[owned[np.asarray(p, dtype=np.int64)]]].astype(np.uint32)
                   for p in case.patches]
        pts = np.asarray(case.points)[gidx]
        local = Case(f"{case.name}_slab{r}", case.lattice, tuple(case.dims[:-1]) + (len(planes),),
                     tuple(case.periodic[:-1]) + (False,), nb, pts.astype(np.int32), patches,
                     list(case.patch_names), case.eos, case.f, case.g, np.asarray(case.rho)[gidx],
                     np.asarray(case.U)[gidx], np.asarray(case.T)[gidx], meta=dict(case.meta, box=False, rank=rank0 + r))
        slabs.append(Slab(r, planes, own_lo, own_hi, local, gidx))
    return slabs


def ghost_sources(slabs: List[Slab]):
    """(slab, ghost plane, owner slab, owner's plane) of every ghost plane,
    all in local plane indices, in a fixed order (every rank lists them the
    same way)."""
    def owner(plane):
        for s in slabs:
            if s.planes[s.own_lo] <= plane < s.planes[s.own_lo] + (s.own_hi - s.own_lo):
                return s
        raise AssertionError(plane)
    out = []
    for s in slabs:
        for j in range(len(s.planes)):
            if not s.own_lo <= j < s.own_hi:
                o = owner(s.planes[j])
                out.append((s, j, o, o.planes.index(s.planes[j], o.own_lo, o.own_hi)))
    return out


class _SlabSteps:
    """The reference's step on the slabs this process drives (self.local:
    (slab, handle) pairs), with exchange(names) refreshing ghost planes."""

    def _setup(self, case):
        self.case = case
        _, self.P, _ = _box_geometry(case)
        self.has_g = case.g is not None
        self.f_on = case.f is not None and bool(case.f.get("update", 1))
        self.f_st = self.f_on and bool(case.f.get("surface_tension", 0))
        self.g_on = self.has_g and bool(case.g.get("update", 1))

    def _all(self, name, field=None):
        for _, h in self.local:
            h.op(name, field)

    def _upload_fields(self, h, st):
        h.upload(**{nm: st[nm] for nm in FIELDS if not (nm == "g" and not self.has_g)})

    def initialize(self):
        """multiPhasePP.c:122-147 on every slab, ghosts exchanged."""
        for s, h in self.local:
            h.upload(rho=s.case.rho, U=s.case.U, T=s.case.T)
        self._all("equilibrium", abi.FIELD_F)
        if self.has_g:
            self._all("equilibrium", abi.FIELD_G)
        self._all("inter_force")
        self.exchange(("Fi", "Ft"))
        if self.g_on:
            self._all("heat_source")
            self.exchange(("S",))

    def step(self, n=1):
        """multiPhasePP.c:157-240 with the ghost exchanges of the reference."""
        for _ in range(n):
            for _, h in self.local:
                h.set_time(h.get_time() + 1)
            for fi, on, name in ((abi.FIELD_F, self.f_on, "f"), (abi.FIELD_G, self.g_on, "g")):
                if not on:
                    continue
                self._all("collision", fi)
                if fi == abi.FIELD_F and self.f_st:
                    self.exchange(("f",))
                self._all("lbstream", fi)
                self._all("update_boundaries", fi)
                self.exchange((name,))
            self._all("macro_density")
            if self.g_on:
                self._all("heat_source")
                self.exchange(("S",))
            self._all("macro_temperature")
            if self.f_on:
                self._all("inter_force")
                self.exchange(("Fi", "Ft"))
            self._all("macro_velocity")

    def owned(self):
        """(global node indices, fields) of the owned planes of this
        process's slabs."""
        out = []
        for s, h in self.local:
            st = h.download()
            lo, hi = s.own_lo * self.P, s.own_hi * self.P
            out.append((s.gidx[lo:hi], {k: v[lo:hi] for k, v in st.items()}))
        return out

    def _assemble(self, parts):
        n = self.case.n
        out = {}
        for gi, st in parts:
            for k, v in st.items():
                if k not in out:
                    out[k] = np.zeros((n,) + v.shape[1:])
                out[k][gi] = v
        return out


class SlabRun(_SlabSteps):
    """Step a split box case on `ranks` handles, all driven by this process.

    make_handle(case) -> an object with upload(**fields), download() -> dict
    of the fields in the reference layouts, set_time(t), get_time() and
    op(name, field=None) for the reference operators named as the Lattice
    methods (equilibrium, collision, lbstream, update_boundaries,
    macro_density, heat_source, macro_temperature, inter_force,
    macro_velocity).  See LatticeHandle for device handles.
    """

    def __init__(self, case: Case, ranks: int, make_handle: Callable, rank0: int = 0, staged: bool = False):
        self._setup(case)
        self.slabs = split(case, ranks, rank0)
        self.handles = [make_handle(s.case) for s in self.slabs]
        self.local = list(zip(self.slabs, self.handles))
        # device-to-device ghost copies when every handle offers them
        self.direct = not staged and all(hasattr(h, "copy_from") for h in self.handles)

    def exchange(self, names):
        """Ghost planes of the fields `names` from their owners."""
        P = self.P
        if self.direct:
            for s, j, o, oj in ghost_sources(self.slabs):
                self.handles[s.rank].copy_from(self.handles[o.rank], j * P, oj * P, P, names)
            return
        states = [h.download() for h in self.handles]
        for s, j, o, oj in ghost_sources(self.slabs):
            st, src = states[s.rank], states[o.rank]
            for nm in names:
                st[nm][j * P:(j + 1) * P] = src[nm][oj * P:(oj + 1) * P]
        for h, st in zip(self.handles, states):
            self._upload_fields(h, st)

    def gather(self):
        """The owned planes of every slab, as the single-domain fields."""
        return self._assemble(self.owned())


class DistSlabRun(_SlabSteps):
    """One slab per process of a torch.distributed group, as one reference
    MPI rank per process: the ghost planes travel by point-to-point messages
    (isend / irecv of the planes' values, in the order ghost_sources lists
    them; tensors on `device`, e.g. CUDA for NCCL, CPU for gloo).  The group's
    rank r holds slab r and runs as reference rank rank0 + r."""

    def __init__(self, case: Case, make_handle: Callable, group=None, rank0: int = 0, device="cpu"):
        import torch
        import torch.distributed as dist
        self._torch, self._dist, self.group = torch, dist, group
        self._setup(case)
        self.rank = dist.get_rank(group)
        self.slabs = split(case, dist.get_world_size(group), rank0)
        self.slab = self.slabs[self.rank]
        self.handle = make_handle(self.slab.case)
        self.local = [(self.slab, self.handle)]
        self.device = torch.device(device)

    def _peer(self, r):
        return r if self.group is None else self._dist.get_global_rank(self.group, r)

    def exchange(self, names):
        torch, dist, P = self._torch, self._dist, self.P
        st = self.handle.download()
        ops, recvs = [], []
        for tag, (s, j, o, oj) in enumerate(ghost_sources(self.slabs)):
            if o.rank == self.rank and s.rank != self.rank:
                buf = np.concatenate([st[nm][oj * P:(oj + 1) * P].reshape(-1) for nm in names])
                t = torch.from_numpy(buf).to(self.device)
                ops.append(dist.P2POp(dist.isend, t, self._peer(s.rank), self.group, tag))
            elif s.rank == self.rank and o.rank != self.rank:
                size = sum(st[nm][j * P:(j + 1) * P].size for nm in names)
                t = torch.empty(size, dtype=torch.float64, device=self.device)
                ops.append(dist.P2POp(dist.irecv, t, self._peer(o.rank), self.group, tag))
                recvs.append((j, t))
        # one group of sends and receives: two ranks that send to each other
        # do not wait on each other's receive
        if ops:
            for r in dist.batch_isend_irecv(ops):
                r.wait()
        for j, t in recvs:
            buf, off = t.cpu().numpy(), 0
            for nm in names:
                dst = st[nm][j * P:(j + 1) * P]
                dst[...] = buf[off:off + dst.size].reshape(dst.shape)
                off += dst.size
        self._upload_fields(self.handle, st)

    def gather(self):
        """Every rank's owned planes, as the single-domain fields (on every rank)."""
        parts = [None] * self._dist.get_world_size(self.group)
        self._dist.all_gather_object(parts, self.owned(), group=self.group)
        return self._assemble([p for ps in parts for p in ps])


class LatticeHandle:
    """Operator-interface adapter of a device Lattice (operator path)."""

    def __init__(self, case, device=-1):
        from . import PATH_OPERATORS, Lattice
        self.lat = Lattice(case, path=PATH_OPERATORS, device=device)

    def upload(self, **fields):
        self.lat.upload(**fields)

    def download(self):
        return self.lat.download()

    def set_time(self, t):
        self.lat.set_time(t)

    def get_time(self):
        return self.lat.info()["current_time"]

    def op(self, name, field=None):
        m = getattr(self.lat, name)
        return m(field) if field is not None else m()

    def copy_from(self, src, dst_start, src_start, count, names):
        self.lat.copy_nodes(src.lat, dst_start, src_start, count, names)

    def close(self):
        self.lat.close()
