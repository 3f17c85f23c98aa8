"""Multi-rank runs of a lattice: the mesh split over ranks (one handle per
rank, on one device or several), with the reference's ghost-node exchange.

The reference runs each MPI rank on its part of the mesh plus ghost nodes
and exchanges them inside the time step (multiPhasePP.c:163-240):
sendPdfField / recvPdfField after each field's boundaries, syncScalarField
of the heat source and syncVectorField of the interaction force.  Every rank
here holds its owned nodes and its ghost nodes, with per-peer lists of the
ghost nodes it receives and of the owned nodes it sends (the
recvGhosts / sendGhosts of the reference's partitioned meshes), and a step
runs the reference's operators with the ghosts refreshed at the same points:

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
with the rank.

Three ways to get the ranks' parts:
  split(case, R)          a box cut into R slabs along its slowest axis
                          (y in 2D, z in 3D), one ghost plane per cut
  partition(case, owner)  any mesh and an owner rank per node, indexed as the
                          reference's partitioner does (localIndexing.c);
                          standard_owner(n, R) is the owner array of the
                          partitioner's default method
  from_meshes(meshes,...) the reference's per-rank mesh files, read with
                          mesh.read_lattice_mesh

RankRun drives every part from one process.  Between device handles
(LatticeHandle) the exchange moves only the ghost nodes, device to device
(mplb_gpu_copy_nodes: one strided copy per field and contiguous run of
nodes, peer to peer between GPUs, ordered on the handles' streams without a
host synchronisation), and the whole step runs in the library
(mplb_ranks_step); other handles (a CPU checker in the tests) exchange
through host copies of their fields.  DistRankRun is one part per process of
a torch.distributed group, the ghosts sent as point-to-point messages.
"""
import ctypes as C
from dataclasses import dataclass, field
from typing import Callable, List, Optional

import numpy as np

from . import abi
from .cases import Case

FIELDS = ("rho", "U", "T", "Fi", "Ft", "S", "f", "g")


@dataclass
class Part:
    """One rank's lattice: owned nodes and ghost nodes."""
    rank: int                    # index in the group
    case: Case                   # the rank's nodes, neighbour table, patches and fields
    own: np.ndarray              # local indices of the owned nodes
    recv: List[np.ndarray]       # per peer: local ghost nodes filled from that peer, in message order
    send: List[np.ndarray]       # per peer: local owned nodes sent to that peer, in message order
    gidx: Optional[np.ndarray] = None   # global node of every local node, where known


@dataclass
class Slab(Part):
    planes: List[int] = field(default_factory=list)  # global plane of every local plane
    own_lo: int = 0              # local index of the first owned plane
    own_hi: int = 0              # one past the last owned plane


def _box_geometry(case):
    d3 = case.lattice == abi.D3Q15
    dims = tuple(case.dims)
    nplanes = dims[2] if d3 else dims[1]
    plane = int(np.prod(dims[:-1]))
    periodic = bool(case.periodic[-1])
    return nplanes, plane, periodic


def _local_case(case, name, gidx, own_mask_local, local_of, owned_global, rank, dims=None, periodic=None):
    """The Case of one rank: nodes gidx (owned ones first or not), neighbour
    rows of the owned nodes mapped through local_of, ghost rows empty, and
    the owned part of every patch."""
    Q = case.Q
    gnb = np.asarray(case.nb, dtype=np.int64)[gidx]
    nb = np.where(gnb >= 0, local_of[np.maximum(gnb, 0)], -1)
    nb[~own_mask_local] = -1
    patches = []
    for p in case.patches:
        p = np.asarray(p, dtype=np.int64)
        patches.append(local_of[p[owned_global[p]]].astype(np.uint32))
    pts = np.asarray(case.points)[gidx].astype(np.int32)
    d = 3 if case.lattice == abi.D3Q15 else 2
    if dims is None:
        dims = tuple(int(pts[:, j].max() - pts[:, j].min() + 1) for j in range(d))
    if periodic is None:
        periodic = (False,) * d
    assert nb.shape == (len(gidx), Q)
    return Case(name, case.lattice, tuple(dims), tuple(periodic), nb.astype(np.int32), pts, patches,
                list(case.patch_names), case.eos, case.f, case.g, np.asarray(case.rho)[gidx],
                np.asarray(case.U)[gidx], np.asarray(case.T)[gidx], meta=dict(case.meta, box=False, rank=rank))


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
        gidx = np.concatenate([p * P + np.arange(P) for p in planes]).astype(np.int64)
        local_of = np.full(case.n, -1, dtype=np.int64)
        local_of[gidx] = np.arange(len(gidx))
        own_mask = np.zeros(len(gidx), dtype=bool)
        own_mask[own_lo * P:own_hi * P] = True
        owned_global = np.zeros(case.n, dtype=bool)
        owned_global[a * P:b * P] = True
        local = _local_case(case, f"{case.name}_slab{r}", gidx, own_mask, local_of, owned_global, rank0 + r,
                            dims=tuple(case.dims[:-1]) + (len(planes),),
                            periodic=tuple(case.periodic[:-1]) + (False,))
        empty = [np.zeros(0, dtype=np.int64) for _ in range(ranks)]
        slabs.append(Slab(r, local, np.arange(own_lo * P, own_hi * P), list(empty), list(empty), gidx,
                          planes, own_lo, own_hi))
    # message lists, in ghost_sources order on both sides
    for s, j, o, oj in ghost_sources(slabs):
        s.recv[o.rank] = np.concatenate([s.recv[o.rank], np.arange(j * P, (j + 1) * P)])
        o.send[s.rank] = np.concatenate([o.send[s.rank], np.arange(oj * P, (oj + 1) * P)])
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


def standard_owner(n: int, ranks: int) -> np.ndarray:
    """Owner rank per node of the reference partitioner's default method
    ("standard", standardDecomp.c:5-48): consecutive blocks of n // ranks
    nodes in global node order, the last rank also taking the remainder.
    The reference's unsigned arithmetic breaks when ranks > n (its first
    block would end at node -1); that is refused here."""
    n, ranks = int(n), int(ranks)
    if ranks < 1 or ranks > n:
        raise ValueError(f"standard decomposition of {n} nodes needs 1 <= ranks <= {n}, got {ranks}")
    owner = np.minimum(np.arange(n, dtype=np.int64) // (n // ranks), ranks - 1)
    return owner


def partition(case: Case, owner, rank0: int = 0) -> List[Part]:
    """Split any mesh by an owner rank per node, as the reference's
    partitioner does: a rank's local nodes are its owned nodes in global
    order, then its ghosts (every pull source of an owned node owned
    elsewhere) in the order a scan of the owned nodes and their velocities
    first meets them (localIndexing.c:7-95); the ghost lists pair the
    receiving rank's ghost with the owner's node, in global node order
    (latticeMeshPartition.c:745-770).  Rank r runs as rank0 + r."""
    owner = np.asarray(owner, dtype=np.int64)
    n = case.n
    if owner.shape != (n,) or owner.min() < 0:
        raise ValueError("owner needs one rank >= 0 per node")
    ranks = int(owner.max()) + 1
    nb = np.asarray(case.nb, dtype=np.int64)
    locals_, gidxs, nlocal = [], [], []
    for r in range(ranks):
        own = np.nonzero(owner == r)[0]
        if len(own) == 0:
            raise ValueError(f"rank {r} owns no node")
        local_of = np.full(n, -1, dtype=np.int64)
        local_of[own] = np.arange(len(own))
        cand = nb[own].reshape(-1)
        cand = cand[cand >= 0]
        cand = cand[local_of[cand] < 0]
        _, first = np.unique(cand, return_index=True)
        ghosts = cand[np.sort(first)]
        local_of[ghosts] = len(own) + np.arange(len(ghosts))
        locals_.append(local_of)
        gidxs.append(np.concatenate([own, ghosts]))
        nlocal.append(len(own))
    parts = []
    for r in range(ranks):
        gidx = gidxs[r]
        own_mask = np.zeros(len(gidx), dtype=bool)
        own_mask[:nlocal[r]] = True
        local = _local_case(case, f"{case.name}_rank{r}", gidx, own_mask, locals_[r], owner == r, rank0 + r)
        parts.append(Part(r, local, np.arange(nlocal[r]), [None] * ranks, [None] * ranks, gidx))
    for r in range(ranks):
        ghosts = np.sort(gidxs[r][nlocal[r]:])       # global node order
        for s in range(ranks):
            sel = ghosts[owner[ghosts] == s] if s != r else ghosts[:0]
            parts[r].recv[s] = locals_[r][sel]
            parts[s].send[r] = locals_[s][sel]
    return parts


def from_meshes(meshes, name, eos, f, g, fields, rank0: int = 0) -> List[Part]:
    """Parts from the reference's per-rank mesh files (mesh.LatticeMesh of
    every rank, as read_lattice_mesh returns them) and each rank's initial
    (rho, U, T) over its nlocal + nghosts nodes.  Rank r runs as rank0 + r."""
    parts = []
    ranks = len(meshes)
    for r, (m, (rho, U, T)) in enumerate(zip(meshes, fields)):
        npts = m.nlocal + m.nghosts
        nb = np.full((npts, m.Q), -1, dtype=np.int32)
        nb[:m.nlocal] = np.asarray(m.nb, dtype=np.int32)
        pts = np.asarray(m.points, dtype=np.int32)
        d = 3 if m.lattice == abi.D3Q15 else 2
        dims = tuple(int(pts[:, j].max() - pts[:, j].min() + 1) for j in range(d))
        case = Case(f"{name}_rank{r}", m.lattice, dims, (False,) * d, nb, pts, list(m.patches),
                    list(m.patch_names), eos, f, g, np.asarray(rho, dtype=np.float64),
                    np.asarray(U, dtype=np.float64), np.asarray(T, dtype=np.float64),
                    meta=dict(box=False, rank=rank0 + r))
        lists = lambda ls: [np.asarray(ls[s], dtype=np.int64) if s < len(ls) else np.zeros(0, dtype=np.int64)
                            for s in range(ranks)]
        parts.append(Part(r, case, np.arange(m.nlocal), lists(m.recv_ghosts), lists(m.send_ghosts)))
    for r, p in enumerate(parts):
        for s, q in enumerate(parts):
            if len(p.recv[s]) != len(q.send[r]):
                raise ValueError(f"rank {r} receives {len(p.recv[s])} ghosts from rank {s}, which sends "
                                 f"{len(q.send[r])}")
    return parts


def node_runs(dst, src):
    """Pairs of local node lists -> (dst_start, src_start, count) runs where
    both lists step by one."""
    dst, src = np.asarray(dst, dtype=np.int64), np.asarray(src, dtype=np.int64)
    if len(dst) == 0:
        return []
    brk = np.nonzero((np.diff(dst) != 1) | (np.diff(src) != 1))[0] + 1
    starts = np.concatenate([[0], brk])
    ends = np.concatenate([brk, [len(dst)]])
    return [(int(dst[a]), int(src[a]), int(b - a)) for a, b in zip(starts, ends)]


class _Steps:
    """The reference's step on the parts this process drives (self.local:
    (part, handle) pairs), with exchange(names) refreshing ghost nodes."""

    def _setup(self, case_like):
        self.rho_0 = float(case_like.eos.get("rho_0", 0.0))
        self.has_g = case_like.g is not None
        self.f_on = case_like.f is not None and bool(case_like.f.get("update", 1))
        self.f_st = self.f_on and bool(case_like.f.get("surface_tension", 0))
        self.g_on = self.has_g and bool(case_like.g.get("update", 1))

    def _all(self, name, field=None):
        for _, h in self.local:
            h.op(name, field)

    def _upload_fields(self, h, st):
        h.upload(**{nm: st[nm] for nm in FIELDS if not (nm == "g" and not self.has_g)})

    def initialize(self):
        """multiPhasePP.c:122-147 on every rank, ghosts exchanged."""
        for p, h in self.local:
            h.upload(rho=p.case.rho, U=p.case.U, T=p.case.T)
        self.exchange(("rho", "U", "T"))
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

    def _local_rho_sums(self):
        """(rank, serial sum of rho over its owned nodes in node order, owned
        count) of every part of this process: the local half of
        averageScalarField (averageScalarField.c, localSum += fld[i])."""
        out = []
        for p, h in self.local:
            rho = np.asarray(h.download()["rho"], dtype=np.float64)[p.own]
            out.append((p.rank, float(np.cumsum(rho)[-1]) if len(rho) else 0.0, len(rho)))
        return out

    @staticmethod
    def _fold_rho_sums(sums):
        """The global half of averageScalarField: MPI_Allreduce of the local
        sums and counts, folded in rank order (((s0 + s1) + s2) + ...; an MPI
        library may fold in another order, and with two ranks every order
        gives the same bits), then the division."""
        sums = sorted(sums)
        total, count = sums[0][1], sums[0][2]
        for _, s, c in sums[1:]:
            total += s
            count += c
        return total / count

    def _average(self, sums):
        return 0.0 if self.rho_0 <= 0 else self._fold_rho_sums(sums)

    def average_rho0(self):
        """The write step's buoyancy reference (multiPhasePP.c:271,
        averageScalarField.c): 0 when the configured rho_0 is <= 0, else
        the mean density over every rank's owned nodes.  Set it with
        set_rho0, as the solver does."""
        return self._average(self._local_rho_sums())

    def set_rho0(self, rho_0):
        """rho_0 on every rank's lattice (the Ft buoyancy term, interForce.c:33)."""
        self.rho_0 = float(rho_0)
        for _, h in self.local:
            h.set_rho0(self.rho_0)

    def owned(self):
        """(part, fields of its owned nodes) of every part of this process."""
        out = []
        for p, h in self.local:
            st = h.download()
            out.append((p, {k: v[p.own] for k, v in st.items()}))
        return out

    @staticmethod
    def _assemble(parts, n):
        out = {}
        for p, st in parts:
            if p.gidx is None:
                raise ValueError("parts read from mesh files have no global numbering")
            for k, v in st.items():
                if k not in out:
                    out[k] = np.zeros((n,) + v.shape[1:])
                out[k][p.gidx[p.own]] = v
        return out


class RankRun(_Steps):
    """Step every part from this process.

    make_handle(case) -> an object with upload(**fields), download() -> dict
    of the fields in the reference layouts, set_time(t), get_time() and
    op(name, field=None) for the reference operators named as the Lattice
    methods (equilibrium, collision, lbstream, update_boundaries,
    macro_density, heat_source, macro_temperature, inter_force,
    macro_velocity); with copy_from(src, dst_start, src_start, count, names)
    the ghosts move handle to handle (LatticeHandle does this on the
    devices), else through host copies.
    """

    def __init__(self, parts: List[Part], make_handle: Callable, staged: bool = False, n_global=None,
                 native: bool = True):
        self.parts = parts
        self._setup(parts[0].case)
        self.n_global = n_global
        self.handles = [make_handle(p.case) for p in parts]
        self.local = list(zip(parts, self.handles))
        # (dst rank, dst start, src rank, src start, count) of every run of ghosts
        self.transfers = []
        for p in parts:
            for s, q in enumerate(parts):
                for d0, s0, c in node_runs(p.recv[s], q.send[p.rank]):
                    self.transfers.append((p.rank, d0, s, s0, c))
        self.direct = not staged and all(hasattr(h, "copy_from") for h in self.handles)
        # device lattices: the whole step in the library (mplb_ranks_step)
        self.native = native and self.direct and all(isinstance(h, LatticeHandle) for h in self.handles)
        if self.native:
            self._lib = self.handles[0].lat.lib
            self._harr = (C.c_void_p * len(self.handles))(*[h.lat.h.value for h in self.handles])
            self._runs = (abi.GhostRun * max(1, len(self.transfers)))(
                *[abi.GhostRun(d, d0, s, s0, c) for d, d0, s, s0, c in self.transfers])

    def initialize(self):
        if not self.native:
            return super().initialize()
        for p, h in self.local:
            h.upload(rho=p.case.rho, U=p.case.U, T=p.case.T)
        self.handles[0].lat._check(self._lib.mplb_ranks_initialize(self._harr, len(self.handles), self._runs,
                                                                   len(self.transfers)))

    def step(self, n=1):
        if not self.native:
            return super().step(n)
        self.handles[0].lat._check(self._lib.mplb_ranks_step(self._harr, len(self.handles), self._runs,
                                                             len(self.transfers), n))

    def exchange(self, names):
        """Ghost nodes of the fields `names` from their owners."""
        if self.direct:
            for d, d0, s, s0, c in self.transfers:
                self.handles[d].copy_from(self.handles[s], d0, s0, c, names)
            return
        states = [h.download() for h in self.handles]
        for d, d0, s, s0, c in self.transfers:
            for nm in names:
                states[d][nm][d0:d0 + c] = states[s][nm][s0:s0 + c]
        for h, st in zip(self.handles, states):
            self._upload_fields(h, st)

    def gather(self):
        """The owned nodes of every part, as the single-domain fields."""
        n = self.n_global
        if n is None:
            n = sum(len(p.own) for p in self.parts)
        return self._assemble(self.owned(), n)

    def close(self):
        for h in self.handles:
            if hasattr(h, "close"):
                h.close()


class SlabRun(RankRun):
    """A box case cut into `ranks` slabs (split) and stepped from this
    process; slab r runs as rank rank0 + r."""

    def __init__(self, case: Case, ranks: int, make_handle: Callable, rank0: int = 0, staged: bool = False,
                 native: bool = True):
        self.case = case
        self.slabs = split(case, ranks, rank0)
        super().__init__(self.slabs, make_handle, staged=staged, n_global=case.n, native=native)


class DistRankRun(_Steps):
    """One part per process of a torch.distributed group, as one reference
    MPI rank per process: the ghosts travel as one message per peer and
    exchange (isend / irecv of the listed nodes' values, grouped so that two
    ranks sending to each other do not wait on each other's receive; tensors
    on `device`, e.g. CUDA for NCCL, CPU for gloo).  `part` is this rank's
    (its recv / send lists are all the exchange needs)."""

    def __init__(self, part: Part, make_handle: Callable, group=None, device="cpu", n_global=None):
        import torch
        import torch.distributed as dist
        self._torch, self._dist, self.group = torch, dist, group
        if part.rank != dist.get_rank(group):
            raise ValueError(f"part of rank {part.rank} given to rank {dist.get_rank(group)}")
        self.part = part
        self._setup(part.case)
        self.handle = make_handle(part.case)
        self.local = [(part, self.handle)]
        self.device = torch.device(device)
        self.n_global = n_global

    def _peer(self, r):
        return r if self.group is None else self._dist.get_global_rank(self.group, r)

    def exchange(self, names):
        torch, dist, p = self._torch, self._dist, self.part
        st = self.handle.download()
        ops, recvs = [], []
        for peer in range(len(p.send)):
            idx = p.send[peer]
            if peer != p.rank and len(idx):
                buf = np.concatenate([st[nm][idx].reshape(-1) for nm in names])
                ops.append(dist.P2POp(dist.isend, torch.from_numpy(buf).to(self.device), self._peer(peer),
                                      self.group))
        for peer in range(len(p.recv)):
            idx = p.recv[peer]
            if peer != p.rank and len(idx):
                size = sum(st[nm][idx].size for nm in names)
                t = torch.empty(size, dtype=torch.float64, device=self.device)
                ops.append(dist.P2POp(dist.irecv, t, self._peer(peer), self.group))
                recvs.append((idx, t))
        if ops:
            for r in dist.batch_isend_irecv(ops):
                r.wait()
        for idx, t in recvs:
            buf, off = t.cpu().numpy(), 0
            for nm in names:
                shape = st[nm][idx].shape
                size = int(np.prod(shape))
                st[nm][idx] = buf[off:off + size].reshape(shape)
                off += size
        self._upload_fields(self.handle, st)

    def average_rho0(self):
        """averageScalarField over the group: every rank's local sum and
        count gathered, folded in rank order on every rank."""
        sums = [None] * self._dist.get_world_size(self.group)
        self._dist.all_gather_object(sums, self._local_rho_sums(), group=self.group)
        return self._average([x for ss in sums for x in ss])

    def gather(self):
        """Every rank's owned nodes, as the single-domain fields (on every rank)."""
        parts = [None] * self._dist.get_world_size(self.group)
        self._dist.all_gather_object(parts, self.owned(), group=self.group)
        flat = [x for ps in parts for x in ps]
        n = self.n_global if self.n_global is not None else sum(len(p.own) for p, _ in flat)
        return self._assemble(flat, n)


class DistSlabRun(DistRankRun):
    """One slab of a box case per process: rank r of the group holds slab r
    and runs as reference rank rank0 + r."""

    def __init__(self, case: Case, make_handle: Callable, group=None, rank0: int = 0, device="cpu"):
        import torch.distributed as dist
        slabs = split(case, dist.get_world_size(group), rank0)
        super().__init__(slabs[dist.get_rank(group)], make_handle, group=group, device=device, n_global=case.n)


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

    def set_rho0(self, rho_0):
        self.lat.set_rho0(rho_0)

    def op(self, name, field=None):
        m = getattr(self.lat, name)
        return m(field) if field is not None else m()

    def copy_from(self, src, dst_start, src_start, count, names):
        self.lat.copy_nodes(src.lat, dst_start, src_start, count, names)

    def close(self):
        self.lat.close()


class FusedSlabRun:
    """A box lattice cut into slabs along its slowest axis (y in 2D, z in 3D),
    every slab a handle on the fused FP64 path: one kernel per slab and step,
    and before each step a halo exchange device to device.

    Slab r owns planes [a_r, b_r) and holds HALO more planes on each side
    that faces another slab (wrapping on a periodic axis; none on a walled
    face of the box).  A fused step needs, for a node, its pull sources one
    plane away and, for the psi / 1/rho / T / U ring of its tile, the pull
    sources of the ring one plane further: so the halo holds two planes of
    the fused state (post-collision populations, T and U of the last step),
    copied from the neighbouring slabs' owned planes before every step
    (mplb_gpu_copy_state, two copies per cut and direction).  The kernel also
    updates the halo planes; what it writes there is never read before the
    next exchange overwrites it.  The owned planes are then bit-identical to
    the single domain (tests/test_gpu_slabs.py).  This is the multi-rank form
    of the fused path: the reference's exchange inside its operator sequence
    (sendPdfField.c, recvPdfField.c, multiPhasePP.c:163-240) becomes one
    exchange of the fused state per step, which for walls that do not cross a
    cut gives the single domain's result (for a fixedT wall across a cut the
    reference's multi-rank run deviates from its single domain; the operator
    runner RankRun reproduces that deviation, this one does not take such
    cases: the cut is always across the slab axis, walls of that axis lie in
    the first and last slab).
    """

    HALO = 2

    def __init__(self, case: Case, nslabs: int, device: int = -1, stream=None, tile_config: int = 0,
                 mirror: bool = False):
        """mirror=True: the step kernels write the halo themselves
        (mplb_gpu_set_owned, mplb_gpu_add_mirror): every slab stores its owned
        nodes only and also stores its two planes next to each cut into the
        neighbour's next-step input, so a step is one kernel per slab and no
        copies; the halo is exchanged with copies only before the first step
        and after a gather (which brings the handles back to the reference's
        state)."""
        from . import Lattice, PATH_FUSED
        self.case, self.nslabs = case, nslabs
        self.nplanes, self.plane, self.periodic = _box_geometry(case)
        self.slabs = fused_slab_parts(case, nslabs, self.HALO)
        self.mirror = mirror
        self._primed = False
        for s in self.slabs:
            s["lat"] = Lattice(s["case"], path=PATH_FUSED, device=device, stream=stream, tile_config=tile_config)
        if mirror:
            for s in self.slabs:
                s["lat"].set_owned(s["own0"], s["nown"])
            for d, dn, src, sn, cnt in self.exchanges():
                self.slabs[src]["lat"].add_mirror(sn, cnt, self.slabs[d]["lat"], dn)

    def exchanges(self):
        """(destination slab, destination node, source slab, source node, nodes)
        of every halo copy of a step."""
        return halo_copies(self.slabs, self.nslabs, self.plane, self.HALO)

    def initialize(self):
        for s in self.slabs:
            s["lat"].upload_case()
            s["lat"].initialize()
        self._primed = False

    def exchange(self):
        """Halo planes of every slab from its neighbours' owned planes."""
        for d, dn, src, sn, cnt in self.exchanges():
            self.slabs[d]["lat"].copy_state(self.slabs[src]["lat"], dn, sn, cnt)

    def step(self, n=1):
        for _ in range(n):
            if not self.mirror or not self._primed:
                self.exchange()
                self._primed = True
            for s in self.slabs:
                s["lat"].step(1)

    def sync(self):
        for s in self.slabs:
            s["lat"].sync()

    def gather(self):
        """The reference state of the whole box: every slab's owned planes."""
        self._primed = False  # the downloads bring the handles back to the reference's state
        out = {}
        for s in self.slabs:
            d = s["lat"].download()
            for k, v in d.items():
                out.setdefault(k, []).append(v[s["own0"]:s["own0"] + s["nown"]])
        return {k: np.concatenate(v, axis=0) for k, v in out.items()}

    def close(self):
        for s in self.slabs:
            s["lat"].close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def fused_slab_parts(case: Case, nslabs: int, halo: int):
    """The slabs of FusedSlabRun: per slab its owned planes [a, b), its local
    planes [lo, hi) (global planes mod the extent), the global node of every
    local node (gidx), the first owned local node and the owned node count,
    and its local box case (halo faces carry no boundary condition)."""
    from .cases import box_mesh
    if nslabs < 2:
        raise ValueError("at least two slabs")
    nplanes, plane, periodic = _box_geometry(case)
    if nplanes < nslabs * (halo + 1):
        raise ValueError(f"{nplanes} planes cannot give {nslabs} slabs of at least {halo + 1} planes")
    bounds = [round(r * nplanes / nslabs) for r in range(nslabs + 1)]
    axis_name = "Z" if case.lattice == abi.D3Q15 else "Y"
    names_g = list(case.patch_names)
    parts = []
    for r in range(nslabs):
        a, b = bounds[r], bounds[r + 1]
        lo = a - halo if (periodic or r > 0) else a
        hi = b + halo if (periodic or r < nslabs - 1) else b
        gplanes = np.arange(lo, hi) % nplanes
        gidx = (gplanes[:, None] * plane + np.arange(plane)[None, :]).ravel()
        dims = tuple(case.dims[:-1]) + (hi - lo,)
        per = tuple(case.periodic[:-1]) + (False,)
        nb, points, patches, names = box_mesh(case.lattice, dims, per)
        # patch types by face name: the box's own faces keep the case's
        # conditions; a slab face on the cut axis is a wall only where the box
        # has one, else it carries a halo and no condition (periodic)
        fields = {}
        for key, fd in (("f", case.f), ("g", case.g)):
            if fd is None:
                fields[key] = None
                continue
            bt, bv = [], []
            for nm in names:
                cut_face = nm[0] == axis_name and ((nm[1] == "0" and lo != 0) or
                                                   (nm[1] == "1" and hi != nplanes) or periodic)
                if cut_face or nm not in names_g:
                    bt.append(abi.BC_PERIODIC)
                    bv.append((0.0, 0.0, 0.0))
                else:
                    j = names_g.index(nm)
                    bt.append(int(fd["bc_type"][j]))
                    bv.append(tuple(np.asarray(fd["bc_value"], dtype=np.float64).reshape(-1, 3)[j]))
            fields[key] = dict(fd, bc_type=bt, bc_value=np.array(bv, dtype=np.float64).reshape(-1, 3))
        lc = Case(f"{case.name}_slab{r}", case.lattice, dims, per, nb, points, patches, names, case.eos,
                  fields["f"], fields["g"], np.asarray(case.rho)[gidx], np.asarray(case.U)[gidx],
                  np.asarray(case.T)[gidx], meta=dict(case.meta, box=True))
        parts.append(dict(case=lc, a=a, b=b, lo=lo, hi=hi, gidx=gidx, own0=(a - lo) * plane, nown=(b - a) * plane))
    return parts


def halo_copies(parts, nslabs: int, plane: int, halo: int):
    """Every halo copy of a FusedSlabRun step: (destination slab, first
    destination node, source slab, first source node, node count)."""
    out = []
    for r, s in enumerate(parts):
        if s["a"] != s["lo"]:   # halo below <- the top owned planes of the slab below
            nbr = parts[(r - 1) % nslabs]
            out.append((r, 0, (r - 1) % nslabs, nbr["own0"] + nbr["nown"] - halo * plane, halo * plane))
        if s["b"] != s["hi"]:   # halo above <- the bottom owned planes of the slab above
            nbr = parts[(r + 1) % nslabs]
            out.append((r, s["own0"] + s["nown"], (r + 1) % nslabs, nbr["own0"], halo * plane))
    return out
