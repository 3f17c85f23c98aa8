"""Slab decomposition (multiphaselb_b200.slabs) against the single domain:
a box cut into 2 or 3 slabs along its slowest axis, each slab on its own
oracle lattice with one ghost plane per cut, the ghost planes exchanged at
the reference's points in the step (multiPhasePP.c:163-240).  The owned
nodes of the slabs, gathered, are bit-identical to the single-domain run.
Host code and the CPU oracle only."""
import numpy as np
import pytest

from multiphaselb_b200 import abi, slabs
from oracle import oracle as orc
from tests.helpers import FIELDS, assert_same, run_checker, small_cases

OPS = {"equilibrium": orc.OP_EQUILIBRIUM, "collision": orc.OP_COLLISION, "lbstream": orc.OP_LBSTREAM,
       "update_boundaries": orc.OP_BOUNDARIES, "macro_density": orc.OP_DENSITY,
       "macro_velocity": orc.OP_VELOCITY, "macro_temperature": orc.OP_TEMPERATURE,
       "inter_force": orc.OP_INTERFORCE, "heat_source": orc.OP_HEATSOURCE}


class CheckerHandle:
    """The slab runner's operator interface over a CPU checker."""

    def __init__(self, case):
        self.k = orc.Checker("port", case)

    def upload(self, **fields):
        self.k.upload(**fields)

    def download(self):
        return self.k.download()

    def set_time(self, t):
        self.k.set_time(t)

    def get_time(self):
        return self.k.get_time()

    def set_rho0(self, r):
        self.k.set_rho0(r)

    def op(self, name, field=None):
        self.k.op(OPS[name], abi.FIELD_F if field is None else field)


def fields_of(case):
    return [f for f in FIELDS if not (f == "g" and case.g is None)]


@pytest.mark.parametrize("name,ranks", [
    ("column_d2q9", 2), ("column_d2q9", 3),      # fixedT / bounce-back walls at the ends
    ("bubble_d2q9", 2), ("bubble_d2q9", 3),      # periodic: the ghost planes wrap
    ("lid_d2q9", 2),                             # fixedU lid
    ("my_column_d2q9", 3),                       # myMRT heat
    ("outflow_d2q9", 2),                         # outflow top, fixedRandomT bottom
    ("st_d2q9", 2), ("st_d2q9", 3),              # surface tension: post-collision sync
    ("st_d3q15", 2),
    ("bubble_d3q15", 3),                         # D3Q15, cut along z
    ("walls_d3q15", 2),
    ("my_slab_d3q15", 2),
])
def test_slabs_equal_single_domain(name, ranks):
    case = small_cases()[name]
    steps = 6
    want = run_checker("port", case, steps)
    # the bottom slab takes the single domain's pid, which seeds fixedRandomT
    run = slabs.SlabRun(case, ranks, CheckerHandle, rank0=case.meta.get("rank", 0))
    run.initialize()
    run.step(steps)
    assert_same(run.gather(), want, fields=fields_of(case), ctx=f"{name} in {ranks} slabs")


def test_cut_deviation_of_the_reference():
    """Where the reference's multi-rank run differs from its single-domain
    run, the split differs the same way and nowhere else: a ghost node does
    not stream (lbstream.c loops over the local nodes), and a fixedT wall node
    next to a cut extrapolates from the ghost's post-collision PDF (the
    exchange follows the boundaries) where the single domain reads the
    streamed one.  After one step the differing PDFs are exactly those."""
    # fixedT side wall, 10 x 12 walled box in 3 slabs: cuts at y = 4 and 8
    case = small_cases()["outflow_corner_d2q9"]
    nx = case.dims[0]
    want = run_checker("port", case, 1)
    run = slabs.SlabRun(case, 3, CheckerHandle, rank0=case.meta.get("rank", 0))
    run.initialize()
    run.step(1)
    got = run.gather()
    assert np.array_equal(got["f"], want["f"])
    node, k = np.nonzero(got["g"] != want["g"])
    assert len(node) > 0
    rev = np.asarray(orc_rev(case))
    assert (case.nb[node, k] == -1).all()                      # unknown populations of wall nodes
    slab_of = np.searchsorted([4, 8], node // nx, side="right")
    xsrc = case.nb[node, rev[k]]
    assert (slab_of != np.searchsorted([4, 8], xsrc // nx, side="right")).all()   # extrapolated from a ghost


def orc_rev(case):
    """Index of the opposite velocity of each lattice velocity."""
    from multiphaselb_b200 import cases as cs
    c = np.asarray(cs.VEL[case.lattice])
    return [int(np.nonzero((c == -c[k]).all(1))[0][0]) for k in range(len(c))]


def test_split_layout():
    """Planes, owned ranges and the neighbour table of a periodic 2D split."""
    case = small_cases()["bubble_d2q9"]          # 24 x 20, periodic in x and y
    ss = slabs.split(case, 3)
    nx = case.dims[0]
    assert [s.planes[s.own_lo] for s in ss] == [0, 7, 13]
    assert [s.own_hi - s.own_lo for s in ss] == [7, 6, 7]
    assert ss[0].planes[0] == 19 and ss[2].planes[-1] == 0           # wrapped ghosts
    for s in ss:
        lc = s.case
        assert lc.n == len(s.planes) * nx and lc.meta["rank"] == s.rank
        own = slice(s.own_lo * nx, s.own_hi * nx)
        # an owned node pulls from the node the single domain pulls from
        g = case.nb[s.gidx[own]]
        got = lc.nb[own]
        assert (got >= 0).all()
        assert np.array_equal(s.gidx[got], g)
        assert (np.delete(lc.nb, np.arange(own.start, own.stop), axis=0) == -1).all()   # ghosts


def test_split_walls_patches_and_refusals():
    case = small_cases()["column_d2q9"]          # 12 x 24, walls at y = 0 and 23
    ss = slabs.split(case, 2)
    nx = case.dims[0]
    assert ss[0].own_lo == 0 and ss[0].planes == list(range(0, 13))   # no ghost below the wall
    assert ss[1].own_hi == len(ss[1].planes)
    # every wall node lands in exactly one slab, as an owned node
    for p, pts in enumerate(case.patches):
        got = np.concatenate([s.gidx[s.case.patches[p].astype(np.int64)] for s in ss])
        assert np.array_equal(np.sort(got), np.sort(pts.astype(np.int64)))
        for s in ss:
            loc = s.case.patches[p].astype(np.int64)
            assert ((loc >= s.own_lo * nx) & (loc < s.own_hi * nx)).all()
    with pytest.raises(ValueError):
        slabs.split(case, 1)
    with pytest.raises(ValueError):
        slabs.split(case, 13)


DIST_WORKER = r"""
import os, sys, json, pickle
sys.path.insert(0, {root!r})
import numpy as np
import torch.distributed as dist
dist.init_process_group("gloo", init_method="tcp://127.0.0.1:{port}", rank=int(os.environ["RANK"]),
                        world_size=int(os.environ["WORLD_SIZE"]))
from multiphaselb_b200 import slabs
from tests.helpers import small_cases
from tests.test_slabs import CheckerHandle
case = small_cases()[{name!r}]
run = slabs.DistSlabRun(case, CheckerHandle, rank0=case.meta.get("rank", 0))
run.initialize()
run.step({steps})
out = run.gather()
if dist.get_rank() == 0:
    with open({path!r}, "wb") as fh:
        pickle.dump(out, fh)
dist.barrier()
dist.destroy_process_group()
"""


@pytest.mark.parametrize("name,world", [("column_d2q9", 2), ("bubble_d2q9", 3), ("outflow_d2q9", 2),
                                        ("st_d2q9", 3), ("bubble_d3q15", 2)])
def test_one_process_per_slab_gloo(tmp_path, name, world):
    """DistSlabRun: one slab per gloo rank, ghost planes by point-to-point
    messages; the gathered fields equal the single-domain run bitwise."""
    import pickle
    from tests.test_multirank import ROOT, free_port, run_ranks
    path = str(tmp_path / "out.pkl")
    code = DIST_WORKER.format(root=ROOT, port=free_port(), name=name, steps=6, path=path)
    run_ranks(code, world=world)
    with open(path, "rb") as fh:
        got = pickle.load(fh)
    case = small_cases()[name]
    assert_same(got, run_checker("port", case, 6), fields=fields_of(case), ctx=f"{name} on {world} gloo ranks")


@pytest.mark.parametrize("R", [2, 3, 4])
@pytest.mark.parametrize("name", ["column_d2q9", "bubble_d2q9", "walls_d3q15"])
def test_fused_slab_mirror_plan(name, R):
    """FusedSlabRun(mirror=True) turns every halo copy into a mirrored range
    of its source slab (mplb_gpu_add_mirror): at most two per slab (the
    library's limit), each inside its slab's owned nodes, each target outside
    the destination's owned nodes, and every halo node of every slab written
    by exactly one range, so no two kernels store the same node in a step."""
    case = small_cases()[name]
    nplanes, plane, periodic = slabs._box_geometry(case)
    if nplanes < 3 * R:
        return
    parts = slabs.fused_slab_parts(case, R, 2)
    per_src = [0] * R
    writes = [np.zeros(p["case"].n, dtype=int) for p in parts]
    for d, dn, s, sn, c in slabs.halo_copies(parts, R, plane, 2):
        per_src[s] += 1
        assert parts[s]["own0"] <= sn and sn + c <= parts[s]["own0"] + parts[s]["nown"]
        assert dn + c <= parts[d]["own0"] or dn >= parts[d]["own0"] + parts[d]["nown"]
        writes[d][dn:dn + c] += 1
    assert max(per_src) <= 2
    for p, w in zip(parts, writes):
        own = np.zeros(p["case"].n, dtype=bool)
        own[p["own0"]:p["own0"] + p["nown"]] = True
        assert np.all(w[own] == 0) and np.all(w[~own] == 1)


@pytest.mark.parametrize("R", [2, 3, 4])
@pytest.mark.parametrize("name", ["column_d2q9", "bubble_d2q9", "walls_d3q15"])
def test_fused_slab_plan(name, R):
    """FusedSlabRun's plan: the owned planes cover the box once in order,
    every halo copy fills halo nodes from owned nodes of the same global
    nodes, each local case is a box whose halo faces carry no condition, and
    its fields are the box's fields of its nodes."""
    case = small_cases()[name]
    nplanes, plane, periodic = slabs._box_geometry(case)
    if nplanes < 3 * R:
        with pytest.raises(ValueError, match="cannot give"):
            slabs.fused_slab_parts(case, R, 2)
        return
    parts = slabs.fused_slab_parts(case, R, 2)
    own = np.concatenate([p["gidx"][p["own0"]:p["own0"] + p["nown"]] for p in parts])
    assert np.array_equal(own, np.arange(case.n))
    copies = slabs.halo_copies(parts, R, plane, 2)
    filled = [set() for _ in parts]
    for d, dn, s, sn, c in copies:
        assert np.array_equal(parts[d]["gidx"][dn:dn + c], parts[s]["gidx"][sn:sn + c])
        assert parts[s]["own0"] <= sn and sn + c <= parts[s]["own0"] + parts[s]["nown"]
        filled[d].update(range(dn, dn + c))
    for p, f in zip(parts, filled):
        halo = set(range(p["case"].n)) - set(range(p["own0"], p["own0"] + p["nown"]))
        assert f == halo
        lc = p["case"]
        assert np.array_equal(lc.rho, np.asarray(case.rho)[p["gidx"]])
        for nm, t in zip(lc.patch_names, lc.f["bc_type"]):
            wall = nm in case.patch_names and not (
                nm[0] in "YZ" and ((nm[1] == "0" and p["lo"] != 0) or (nm[1] == "1" and p["hi"] != nplanes) or periodic))
            if not wall:
                assert t == abi.BC_PERIODIC
