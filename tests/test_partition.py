"""Multi-rank runs of any mesh (multiphaselb_b200.slabs.partition and
from_meshes): an owner rank per node, the local numbering and ghost lists
of the reference's partitioner, the ranks stepped on CPU checkers with the
reference's exchanges, and the reference's per-rank mesh files written and
read back.  Owned nodes against the single-domain run, bitwise.  Host code
and the CPU oracle only."""
import numpy as np
import pytest

from multiphaselb_b200 import abi, mesh, slabs
from tests.helpers import assert_same, run_checker, small_cases
from tests.test_slabs import CheckerHandle, fields_of


def blocks(case, fn):
    pts = np.asarray(case.points)
    return np.array([fn(*p) for p in pts.tolist()], dtype=np.int64)


def cylinder_bounceback():
    """The channel with a cylinder, the heat's cylinder patch bounce-back (a
    wall crossing a cut that extrapolates would differ as in the reference)."""
    c = small_cases()["cylinder_d2q9"]
    c.g = dict(c.g, bc_type=[abi.BC_FIXEDT, abi.BC_FIXEDT, abi.BC_BOUNCEBACK])
    return c


OWNERS = {
    # irregular blocks over a periodic bubble, 24 x 20, three ranks
    "bubble_d2q9": lambda c: blocks(c, lambda x, y, z: ((x // 5) + 2 * (y // 7)) % 3),
    # x halves of the surface-tension channel: the cut crosses its walls
    "st_d2q9": lambda c: blocks(c, lambda x, y, z: int(x >= 9)),
    # y halves of the channel with a cylinder: the cut crosses the cylinder
    "cylinder": lambda c: blocks(c, lambda x, y, z: int(y >= 7)),
    # D3Q15 in x halves and z thirds
    "bubble_d3q15": lambda c: blocks(c, lambda x, y, z: int(x >= 5) * 3 + z // 2),
}


def get_case(name):
    return cylinder_bounceback() if name == "cylinder" else small_cases()[name]


@pytest.mark.parametrize("name", sorted(OWNERS))
def test_partitioned_run_equals_single_domain(name):
    case = get_case(name)
    owner = OWNERS[name](case)
    parts = slabs.partition(case, owner, rank0=case.meta.get("rank", 0))
    run = slabs.RankRun(parts, CheckerHandle, n_global=case.n)
    run.initialize()
    run.step(6)
    assert_same(run.gather(), run_checker("port", case, 6), fields=fields_of(case),
                ctx=f"{name} on {len(parts)} ranks")


def test_partition_numbering_and_ghost_lists():
    """Local numbering of localIndexing.c (owned nodes in global order, then
    ghosts as a scan of the owned nodes' pull sources first meets them) and
    the ghost lists of latticeMeshPartition.c (paired, in global order)."""
    case = small_cases()["bubble_d2q9"]
    owner = OWNERS["bubble_d2q9"](case)
    parts = slabs.partition(case, owner)
    for p in parts:
        own = np.nonzero(owner == p.rank)[0]
        assert np.array_equal(p.gidx[:len(own)], own) and np.array_equal(p.own, np.arange(len(own)))
        seen, order = set(own.tolist()), []
        for i in own:
            for s in case.nb[i]:
                if s >= 0 and s not in seen:
                    seen.add(int(s))
                    order.append(int(s))
        assert p.gidx[len(own):].tolist() == order
        # ghost rows have no neighbours; owned rows pull from the same nodes as the single domain
        assert (p.case.nb[len(own):] == -1).all()
        assert np.array_equal(p.gidx[p.case.nb[:len(own)]], case.nb[own])
        got = np.concatenate([p.recv[s] for s in range(len(parts))])
        assert sorted(got.tolist()) == list(range(len(own), len(p.gidx)))
    for r, p in enumerate(parts):
        for s, q in enumerate(parts):
            g = p.gidx[p.recv[s]]
            assert np.array_equal(g, q.gidx[q.send[r]]) and np.all(np.diff(g) > 0) and (owner[g] == s).all()


def test_mesh_files_round_trip_run(tmp_path):
    """Each rank's part written as the reference's processor<pid>/lattice
    files (points, ghosts, neighbours of the local nodes, boundary,
    recvGhosts, sendGhosts), read back and run: the same owned fields."""
    case = cylinder_bounceback()
    owner = OWNERS["cylinder"](case)
    parts = slabs.partition(case, owner)
    for p in parts:
        nl = len(p.own)
        m = mesh.LatticeMesh(case.lattice, p.case.points, p.case.nb[:nl], list(case.patch_names),
                             p.case.patches, nl, len(p.gidx) - nl, None, p.recv, p.send)
        mesh.write_lattice_mesh(m, str(tmp_path), pid=p.rank)
    meshes = [mesh.read_lattice_mesh(str(tmp_path), pid=r) for r in range(len(parts))]
    fields = [(p.case.rho, p.case.U, p.case.T) for p in parts]
    back = slabs.from_meshes(meshes, case.name, case.eos, case.f, case.g, fields)
    outs = []
    for ps in (parts, back):
        run = slabs.RankRun(ps, CheckerHandle)
        run.initialize()
        run.step(4)
        outs.append(run.owned())
    for (p, a), (q, b) in zip(*outs):
        assert_same(b, a, fields=fields_of(case), ctx=f"rank {p.rank} from files")


def _ref_standard(n, ranks):
    import ctypes as C
    import os
    from oracle import oracle as orc
    if not orc.available("ref") and not orc.ref_tree_present():
        pytest.skip("reference build absent")
    lib = orc._lib("ref")
    fn = lib.ref_standard_decomp
    fn.argtypes = [C.c_uint32, C.c_uint32, C.c_void_p]
    out = np.full(n, 0xFFFFFFFF, dtype=np.uint32)
    fn(n, ranks, out.ctypes.data)
    return out.astype(np.int64)


@pytest.mark.parametrize("n,ranks", [(480, 3), (481, 7), (10, 10), (7, 1), (65536, 148), (7_077_888, 8)])
def test_standard_owner_is_the_reference_decomposition(n, ranks):
    """slabs.standard_owner equals the reference partitioner's default method
    (standardDecomp.c, compiled from the reference's source)."""
    assert np.array_equal(slabs.standard_owner(n, ranks), _ref_standard(n, ranks))


@pytest.mark.parametrize("name,ranks", [("bubble_d2q9", 3), ("bubble_d3q15", 4), ("st_d2q9", 2)])
def test_standard_partition_run_equals_single_domain(name, ranks):
    """The reference's default partition of a periodic mesh, stepped rank by
    rank with its ghost exchange, is the single-domain run bit for bit."""
    case = get_case(name)
    parts = slabs.partition(case, slabs.standard_owner(case.n, ranks), rank0=case.meta.get("rank", 0))
    assert len(parts) == ranks
    run = slabs.RankRun(parts, CheckerHandle, n_global=case.n)
    run.initialize()
    run.step(6)
    assert_same(run.gather(), run_checker("port", case, 6), fields=fields_of(case),
                ctx=f"{name} standard decomposition on {ranks} ranks")


def test_refusals():
    case = small_cases()["bubble_d2q9"]
    with pytest.raises(ValueError):
        slabs.partition(case, np.zeros(case.n - 1, dtype=int))
    with pytest.raises(ValueError):
        slabs.partition(case, np.where(np.arange(case.n) < 10, 0, 2))    # rank 1 owns nothing
    for ranks in (0, case.n + 1):                                         # the reference's block of 0 nodes
        with pytest.raises(ValueError):
            slabs.standard_owner(case.n, ranks)
    parts = slabs.partition(case, OWNERS["bubble_d2q9"](case))
    m = [mesh.LatticeMesh(case.lattice, p.case.points, p.case.nb[:len(p.own)], [], [], len(p.own),
                          len(p.gidx) - len(p.own), None, p.recv, p.send) for p in parts]
    m[1].send_ghosts = [s[:-1] if len(s) else s for s in m[1].send_ghosts]
    with pytest.raises(ValueError):
        slabs.from_meshes(m, "x", case.eos, case.f, case.g, [(p.case.rho, p.case.U, p.case.T) for p in parts])


DIST_WORKER = r"""
import os, sys, pickle
sys.path.insert(0, {root!r})
import numpy as np
import torch.distributed as dist
dist.init_process_group("gloo", init_method="tcp://127.0.0.1:{port}", rank=int(os.environ["RANK"]),
                        world_size=int(os.environ["WORLD_SIZE"]))
from multiphaselb_b200 import slabs
from tests.test_partition import OWNERS, get_case
from tests.test_slabs import CheckerHandle
case = get_case({name!r})
parts = slabs.partition(case, OWNERS[{name!r}](case))
run = slabs.DistRankRun(parts[dist.get_rank()], CheckerHandle, n_global=case.n)
run.initialize()
run.step({steps})
out = run.gather()
if dist.get_rank() == 0:
    with open({path!r}, "wb") as fh:
        pickle.dump(out, fh)
dist.barrier()
dist.destroy_process_group()
"""


def test_partitioned_gloo_ranks(tmp_path):
    """One partitioned rank per gloo process (irregular blocks, 3 ranks)."""
    import pickle
    from tests.test_multirank import ROOT, free_port, run_ranks
    path = str(tmp_path / "out.pkl")
    run_ranks(DIST_WORKER.format(root=ROOT, port=free_port(), name="bubble_d2q9", steps=5, path=path), world=3)
    with open(path, "rb") as fh:
        got = pickle.load(fh)
    case = get_case("bubble_d2q9")
    assert_same(got, run_checker("port", case, 5), fields=fields_of(case), ctx="bubble_d2q9 on 3 gloo ranks")
