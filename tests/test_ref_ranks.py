"""Multi-rank runs against the reference's own exchange code.

The reference build under oracle/_ref runs every rank of a partitioned mesh
in one process, one thread per rank: its sendPdfField / recvPdfField,
syncScalarField, syncVectorField (and syncPdfField inside the
surface-tension collisions) pass their messages through the MPI stand-in's
in-process mailbox.  The multi-rank runner (multiphaselb_b200.slabs.RankRun,
the same exchange points and lists as mplb_ranks_step) must give every
rank's owned nodes bit for bit, including where the reference's multi-rank
run is not its single-domain run (a fixedT wall across a cut).

fixedRandomT draws from the C library's one rand() state, seeded with the
rank's pid at every application; the harness runs each rank thread's
boundary update alone so that every rank draws what it would draw in its
own process."""
import ctypes as C
import os

import numpy as np
import pytest

from multiphaselb_b200 import slabs
from oracle import oracle as orc
from tests.helpers import assert_same, small_cases
from tests.test_partition import blocks as blocks_owner
from tests.test_slabs import CheckerHandle, fields_of


def RefRanks(parts):
    if not orc.available("ref") and not orc.ref_tree_present():
        pytest.skip("reference build absent")
    return orc.RefRanks(parts)


def x_halves(c):
    return blocks_owner(c, lambda x, y, z: int(x >= c.dims[0] // 2))


CASES = {
    # irregular blocks over a periodic bubble, three ranks
    "bubble_d2q9": lambda c: blocks_owner(c, lambda x, y, z: ((x // 5) + 2 * (y // 7)) % 3),
    # x halves of the thermal column: the cuts cross both fixedT walls
    "column_d2q9": x_halves,
    # surface tension: the collision itself syncs f (liMRTCollision.c:126-131)
    "st_d2q9": x_halves,
    "st_d3q15": x_halves,
    # the reference partitioner's default decomposition
    "lid_d2q9": lambda c: slabs.standard_owner(c.n, 3),
    "walls_d3q15": lambda c: slabs.standard_owner(c.n, 4),
    "my_column_d2q9": x_halves,
    "cylinder_d2q9": lambda c: blocks_owner(c, lambda x, y, z: int(y >= 7)),
    # outflow with fixedRandomT walls (myMRT): every rank seeds with its pid
    "outflow_d2q9": x_halves,
    "outflow_d3q15": lambda c: slabs.standard_owner(c.n, 3),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_runner_equals_reference_ranks(name):
    case = small_cases()[name]
    parts = slabs.partition(case, CASES[name](case))
    ref = RefRanks(parts)
    ref.run(init=True)
    ref.run(init=False, nsteps=6)
    run = slabs.RankRun(parts, CheckerHandle, n_global=case.n)
    run.initialize()
    run.step(6)
    for (p, want), (_, got) in zip(ref.owned(), run.owned()):
        assert_same(got, want, fields=fields_of(case), ctx=f"{name} rank {p.rank} of {len(parts)}")


@pytest.mark.parametrize("name", ["bubble_d2q9", "column_d2q9", "walls_d3q15"])
def test_adapter_on_reference_ranks(name):
    """include/mplb_gpu_reference.h on the reference's own multi-rank
    structures: every rank packs (ghost rows without neighbours) and the
    ghost runs built from their mpiInfo are the runner's transfers, i.e. the
    exchange mplb_ranks_step is given."""
    from tests.test_adapter import adapter_lib
    lib = adapter_lib()
    lib.adapter_ghost_runs_of_ranks.argtypes = [C.POINTER(C.c_void_p), C.c_uint32, C.c_void_p, C.c_uint32,
                                                C.POINTER(C.c_uint32)]
    lib.adapter_ghost_runs_of_ranks.restype = C.c_int
    case = small_cases()[name]
    parts = slabs.partition(case, CASES[name](case))
    ref = RefRanks(parts)
    cap = sum(len(p.recv[s]) for p in parts for s in range(len(parts))) + 1
    out = np.zeros((cap, 5), dtype=np.uint32)
    n = C.c_uint32(0)
    assert lib.adapter_ghost_runs_of_ranks(ref.harr, len(parts), out.ctypes.data, cap, C.byref(n)) == 0
    run = slabs.RankRun(parts, lambda c: None, staged=True)
    assert [tuple(int(v) for v in row) for row in out[:n.value]] == [tuple(t) for t in run.transfers]


DIST_WORKER = r"""
import os, sys, pickle
sys.path.insert(0, {root!r})
import torch.distributed as dist
dist.init_process_group("gloo", init_method="tcp://127.0.0.1:{port}", rank=int(os.environ["RANK"]),
                        world_size=int(os.environ["WORLD_SIZE"]))
from multiphaselb_b200 import slabs
from tests.helpers import small_cases
from tests.test_ref_ranks import CASES, with_rho0
from tests.test_slabs import CheckerHandle
case = with_rho0(small_cases()[{name!r}], 1.0)
parts = slabs.partition(case, CASES[{name!r}](case))
run = slabs.DistRankRun(parts[dist.get_rank()], CheckerHandle, n_global=case.n)
run.initialize()
run.step({steps})
avg = run.average_rho0()
run.set_rho0(avg)
run.step(2)
out = run.gather()
if dist.get_rank() == 0:
    with open({path!r}, "wb") as fh:
        pickle.dump((out, avg), fh)
dist.barrier()
dist.destroy_process_group()
"""


def test_gloo_ranks_equal_reference_ranks(tmp_path):
    """One process per rank (DistRankRun over gloo) against the reference's
    multi-rank run, on the thermal column cut across its fixedT walls, where
    the reference's multi-rank result is not its single-domain result, with
    a write step's rho_0 update between the steps."""
    import pickle
    from tests.test_multirank import ROOT, free_port, run_ranks
    name, steps = "column_d2q9", 6
    case = with_rho0(small_cases()[name], 1.0)
    parts = slabs.partition(case, CASES[name](case))
    ref = RefRanks(parts)
    ref.run(init=True)
    ref.run(init=False, nsteps=steps)
    avg = ref.average_rho0()
    ref.run(init=False, nsteps=2)
    want = {}
    for p, fields in ref.owned():
        for n, v in fields.items():
            want.setdefault(n, np.zeros((case.n,) + v.shape[1:], dtype=v.dtype))[p.gidx[:len(p.own)]] = v
    path = str(tmp_path / "out.pkl")
    run_ranks(DIST_WORKER.format(root=ROOT, port=free_port(), name=name, steps=steps, path=path), world=len(parts))
    with open(path, "rb") as fh:
        got, got_avg = pickle.load(fh)
    assert all(a == got_avg for a in avg), (got_avg, avg)
    assert_same(got, want, fields=fields_of(case), ctx=f"{name} on {len(parts)} gloo ranks vs reference ranks")


def with_rho0(case, rho_0):
    import dataclasses
    return dataclasses.replace(case, eos=dict(case.eos, rho_0=rho_0))


@pytest.mark.parametrize("name,ranks", [("column_d2q9", None), ("bubble_d2q9", 3), ("walls_d3q15", 4)])
def test_write_step_rho0_equals_reference_ranks(name, ranks):
    """The write step's rho_0 (averageScalarField: local serial sums, then
    MPI_Allreduce of sums and counts) on every rank, and the steps after it
    with the new buoyancy reference, bit for bit against the reference's
    own function on its rank threads."""
    case = with_rho0(small_cases()[name], 1.0)
    owner = CASES[name](case) if ranks is None else slabs.standard_owner(case.n, ranks)
    parts = slabs.partition(case, owner)
    ref = RefRanks(parts)
    ref.run(init=True)
    ref.run(init=False, nsteps=4)
    want = ref.average_rho0()
    # the adapter's helper for C drivers, on the same reference structures
    from tests.test_adapter import adapter_lib
    lib = adapter_lib()
    lib.adapter_average_rho0_of_ranks.argtypes = [C.POINTER(C.c_void_p), C.c_uint32]
    lib.adapter_average_rho0_of_ranks.restype = C.c_double
    assert lib.adapter_average_rho0_of_ranks(ref.harr, len(parts)) == want[0]
    ref.run(init=False, nsteps=4)
    run = slabs.RankRun(parts, CheckerHandle, n_global=case.n)
    run.initialize()
    run.step(4)
    got = run.average_rho0()
    assert all(w == got for w in want), (got, want)
    assert got != 1.0
    run.set_rho0(got)
    run.step(4)
    for (p, w), (_, g) in zip(ref.owned(), run.owned()):
        assert_same(g, w, fields=fields_of(case), ctx=f"{name} rank {p.rank} after the rho_0 update")


def test_rho0_off_when_not_configured():
    """rho_0 <= 0 keeps the average at 0, as averageScalarField does."""
    case = small_cases()["column_d2q9"]
    parts = slabs.partition(case, CASES["column_d2q9"](case))
    ref = RefRanks(parts)
    ref.run(init=True)
    run = slabs.RankRun(parts, CheckerHandle, n_global=case.n)
    run.initialize()
    assert ref.average_rho0() == [0.0] * len(parts) and run.average_rho0() == 0.0
