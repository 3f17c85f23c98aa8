"""Multi-rank runs against the reference's own exchange code.

The reference build under oracle/_ref runs every rank of a partitioned mesh
in one process, one thread per rank: its sendPdfField / recvPdfField,
syncScalarField, syncVectorField (and syncPdfField inside the
surface-tension collisions) pass their messages through the MPI stand-in's
in-process mailbox.  The multi-rank runner (multiphaselb_b200.slabs.RankRun,
the same exchange points and lists as mplb_ranks_step) must give every
rank's owned nodes bit for bit, including where the reference's multi-rank
run is not its single-domain run (a fixedT wall across a cut).

fixedRandomT cases are left out: the reference draws its wall values from
the C library's one rand() state, which rank threads would share."""
import ctypes as C
import os

import numpy as np
import pytest

from multiphaselb_b200 import slabs
from oracle import oracle as orc
from tests.helpers import assert_same, small_cases
from tests.test_partition import blocks as blocks_owner
from tests.test_slabs import CheckerHandle, fields_of


def ref_lib():
    if not orc.available("ref") and not os.path.isdir("/root/reference/src"):
        pytest.skip("reference build absent")
    lib = orc._lib("ref")
    if not hasattr(lib, "ref_ranks_run"):
        pytest.skip("reference build predates the multi-rank harness")
    lib.ref_set_parallel.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32] + [C.c_void_p] * 4
    lib.ref_set_parallel.restype = C.c_int
    lib.ref_ranks_run.argtypes = [C.POINTER(C.c_void_p), C.c_uint32, C.c_int, C.c_uint32]
    lib.ref_ranks_run.restype = C.c_int
    return lib


class RefRanks:
    """Every part as a reference case with its mpiInfo, stepped together."""

    def __init__(self, parts):
        self.lib = ref_lib()
        self.parts = parts
        R = len(parts)
        self.k = [orc.Checker("ref", p.case, rank=p.rank) for p in parts]
        u32 = lambda a: np.ascontiguousarray(np.concatenate([np.asarray(x, dtype=np.uint32) for x in a]
                                                            + [np.zeros(1, np.uint32)]))
        for k, p in zip(self.k, parts):
            nrg = np.array([len(p.recv[s]) for s in range(R)], dtype=np.uint32)
            nsg = np.array([len(p.send[s]) for s in range(R)], dtype=np.uint32)
            recv, send = u32(p.recv), u32(p.send)
            rc = self.lib.ref_set_parallel(k.h, p.rank, R, len(p.own), nrg.ctypes.data, recv.ctypes.data,
                                           nsg.ctypes.data, send.ctypes.data)
            assert rc == 0, rc
            k.upload(rho=p.case.rho, U=p.case.U, T=p.case.T)
        self.harr = (C.c_void_p * R)(*[k.h for k in self.k])

    def run(self, init, nsteps=0):
        rc = self.lib.ref_ranks_run(self.harr, len(self.k), int(init), nsteps)
        assert rc == 0, f"reference ranks: {rc}"

    def owned(self):
        return [(p, {n: v[:len(p.own)] for n, v in k.download().items()}) for p, k in zip(self.parts, self.k)]


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
