"""include/mplb_gpu_reference.h on the reference's own structures.

CPU: the descriptors packed from latticeMesh / lbeField / EOSInfo equal the
structures field by field.  GPU: the drop-in loop (reference structs -> GPU
handle -> steps -> results written back into the reference structs) leaves
exactly the state the reference's own CPU loop produces."""
import ctypes as C
import os

import numpy as np
import pytest

from multiphaselb_b200 import abi
from oracle import oracle as orc
from tests.helpers import FIELDS, assert_same, small_cases

HERE = os.path.dirname(os.path.abspath(__file__))
ADAPTER = os.path.join(HERE, "..", "oracle", "_ref", "libmplb_adapter_check.so")


def adapter_lib():
    if not os.path.exists(ADAPTER):
        if not orc.ref_tree_present():
            pytest.skip("adapter checker not built and the reference tree is absent")
        from multiphaselb_b200 import build
        build.build()
        orc.make("adapter")
    orc._lib("ref")  # load the harness first (same file the adapter links)
    lib = C.CDLL(ADAPTER)
    lib.adapter_pack_check.argtypes = [C.c_void_p]
    lib.adapter_pack_check.restype = C.c_int
    lib.adapter_gpu_run.argtypes = [C.c_void_p, C.c_uint32, C.c_int, C.c_uint32]
    lib.adapter_gpu_run.restype = C.c_int
    return lib


@pytest.mark.parametrize("name", list(small_cases().keys()))
def test_adapter_packs_reference_structs(name):
    lib = adapter_lib()
    k = orc.Checker("ref", small_cases()[name])
    k.upload_case()
    k.initialize()
    assert lib.adapter_pack_check(k.h) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(small_cases().keys()))
@pytest.mark.parametrize("path", [abi.PATH_AUTO, abi.PATH_OPERATORS])
def test_adapter_dropin_loop_matches_reference(gpu_lib, name, path):
    lib = adapter_lib()
    case = small_cases()[name]
    cpu, gpu = orc.Checker("ref", case), orc.Checker("ref", case)
    for k in (cpu, gpu):
        k.upload_case()
        k.initialize()
    cpu.step(6)
    assert lib.adapter_gpu_run(gpu.h, 6, path, 0) == 0
    fields = [f for f in FIELDS if not (f == "g" and case.g is None)]
    assert_same(gpu.download(), cpu.download(), fields=fields, ctx=f"adapter {name} path {path}")


def _partition(name):
    from multiphaselb_b200 import slabs
    from tests.test_partition import OWNERS, get_case
    case = get_case(name)
    return case, slabs.partition(case, OWNERS[name](case))


@pytest.mark.parametrize("name", ["bubble_d2q9", "bubble_d3q15"])
def test_adapter_packs_partitioned_ranks(name):
    """A rank of a partitioned mesh (owned nodes, then ghosts, neighbours for
    the owned nodes only, as readLatticeMesh reads them) packs into a
    descriptor whose ghost rows have no neighbours."""
    lib = adapter_lib()
    lib.adapter_pack_part_check.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p,
                                            C.c_uint32, C.c_uint32]
    lib.adapter_pack_part_check.restype = C.c_int
    case, parts = _partition(name)
    k = orc.Checker("ref", case)
    for p in parts:
        nlocal = len(p.own)
        nb = np.ascontiguousarray(p.case.nb[:nlocal], dtype=np.int32)
        pts = np.ascontiguousarray(p.case.points, dtype=np.int32)
        assert lib.adapter_pack_part_check(k.h, p.case.n, nlocal, nb.ctypes.data, pts.ctypes.data,
                                           p.rank, len(parts)) == 0
        # the descriptor the adapter packs is the one the Python runner creates its handle from
        assert (p.case.nb[nlocal:] == -1).all()
    # a single rank with ghosts is refused
    p = parts[0]
    nb = np.ascontiguousarray(p.case.nb[:len(p.own)], dtype=np.int32)
    pts = np.ascontiguousarray(p.case.points, dtype=np.int32)
    assert lib.adapter_pack_part_check(k.h, p.case.n, len(p.own), nb.ctypes.data, pts.ctypes.data,
                                       0, 1) == 1000 - abi.E_UNSUPPORTED


def _ghost_runs(lib, parts, pid_of=None):
    R = len(parts)
    lib.adapter_ghost_runs.argtypes = [C.c_uint32] + [C.c_void_p] * 6 + [C.c_uint32, C.POINTER(C.c_uint32)]
    lib.adapter_ghost_runs.restype = C.c_int
    u32 = lambda a: np.ascontiguousarray(a, dtype=np.uint32)
    pid = u32(range(R) if pid_of is None else pid_of)
    nrg = u32([[len(p.recv[s]) for s in range(R)] for p in parts])
    nsg = u32([[len(p.send[s]) for s in range(R)] for p in parts])
    recv = u32(np.concatenate([np.asarray(p.recv[s]) for p in parts for s in range(R)] + [np.zeros(1)]))
    send = u32(np.concatenate([np.asarray(p.send[s]) for p in parts for s in range(R)] + [np.zeros(1)]))
    cap = int(nrg.sum()) + 1
    out = np.zeros((cap, 5), dtype=np.uint32)
    n = C.c_uint32(0)
    rc = lib.adapter_ghost_runs(R, pid.ctypes.data, nrg.ctypes.data, recv.ctypes.data, nsg.ctypes.data,
                                send.ctypes.data, out.ctypes.data, cap, C.byref(n))
    return rc, [tuple(int(v) for v in row) for row in out[:n.value]]


@pytest.mark.parametrize("name", sorted(["bubble_d2q9", "st_d2q9", "cylinder", "bubble_d3q15"]))
def test_adapter_ghost_runs_match_runner(name):
    """The exchange built in C from the ranks' recvGhosts / sendGhosts is the
    one the multi-rank runner passes to mplb_ranks_step (the runner is
    bitwise against the single domain, tests/test_partition.py)."""
    from multiphaselb_b200 import slabs
    lib = adapter_lib()
    case, parts = _partition(name)
    rc, runs = _ghost_runs(lib, parts)
    assert rc == 0
    run = slabs.RankRun(parts, lambda c: None, staged=True)
    assert runs == [tuple(t) for t in run.transfers]
    assert sum(r[4] for r in runs) == sum(len(p.recv[s]) for p in parts for s in range(len(parts)))


def test_adapter_ghost_runs_refusals():
    """Lists that do not pair, or meshes out of pid order, are refused."""
    lib = adapter_lib()
    case, parts = _partition("bubble_d2q9")
    R = len(parts)
    rc, _ = _ghost_runs(lib, parts, pid_of=list(range(R))[::-1])
    assert rc == abi.E_ARG
    # drop one ghost from rank 0's list from rank 1
    import copy
    bad = copy.deepcopy(parts)
    bad[0].recv[1] = bad[0].recv[1][:-1]
    rc, _ = _ghost_runs(lib, bad)
    assert rc == abi.E_ARG
