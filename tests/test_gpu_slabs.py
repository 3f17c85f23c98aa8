"""Slab decomposition on the device: every slab a device lattice on the
operator path (multiphaselb_b200.slabs.LatticeHandle), the ghost planes
exchanged at the reference's points, against the same split run on CPU
checkers; the whole step in the library (mplb_ranks_step), the ghost
exchange device to device driven from Python (mplb_gpu_copy_nodes), and
through the host.  Bitwise.  Also mplb_gpu_copy_nodes itself: what it
copies and what it refuses."""
import numpy as np
import pytest

from multiphaselb_b200 import Lattice, MplbError, abi, slabs
from tests.helpers import assert_same, small_cases
from tests.test_slabs import CheckerHandle, fields_of

pytestmark = pytest.mark.gpu


def run_split(case, ranks, make, staged=False, native=True):
    run = slabs.SlabRun(case, ranks, make, rank0=case.meta.get("rank", 0), staged=staged, native=native)
    assert run.direct == (make is slabs.LatticeHandle and not staged)
    assert run.native == (run.direct and native)
    run.initialize()
    run.step(5)
    out = run.gather()
    for h in run.handles:
        if hasattr(h, "close"):
            h.close()
    return out


@pytest.mark.parametrize("name,ranks", [("column_d2q9", 3), ("bubble_d2q9", 2), ("outflow_corner_d2q9", 3),
                                        ("st_d2q9", 2), ("my_slab_d3q15", 2), ("bubble_d3q15", 3)])
def test_device_slabs_match_checker_slabs(gpu_lib, name, ranks):
    case = small_cases()[name]
    want = run_split(case, ranks, CheckerHandle)
    fields = fields_of(case)
    assert_same(run_split(case, ranks, slabs.LatticeHandle), want, fields=fields,
                ctx=f"{name} in {ranks} slabs, whole step in the library vs checker")
    assert_same(run_split(case, ranks, slabs.LatticeHandle, native=False), want, fields=fields,
                ctx=f"{name} in {ranks} slabs, device-to-device exchange driven from Python vs checker")
    assert_same(run_split(case, ranks, slabs.LatticeHandle, staged=True), want, fields=fields,
                ctx=f"{name} in {ranks} slabs, host-staged exchange vs checker")


def test_copy_nodes_copies_ranges_of_every_field(gpu_lib):
    case = small_cases()["column_d2q9"]
    rng = np.random.default_rng(7)
    n, Q = case.n, case.Q
    a_fields = dict(rho=rng.random(n), U=rng.random((n, 3)), T=rng.random(n), f=rng.random((n, Q)),
                    g=rng.random((n, Q)), S=rng.random(n), Fi=rng.random((n, 3)), Ft=rng.random((n, 3)))
    b_fields = {k: np.zeros_like(v) for k, v in a_fields.items()}
    with Lattice(case, path=abi.PATH_OPERATORS) as a, Lattice(case, path=abi.PATH_OPERATORS) as b:
        a.upload(**a_fields)
        b.upload(**b_fields)
        b.copy_nodes(a, 30, 100, 17, fields=("f", "S", "U"))
        b.copy_nodes(b, 200, 30, 5, fields=("f",))          # on one handle, after the first copy
        got = b.download()
        for k in a_fields:
            want = b_fields[k].copy()
            if k in ("f", "S", "U"):
                want[30:47] = a_fields[k][100:117]
            if k == "f":
                want[200:205] = a_fields[k][100:105]
            assert np.array_equal(got[k], want), k
        with pytest.raises(MplbError) as e:
            b.copy_nodes(a, n - 3, 0, 4)
        assert e.value.code == abi.E_ARG
        with pytest.raises(MplbError) as e:
            b.copy_nodes(b, 10, 12, 4)
        assert e.value.code == abi.E_ARG
        assert b.lib.mplb_gpu_copy_nodes(b.h, 0, a.h, 0, 1, 256) == abi.E_ARG


@pytest.mark.parametrize("name", ["bubble_d2q9", "cylinder", "bubble_d3q15"])
def test_device_partition_matches_checker_partition(gpu_lib, name):
    """Irregular partitions: the ghosts of a rank form many short runs of
    nodes, each one device copy per field."""
    from tests.test_partition import OWNERS, get_case
    case = get_case(name)
    parts = slabs.partition(case, OWNERS[name](case))
    outs = []
    for make in (CheckerHandle, slabs.LatticeHandle):
        run = slabs.RankRun(parts, make, n_global=case.n)
        assert run.native == (make is slabs.LatticeHandle)
        run.initialize()
        run.step(5)
        outs.append(run.gather())
        run.close()
    assert_same(outs[1], outs[0], fields=fields_of(case), ctx=f"{name} partitioned, device vs checker")


# ---------------------------------------------------------------- fused slabs
def bubble_d3q15_z12():
    from multiphaselb_b200 import cases
    return cases.perturbed(cases.bubble_case(abi.D3Q15, 10, 3.0, 2.0, 0.75, dims=(10, 8, 12)), du=1e-3)


FUSED_SLAB_CASES = [("column_d2q9", 2), ("column_d2q9", 4), ("bubble_d2q9", 3), ("st_d2q9", 3),
                    ("walls_d3q15", 2), ("bubble_d3q15_z12", 4)]


def fused_case(name):
    return bubble_d3q15_z12() if name == "bubble_d3q15_z12" else small_cases()[name]


@pytest.mark.parametrize("name,ranks", FUSED_SLAB_CASES)
def test_fused_slabs_match_oracle(gpu_lib, name, ranks):
    """Slabs on the fused path, the halo exchanged as fused state
    (mplb_gpu_copy_state), against the single-domain oracle run: the owned
    planes bit for bit after 12 steps, and after 12 more with the reference
    state rebuilt in between."""
    from tests.helpers import run_checker
    case = fused_case(name)
    fields = [f for f in fields_of(case) if f != "S" or case.g is not None]
    with slabs.FusedSlabRun(case, ranks) as run:
        assert all(s["lat"].info()["path"] == abi.PATH_FUSED for s in run.slabs)
        run.initialize()
        run.step(12)
        assert_same(run.gather(), run_checker("port", case, 12), fields=fields, ctx=f"{name} in {ranks} fused slabs @12")
        run.step(12)
        assert_same(run.gather(), run_checker("port", case, 24), fields=fields, ctx=f"{name} in {ranks} fused slabs @24")


@pytest.mark.parametrize("name,ranks", FUSED_SLAB_CASES)
def test_fused_slabs_mirror_match_oracle(gpu_lib, name, ranks):
    """Slabs whose step kernels write the neighbours' halos themselves
    (mplb_gpu_set_owned, mplb_gpu_add_mirror: no copies between the steps,
    one exchange before the first step and after each gather) against the
    single-domain oracle run: the owned planes bit for bit after 12 steps, and
    after 12 more with the reference state rebuilt in between."""
    from tests.helpers import run_checker
    case = fused_case(name)
    fields = [f for f in fields_of(case) if f != "S" or case.g is not None]
    with slabs.FusedSlabRun(case, ranks, mirror=True) as run:
        run.initialize()
        run.step(12)
        assert_same(run.gather(), run_checker("port", case, 12), fields=fields,
                    ctx=f"{name} in {ranks} mirrored slabs @12")
        run.step(12)
        assert_same(run.gather(), run_checker("port", case, 24), fields=fields,
                    ctx=f"{name} in {ranks} mirrored slabs @24")


def test_mirrors_refuse(gpu_lib):
    """Mirrored ranges: owned sources, targets outside the neighbour's owned
    nodes, at most two, one step per call, neighbours in turn."""
    case = small_cases()["column_d2q9"]
    with slabs.FusedSlabRun(case, 2, mirror=True) as run:
        a, b = run.slabs[0]["lat"], run.slabs[1]["lat"]
        sa, sb = run.slabs[0], run.slabs[1]
        with pytest.raises(MplbError, match="into itself"):
            a.add_mirror(sa["own0"], 1, a, 0)
        with pytest.raises(MplbError, match="outside this handle's owned range"):
            a.add_mirror(sa["own0"] + sa["nown"], 1, b, 0)
        with pytest.raises(MplbError, match="overlaps the neighbour's owned range"):
            a.add_mirror(sa["own0"], 1, b, sb["own0"])
        run.initialize()
        run.step(2)
        with pytest.raises(MplbError, match="one step per call"):
            a.step(2)
        a.step(1)
        with pytest.raises(MplbError, match="one step ahead"):
            a.step(1)
        a.add_mirror(sa["own0"], 1, b, 0)  # the second range of slab 0 (slab 0 of a walled column has one)
        with pytest.raises(MplbError, match="at most two"):
            a.add_mirror(sa["own0"], 1, b, 0)
        b.set_owned(0, sb["own0"] + sb["nown"])  # now the targets lie in b's owned nodes
        with pytest.raises(MplbError, match="overlaps the neighbour's owned range"):
            b.step(1)
            a.step(1)
    with Lattice(case, path=abi.PATH_OPERATORS) as op:
        with pytest.raises(MplbError, match="fused FP64 path"):
            op.set_owned(0, 1)


def test_copy_state_refuses(gpu_lib):
    """State copies need two fused FP64 handles of the same lattice and options."""
    a_case = small_cases()["column_d2q9"]
    with Lattice(a_case, path=abi.PATH_FUSED) as a, Lattice(a_case, path=abi.PATH_OPERATORS) as b, \
            Lattice(small_cases()["bubble_d2q9"], path=abi.PATH_FUSED) as c:
        for lat in (a, b, c):
            lat.upload_case()
            lat.initialize()
        with pytest.raises(MplbError, match="fused FP64 path"):
            a.copy_state(b, 0, 0, 10)
        with pytest.raises(MplbError, match="differ"):
            a.copy_state(c, 0, 0, 10)
        with pytest.raises(MplbError, match="out of bounds"):
            a.copy_state(a, 0, a_case.n - 5, 10)
        with pytest.raises(MplbError, match="overlapping"):
            a.copy_state(a, 0, 5, 10)
