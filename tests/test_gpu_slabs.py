"""Slab decomposition on the device: every slab a device lattice on the
operator path (multiphaselb_b200.slabs.LatticeHandle), the ghost planes
exchanged at the reference's points, against the same split run on CPU
checkers.  Bitwise."""
import pytest

from multiphaselb_b200 import slabs
from tests.helpers import assert_same, small_cases
from tests.test_slabs import CheckerHandle, fields_of

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,ranks", [("column_d2q9", 3), ("bubble_d2q9", 2), ("outflow_corner_d2q9", 3),
                                        ("st_d2q9", 2), ("my_slab_d3q15", 2)])
def test_device_slabs_match_checker_slabs(gpu_lib, name, ranks):
    case = small_cases()[name]
    rank0 = case.meta.get("rank", 0)
    runs = []
    for make in (CheckerHandle, slabs.LatticeHandle):
        run = slabs.SlabRun(case, ranks, make, rank0=rank0)
        run.initialize()
        run.step(5)
        runs.append(run.gather())
        for h in run.handles:
            if hasattr(h, "close"):
                h.close()
    assert_same(runs[1], runs[0], fields=fields_of(case), ctx=f"{name} in {ranks} slabs, device vs checker")
