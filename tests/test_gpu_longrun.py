"""Long runs on the GPU against the CPU oracle, bit for bit.

Every small case runs 1000 steps (the outflow channels, whose tiny lattices
blow up in the reference's own solver after 30 to 60 steps, run 25) on the
default path (fused where the mesh is a box, multiPhasePP.c:157-240 as one
kernel per step) and on the operator path (one kernel per reference
operator), each compared with the oracle run of the same steps.  The named
workloads run at their full sizes for 50 steps (3 at 192^3, where the
oracle takes about 4 s per step), and the long fixtures made by the
reference build (tests/golden/long_*.npz) are checked where the reference
tree is absent.
"""
import functools
import os

import pytest

from multiphaselb_b200 import Lattice, abi, cases
from tests.helpers import FIELDS, assert_same, run_checker, run_gpu, small_cases
from tests.test_oracle import LONG_STEPS

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@functools.lru_cache(maxsize=None)
def oracle_long(name):
    return run_checker("port", small_cases()[name], LONG_STEPS[name])


def fields_of(case):
    return [f for f in FIELDS if not (f == "g" and case.g is None)]


@pytest.mark.parametrize("path", [abi.PATH_AUTO, abi.PATH_OPERATORS])
@pytest.mark.parametrize("name", list(small_cases().keys()))
def test_long_run_matches_oracle(gpu_lib, name, path):
    case, steps = small_cases()[name], LONG_STEPS[name]
    got, info = run_gpu(case, steps, path=path)
    if path == abi.PATH_OPERATORS:
        assert info["path"] == abi.PATH_OPERATORS
    assert_same(got, oracle_long(name), fields=fields_of(case), ctx=f"{name}@{steps} path {info['path']}")


@pytest.mark.parametrize("name", list(small_cases().keys()))
def test_long_run_in_chunks_matches_oracle(gpu_lib, name):
    """The same run cut into uneven calls (download in between), so the fused
    path's lazily rebuilt state is taken and dropped many times."""
    case, steps = small_cases()[name], LONG_STEPS[name]
    chunks, left, c = [], steps, 1
    while left:
        chunks.append(min(c, left))
        left -= chunks[-1]
        c = c * 3 % 97 + 1
    with Lattice(case) as lat:
        lat.upload_case()
        lat.initialize()
        for c in chunks:
            lat.step(c)
            lat.download()
        got = lat.download()
    assert_same(got, oracle_long(name), fields=fields_of(case), ctx=f"{name}@{steps} in {len(chunks)} calls")


@pytest.mark.parametrize("name,steps", [("column_d2q9_128x512", 50), ("bubble_d2q9_256", 50),
                                        ("bubble_d3q15_192", 3)])
def test_fullsize_long_run_matches_oracle(gpu_lib, name, steps):
    case = cases.standard_cases()[name]()
    got, info = run_gpu(case, steps)
    assert info["path"] == abi.PATH_FUSED
    assert_same(got, run_checker("port", case, steps), fields=fields_of(case), ctx=f"{name}@{steps}")


@pytest.mark.parametrize("path", [abi.PATH_AUTO, abi.PATH_OPERATORS])
@pytest.mark.parametrize("fname", sorted(f for f in os.listdir(GOLDEN) if f.startswith("long_")))
def test_long_golden_vectors_on_gpu(gpu_lib, fname, path):
    """The reference build's own state after 1000 steps."""
    from tests.golden.make_golden import load_case
    case, steps, want = load_case(os.path.join(GOLDEN, fname))
    got, _ = run_gpu(case, steps, path=path)
    assert_same(got, want, fields=list(want.keys()), ctx=f"{fname} path {path}")
