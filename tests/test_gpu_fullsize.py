"""The named workloads at their full sizes (thermal column 128 x 512, bubble
256^2, bubble 192^3): the GPU against the CPU oracle for a few steps, the
fused path against the operator path over a longer run, and the mass and
energy a step must conserve.  All comparisons are bitwise except the
conservation sums."""
import numpy as np
import pytest

from multiphaselb_b200 import Lattice, abi, cases
from tests.helpers import assert_same, run_checker

pytestmark = pytest.mark.gpu

WORKLOADS = {name: build for name, build in cases.standard_cases().items()}


def gpu_run(case, steps, path):
    with Lattice(case, path=path) as lat:
        lat.upload_case()
        lat.initialize()
        lat.step(steps)
        return lat.download(), lat.info()


@pytest.mark.parametrize("name,steps", [("column_d2q9_128x512", 4), ("bubble_d2q9_256", 4),
                                        ("bubble_d3q15_192", 1)])
def test_fullsize_fused_matches_oracle(gpu_lib, name, steps):
    case = WORKLOADS[name]()
    got, info = gpu_run(case, steps, abi.PATH_AUTO)
    assert info["path"] == abi.PATH_FUSED
    want = run_checker("port", case, steps)
    fields = [f for f in ("rho", "U", "T", "Fi", "Ft", "S", "f", "g") if not (f == "g" and case.g is None)]
    assert_same(got, want, fields=fields, ctx=f"{name} fused vs oracle, {steps} steps")


@pytest.mark.parametrize("name,steps", [("column_d2q9_128x512", 200), ("bubble_d2q9_256", 200),
                                        ("bubble_d3q15_192", 12)])
def test_fullsize_fused_equals_operators(gpu_lib, name, steps):
    """Two independent GPU implementations of the same steps: one kernel per
    step against one kernel per reference operator."""
    case = WORKLOADS[name]()
    a, ia = gpu_run(case, steps, abi.PATH_FUSED)
    b, ib = gpu_run(case, steps, abi.PATH_OPERATORS)
    assert ia["path"] == abi.PATH_FUSED and ib["path"] == abi.PATH_OPERATORS
    fields = [f for f in ("rho", "U", "T", "Fi", "Ft", "S", "f", "g") if not (f == "g" and case.g is None)]
    assert_same(a, b, fields=fields, ctx=f"{name} fused vs operators, {steps} steps")


def test_fullsize_bubble_conserves_mass(gpu_lib):
    """A fully periodic bubble keeps its mass to rounding (1e-11 relative)
    over 500 fused steps."""
    case = WORKLOADS["bubble_d2q9_256"]()
    with Lattice(case, path=abi.PATH_FUSED) as lat:
        lat.upload_case()
        lat.initialize()
        lat.step(1)
        m0 = lat.download()["rho"].sum()
        lat.step(500)
        m1 = lat.download()["rho"].sum()
    assert abs(m1 - m0) <= 1e-11 * m0, (m0, m1)
