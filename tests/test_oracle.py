"""The CPU restatement (oracle/mplb_oracle.c) against the reference's own
sources compiled in place (oracle/_ref) and against committed golden vectors
made by that reference build (tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

from multiphaselb_b200 import abi, cases
from oracle import oracle as orc
from tests.helpers import FIELDS, assert_same, run_checker, small_cases

def ref_available():
    if orc.available("ref"):
        return True
    if orc.ref_tree_present():
        orc.build("ref")
        return orc.available("ref")
    return False


@pytest.mark.parametrize("name", list(small_cases().keys()))
@pytest.mark.parametrize("steps", [0, 1, 7])
def test_port_matches_reference_bitwise(name, steps):
    if not ref_available():
        pytest.skip("reference build not present (pinned by the golden vectors instead)")
    case = small_cases()[name]
    assert_same(run_checker("port", case, steps), run_checker("ref", case, steps), ctx=f"{name}@{steps}")


# Long runs: every small case for 1000 steps (the outflow channels, whose
# tiny lattices blow up in the reference itself after 30 to 60 steps, for 25).
LONG_STEPS = {name: 25 if name.startswith("outflow") else 1000 for name in small_cases()}


@pytest.mark.parametrize("name", list(small_cases().keys()))
def test_port_matches_reference_long_run(name):
    if not ref_available():
        pytest.skip("reference build not present (pinned by the long golden vectors instead)")
    case, steps = small_cases()[name], LONG_STEPS[name]
    assert_same(run_checker("port", case, steps), run_checker("ref", case, steps), ctx=f"{name}@{steps}")


@pytest.mark.parametrize("name", list(small_cases().keys()))
def test_port_operators_match_reference(name):
    """Each reference operator, one at a time, from the same state."""
    if not ref_available():
        pytest.skip("reference build not present")
    case = small_cases()[name]
    ks = {k: orc.Checker(k, case) for k in ("port", "ref")}
    for k in ks.values():
        k.upload_case()
        k.initialize()
        k.step(2)
    seq = [(orc.OP_COLLISION, abi.FIELD_F), (orc.OP_LBSTREAM, abi.FIELD_F), (orc.OP_BOUNDARIES, abi.FIELD_F)]
    if case.g is not None:
        seq += [(orc.OP_COLLISION, abi.FIELD_G), (orc.OP_LBSTREAM, abi.FIELD_G), (orc.OP_BOUNDARIES, abi.FIELD_G)]
    seq += [(orc.OP_DENSITY, abi.FIELD_F)]
    if case.g is not None:
        seq += [(orc.OP_HEATSOURCE, abi.FIELD_G), (orc.OP_TEMPERATURE, abi.FIELD_G)]
    seq += [(orc.OP_INTERFORCE, abi.FIELD_F), (orc.OP_VELOCITY, abi.FIELD_F)]
    for op, fld in seq:
        for k in ks.values():
            k.op(op, fld)
        assert_same(ks["port"].download(), ks["ref"].download(), ctx=f"{name} op {op}/{fld}")


def test_eos_and_potential_match_reference():
    if not ref_available():
        pytest.skip("reference build not present")
    rng = np.random.Generator(np.random.PCG64(cases.SEED))
    for eos in (dict(type=abi.EOS_IDEAL, R=1.0), dict(type=abi.EOS_CS, a=1.0, b=4.0, R=1.0),
                dict(type=abi.EOS_PR, a=2.0 / 49.0, b=2.0 / 21.0, w=0.344, R=1.0),
                dict(type=abi.EOS_VDW, a=9.0 / 392.0, b=2.0 / 21.0, R=1.0, M=1.0)):
        c = cases.bubble_case(abi.D2Q9, 6, 2.0, 1.0, 0.8)
        c.eos = dict(c.eos, **eos)
        ks = {k: orc.Checker(k, c) for k in ("port", "ref")}
        for rho, T in zip(rng.uniform(0.01, 0.9, 64), rng.uniform(0.03, 0.1, 64)):
            rho = rho * (8.0 if eos["type"] == abi.EOS_VDW else 1.0)
            for fn in ("p_eos", "potential"):
                a, b = getattr(ks["port"], fn)(rho, T), getattr(ks["ref"], fn)(rho, T)
                assert a == b or (np.isnan(a) and np.isnan(b)), (eos, fn, rho, T, a, b)


def test_average_rho0_matches_reference():
    if not ref_available():
        pytest.skip("reference build not present")
    case = small_cases()["column_d2q9"]
    ks = {k: orc.Checker(k, case) for k in ("port", "ref")}
    for k in ks.values():
        k.upload_case()
        k.initialize()
        k.step(3)
    assert ks["port"].average_rho0() == ks["ref"].average_rho0() == 0.0
    for k in ks.values():
        k.set_rho0(1.0)
    a, b = ks["port"].average_rho0(), ks["ref"].average_rho0()
    assert a == b and a > 0


GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def golden_files():
    return sorted(f for f in os.listdir(GOLDEN) if f.endswith("steps.npz"))


@pytest.mark.parametrize("fname", golden_files())
def test_port_matches_golden(fname):
    from tests.golden.make_golden import load_case
    case, steps, want = load_case(os.path.join(GOLDEN, fname))
    got = run_checker("port", case, steps)
    assert_same(got, want, fields=[k for k in FIELDS if k in want], ctx=fname)


@pytest.mark.parametrize("name", list(small_cases().keys()))
def test_port_pressure_matches_reference(name):
    if not ref_available():
        pytest.skip("reference build not present")
    case = small_cases()[name]
    ks = {k: orc.Checker(k, case) for k in ("port", "ref")}
    for k in ks.values():
        k.upload_case()
        k.initialize()
        k.step(3)
    assert np.array_equal(ks["port"].pressure(), ks["ref"].pressure())
