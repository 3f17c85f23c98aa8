"""Host-side case builders: EOS coexistence (Maxwell) and critical point."""
import numpy as np
import pytest

from multiphaselb_b200 import abi, cases

CS = dict(type=abi.EOS_CS, a=1.0, b=4.0, R=1.0, G=-1.0, M=1.0, Cv=1.0)
VDW = dict(type=abi.EOS_VDW, a=9.0 / 392.0, b=2.0 / 21.0, R=1.0, G=-1.0, M=1.0, Cv=1.0)


def equal_area(eos, T, rv, rl):
    v = np.linspace(1.0 / rl, 1.0 / rv, 2000001)
    P = cases.p_eos(eos, rv, T)
    f = cases.p_eos(eos, 1.0 / v, T) - P
    return float(np.sum(0.5 * (f[1:] + f[:-1]) * np.diff(v))), P


@pytest.mark.parametrize("eos", [CS, VDW], ids=["cs", "vdw"])
def test_coexistence_curve(eos):
    tc = cases.critical_temperature(eos)
    prev = None
    for t in (0.6, 0.65, 0.7, 0.75, 0.8, 0.85, 0.9, 0.95):
        T = t * tc
        rv, rl = cases.maxwell_densities(eos, T)
        assert 0 < rv < rl
        # equal pressures and equal areas
        assert abs(cases.p_eos(eos, rv, T) - cases.p_eos(eos, rl, T)) < 1e-12
        area, P = equal_area(eos, T, rv, rl)
        assert abs(area) < 1e-6 * P * (1.0 / rv - 1.0 / rl), (t, area)
        # both branches move toward each other as T rises
        if prev is not None:
            assert rv > prev[0] and rl < prev[1], (t, rv, rl, prev)
        prev = (rv, rl)


def test_vapour_far_below_spinodal_at_low_temperature():
    """At 0.6 Tc the CS vapour density is ~3e-3, an order of magnitude below
    the vapour spinodal (a root bracket that started above the true root
    once returned the spinodal instead)."""
    T = 0.6 * cases.critical_temperature(CS)
    rv, rl = cases.maxwell_densities(CS, T)
    assert 2e-3 < rv < 5e-3 and 0.39 < rl < 0.42
