"""Time-averaging filter of the batched ensemble (mplb_batch_filter /
mplb_batch_average): a window replaces each filtered lattice's populations by
their mean over its last `window` steps.

* The mean is the mean: lone lattices stepped to each time of the window
  give the states, the host averages them, the batch's filtered state must match to
  the rounding of one FP32 value (and differ from the mean of a window one
  step shorter or longer by far more).
* A window of one step changes nothing (bitwise).
* On a lattice whose slow acoustic mode dominates the approach to
  equilibrium, a filtered run needs far fewer steps than plain FP64 and ends
  at its coexistence densities.
"""
import numpy as np
import pytest

from multiphaselb_b200 import Batch, Lattice, MplbError, abi, cases, ensemble, warmstart

pytestmark = pytest.mark.gpu


def bubbles():
    return [cases.bubble_case(abi.D2Q9, dims=(48, 40), radius=10.0, width=4.0, t_ratio=0.7, name="a"),
            cases.bubble_case(abi.D2Q9, dims=(64, 32), radius=9.0, width=4.0, t_ratio=0.85, name="b")]


def make(cs):
    lats = []
    for c in cs:
        lat = Lattice(c, path=abi.PATH_FUSED, precision=abi.FP32_DEV)
        lat.upload_case()
        lat.initialize()
        lats.append(lat)
    return lats


def lone_at(case, steps):
    """f of a lone lattice after `steps` steps, downloaded once (a download
    between steps would re-enter the FP32 form from the FP64 state)."""
    with Lattice(case, path=abi.PATH_FUSED, precision=abi.FP32_DEV) as lat:
        lat.upload_case()
        lat.initialize()
        lat.step(steps)
        return lat.download()["f"]


def test_window_state_is_the_mean_of_the_last_states():
    """Windows of 7 and 3 states: an 8-step window (the smallest even count
    above 7).  Lattice i averages the states after window steps 7-N .. 6 and
    window step 7 runs from the mean, so the f a download emits after the
    window (f streamed from the state before the last step) is the mean of
    the f a lone lattice emits at times pre+9-N .. pre+8."""
    cs = bubbles()
    windows = [7, 3]
    pre = 40
    lats = make(cs)
    try:
        with Batch(lats, check_interval=10) as b:
            b.step(pre)
            b.filter(windows)
            assert b.average() == 8
        got = [lat.download()["f"] for lat in lats]
    finally:
        for lat in lats:
            lat.close()
    for c, N, g in zip(cs, windows, got):
        emitted = {t: lone_at(c, pre + t) for t in range(1, 9)}
        want = np.mean([emitted[t] for t in range(9 - N, 9)], axis=0)
        tol = 2.0 ** -23 * np.abs(want).max()  # one FP32 rounding of the mean deviation
        err = np.abs(g - want).max()
        assert err <= tol, (c.name, err, tol)
        for other in (N - 1, N + 1):  # the neighbouring windows are far off
            alt = np.mean([emitted[t] for t in range(9 - other, 9)], axis=0)
            assert np.abs(g - alt).max() > 20 * tol, (c.name, other)


def test_window_of_one_step_changes_nothing():
    cs = bubbles()
    lats = make(cs)
    try:
        with Batch(lats, check_interval=10) as b:
            b.step(12)
            b.filter([1, 0])
            assert b.average() == 2
        got = [lat.download() for lat in lats]
    finally:
        for lat in lats:
            lat.close()
    for c, g in zip(cs, got):
        with Lattice(c, path=abi.PATH_FUSED, precision=abi.FP32_DEV) as lat:
            lat.upload_case()
            lat.initialize()
            lat.step(14)
            want = lat.download()
        for k in ("f", "rho", "U"):
            assert np.array_equal(g[k], want[k]), (c.name, k)


def test_filter_arguments():
    lats = make(bubbles()[:1])
    try:
        with Batch(lats, check_interval=10) as b:
            with pytest.raises(MplbError) as e:
                b.average()
            assert e.value.code == abi.E_STATE
            with pytest.raises(MplbError) as e:
                b.filter([abi.BATCH_MAX_WINDOW + 1])
            assert e.value.code == abi.E_ARG
            with pytest.raises(ValueError):
                b.filter([4, 4])
            b.filter([0])  # nothing filtered: a window is empty
            assert b.average() == 0
            b.filter(None)
    finally:
        for lat in lats:
            lat.close()


def run(case, filt, max_steps=200000):
    lat = make([case])[0]
    try:
        with Batch([lat], check_interval=1000, tol=1e-9) as b:
            if filt:
                b.filter(ensemble.filter_windows([case], filt[0]), filt[1], filt[2])
            steps, rate, conv = b.run(max_steps)
        rho = lat.download()["rho"]
    finally:
        lat.close()
    return int(steps[0]), float(rate[0]), conv, rho


def test_filtered_run_reaches_the_plain_equilibrium_in_fewer_steps():
    """256^2 bubble at 0.7 Tc: plain FP64 takes about 68,000 steps to
    |drho/dt| < 1e-9; the FP32-deviation batch without the filter stalls
    above the tolerance (its rounding keeps the slow acoustic mode alive);
    with windows of 1.6 sound crossing times it converges in under half the
    FP64 steps to the FP64 coexistence densities."""
    c = cases.bubble_case(abi.D2Q9, 256, 60.0, 5.0, 0.7)
    rho64, s64, r64, _ = warmstart.converge(c, K=1000, tol=1e-9, max_steps=200000)
    assert r64 < 1e-9
    s1, r1, c1, rho1 = run(c, (1.6, 2000, 10000))
    assert c1 == 1 and r1 < 1e-9, (s1, r1)
    assert s1 < 0.5 * s64, (s64, s1)
    s0, r0, c0, _ = run(c, None, max_steps=s1)
    assert c0 == 0 and r0 > 1e-9, (s0, r0)  # the same steps without the filter: not there
    v64, l64 = ensemble.coexistence(c, rho64)
    v1, l1 = ensemble.coexistence(c, rho1)
    assert abs(v1 - v64) < 1e-3 * v64 and abs(l1 - l64) < 1e-3 * l64, (v64, v1, l64, l1)
