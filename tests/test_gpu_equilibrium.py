"""Equilibrium monitor and run-to-equilibrium (mplb_gpu_monitor,
mplb_gpu_run_to_equilibrium), and mass conservation of the FP32-deviation
collision."""
import numpy as np
import pytest

from multiphaselb_b200 import Lattice, MplbError, abi, cases

pytestmark = pytest.mark.gpu


def bubble(L=48, R=10.0, t=0.8):
    return cases.bubble_case(abi.D2Q9, L=L, radius=R, width=4.0, t_ratio=t)


def fresh(case, precision=abi.FP64):
    lat = Lattice(case, path=abi.PATH_FUSED, precision=precision)
    lat.upload_case()
    lat.initialize()
    return lat


def test_monitor_mass_matches_density_sum(gpu_lib):
    """After a fused step the current populations are post-collision; the
    collision conserves mass, so their node sums are the step's densities."""
    c = bubble()
    with fresh(c) as lat:
        lat.step(30)
        d, m = lat.monitor(reset=True)
        assert d == 0.0
        rho = lat.download()["rho"]
        assert abs(m - rho.sum()) <= 1e-12 * rho.sum(), (m, rho.sum())


def test_monitor_does_not_change_the_state(gpu_lib):
    c = bubble()
    with fresh(c) as a, fresh(c) as b:
        a.step(20)
        a.monitor(reset=True)
        a.step(20)
        a.monitor()
        b.step(40)
        da, db = a.download(), b.download()
        for k in ("rho", "U", "f"):
            assert np.array_equal(da[k], db[k]), k


def test_fp32dev_equilibrium_run_keeps_total_momentum(gpu_lib):
    """Equilibrium runs of the FP32 form reset the total momentum at every
    check: after many checks the net flow of a static bubble stays at the
    FP64 level instead of drifting."""
    c = bubble(L=64, R=12.0, t=0.8)
    with fresh(c, abi.FP32_DEV) as lat:
        lat.run_to_equilibrium(20000, 500, 0.0)
        U = lat.download()["U"]
        rho = lat.download()["rho"]
    J = (rho[:, None] * U).sum(axis=0)
    print("net momentum", J)
    assert np.abs(J).max() < 1e-9 * c.n


@pytest.mark.parametrize("precision", [abi.FP64, abi.FP32_DEV])
def test_run_to_equilibrium(gpu_lib, precision):
    c = bubble(L=40, R=8.0, t=0.85)
    K, tol = 200, 1e-7
    with fresh(c, precision) as lat:
        steps, rate = lat.run_to_equilibrium(20000, K, tol)
        assert steps % K == 0 and 0 < steps < 20000, (steps, rate)
        assert 0 <= rate < tol
        assert lat.info()["current_time"] == steps
        got = lat.download()
    if precision == abi.FP64:
        # the FP64 form's equilibrium run is plain stepping plus read-only checks
        with fresh(c, precision) as ref:
            ref.step(steps)
            want = ref.download()
        for k in ("rho", "U", "f"):
            assert np.array_equal(got[k], want[k]), k


def test_run_to_equilibrium_stops_at_max_steps(gpu_lib):
    with fresh(bubble()) as lat:
        steps, rate = lat.run_to_equilibrium(1000, 300, 1e-30)
        assert steps == 1200 and rate > 0


def test_monitor_rejects_frozen_flow(gpu_lib):
    c = cases.column_case(16, 32)
    c.f = dict(c.f, update=0)
    with Lattice(c, path=abi.PATH_FUSED) as lat:
        lat.upload_case()
        lat.initialize()
        with pytest.raises(MplbError) as e:
            lat.monitor()
        assert e.value.code == abi.E_UNSUPPORTED


def test_fp32dev_conserves_mass(gpu_lib):
    """The FP32 collision used to gain about 2.7e-10 per node and step at a
    steady bubble (its rounded mass moment is not the exact input sum); with
    exact mass bookkeeping the lattice mass only wanders by roundings of
    either sign."""
    c = bubble(L=64, R=12.0, t=0.8)
    with fresh(c, abi.FP32_DEV) as lat:
        lat.step(2000)
        _, m0 = lat.monitor(reset=True)
        lat.step(8000)
        _, m1 = lat.monitor()
    drift_per_node_step = abs(m1 - m0) / (c.n * 8000)
    print("mass", m0, m1, drift_per_node_step)
    assert drift_per_node_step < 1e-12


@pytest.mark.parametrize("precision", [abi.FP64, abi.FP32_DEV])
def test_run_to_equilibrium_reports_divergence(gpu_lib, precision):
    """A non-finite density (here: planted in the initial state on the host)
    stops the run with MPLB_E_NONFINITE instead of passing for converged
    (NaN drops out of a max)."""
    c = bubble(L=32, R=7.0)
    c.rho = c.rho.copy()
    c.rho[100] = np.nan
    with Lattice(c, path=abi.PATH_FUSED, precision=precision) as lat:
        lat.upload_case()
        lat.initialize()
        with pytest.raises(MplbError) as e:
            lat.run_to_equilibrium(1000, 10, 1e-9)
        assert e.value.code == abi.E_NONFINITE
