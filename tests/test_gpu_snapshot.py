"""Write-step snapshots (mplb_gpu_snapshot / _wait): the copy taken at step s
equals a synchronous download at step s, the handle keeps stepping while it
travels, and taking it does not change the run."""
import numpy as np
import pytest

from multiphaselb_b200 import Lattice, MplbError, abi
from tests.helpers import small_cases

pytestmark = pytest.mark.gpu


def fresh(case, precision=abi.FP64):
    lat = Lattice(case, path=abi.PATH_FUSED, precision=precision)
    lat.upload_case()
    lat.initialize()
    return lat


@pytest.mark.parametrize("name,precision", [("column_d2q9", abi.FP64), ("bubble_d3q15", abi.FP64),
                                            ("bubble_d2q9", abi.FP32_DEV)])
def test_snapshot_equals_download_and_does_not_disturb(gpu_lib, name, precision):
    case = small_cases()[name]
    with fresh(case, precision) as a, fresh(case, precision) as b:
        a.step(7)
        a.snapshot(pressure=True)
        a.step(5)                      # stepping goes on while the copy travels
        snap = a.snapshot_wait()
        b.step(7)
        want = b.download()
        want_p = b.macro_pressure()
        for k in ("rho", "U", "T"):
            assert np.array_equal(snap[k], want[k]), k
        assert np.array_equal(snap["p"], want_p)
        b.step(5)
        got, ref = a.download(), b.download()
        for k in ("rho", "U", "T", "f"):
            assert np.array_equal(got[k], ref[k]), k


def test_second_snapshot_replaces_the_first(gpu_lib):
    case = small_cases()["bubble_d2q9"]
    with fresh(case) as a, fresh(case) as b:
        a.step(3)
        a.snapshot()
        a.step(3)
        a.snapshot()
        snap = a.snapshot_wait()
        b.step(6)
        assert np.array_equal(snap["rho"], b.download()["rho"])


def test_snapshot_wait_needs_a_snapshot(gpu_lib):
    with fresh(small_cases()["bubble_d2q9"]) as a:
        with pytest.raises(MplbError) as e:
            a.snapshot_wait()
        assert e.value.code == abi.E_STATE
