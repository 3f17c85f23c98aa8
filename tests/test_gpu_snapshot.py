"""Write-step snapshots (mplb_gpu_snapshot / _wait / _write / _join): the
copy taken at step s equals a synchronous download at step s, the handle
keeps stepping while it travels and while its files are written, taking it
does not change the run, and the files hold the reference writers' bytes
(checked with the restatement in oracle/oracle.py, itself pinned to the
reference's writers by tests/test_writers.py)."""
import os

import numpy as np
import pytest

from multiphaselb_b200 import Lattice, MplbError, abi
from oracle import oracle
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


def tree(root, time, pid=0):
    d = os.path.join(root, f"processor{pid}", str(time))
    return {f: open(os.path.join(d, f), "rb").read() for f in sorted(os.listdir(d))}


@pytest.mark.parametrize("name,precision,fmt", [("column_d2q9", abi.FP64, abi.FMT_ASCII_RAW),
                                                ("bubble_d3q15", abi.FP64, abi.FMT_BINARY_RAW),
                                                ("bubble_d2q9", abi.FP32_DEV, abi.FMT_ASCII_RAW),
                                                ("bubble_d2q9", abi.FP64, abi.FMT_PVTU)])
def test_snapshot_files_are_the_reference_write_block(gpu_lib, tmp_path, name, precision, fmt):
    """The writer thread's files for a snapshot at step s hold the bytes the
    reference's writers would give for the state at step s (rho, T, p, U, f,
    g, as multiPhasePP.c:289-301 writes them), although the handle stepped on
    while they were written."""
    case = small_cases()[name]
    root = str(tmp_path / "run")
    if fmt == abi.FMT_PVTU:
        os.makedirs(os.path.join(root, "processor0", "9"))
        open(os.path.join(root, "processor0", "9", "fields.vtu"), "w").close()
    with fresh(case, precision) as a, fresh(case, precision) as b:
        a.step(9)
        a.snapshot(pressure=True, pdfs=True)
        a.snapshot_write(root, 0, fmt)
        a.step(4)
        a.snapshot_join()
        b.step(9)
        want = b.download()
        want["p"] = b.macro_pressure()
    got = tree(root, 9)
    order = [("rho", True), ("T", True), ("p", True), ("U", False), ("f", False), ("g", False)]
    if fmt == abi.FMT_PVTU:
        body = b"".join(oracle.field_file_bytes(fmt, k, want[k], s) for k, s in order)
        assert got == {"fields.vtu": body}
    else:
        assert sorted(got) == sorted(k for k, _ in order)
        for k, s in order:
            assert got[k] == oracle.field_file_bytes(fmt, k, want[k], s), k


def test_snapshot_writer_reports_nan(gpu_lib, tmp_path):
    case = small_cases()["bubble_d2q9"]
    case.rho = case.rho.copy()
    case.rho[3] = np.nan
    lat = Lattice(case, path=abi.PATH_FUSED)
    lat.upload_case()
    with lat:
        lat.snapshot()
        lat.snapshot_write(str(tmp_path), 0, "asciiRaw")
        with pytest.raises(MplbError) as e:
            lat.snapshot_join()
        assert e.value.code == abi.E_NONFINITE
        lat.snapshot_join()           # the error is reported once
    assert not (tmp_path / "processor0" / "0" / "rho").exists()


def test_snapshot_without_pdfs_writes_four_fields(gpu_lib, tmp_path):
    with fresh(small_cases()["bubble_d2q9"]) as a:
        a.step(2)
        a.snapshot()
        a.snapshot_write(str(tmp_path), 1, "binaryRaw")
        a.snapshot(pressure=True)      # waits for the writer before reusing the host copy
        a.snapshot_join()
    assert sorted(tree(str(tmp_path), 2, pid=1)) == ["T", "U", "rho"]
