"""Field files (mplb_write_scalar_field / mplb_write_vector_field): the
library's bytes against the reference's own writers (asciiRaw, binaryRaw and
pvtu sources compiled into oracle/_ref) and against the Python restatement in
oracle/oracle.py.  Host code only: these run without a GPU."""
import os

import numpy as np
import pytest

from multiphaselb_b200 import MplbError, abi, write_field
from oracle import oracle
from tests.golden.make_writer_golden import CASES, golden_values
from tests.test_oracle import ref_available

FORMATS = [abi.FMT_ASCII_RAW, abi.FMT_BINARY_RAW, abi.FMT_PVTU]


def values(n, vs, seed):
    """Magnitudes from 1e-300 to 1e300, both signs, zeros, -0, infinities,
    subnormals and six-digit rounding ties of the decimal text."""
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(n * vs) * 10.0 ** rng.integers(-12, 6, n * vs)
    special = [0.0, -0.0, 1.0, -1.0, 0.5, 1e-300, -1e300, 5e-324, np.inf, -np.inf, 0.1234565, 1.0000005,
               999999.5, 9999995.0, 1e-5, 1e-4, 123456.5, 2.5e-5, 65504.0, 3.4028235e38, 1e39, 1e-46]
    k = min(len(special), a.size)
    a[:k] = special[:k]
    return a.reshape(n, vs)


def read_tree(root, pid, time):
    d = os.path.join(root, f"processor{pid}", str(time))
    return {f: open(os.path.join(d, f), "rb").read() for f in sorted(os.listdir(d))}


def pvtu_dir(root, pid, time):
    d = os.path.join(root, f"processor{pid}", str(time))
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "fields.vtu"), "w") as fp:
        fp.write("<!-- mesh part -->\n")


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "writers.npz")


def ref_writers():
    return ref_available() and hasattr(oracle._lib("ref"), "ref_write_field")


@pytest.mark.parametrize("fmt", FORMATS)
@pytest.mark.parametrize("n,vs", [(0, 1), (1, 1), (7, 1), (70001, 1), (5, 3), (40000, 9), (3001, 15)])
def test_bytes_match_reference_writers(tmp_path, monkeypatch, fmt, n, vs):
    if not ref_writers():
        pytest.skip("reference build not present (pinned by tests/golden/writers.npz instead)")
    scalar = vs == 1
    a = values(n, vs, seed=n * 31 + vs)
    field = a[:, 0] if scalar else a
    name = "rho" if scalar else "f"
    pid, time = 3, 1250
    ref_root, lib_root = tmp_path / "ref", tmp_path / "lib"
    ref_root.mkdir()
    lib_root.mkdir()
    if fmt == abi.FMT_PVTU:
        pvtu_dir(ref_root, pid, time)
        pvtu_dir(lib_root, pid, time)
    monkeypatch.chdir(ref_root)
    oracle.ref_write_field(fmt, name, field, scalar, pid, time)
    monkeypatch.chdir(tmp_path)
    write_field(name, field, time, root=str(lib_root), pid=pid, fmt=fmt, scalar=scalar)
    want, got = read_tree(ref_root, pid, time), read_tree(lib_root, pid, time)
    assert want.keys() == got.keys()
    for f in want:
        assert got[f] == want[f], f
    # the Python restatement (the checker used on machines without the
    # reference build) says the same
    fname = "fields.vtu" if fmt == abi.FMT_PVTU else name
    body = oracle.field_file_bytes(fmt, name, field, scalar)
    head = b"<!-- mesh part -->\n" if fmt == abi.FMT_PVTU else b""
    assert head + body == want[fname]


@pytest.mark.parametrize("key", sorted(CASES))
def test_bytes_match_golden_files(tmp_path, key):
    """Files the reference's writers made (tests/golden/make_writer_golden.py)."""
    fmt, name, n, vs = CASES[key]
    scalar = vs == 1
    want = bytes(np.load(GOLDEN)[key])
    field = golden_values(n, vs)
    field = field[:, 0] if scalar else field
    if fmt == abi.FMT_PVTU:
        pvtu_dir(tmp_path, 0, 5)
    write_field(name, field, 5, root=str(tmp_path), fmt=fmt, scalar=scalar)
    got = read_tree(tmp_path, 0, 5)["fields.vtu" if fmt == abi.FMT_PVTU else name]
    head = b"<!-- mesh part -->\n" if fmt == abi.FMT_PVTU else b""
    assert got == head + want
    assert oracle.field_file_bytes(fmt, name, field, scalar) == want


def test_thread_count_does_not_change_bytes(tmp_path, monkeypatch):
    a = values(150001, 9, seed=5)
    out = {}
    for t in ("1", "3", "16"):
        monkeypatch.setenv("MPLB_IO_THREADS", t)
        root = tmp_path / t
        write_field("g", a, 10, root=str(root))
        write_field("T", a[:, 4], 10, root=str(root))
        write_field("g", a, 11, root=str(root), fmt="binaryRaw")
        out[t] = read_tree(root, 0, 10), read_tree(root, 0, 11)
    assert out["1"] == out["3"] == out["16"]


def test_scalar_and_one_column_array_differ(tmp_path):
    """writeScalarField prints "%g\\n", writeVectorField with vsize 1 "%g \\n"."""
    x = np.array([0.25, 2.0])
    write_field("s", x, 0, root=str(tmp_path))
    write_field("v", x.reshape(2, 1), 0, root=str(tmp_path), scalar=False)
    t = read_tree(tmp_path, 0, 0)
    assert t["s"] == b"0.25\n2\n" and t["v"] == b"0.25 \n2 \n"


def test_nan_is_refused_and_nothing_written(tmp_path):
    x = np.ones((10, 3))
    x[7, 2] = np.nan
    with pytest.raises(MplbError) as e:
        write_field("U", x, 4, root=str(tmp_path))
    assert e.value.code == abi.E_NONFINITE
    assert not (tmp_path / "processor0" / "4" / "U").exists()
    # infinities pass, as in the reference (isnan only)
    write_field("U", np.full((2, 3), np.inf), 4, root=str(tmp_path))
    assert read_tree(tmp_path, 0, 4)["U"] == b"inf inf inf \ninf inf inf \n"


def test_errors(tmp_path):
    x = np.ones(4)
    for fmt, code in ((abi.FMT_ENSIGHT, abi.E_UNSUPPORTED), (9, abi.E_ARG)):
        with pytest.raises(MplbError) as e:
            write_field("rho", x, 0, root=str(tmp_path), fmt=fmt)
        assert e.value.code == code
    with pytest.raises(MplbError) as e:
        write_field("a/b", x, 0, root=str(tmp_path))
    assert e.value.code == abi.E_ARG
    blocker = tmp_path / "file"
    blocker.write_text("")
    with pytest.raises(MplbError) as e:
        write_field("rho", x, 0, root=str(blocker))
    assert e.value.code == abi.E_IO
    # pvtu appends to the mesh writer's file: no folder, no file
    with pytest.raises(MplbError) as e:
        write_field("rho", x, 0, root=str(tmp_path / "none"), fmt="pvtu")
    assert e.value.code == abi.E_IO
