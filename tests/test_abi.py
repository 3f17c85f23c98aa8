"""The C-ABI library without a GPU: it loads, exports every function that
include/mplb_gpu.h declares, reports the header's ABI version, and the ctypes
mirror in multiphaselb_b200/abi.py matches the header's struct layouts (sizes
and field offsets from a C compile of the header)."""
import ctypes as C
import os
import re
import subprocess

import pytest

from multiphaselb_b200 import abi, load_library

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mplb_gpu.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", " ", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\*?\s+\*?(mplb_\w+)\s*\(", src, flags=re.M)))


def test_library_exports_every_declared_function():
    names = declared_functions()
    assert len(names) > 40, names
    lib = load_library()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", lib._name], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    assert not [n for n in names if n not in exported]


def test_version_reports_the_header_abi():
    m = re.search(r"#define MPLB_ABI_VERSION (\d+)", open(HEADER).read())
    v = load_library().mplb_gpu_version().decode()
    assert f"ABI {m.group(1)} " in v, v


def test_constants_mirror_the_header():
    h = open(HEADER).read()
    assert int(re.search(r"#define MPLB_BATCH_MAX_WINDOW (\d+)u", h).group(1)) == abi.BATCH_MAX_WINDOW


STRUCTS = {
    "mplb_mesh_desc": abi.MeshDesc,
    "mplb_eos_desc": abi.EosDesc,
    "mplb_field_desc": abi.FieldDesc,
    "mplb_opts": abi.Opts,
    "mplb_info": abi.Info,
    "mplb_batch_opts": abi.BatchOpts,
    "mplb_batch_info": abi.BatchInfo,
    "mplb_ghost_run": abi.GhostRun,
}


@pytest.fixture(scope="module")
def c_layouts(tmp_path_factory):
    """sizeof and offsetof of every mirrored struct, from gcc on the header."""
    d = tmp_path_factory.mktemp("abi")
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    for cname, py in STRUCTS.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'  printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    (d / "layout.c").write_text("\n".join(lines) + "\n")
    exe = d / "layout"
    subprocess.run(["gcc", "-std=c11", "-o", str(exe), str(d / "layout.c")], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    res = {}
    for line in out.splitlines():
        key, val = line.rsplit(" ", 1)
        res[key] = int(val)
    return res


@pytest.mark.parametrize("cname", sorted(STRUCTS))
def test_ctypes_mirror_matches_header(c_layouts, cname):
    py = STRUCTS[cname]
    assert C.sizeof(py) == c_layouts[f"{cname} size"], cname
    for fname, _ in py._fields_:
        assert getattr(py, fname).offset == c_layouts[f"{cname}.{fname}"], (cname, fname)
