"""Each kernel with external linkage is defined in exactly one translation unit.

The FP64 unit is compiled without multiply-add contraction (bitwise parity),
the FP32-deviation unit with it.  If a kernel template were instantiated in
both, two modules would register the same kernel name and which copy runs
would depend on load order, so the FP64 results could pick up contracted
arithmetic."""
import collections
import shutil
import subprocess
import tempfile

import pytest


def test_no_kernel_in_two_objects():
    if not shutil.which("nm"):
        pytest.skip("nm not available")
    from multiphaselb_b200 import build
    with tempfile.TemporaryDirectory() as d:
        objs = build.compile_objects(d)
        owners = collections.defaultdict(set)
        for o in objs:
            out = subprocess.run(["nm", "-C", "--defined-only", o], capture_output=True, text=True, check=True).stdout
            for line in out.splitlines():
                parts = line.split(" ", 2)
                # global (T) and weak/COMDAT (W) kernel stubs; file-local
                # (static, 't') kernels bind to their own unit and cannot clash
                if len(parts) == 3 and parts[1] in ("T", "W") and "mplb::k_" in parts[2]:
                    owners[parts[2].split("(")[0]].add(o)
    shared = {k: v for k, v in owners.items() if len(v) > 1}
    assert not shared, shared
