"""include/mplb_gpu_reference.h on the reference's own structures.

CPU: the descriptors packed from latticeMesh / lbeField / EOSInfo equal the
structures field by field.  GPU: the drop-in loop (reference structs -> GPU
handle -> steps -> results written back into the reference structs) leaves
exactly the state the reference's own CPU loop produces."""
import ctypes as C
import os
import subprocess

import pytest

from multiphaselb_b200 import abi
from oracle import oracle as orc
from tests.helpers import FIELDS, assert_same, small_cases

HERE = os.path.dirname(os.path.abspath(__file__))
ADAPTER = os.path.join(HERE, "..", "oracle", "_ref", "libmplb_adapter_check.so")


def adapter_lib():
    if not os.path.exists(ADAPTER):
        if not os.path.isdir("/root/reference/src"):
            pytest.skip("adapter checker not built and the reference tree is absent")
        from multiphaselb_b200 import build
        build.build()
        subprocess.run(["make", "-s", "-C", os.path.join(HERE, "..", "oracle"), "adapter"], check=True)
    orc._lib("ref")  # load the harness first (same file the adapter links)
    lib = C.CDLL(ADAPTER)
    lib.adapter_pack_check.argtypes = [C.c_void_p]
    lib.adapter_pack_check.restype = C.c_int
    lib.adapter_gpu_run.argtypes = [C.c_void_p, C.c_uint32, C.c_int, C.c_uint32]
    lib.adapter_gpu_run.restype = C.c_int
    return lib


@pytest.mark.parametrize("name", list(small_cases().keys()))
def test_adapter_packs_reference_structs(name):
    lib = adapter_lib()
    k = orc.Checker("ref", small_cases()[name])
    k.upload_case()
    k.initialize()
    assert lib.adapter_pack_check(k.h) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(small_cases().keys()))
@pytest.mark.parametrize("path", [abi.PATH_AUTO, abi.PATH_OPERATORS])
def test_adapter_dropin_loop_matches_reference(gpu_lib, name, path):
    lib = adapter_lib()
    case = small_cases()[name]
    cpu, gpu = orc.Checker("ref", case), orc.Checker("ref", case)
    for k in (cpu, gpu):
        k.upload_case()
        k.initialize()
    cpu.step(6)
    assert lib.adapter_gpu_run(gpu.h, 6, path, 0) == 0
    fields = [f for f in FIELDS if not (f == "g" and case.g is None)]
    assert_same(gpu.download(), cpu.download(), fields=fields, ctx=f"adapter {name} path {path}")
