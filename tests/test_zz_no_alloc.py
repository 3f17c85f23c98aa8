"""mplb_mass_energy_noalloc: the mass/energy check for callers that may not
allocate device memory (framework-owned allocators, no-allocation time loops,
code that must not synchronise).  Its sums must match the handle-based
mplb_gpu_mass_energy on the same fields, call after call, although every call
reuses the same fixed scratch array inside the library.

This file is collected last on purpose: if it fails, a run that stops at the
first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from multiphaselb_b200 import Lattice, abi
from tests.helpers import small_cases

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # same bound as the other reduction checks (different summation tree)


def _bind(lib):
    fn = lib.mplb_mass_energy_noalloc
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
    fn.restype = C.c_int
    return fn


def test_noalloc_matches_handle_sums_twice(gpu_lib):
    import torch
    fn = _bind(gpu_lib)
    case = small_cases()["column_d2q9"]
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream), Lattice(case, stream=stream.cuda_stream) as lat:
        lat.upload_case()
        lat.initialize()
        out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
        for call in range(2):
            lat.step(3 + call)  # a different state for each call
            want_m, want_e = lat.mass_energy()
            d = lat.download()
            rho = torch.tensor(d["rho"], dtype=torch.float64, device="cuda")
            T = torch.tensor(d["T"], dtype=torch.float64, device="cuda")
            rc = fn(rho.data_ptr(), T.data_ptr(), case.n, out.data_ptr(), C.c_void_p(stream.cuda_stream))
            assert rc == 0, gpu_lib.mplb_gpu_last_error().decode()
            stream.synchronize()
            m, e = out.tolist()
            assert abs(m - want_m) <= RTOL * abs(want_m), (call, m, want_m)
            assert abs(e - want_e) <= RTOL * abs(want_e), (call, e, want_e)


def test_noalloc_rejects_oversized_input(gpu_lib):
    import torch
    fn = _bind(gpu_lib)
    x = torch.zeros(4, dtype=torch.float64, device="cuda")
    rc = fn(x.data_ptr(), None, 16_777_217, x.data_ptr(), None)
    assert rc == abi.E_ARG
    assert "exceeds the fixed scratch limit" in gpu_lib.mplb_gpu_last_error().decode()
