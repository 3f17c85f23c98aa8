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


def test_noalloc_many_blocks_then_fewer_then_no_energy(gpu_lib):
    """Plain device arrays of a few million nodes (over a thousand partial
    blocks, summed again by the final pass) against torch.sum; then a call on
    fewer nodes, which must not pick up partials the larger call left in the
    shared scratch; then a call without T, whose energy is 0."""
    import torch
    fn = _bind(gpu_lib)
    g = torch.Generator(device="cuda").manual_seed(20261203)
    n_big, n_small = 5_000_000, 70_001
    rho = torch.rand(n_big, dtype=torch.float64, device="cuda", generator=g) + 0.5
    T = torch.rand(n_big, dtype=torch.float64, device="cuda", generator=g) * 0.1 + 0.05
    out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
    for n in (n_big, n_small):
        rc = fn(rho.data_ptr(), T.data_ptr(), n, out.data_ptr(), None)
        assert rc == 0, gpu_lib.mplb_gpu_last_error().decode()
        torch.cuda.synchronize()
        m, e = out.tolist()
        want_m, want_e = rho[:n].sum().item(), T[:n].sum().item()
        assert abs(m - want_m) <= RTOL * abs(want_m), (n, m, want_m)
        assert abs(e - want_e) <= RTOL * abs(want_e), (n, e, want_e)
    rc = fn(rho.data_ptr(), None, n_small, out.data_ptr(), None)
    assert rc == 0, gpu_lib.mplb_gpu_last_error().decode()
    torch.cuda.synchronize()
    m, e = out.tolist()
    assert abs(m - rho[:n_small].sum().item()) <= RTOL * abs(m)
    assert e == 0.0


def test_noalloc_rejects_oversized_input(gpu_lib):
    import torch
    fn = _bind(gpu_lib)
    x = torch.zeros(4, dtype=torch.float64, device="cuda")
    rc = fn(x.data_ptr(), None, 16_777_217, x.data_ptr(), None)
    assert rc == abi.E_ARG
    assert "exceeds the fixed scratch limit" in gpu_lib.mplb_gpu_last_error().decode()
