"""Descriptor validation of mplb_gpu_create, which runs before any device
work and so needs no GPU: each malformed or unsupported descriptor returns its
error code and message, and NULL handles are refused by every entry point.
Host logic only."""
import ctypes as C

import numpy as np
import pytest

from multiphaselb_b200 import abi, cases, load_library
from tests.helpers import mymrt, small_cases


def create(case, opts=None, mutate=None):
    lib = load_library()
    d = abi.Descriptors(case)
    if mutate:
        mutate(d)
    h = C.c_void_p()
    rc = lib.mplb_gpu_create(C.byref(d.mesh), C.byref(d.eos), C.byref(d.f), C.byref(d.g),
                             C.byref(opts) if opts is not None else None, C.byref(h))
    msg = lib.mplb_gpu_last_error().decode()
    if rc == 0:
        lib.mplb_gpu_destroy(h)  # a machine with a GPU gets this far
    return rc, msg


def column():
    return cases.column_case(8, 12)


def test_null_out_and_descriptors():
    lib = load_library()
    assert lib.mplb_gpu_create(None, None, None, None, None, None) == abi.E_ARG
    h = C.c_void_p()
    assert lib.mplb_gpu_create(None, None, None, None, None, C.byref(h)) == abi.E_ARG
    assert "required" in lib.mplb_gpu_last_error().decode()


@pytest.mark.parametrize("what,mutate,needle", [
    ("lattice", lambda d: setattr(d.mesh, "lattice", 7), "unknown lattice"),
    ("empty", lambda d: setattr(d.mesh, "n_points", 0), "empty mesh"),
    ("patches", lambda d: setattr(d.mesh, "n_patches", abi.MAX_PATCHES + 1), "too many"),
    ("eos", lambda d: setattr(d.eos, "type", 9), "unknown EOS"),
])
def test_malformed_mesh_and_eos(what, mutate, needle):
    rc, msg = create(column(), mutate=mutate)
    assert rc == abi.E_ARG and needle in msg, (what, rc, msg)


def test_unknown_precision():
    rc, msg = create(column(), opts=abi.Opts(7, abi.PATH_AUTO, -1, None, 0, 0, 0))
    assert rc == abi.E_ARG and "precision" in msg


def test_neighbour_and_boundary_indices_out_of_range():
    c = column()
    c.nb = c.nb.copy()
    c.nb[5, 3] = c.n
    rc, msg = create(c)
    assert rc == abi.E_ARG and "neighbour index out of range at entry 48" in msg
    c = column()
    c.patches = [c.patches[0].copy(), c.patches[1].copy()]
    c.patches[1][0] = c.n + 3
    rc, msg = create(c)
    assert rc == abi.E_ARG and "boundary node out of range" in msg


@pytest.mark.parametrize("name,edit,code,needle", [
    ("limrt_on_d3q15", lambda c: setattr(c, "f", dict(c.f, model=abi.LIMRT)), abi.E_UNSUPPORTED, "liMRT is D2Q9 only"),
    ("xumrt_on_d2q9", lambda c: setattr(c, "f", dict(c.f, model=abi.XUMRT)), abi.E_UNSUPPORTED, "xuMRT is D3Q15 only"),
    ("mymrt_on_flow", lambda c: setattr(c, "f", dict(c.f, model=abi.MYMRT)), abi.E_UNSUPPORTED, "f model"),
    ("litemp_on_d3q15", None, abi.E_UNSUPPORTED, "liTempMRT is D2Q9 only"),
    ("frdt_on_litemp", None, abi.E_UNSUPPORTED, "fixedRandomT needs the myMRT field"),
    ("fixedt_without_values", None, abi.E_ARG, "bc_value missing"),
    ("fixedgradt", None, abi.E_UNSUPPORTED, "outside this path"),
    ("st_on_thermal", None, abi.E_UNSUPPORTED, "surface tension"),
])
def test_unsupported_field_options(name, edit, code, needle):
    if name == "limrt_on_d3q15":
        c = small_cases()["bubble_d3q15"]
        edit(c)
    elif name == "xumrt_on_d2q9":
        c = small_cases()["bubble_d2q9"]
        edit(c)
    elif name == "mymrt_on_flow":
        c = column()
        edit(c)
    elif name == "litemp_on_d3q15":
        c = small_cases()["my_slab_d3q15"]
        c.g = dict(c.g, model=abi.LITEMPMRT)
    elif name == "frdt_on_litemp":
        c = column()
        c.g = dict(c.g, bc_type=[abi.BC_FIXEDRANDOMT, abi.BC_FIXEDT])
    elif name == "fixedt_without_values":
        c = column()
        c.g = {k: v for k, v in c.g.items() if k != "bc_value"}

        def drop(d):
            d.g.bc_value = None
        rc, msg = create(c, mutate=drop)
        assert rc == code and needle in msg, (rc, msg)
        return
    elif name == "fixedgradt":
        c = column()
        c.g = dict(c.g, bc_type=[abi.BC_FIXEDGRADT, abi.BC_FIXEDT])
    else:
        c = column()
        c.g = dict(c.g, surface_tension=1)
    rc, msg = create(c)
    assert rc == code and needle in msg, (name, rc, msg)


def test_frozen_field_accepts_any_model():
    """A frozen field (update 0) is never touched by the reference, so its
    model and boundaries are not checked: creation proceeds to the device
    (which this CPU test then lacks)."""
    c = column()
    c.g = dict(c.g, update=0, model=abi.XUMRT, bc_type=[abi.BC_FIXEDGRADT, abi.BC_FIXEDGRADT])
    rc, msg = create(c)
    assert rc in (0, abi.E_CUDA), (rc, msg)
    assert "outside this path" not in msg and "g model" not in msg


def test_null_handles_are_refused():
    lib = load_library()
    calls = [
        lambda: lib.mplb_gpu_step(None, 1),
        lambda: lib.mplb_gpu_initialize(None),
        lambda: lib.mplb_gpu_download(None, *([None] * 8)),
        lambda: lib.mplb_gpu_snapshot(None, 0),
        lambda: lib.mplb_gpu_snapshot_wait(None, None, None, None, None),
        lambda: lib.mplb_gpu_snapshot_write(None, b"", 0, 0),
        lambda: lib.mplb_gpu_snapshot_join(None),
        lambda: lib.mplb_gpu_collision(None, 0),
        lambda: lib.mplb_gpu_macro_pressure(None),
        lambda: lib.mplb_gpu_copy_nodes(None, 0, None, 0, 1, 64),
        lambda: lib.mplb_ranks_initialize(None, 0, None, 0),
        lambda: lib.mplb_ranks_step(None, 2, None, 0, 1),
    ]
    for call in calls:
        assert call() == abi.E_ARG
    assert lib.mplb_gpu_destroy(None) == 0


def test_mymrt_descriptor_fields_reach_the_field():
    """alpha_1 / alpha_2 travel in the descriptor (ABI 2)."""
    c = column()
    c.g = mymrt(abi.D2Q9, [abi.BC_FIXEDT, abi.BC_FIXEDT], c.g["bc_value"])
    d = abi.Descriptors(c)
    assert d.g.model == abi.MYMRT and d.g.alpha_1 == 1.0 and d.g.alpha_2 == -1.0
    assert np.isclose(d.g.Lambda[3], 0.9)
