"""GPU library (through the C-ABI) against the CPU oracle.

Bar: bit-identical binary64 results.  The device code keeps the reference's
operation order and is compiled without multiply-add contraction; IEEE
division and square root are correctly rounded on both sides.
"""
import os

import numpy as np
import pytest

from multiphaselb_b200 import abi
from oracle import oracle as orc
from tests.helpers import FIELDS, assert_same, run_checker, run_gpu, small_cases

pytestmark = pytest.mark.gpu

CASES = list(small_cases().keys())


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("steps", [0, 1, 10])
def test_operator_path_matches_oracle(gpu_lib, name, steps):
    case = small_cases()[name]
    want = run_checker("port", case, steps)
    got, info = run_gpu(case, steps, path=abi.PATH_OPERATORS)
    assert info["path"] == abi.PATH_OPERATORS
    assert_same(got, want, ctx=f"operators {name}@{steps}")


@pytest.mark.parametrize("name", CASES)
def test_each_operator_matches_oracle(gpu_lib, name):
    """Reference operators one at a time through the per-operator entry points."""
    from multiphaselb_b200 import Lattice
    case = small_cases()[name]
    k = orc.Checker("port", case)
    k.upload_case()
    k.initialize()
    k.step(2)
    state = k.download()
    # the checker has made 2 boundary updates: a fresh handle's fixedRandomT
    # patches have 2 fewer perturbed updates left (psteps - localTStep)
    gcase = case
    if case.g is not None and abi.BC_FIXEDRANDOMT in list(case.g["bc_type"]):
        gcase = type(case)(**{**case.__dict__})
        bcv = np.array(case.g["bc_value"], dtype=float).copy()
        for p, t in enumerate(case.g["bc_type"]):
            if t == abi.BC_FIXEDRANDOMT:
                bcv[p, 2] -= 2
        gcase.g = dict(case.g, bc_value=bcv)
    with Lattice(gcase, path=abi.PATH_OPERATORS) as lat:
        lat.upload(rho=state["rho"], U=state["U"], T=state["T"], f=state["f"],
                   g=state["g"] if case.g is not None else None, S=state["S"], Fi=state["Fi"], Ft=state["Ft"])
        lat.set_time(k.get_time())
        seq = [("collision", orc.OP_COLLISION, abi.FIELD_F), ("lbstream", orc.OP_LBSTREAM, abi.FIELD_F),
               ("update_boundaries", orc.OP_BOUNDARIES, abi.FIELD_F)]
        if case.g is not None:
            seq += [("collision", orc.OP_COLLISION, abi.FIELD_G), ("lbstream", orc.OP_LBSTREAM, abi.FIELD_G),
                    ("update_boundaries", orc.OP_BOUNDARIES, abi.FIELD_G)]
        seq += [("macro_density", orc.OP_DENSITY, None)]
        if case.g is not None:
            seq += [("heat_source", orc.OP_HEATSOURCE, None), ("macro_temperature", orc.OP_TEMPERATURE, None)]
        seq += [("inter_force", orc.OP_INTERFORCE, None), ("macro_velocity", orc.OP_VELOCITY, None),
                ("equilibrium", orc.OP_EQUILIBRIUM, abi.FIELD_F)]
        for meth, op, fld in seq:
            k.op(op, abi.FIELD_F if fld is None else fld)
            getattr(lat, meth)(*([] if fld is None else [fld]))
            fields = [f for f in FIELDS if not (f == "g" and case.g is None)]
            assert_same(lat.download(), k.download(), fields=fields, ctx=f"{name} {meth}")


def test_macro_ranges_match_oracle(gpu_lib):
    """macroDensity / macroVelocity / macroTemperature over partial node ranges."""
    from multiphaselb_b200 import Lattice
    case = small_cases()["column_d2q9"]
    k = orc.Checker("port", case)
    k.upload_case()
    k.initialize()
    k.step(1)
    k.op(orc.OP_COLLISION, abi.FIELD_F)
    k.op(orc.OP_LBSTREAM, abi.FIELD_F)
    s = k.download()
    with Lattice(case, path=abi.PATH_OPERATORS) as lat:
        lat.upload(rho=s["rho"], U=s["U"], T=s["T"], f=s["f"], g=s["g"], S=s["S"], Fi=s["Fi"], Ft=s["Ft"])
        for a, b in ((0, 17), (17, 100), (100, case.n)):
            k.op(orc.OP_DENSITY, abi.FIELD_F, a, b)
            lat.macro_density(a, b)
            k.op(orc.OP_VELOCITY, abi.FIELD_F, a, b)
            lat.macro_velocity(a, b)
            k.op(orc.OP_TEMPERATURE, abi.FIELD_G, a, b)
            lat.macro_temperature(a, b)
            assert_same(lat.download(), k.download(), ctx=f"range {a}:{b}")


@pytest.mark.parametrize("name", CASES)
def test_golden_vectors_on_gpu(gpu_lib, name):
    """GPU against the reference's own outputs committed as golden vectors."""
    from tests.golden.make_golden import load_case
    gdir = os.path.join(os.path.dirname(__file__), "golden")
    fname = [f for f in os.listdir(gdir) if f.startswith(name + "_") and f.endswith(".npz")][0]
    case, steps, want = load_case(os.path.join(gdir, fname))
    got, _ = run_gpu(case, steps, path=abi.PATH_OPERATORS)
    assert_same(got, want, fields=list(want.keys()), ctx=fname)


def test_restart_time_and_flags(gpu_lib):
    """Start time > 0 (heat-source history kept) and the frozen / no-heat switches."""
    case = small_cases()["column_d2q9"]
    assert_same(run_gpu(case, 4, path=abi.PATH_OPERATORS, start_time=7)[0],
                run_checker("port", case, 4, start_time=7), ctx="start_time 7")
    for fu, gu in ((0, 1), (1, 0)):
        c2 = type(case)(**{**case.__dict__})
        c2.f = dict(case.f, update=fu)
        c2.g = dict(case.g, update=gu)
        assert_same(run_gpu(c2, 5, path=abi.PATH_OPERATORS)[0], run_checker("port", c2, 5),
                    ctx=f"update f={fu} g={gu}")


def test_average_rho0_and_reductions(gpu_lib):
    from multiphaselb_b200 import Lattice
    case = small_cases()["column_d2q9"]
    k = orc.Checker("port", case)
    k.upload_case()
    k.initialize()
    k.step(3)
    with Lattice(case, path=abi.PATH_OPERATORS) as lat:
        lat.upload_case()
        lat.initialize()
        lat.step(3)
        assert lat.average_rho0() == k.average_rho0() == 0.0
        lat.set_rho0(1.0)
        k.set_rho0(1.0)
        assert lat.average_rho0() == k.average_rho0()
        d = lat.download()
        m, e = lat.mass_energy()
        assert abs(m - d["rho"].sum()) <= 1e-12 * abs(d["rho"].sum())
        assert abs(e - d["T"].sum()) <= 1e-12 * abs(d["T"].sum())


def test_serial_boundary_order(gpu_lib):
    """A mesh where a fixedU node reads populations a bounce-back node wrote:
    the library must fall back to the reference's serial boundary order."""
    from multiphaselb_b200 import cases
    case = small_cases()["lid_d2q9"]
    c2 = type(case)(**{**case.__dict__})
    # add the top row's second-to-last row as a bounce-back patch before the lid
    top = np.nonzero(case.points[:, 1] == case.dims[1] - 2)[0].astype(np.uint32)
    c2.patches = [case.patches[0], top, case.patches[1]]
    c2.patch_names = ["Y0", "inner", "Y1"]
    c2.f = dict(case.f, bc_type=[abi.BC_BOUNCEBACK, abi.BC_BOUNCEBACK, abi.BC_FIXEDU],
                bc_value=np.array([[0, 0, 0], [0, 0, 0], [0.02, 0, 0]], dtype=float))
    c2.g = dict(case.g, bc_type=[abi.BC_FIXEDT, abi.BC_PERIODIC, abi.BC_FIXEDT],
                bc_value=np.array([case.g["bc_value"][0], [0, 0, 0], case.g["bc_value"][1]], dtype=float))
    got, info = run_gpu(c2, 6, path=abi.PATH_OPERATORS)
    assert info["bc_sequential"] & 1
    assert_same(got, run_checker("port", c2, 6), ctx="serial bc")


FUSABLE = ["bubble_d2q9", "column_d2q9", "bubble_d3q15", "walls_d3q15", "st_d2q9", "st_d3q15", "my_column_d2q9"]


@pytest.mark.parametrize("name", FUSABLE)
@pytest.mark.parametrize("steps", [1, 2, 11])
def test_fused_path_matches_oracle(gpu_lib, name, steps):
    case = small_cases()[name]
    want = run_checker("port", case, steps)
    got, info = run_gpu(case, steps, path=abi.PATH_FUSED)
    assert info["path"] == abi.PATH_FUSED
    assert_same(got, want, ctx=f"fused {name}@{steps}")


@pytest.mark.parametrize("name", FUSABLE)
def test_fused_interleaved_with_downloads(gpu_lib, name):
    """Materialise the reference state mid-run, then keep stepping."""
    from multiphaselb_b200 import Lattice
    case = small_cases()[name]
    k = orc.Checker("port", case)
    k.upload_case()
    k.initialize()
    with Lattice(case, path=abi.PATH_FUSED) as lat:
        lat.upload_case()
        lat.initialize()
        for chunk in (3, 1, 4):
            k.step(chunk)
            lat.step(chunk)
            assert_same(lat.download(), k.download(), ctx=f"{name} after chunk {chunk}")
        # an operator call on the materialised state, then fused steps again
        k.op(orc.OP_INTERFORCE)
        lat.inter_force()
        k.step(2)
        lat.step(2)
        assert_same(lat.download(), k.download(), ctx=f"{name} after operator + 2 steps")


def test_fused_auto_selects_box_path(gpu_lib):
    _, info = run_gpu(small_cases()["column_d2q9"], 1)
    assert info["path"] == abi.PATH_FUSED
    _, info = run_gpu(small_cases()["lid_d2q9"], 1)
    assert info["path"] == abi.PATH_OPERATORS  # fixedU is an operator-path boundary


@pytest.mark.parametrize("fu,gu", [(0, 1), (1, 0)])
def test_fused_frozen_fields(gpu_lib, fu, gu):
    case = small_cases()["column_d2q9"]
    c2 = type(case)(**{**case.__dict__})
    c2.f = dict(case.f, update=fu)
    c2.g = dict(case.g, update=gu)
    got, info = run_gpu(c2, 6, path=abi.PATH_FUSED)
    assert_same(got, run_checker("port", c2, 6), ctx=f"fused update f={fu} g={gu}")


@pytest.mark.parametrize("name", ["column_d2q9", "bubble_d2q9", "bubble_d3q15", "walls_d3q15", "st_d2q9", "st_d3q15",
                                  "my_column_d2q9"])
def test_every_tile_candidate_is_exact(gpu_lib, name):
    """Each fused tile shape (forced) gives the oracle's bits; the autotuner
    then times them all and picks one."""
    from multiphaselb_b200 import Lattice, MplbError
    case = small_cases()[name]
    want = run_checker("port", case, 4)
    # 2D: 10 shapes (the last two with added ring warps); 3D: 6 shapes, then
    # 4 TMA-staged ones (fully periodic boxes whose extents the tile divides
    # only)
    ncand = 10
    ran = []
    for c in range(1, ncand + 1):
        with Lattice(case, path=abi.PATH_FUSED, tile_config=c) as lat:
            lat.upload_case()
            lat.initialize()
            try:
                lat.step(4)
            except MplbError as e:
                assert "does not take this lattice" in str(e), e
                continue
            assert lat.info()["tile_config"] == c - 1
            assert_same(lat.download(), want, ctx=f"{name} tile candidate {c - 1}")
            ran.append(c)
    assert set(range(1, 7 if case.lattice == abi.D3Q15 else 11)) <= set(ran), ran
    with Lattice(case, path=abi.PATH_FUSED) as lat:
        lat.upload_case()
        lat.initialize()
        lat.step(4)
        info = lat.info()
        assert info["tile_config"] + 1 in ran
        assert all((t > 0) == (c + 1 in ran) for c, t in enumerate(info["tile_ms"][:ncand])), info["tile_ms"]
        assert_same(lat.download(), want, ctx=f"{name} autotuned")


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("path", [abi.PATH_OPERATORS, abi.PATH_AUTO])
def test_pressure_matches_oracle(gpu_lib, name, path):
    """Write-time pressure (macroPressure) after a few steps, bit for bit."""
    from multiphaselb_b200 import Lattice
    case = small_cases()[name]
    k = orc.Checker("port", case)
    k.upload_case()
    k.initialize()
    k.step(5)
    want = k.pressure()
    with Lattice(case, path=path) as lat:
        lat.upload_case()
        lat.initialize()
        lat.step(5)
        got = lat.macro_pressure()
    assert np.array_equal(got, want), float(np.abs(got - want).max())


def test_surface_tension_rejected_in_fp32(gpu_lib):
    """The FP32-deviation collision has no surface-tension term: create says so."""
    from multiphaselb_b200 import Lattice, MplbError
    with pytest.raises(MplbError) as e:
        Lattice(small_cases()["st_d2q9"], path=abi.PATH_FUSED, precision=abi.FP32_DEV)
    assert e.value.code == abi.E_UNSUPPORTED


OPERATOR_ONLY = ["outflow_d2q9", "outflow_corner_d2q9", "outflow_d3q15", "my_slab_d3q15"]


@pytest.mark.parametrize("name", OPERATOR_ONLY)
def test_operator_only_options_select_the_operator_path(gpu_lib, name):
    """Outflow, fixedRandomT and a D3Q15 thermal field run on the operator
    path: AUTO picks it on a box, FUSED and the FP32 form say they cannot."""
    from multiphaselb_b200 import Lattice, MplbError
    case = small_cases()[name]
    _, info = run_gpu(case, 1)
    assert info["path"] == abi.PATH_OPERATORS
    for kw in (dict(path=abi.PATH_FUSED), dict(path=abi.PATH_AUTO, precision=abi.FP32_DEV)):
        with pytest.raises(MplbError) as e:
            Lattice(case, **kw)
        assert e.value.code == abi.E_UNSUPPORTED


def test_outflow_corner_runs_in_serial_order(gpu_lib):
    """A corner node's outflow normal truncates to the rest direction, so it
    reads its own populations, which other patches write: the reference's
    serial boundary order is kept, and the result is the oracle's."""
    case = small_cases()["outflow_corner_d2q9"]
    got, info = run_gpu(case, 5, path=abi.PATH_OPERATORS)
    assert info["bc_sequential"] & 1 and info["bc_sequential"] & 2
    assert_same(got, run_checker("port", case, 5), ctx="outflow corner")


def test_fixedrandomt_follows_the_rank_seed(gpu_lib):
    """srand(pid) at every call: another rank draws other wall temperatures,
    and after the perturbed updates both ranks apply the plain wall value."""
    case = small_cases()["outflow_d2q9"]
    outs = {}
    for rank in (0, 3, 4):
        c2 = type(case)(**{**case.__dict__})
        c2.meta = dict(case.meta, rank=rank)
        got, _ = run_gpu(c2, 2, path=abi.PATH_OPERATORS)
        assert_same(got, run_checker("port", c2, 2), ctx=f"rank {rank}")
        outs[rank] = got["g"]
    assert not np.array_equal(outs[3], outs[4]) and not np.array_equal(outs[0], outs[3])


def test_outflow_without_normal_is_refused(gpu_lib):
    """Outflow on nodes with every neighbour present has no normal (the
    reference stops: outflow.c:67-71); create refuses it."""
    from multiphaselb_b200 import Lattice, MplbError
    case = small_cases()["outflow_d2q9"]
    c2 = type(case)(**{**case.__dict__})
    mid = np.nonzero(case.points[:, 1] == case.dims[1] // 2)[0].astype(np.uint32)
    c2.patches = [case.patches[0], mid]
    c2.f = dict(case.f, bc_type=[abi.BC_BOUNCEBACK, abi.BC_OUTFLOW])
    with pytest.raises(MplbError) as e:
        Lattice(c2, path=abi.PATH_OPERATORS)
    assert e.value.code == abi.E_ARG


@pytest.mark.parametrize("name", ["my_column_d2q9"])
def test_mymrt_takes_the_fused_path(gpu_lib, name):
    """A D2Q9 myMRT thermal field runs fused (a pull-and-sum pre-kernel, then
    the fused step); the FP32 form has no myMRT collision and refuses."""
    from multiphaselb_b200 import Lattice, MplbError
    case = small_cases()[name]
    _, info = run_gpu(case, 1)
    assert info["path"] == abi.PATH_FUSED
    with pytest.raises(MplbError) as e:
        Lattice(case, path=abi.PATH_AUTO, precision=abi.FP32_DEV)
    assert e.value.code == abi.E_UNSUPPORTED
