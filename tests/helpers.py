"""Shared helpers: run a case through a checker or through the GPU library
and compare the reference state fields."""
import numpy as np

from multiphaselb_b200 import abi, cases

FIELDS = ("rho", "U", "T", "Fi", "Ft", "S", "f", "g")


def small_cases():
    """Small seeded cases covering every operator and boundary on the path."""
    return {
        "bubble_d2q9": cases.perturbed(cases.bubble_case(abi.D2Q9, 24, 6.0, 3.0, 0.8, dims=(24, 20)), du=1e-3),
        "column_d2q9": cases.perturbed(cases.column_case(12, 24, amp=1e-3, width=3.0), du=1e-3),
        "lid_d2q9": cases.perturbed(cases.column_case(12, 16, amp=1e-3, width=3.0, wall_u=(0.02, 0.0, 0.0),
                                                      name="lid_d2q9_12x16"), du=1e-3),
        "bubble_d3q15": cases.perturbed(cases.bubble_case(abi.D3Q15, 10, 3.0, 2.0, 0.75, dims=(10, 8, 6)), du=1e-3),
        "walls_d3q15": walled_d3q15(),
        "st_d2q9": surface_tension_d2q9(),
        "st_d3q15": surface_tension_d3q15(),
    }


def surface_tension_d2q9():
    """D2Q9 bubble with the surface-tension term (liMRTSurfaceTension), periodic
    x and bounce-back walls in y (wall nodes take C = 0)."""
    c = cases.bubble_case(abi.D2Q9, 20, 5.0, 3.0, 0.8, dims=(20, 18))
    nb, points, patches, names = cases.box_mesh(abi.D2Q9, c.dims, (True, False))
    c.nb, c.points, c.patches, c.patch_names = nb, points, patches, names
    c.periodic = (True, False)
    c.f = dict(c.f, surface_tension=1, kappa_st=0.4, bc_type=[abi.BC_BOUNCEBACK] * len(patches),
               bc_value=np.zeros((len(patches), 3)))
    c.name = "st_d2q9_20x18"
    return cases.perturbed(c, du=1e-3)


def surface_tension_d3q15():
    """The walled D3Q15 box with the surface-tension term (xuMRTSurfaceTension)."""
    c = walled_d3q15()
    c.f = dict(c.f, surface_tension=1, kappa_st=0.4)
    c.name = "st_d3q15_8x6x7"
    return c


def walled_d3q15():
    """D3Q15 bubble in a box with bounce-back walls on x and z, periodic y."""
    c = cases.bubble_case(abi.D3Q15, 8, 2.5, 2.0, 0.75, dims=(8, 6, 7))
    nb, points, patches, names = cases.box_mesh(abi.D3Q15, c.dims, (False, True, False))
    c.nb, c.points, c.patches, c.patch_names = nb, points, patches, names
    c.periodic = (False, True, False)
    c.f = dict(c.f, bc_type=[abi.BC_BOUNCEBACK] * len(patches), bc_value=np.zeros((len(patches), 3)))
    c.eos = dict(c.eos, g=(0.0, 0.0, -1e-5), fext=(1e-6, 0.0, 0.0), rho_0=0.0)
    c.name = "walls_d3q15_8x6x7"
    return cases.perturbed(c, du=1e-3)


def run_checker(kind, case, steps, start_time=0):
    from oracle.oracle import Checker
    k = Checker(kind, case, start_time=start_time)
    k.upload_case()
    k.initialize()
    if steps:
        k.step(steps)
    out = k.download()
    k.close()
    return out


def run_gpu(case, steps, path=abi.PATH_AUTO, chunks=None, start_time=0):
    from multiphaselb_b200 import Lattice
    with Lattice(case, path=path, start_time=start_time) as lat:
        lat.upload_case()
        lat.initialize()
        if chunks:
            for c in chunks:
                lat.step(c)
        elif steps:
            lat.step(steps)
        out = lat.download()
        info = lat.info()
    return out, info


def assert_same(a, b, fields=FIELDS, rtol=0.0, ctx=""):
    """Bit-identical unless rtol > 0 (then max |a-b| <= rtol * max|b|)."""
    for k in fields:
        x, y = np.asarray(a[k]), np.asarray(b[k])
        assert x.shape == y.shape, (ctx, k, x.shape, y.shape)
        assert np.isfinite(y).all(), f"{ctx}: checker produced non-finite {k}"
        if rtol == 0.0:
            if not np.array_equal(x, y):
                d = np.abs(x - y)
                i = np.unravel_index(np.argmax(d), d.shape)
                raise AssertionError(f"{ctx}: field {k} differs: max |diff| {d.max():.3e} at {i} "
                                     f"({x[i]!r} vs {y[i]!r}); {np.count_nonzero(x != y)} entries")
        else:
            scale = max(np.abs(y).max(), 1e-300)
            err = np.abs(x - y).max() / scale
            assert err <= rtol, f"{ctx}: field {k} relative error {err:.3e} > {rtol:.1e}"
