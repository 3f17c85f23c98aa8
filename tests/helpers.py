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
        "my_column_d2q9": mymrt_column_d2q9(),
        "my_walls_d3q15": mymrt_walls_d3q15(),
        "outflow_d2q9": outflow_d2q9(),
        "outflow_corner_d2q9": outflow_corner_d2q9(),
        "outflow_d3q15": outflow_d3q15(),
        "cylinder_d2q9": cylinder_d2q9(),
        "my_slab_d3q15": mymrt_slab_d3q15(),
    }


def mymrt_slab_d3q15():
    """D3Q15 bubble in a slab: periodic x and y, bounce-back z walls for the
    flow, fixedT z walls (hot bottom, cold top) for the myMRT heat, gravity
    along -z; no node lies on two patches, so the fused path takes it."""
    c = thermal_box(abi.D3Q15, (6, 5, 7), (True, True, False))
    T0 = c.meta["T"]
    c.f = dict(c.f, bc_type=[abi.BC_BOUNCEBACK] * 2, bc_value=np.zeros((2, 3)))
    c.g = mymrt(abi.D3Q15, [abi.BC_FIXEDT, abi.BC_FIXEDT], [(1.02 * T0, 0, 0), (0.98 * T0, 0, 0)])
    c.eos = dict(c.eos, g=(0.0, 0.0, -1e-5), rho_0=0.0)
    c.name = "my_slab_d3q15_6x5x7"
    return cases.perturbed(c, du=1e-3)


def cylinder_d2q9():
    """A non-box mesh: periodic-x channel of 24 x 16 with a disc of radius 3.5
    removed (multiphaselb_b200.mesh.channel_with_cylinder), the thermal VdW
    column's fields on it; bounce-back walls and cylinder for the flow,
    fixedT walls and a hot fixedT cylinder for the heat."""
    from multiphaselb_b200 import mesh as meshmod
    m = meshmod.channel_with_cylinder(24, 16, 11.5, 6.5, 3.5)
    col = cases.column_case(24, 16, amp=1e-3, width=3.0)
    keep = np.array([x + 24 * y for x, y, _ in m.points.tolist()])
    tc = col.meta["Tc"]
    f = dict(col.f, bc_type=[abi.BC_BOUNCEBACK] * 3, bc_value=np.zeros((3, 3)))
    g = dict(col.g, bc_type=[abi.BC_FIXEDT] * 3,
             bc_value=np.array([[0.86 * tc, 0, 0], [0.84 * tc, 0, 0], [0.9 * tc, 0, 0]]))
    c = meshmod.mesh_case(m, "cylinder_d2q9_24x16", col.eos, f, g, col.rho[keep], col.U[keep], col.T[keep],
                          meta=dict(Tc=tc, box=False))
    return cases.perturbed(c, du=1e-3)


LAMBDA_MY2 = [0.0, 1.1, 1.1, 0.9, 1.0, 0.9, 1.0, 1.0, 1.0]
LAMBDA_MY3 = [0.0, 1.0, 1.0, 1.1, 1.0, 1.1, 1.0, 1.1, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0]


def mymrt(lattice, bc_type, bc_value):
    """A myMRT thermal field (myMRTCollision.c) with its own alpha constants."""
    d3 = lattice == abi.D3Q15
    return dict(model=abi.MYMRT, update=1, Lambda=LAMBDA_MY3 if d3 else LAMBDA_MY2,
                alpha_1=0.25 if d3 else 1.0, alpha_2=0.25 if d3 else -1.0,
                bc_type=bc_type, bc_value=np.asarray(bc_value, dtype=np.float64).reshape(-1, 3))


def mymrt_column_d2q9():
    """The thermal column with the myMRT thermal model instead of liTempMRT."""
    c = cases.column_case(12, 24, amp=1e-3, width=3.0, name="my_column_d2q9_12x24")
    c.g = mymrt(abi.D2Q9, [abi.BC_FIXEDT, abi.BC_FIXEDT], c.g["bc_value"])
    return cases.perturbed(c, du=1e-3)


def thermal_box(lattice, dims, periodic, T_noise=1e-3, seed=7):
    c = cases.bubble_case(lattice, 8, 2.5, 2.0, 0.75, dims=dims)
    nb, points, patches, names = cases.box_mesh(lattice, c.dims, periodic)
    c.nb, c.points, c.patches, c.patch_names = nb, points, patches, names
    c.periodic = tuple(periodic[:len(dims)])
    rng = np.random.Generator(np.random.PCG64(seed))
    c.T = c.T * (1.0 + T_noise * rng.uniform(-1.0, 1.0, size=c.n))
    return c


def mymrt_walls_d3q15():
    """D3Q15 bubble between bounce-back x walls and fixedT z walls (hot
    bottom, cold top), myMRT heat, gravity along -z."""
    c = thermal_box(abi.D3Q15, (8, 6, 7), (False, True, False))
    T0 = c.meta["T"]
    bct = {"X0": abi.BC_BOUNCEBACK, "X1": abi.BC_BOUNCEBACK, "Z0": abi.BC_FIXEDT, "Z1": abi.BC_FIXEDT}
    val = {"Z0": (1.02 * T0, 0, 0), "Z1": (0.98 * T0, 0, 0)}
    names = c.patch_names
    c.f = dict(c.f, bc_type=[abi.BC_BOUNCEBACK] * len(names), bc_value=np.zeros((len(names), 3)))
    c.g = mymrt(abi.D3Q15, [bct[n] for n in names], [val.get(n, (0, 0, 0)) for n in names])
    c.eos = dict(c.eos, g=(0.0, 0.0, -1e-5), rho_0=0.0)
    c.name = "my_walls_d3q15_8x6x7"
    return cases.perturbed(c, du=1e-3)


def outflow_d2q9():
    """Periodic-x D2Q9 channel: bounce-back bottom and outflow top for the
    flow; fixedRandomT bottom (perturbed for 3 updates) and outflow top for
    the myMRT heat; rank 3 seeds the perturbation."""
    c = thermal_box(abi.D2Q9, (12, 14), (True, False))
    T0 = c.meta["T"]
    c.f = dict(c.f, bc_type=[abi.BC_BOUNCEBACK, abi.BC_OUTFLOW], bc_value=np.zeros((2, 3)))
    c.g = mymrt(abi.D2Q9, [abi.BC_FIXEDRANDOMT, abi.BC_OUTFLOW], [(1.03 * T0, 5.0, 3.0), (0, 0, 0)])
    c.eos = dict(c.eos, g=(0.0, -1e-5, 0.0), rho_0=0.0)
    c.meta = dict(c.meta, rank=3)
    c.name = "outflow_d2q9_12x14"
    return cases.perturbed(c, du=2e-3)


def outflow_corner_d2q9():
    """Walls on all four sides: outflow on the +x and +y walls (their shared
    corner has a diagonal normal, which truncates to the rest direction), a
    fixedRandomT wall at the bottom (perturbed for 2 updates, rank 0) and a
    fixedT wall at -x."""
    c = thermal_box(abi.D2Q9, (10, 12), (False, False))
    T0 = c.meta["T"]
    bct_f = {"X0": abi.BC_BOUNCEBACK, "X1": abi.BC_OUTFLOW, "Y0": abi.BC_BOUNCEBACK, "Y1": abi.BC_OUTFLOW}
    bct_g = {"X0": abi.BC_FIXEDT, "X1": abi.BC_OUTFLOW, "Y0": abi.BC_FIXEDRANDOMT, "Y1": abi.BC_OUTFLOW}
    val_g = {"X0": (0.99 * T0, 0, 0), "Y0": (1.02 * T0, 10.0, 2.0)}
    names = c.patch_names
    c.f = dict(c.f, bc_type=[bct_f[n] for n in names], bc_value=np.zeros((len(names), 3)))
    c.g = mymrt(abi.D2Q9, [bct_g[n] for n in names], [val_g.get(n, (0, 0, 0)) for n in names])
    c.eos = dict(c.eos, g=(0.0, -1e-5, 0.0), rho_0=0.0)
    c.name = "outflow_corner_d2q9_10x12"
    return cases.perturbed(c, du=2e-3)


def outflow_d3q15():
    """D3Q15, periodic x and y: bounce-back bottom and outflow top for the
    flow, fixedRandomT bottom and outflow top for the myMRT heat, rank 1."""
    c = thermal_box(abi.D3Q15, (6, 5, 8), (True, True, False))
    T0 = c.meta["T"]
    c.f = dict(c.f, bc_type=[abi.BC_BOUNCEBACK, abi.BC_OUTFLOW], bc_value=np.zeros((2, 3)))
    c.g = mymrt(abi.D3Q15, [abi.BC_FIXEDRANDOMT, abi.BC_OUTFLOW], [(1.02 * T0, 4.0, 2.0), (0, 0, 0)])
    c.eos = dict(c.eos, g=(0.0, 0.0, -1e-5), rho_0=0.0)
    c.meta = dict(c.meta, rank=1)
    c.name = "outflow_d3q15_6x5x8"
    return cases.perturbed(c, du=2e-3)


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
