"""Deterministic lattice cases: meshes, boundary patches, EOS and initial fields.

The reference builds meshes with its own pre-processing apps (latticeBox2D /
latticeBox3D, src/applications/mesh/) and writes the initial fields with
setInitialFields.  Those apps are outside the lattice-update path, so the
cases here are built directly, with the same conventions:

* node id = x + Nx*(y + Ny*z), coordinates in ``points`` (readLatticeMesh.c:80-110);
* ``nb[id][k]`` is the node at x - c_k, the pull source of population k,
  -1 when it does not exist (latticeBox2D.c:174, lbstream.c:36-40);
* periodic axes wrap modulo the extent.  This is a true modular wrap: the
  reference's own box mesher duplicates the seam node instead
  (latticeBox2D/periodicXY.c:17-32, period Nx-1), and the solver accepts
  either table unchanged;
* wall faces are boundary patches, in the order X0 X1 Y0 Y1 Z0 Z1 of the
  non-periodic axes, each holding every node of that face (corner nodes sit
  in more than one patch, as in latticeBox2D/periodicX.c:60-66);
* the sphere / disc profile is the reference's tanh form
  (setInitialFields/sphereBoundedScalarField.c:184):
  0.5*(in+out) + 0.5*(out-in)*tanh(2*(r-R)/W).

Random draws use numpy's PCG64 with an explicit seed.
"""
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import abi

VEL = {
    abi.D2Q9: np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [-1, 0, 0], [0, -1, 0],
                        [1, 1, 0], [-1, 1, 0], [-1, -1, 0], [1, -1, 0]], dtype=np.int64),
    abi.D3Q15: np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1],
                         [1, 1, 1], [-1, 1, 1], [1, -1, 1], [-1, -1, 1], [1, 1, -1], [-1, 1, -1],
                         [1, -1, -1], [-1, -1, -1]], dtype=np.int64),
}

SEED = 20261203


@dataclass
class Case:
    name: str
    lattice: int
    dims: tuple
    periodic: tuple
    nb: np.ndarray
    points: np.ndarray
    patches: list
    patch_names: list
    eos: dict
    f: Optional[dict]
    g: Optional[dict]
    rho: np.ndarray
    U: np.ndarray
    T: np.ndarray
    meta: dict = field(default_factory=dict)

    @property
    def n(self):
        return int(self.nb.shape[0])

    @property
    def Q(self):
        return abi.Q_OF[self.lattice]


_MESH_CACHE = {}


def box_mesh(lattice, dims, periodic):
    """Neighbour table, coordinates and wall patches of an Nx x Ny (x Nz) box
    (cached per shape; each call returns fresh copies)."""
    key = (lattice, tuple(dims), tuple(bool(p) for p in periodic))
    if key not in _MESH_CACHE:
        if len(_MESH_CACHE) > 16:
            _MESH_CACHE.clear()
        _MESH_CACHE[key] = _box_mesh(lattice, dims, periodic)
    nb, points, patches, names = _MESH_CACHE[key]
    return nb.copy(), points.copy(), [p.copy() for p in patches], list(names)


def _box_mesh(lattice, dims, periodic):
    nx, ny, nz = (list(dims) + [1, 1])[:3]
    px, py, pz = (list(periodic) + [True, True])[:3]
    if lattice == abi.D2Q9:
        nz, pz = 1, True
    vel = VEL[lattice]
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    x, y, z = x.ravel(), y.ravel(), z.ravel()
    n = x.size
    nb = np.empty((n, len(vel)), dtype=np.int32)
    for k, c in enumerate(vel):
        sx, sy, sz = x - c[0], y - c[1], z - c[2]
        ok = np.ones(n, dtype=bool)
        for s, ext, per in ((sx, nx, px), (sy, ny, py), (sz, nz, pz)):
            if per:
                s %= ext
            else:
                ok &= (s >= 0) & (s < ext)
        nb[:, k] = np.where(ok, sx + nx * (sy + ny * sz), -1)
    points = np.stack([x, y, z], axis=1).astype(np.int32)
    patches, names = [], []
    for axis, (ext, per, nm) in enumerate(((nx, px, "X"), (ny, py, "Y"), (nz, pz, "Z"))):
        if per or (lattice == abi.D2Q9 and axis == 2):
            continue
        coord = (x, y, z)[axis]
        for side, val in (("0", 0), ("1", ext - 1)):
            patches.append(np.nonzero(coord == val)[0].astype(np.uint32))
            names.append(nm + side)
    return nb, points, patches, names


# ----------------------------------------------------------------- EOS helpers
def p_eos(eos, rho, T):
    """Same formulas as the reference's p_eos (src/EOS/p_eos.c:7-64)."""
    t = eos["type"]
    R = eos.get("R", 1.0)
    if t == abi.EOS_IDEAL:
        return rho * R * T
    if t == abi.EOS_CS:
        a, b = eos["a"], eos["b"]
        al = b * rho / 4.0
        be = 1 - al
        return rho * R * T * ((1 + al + al * al - al * al * al) / (be * be * be)) - a * rho * rho
    if t == abi.EOS_VDW:
        a, b, M = eos["a"], eos["b"], eos.get("M", 1.0)
        return rho * R * T / (M - rho * b) - a * rho * rho / (M * M)
    if t == abi.EOS_PR:
        a, b, w = eos["a"], eos["b"], eos["w"]
        tc = 0.170151343 * a / (b * R)
        phi = 1 + (0.37464 + 1.5422 * w - 0.26992 * w * w) * (1 - np.sqrt(T / tc))
        return rho * R * T / (1 - b * rho) - a * phi * phi * rho * rho / (1 + 2 * b * rho - b * rho * b * rho)
    raise ValueError(t)


def _eos_key(eos):
    return tuple(sorted((k, tuple(v) if isinstance(v, (list, tuple)) else v) for k, v in eos.items()))


_TC_CACHE, _MAXWELL_CACHE = {}, {}


def critical_temperature(eos):
    """Tc from dp/drho = d2p/drho2 = 0, by bisection on T (FP64)."""
    key = _eos_key(eos)
    if key not in _TC_CACHE:
        _TC_CACHE[key] = _critical_temperature(eos)
    return _TC_CACHE[key]


def _critical_temperature(eos):
    if eos["type"] == abi.EOS_VDW and eos.get("M", 1.0) == 1.0:
        return 8 * eos["a"] / (27 * eos["b"] * eos.get("R", 1.0))
    rho = np.linspace(1e-4, 0.999 * _rho_max(eos), 20001)

    def has_loop(T):
        return np.any(np.diff(p_eos(eos, rho, T)) < 0)

    lo, hi = 1e-6, 10.0
    while not has_loop(lo):
        lo *= 0.5
    for _ in range(80):
        mid = 0.5 * (lo + hi)
        if has_loop(mid):
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def _rho_max(eos):
    if eos["type"] == abi.EOS_CS:
        return 4.0 / eos["b"]
    if eos["type"] in (abi.EOS_VDW,):
        return eos.get("M", 1.0) / eos["b"]
    if eos["type"] == abi.EOS_PR:
        return 1.0 / eos["b"]
    return 10.0


def maxwell_densities(eos, T):
    """Coexistence (vapour, liquid) densities by the equal-area rule in the
    specific volume: p(v_v) = p(v_l) = P and int_{v_l}^{v_v} p dv = P (v_v - v_l)."""
    key = (_eos_key(eos), float(T))
    if key not in _MAXWELL_CACHE:
        _MAXWELL_CACHE[key] = _maxwell_densities(eos, T)
    return _MAXWELL_CACHE[key]


_GL_X, _GL_W = np.polynomial.legendre.leggauss(96)


def _maxwell_densities(eos, T):
    rmax = _rho_max(eos)
    rho = np.linspace(1e-6, 0.9999 * rmax, 100001)
    p = p_eos(eos, rho, T)
    dp = np.diff(p)
    i_max = np.argmax(dp < 0)                # first local max (vapour spinodal)
    i_min = i_max + np.argmax(dp[i_max:] > 0)  # following local min (liquid spinodal)
    plo, phi = max(p[i_min], 1e-14), p[i_max]

    def roots(P):
        # p(0) = 0 < P: the vapour root may lie below the grid's first point
        rv = _bisect(lambda r: p_eos(eos, r, T) - P, 0.0, rho[i_max], it=200)
        rl = _bisect(lambda r: p_eos(eos, r, T) - P, rho[i_min], rho[-1])
        return rv, rl

    def area(P):
        # split at the spinodals so each Gauss-Legendre piece is smooth, and
        # integrate in s = ln v (dv = v ds): at low T the vapour volume is
        # orders of magnitude above the liquid's and p ~ RT/v there
        rv, rl = roots(P)
        knots = np.log([1.0 / rl, 1.0 / rho[i_min], 1.0 / rho[i_max], 1.0 / rv])
        tot = 0.0
        for a, b in zip(knots[:-1], knots[1:]):
            v = np.exp(0.5 * (b - a) * _GL_X + 0.5 * (a + b))
            tot += 0.5 * (b - a) * np.dot(_GL_W, (p_eos(eos, 1.0 / v, T) - P) * v)
        return tot

    P = _bisect(area, plo, phi, it=80)
    return roots(P)


def _bisect(fn, lo, hi, it=80):
    flo = fn(lo)
    for _ in range(it):
        mid = 0.5 * (lo + hi)
        fm = fn(mid)
        if (fm > 0) == (flo > 0):
            lo, flo = mid, fm
        else:
            hi = mid
    return 0.5 * (lo + hi)


def tanh_profile(r, R, W, rin, rout):
    return 0.5 * (rin + rout) + 0.5 * (rout - rin) * np.tanh(2.0 * (r - R) / W)


# --------------------------------------------------------------- case builders
LAMBDA_C1 = [1.0, 1.5, 1.4, 1.0, 1.2, 1.0, 1.2, 1.0, 1.0]
LAMBDA_XU = [1.0, 1.1, 1.1, 1.0, 1.1, 1.0, 1.1, 1.0, 1.1, 1.0, 1.0, 1.0, 1.0, 1.0, 1.2]
LAMBDA_G = [1.0, 1.0, 1.0, 0.8, 1.0, 0.8, 1.0, 1.0, 1.0]


def bubble_case(lattice=abi.D2Q9, L=256, radius=40.0, width=5.0, t_ratio=0.8,
                a=1.0, b=4.0, sigma=0.125, Lambda=None, name=None, dims=None):
    """Static vapour bubble in liquid, fully periodic, Carnahan-Starling EOS,
    isothermal (the thermal population is absent)."""
    eos = dict(type=abi.EOS_CS, a=a, b=b, R=1.0, G=-1.0, M=1.0, Cv=1.0,
               g=(0.0, 0.0, 0.0), fext=(0.0, 0.0, 0.0), rho_0=0.0)
    d3 = lattice == abi.D3Q15
    if dims is None:
        dims = (L, L, L) if d3 else (L, L)
    nb, points, patches, names = box_mesh(lattice, dims, (True, True, True))
    tc = critical_temperature(eos)
    T0 = t_ratio * tc
    rv, rl = maxwell_densities(eos, T0)
    ctr = [(d - 1) / 2.0 for d in dims]
    r2 = sum((points[:, i] - ctr[i]) ** 2 for i in range(len(dims)))
    rho = tanh_profile(np.sqrt(r2), radius, width, rv, rl)
    n = rho.size
    f = dict(model=abi.XUMRT if d3 else abi.LIMRT, update=1,
             Lambda=Lambda or (LAMBDA_XU if d3 else LAMBDA_C1), sigma=sigma,
             bc_type=[], bc_value=np.zeros((0, 3)))
    return Case(name or f"bubble_{'d3q15' if d3 else 'd2q9'}_{'x'.join(map(str, dims))}",
                lattice, tuple(dims), (True,) * len(dims), nb, points, patches, names, eos, f, None,
                rho.astype(np.float64), np.zeros((n, 3)), np.full(n, T0),
                meta=dict(Tc=tc, T=T0, rho_v=rv, rho_l=rl, radius=radius))


def band_case(lattice=abi.D2Q9, dims=(8, 256), axis=1, height=96.0, width=5.0, t_ratio=0.8,
              a=1.0, b=4.0, sigma=0.125, Lambda=None, name=None):
    """Liquid band (a column or layer with flat interfaces) in vapour, fully
    periodic, Carnahan-Starling EOS, isothermal: along `axis` the band spans
    [c - height/2, c + height/2] around the box centre c, joined to the vapour
    by tanh profiles of width `width` at the Maxwell densities, as the
    reference's tgProfileScalarField builds an axial profile
    (src/applications/fields/setInitialFields/tgProfileScalarField.c:66-76,
    there with the band between z1 and z2)."""
    eos = dict(type=abi.EOS_CS, a=a, b=b, R=1.0, G=-1.0, M=1.0, Cv=1.0,
               g=(0.0, 0.0, 0.0), fext=(0.0, 0.0, 0.0), rho_0=0.0)
    d3 = lattice == abi.D3Q15
    nb, points, patches, names = box_mesh(lattice, tuple(dims), (True,) * len(dims))
    tc = critical_temperature(eos)
    T0 = t_ratio * tc
    rv, rl = maxwell_densities(eos, T0)
    c = (dims[axis] - 1) / 2.0
    z = points[:, axis].astype(np.float64)
    z1, z2 = c - 0.5 * height, c + 0.5 * height
    rho = rv + 0.5 * (rl - rv) * (np.tanh(2.0 * (z - z1) / width) - np.tanh(2.0 * (z - z2) / width))
    n = rho.size
    f = dict(model=abi.XUMRT if d3 else abi.LIMRT, update=1,
             Lambda=Lambda or (LAMBDA_XU if d3 else LAMBDA_C1), sigma=sigma,
             bc_type=[], bc_value=np.zeros((0, 3)))
    return Case(name or f"band_{'d3q15' if d3 else 'd2q9'}_{'x'.join(map(str, dims))}_h{height:g}",
                lattice, tuple(dims), (True,) * len(dims), nb, points, patches, names, eos, f, None,
                rho.astype(np.float64), np.zeros((n, 3)), np.full(n, T0),
                meta=dict(Tc=tc, T=T0, rho_v=rv, rho_l=rl, axis=axis, center=c, height=height))


def column_case(nx=128, ny=512, liquid_frac=0.4, width=4.0, t0=0.85, t_bot=0.86, t_top=0.84,
                gy=-1e-5, amp=1e-4, seed=SEED, name=None, f_bc=abi.BC_BOUNCEBACK, wall_u=None,
                a=9.0 / 392.0, b=2.0 / 21.0):
    """Thermal van der Waals liquid column: periodic in x, walls in y,
    liMRT flow + liTempMRT heat, fixedT bottom/top, gravity along y.

    The attraction defaults to a = 9/392 (Tc = 1/14), not 9/49 (Tc = 4/7):
    with G = -1 the pseudopotential sqrt(2(p - rho/3)/G) needs p < rho/3, and
    at 0.85 Tc with a = 9/49 the coexisting vapour has p - rho/3 = +5.4e-3, so
    psi is NaN there (the reference's own solver produces NaN on that case).
    Scaling a keeps T/Tc, rho_c = 1/(3b) and the coexistence densities
    (van der Waals corresponding states) unchanged."""
    eos = dict(type=abi.EOS_VDW, a=a, b=b, R=1.0, G=-1.0, M=1.0, Cv=1.0,
               g=(0.0, gy, 0.0), fext=(0.0, 0.0, 0.0), rho_0=0.0)
    tc = 8 * a / (27 * b)
    nb, points, patches, names = box_mesh(abi.D2Q9, (nx, ny), (True, False))
    rv, rl = maxwell_densities(eos, t0 * tc)
    y = points[:, 1].astype(np.float64)
    rho = tanh_profile(y, liquid_frac * ny, width, rl, rv)
    rng = np.random.Generator(np.random.PCG64(seed))
    T = t0 * tc + amp * rng.uniform(-1.0, 1.0, size=y.size)
    n = y.size
    # patches: Y0 (bottom), Y1 (top)
    g_bc_val = np.zeros((2, 3))
    g_bc_val[0, 0] = t_bot * tc
    g_bc_val[1, 0] = t_top * tc
    f_bc_val = np.zeros((2, 3))
    if wall_u is not None:
        f_bc_val[1, :] = wall_u
    f = dict(model=abi.LIMRT, update=1, Lambda=LAMBDA_C1, sigma=0.125,
             bc_type=[f_bc, f_bc] if wall_u is None else [abi.BC_BOUNCEBACK, abi.BC_FIXEDU],
             bc_value=f_bc_val)
    g = dict(model=abi.LITEMPMRT, update=1, Lambda=LAMBDA_G,
             bc_type=[abi.BC_FIXEDT, abi.BC_FIXEDT], bc_value=g_bc_val)
    return Case(name or f"column_d2q9_{nx}x{ny}", abi.D2Q9, (nx, ny), (True, False), nb, points,
                patches, names, eos, f, g, rho.astype(np.float64), np.zeros((n, 3)), T,
                meta=dict(Tc=tc, T=t0 * tc, rho_v=rv, rho_l=rl))


def perturbed(case, seed=SEED, du=1e-3, drho=0.0):
    """Copy of a case with a seeded random velocity (and density) perturbation,
    so that every term of the collision and force is exercised."""
    rng = np.random.Generator(np.random.PCG64(seed))
    U = case.U.copy()
    d = 3 if case.lattice == abi.D3Q15 else 2
    U[:, :d] += du * rng.uniform(-1.0, 1.0, size=(case.n, d))
    rho = case.rho * (1.0 + drho * rng.uniform(-1.0, 1.0, size=case.n))
    c = Case(**{**case.__dict__})
    c.U, c.rho = U, rho
    c.name = case.name + "_pert"
    return c


def standard_cases():
    """The workload shapes named for this path (full sizes)."""
    return {
        "bubble_d2q9_256": lambda: bubble_case(abi.D2Q9, 256, 40.0, 5.0, 0.8),
        "column_d2q9_128x512": lambda: column_case(128, 512),
        "bubble_d3q15_192": lambda: bubble_case(abi.D3Q15, 192, 48.0, 5.0, 0.75),
    }
