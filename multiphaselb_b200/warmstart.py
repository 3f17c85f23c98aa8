"""Learned warm start for static bubbles and liquid columns (mplb_mlp_* in
include/mplb_gpu.h).

    python -m multiphaselb_b200.warmstart train --lattice d2q9 --out weights.npz
    python -m multiphaselb_b200.warmstart evaluate --lattice d3q15 --weights weights.npz --cases 64
    python -m multiphaselb_b200.warmstart train --geometry column
    python -m multiphaselb_b200.warmstart evaluate --geometry column --cases 32

Pipeline:
  1. converge a grid of bubbles (T/Tc, R) with the plain FP64 solver
     (mplb_gpu_run_to_equilibrium) and take their radial density profiles;
  2. train the 5-64-64-64-1 network on the device (the library's own forward,
     backward and Adam kernels) on (T/Tc, a, b, r/R, R) -> b * rho samples;
  3. initialise new lattices from the network on the device
     (mplb_mlp_init_bubble) instead of the tanh/Maxwell profile.

The tanh/Maxwell initial state stays the fallback: ``initializer`` returns
None for inputs outside the trained ranges.  The converged plain solver is the
yardstick: ``evaluate`` runs every case from both initial states to equilibrium
and reports the steps, the wall time and the network's initial error against
the converged profile.  One network per lattice family (2D and 3D bubbles
have different Laplace pressures), and one for axial profiles: liquid bands
(a column or layer) with flat interfaces, whose features carry R = +inf and
the signed distance to the interface (mplb_mlp_init_column).
"""
import argparse
import ctypes as C
import json
import os
import sys
import time

import numpy as np

from . import Lattice, MplbError, abi, cases, load_library

NPARAM = 8769
HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = {abi.D2Q9: os.path.join(HERE, "data", "warmstart_d2q9.npz"),
                   abi.D3Q15: os.path.join(HERE, "data", "warmstart_d3q15.npz")}
# axial profiles (liquid bands with flat interfaces), D2Q9
COLUMN_WEIGHTS = os.path.join(HERE, "data", "warmstart_d2q9_column.npz")
T_RANGE = (0.6, 0.95)
CS_A, CS_B = 1.0, 4.0


def _lib():
    lib = load_library()
    if not getattr(lib, "_mlp_sigs", False):
        D = C.POINTER(C.c_double)
        F = C.POINTER(C.c_float)
        H = C.c_void_p
        sig = {
            "mplb_mlp_create": ([C.c_int32, C.c_uint64, C.POINTER(H)], C.c_int),
            "mplb_mlp_destroy": ([H], C.c_int),
            "mplb_mlp_get_params": ([H, F], C.c_int),
            "mplb_mlp_set_params": ([H, F], C.c_int),
            "mplb_mlp_features": ([C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, F], None),
            "mplb_mlp_set_samples": ([H, D, D, D, D, D, D, C.c_uint32], C.c_int),
            "mplb_mlp_gradient": ([H, F, D], C.c_int),
            "mplb_mlp_train": ([H, C.c_uint32, C.c_uint32, C.c_float, D], C.c_int),
            "mplb_mlp_predict": ([H, D, D, D, D, D, C.c_uint32, D], C.c_int),
            "mplb_mlp_init_bubble": ([H, H, C.c_double, D, C.c_double, C.c_double], C.c_int),
            "mplb_mlp_init_bubble_mass": ([H, H, C.c_double, D, C.c_double, C.c_double, C.c_double, D], C.c_int),
            "mplb_mlp_init_column": ([H, H, C.c_double, C.c_int32, C.c_double, C.c_double, C.c_double], C.c_int),
            "mplb_mlp_init_column_mass": ([H, H, C.c_double, C.c_int32, C.c_double, C.c_double, C.c_double,
                                           C.c_double, D], C.c_int),
        }
        for name, (args, res) in sig.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        lib._mlp_sigs = True
    return lib


def _f32(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(C.POINTER(C.c_float))


def _f64(a, n=None):
    a = np.ascontiguousarray(np.broadcast_to(a, (n,)) if n is not None else a, dtype=np.float64)
    return a, a.ctypes.data_as(C.POINTER(C.c_double))


def features(t_ratio, a, b, r, R):
    """The network's normalised inputs for one sample (library host code)."""
    out = np.zeros(5, dtype=np.float32)
    _lib().mplb_mlp_features(t_ratio, a, b, r, R, out.ctypes.data_as(C.POINTER(C.c_float)))
    return out


class Network:
    """A device-resident warm-start network (mplb_mlp_t)."""

    def __init__(self, device=-1, seed=0, params=None):
        self.lib = _lib()
        h = C.c_void_p()
        self._check(self.lib.mplb_mlp_create(device, seed, C.byref(h)))
        self.h = h
        if params is not None:
            self.set_params(params)

    def _check(self, rc):
        if rc != 0:
            raise MplbError(rc, self.lib.mplb_gpu_last_error().decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.mplb_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def params(self):
        p = np.zeros(NPARAM, dtype=np.float32)
        self._check(self.lib.mplb_mlp_get_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float))))
        return p

    def set_params(self, p):
        a, ptr = _f32(p)
        assert a.size == NPARAM
        self._check(self.lib.mplb_mlp_set_params(self.h, ptr))

    def set_samples(self, t_ratio, a, b, r, R, rho):
        n = len(rho)
        keep = [_f64(x, n) for x in (t_ratio, a, b, r, R, rho)]
        self._check(self.lib.mplb_mlp_set_samples(self.h, *[k[1] for k in keep], n))

    def gradient(self):
        g = np.zeros(NPARAM, dtype=np.float32)
        loss = C.c_double()
        self._check(self.lib.mplb_mlp_gradient(self.h, g.ctypes.data_as(C.POINTER(C.c_float)), C.byref(loss)))
        return g, loss.value

    def train(self, steps, batch=1024, lr=1e-3):
        loss = C.c_double()
        self._check(self.lib.mplb_mlp_train(self.h, steps, batch, lr, C.byref(loss)))
        return loss.value

    def predict(self, t_ratio, a, b, r, R):
        n = len(np.atleast_1d(r))
        keep = [_f64(x, n) for x in (t_ratio, a, b, r, R)]
        out = np.zeros(n)
        self._check(self.lib.mplb_mlp_predict(self.h, *[k[1] for k in keep], n, abi.dptr(out)))
        return out

    def init_bubble(self, lat, t_ratio, center, radius, T):
        c, cp = _f64(np.asarray(center, dtype=np.float64).ravel().tolist() + [0.0] * (3 - len(center)))
        self._check(self.lib.mplb_mlp_init_bubble(self.h, lat.h, t_ratio, cp, radius, T))

    def init_column(self, lat, t_ratio, axis, center, height, T):
        self._check(self.lib.mplb_mlp_init_column(self.h, lat.h, t_ratio, axis, center, height, T))

    def save(self, path):
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        np.savez(path, params=self.params())

    @classmethod
    def load(cls, path, device=-1):
        return cls(device=device, params=np.load(path)["params"])


# ------------------------------------------------------------- training data
def centre(case):
    return [(d - 1) / 2.0 for d in case.dims]


def radial(case):
    """Distance of every node to the bubble centre."""
    c = centre(case)
    D = len(case.dims)
    return np.sqrt(sum((case.points[:, i] - c[i]) ** 2 for i in range(D)))


def profile_samples(case, rho, radius, rng, per_bin=48, bins=64):
    """Stratified samples of a converged profile: up to per_bin nodes in each
    of `bins` equal intervals of r - R on [-30, 30] (the network's clamped
    range, 6 interface widths), plus some bulk nodes on either side beyond.
    Returns (r, rho)."""
    r = radial(case)
    d = r - radius
    idx = []
    edges = np.linspace(-30.0, 30.0, bins + 1)
    which = np.digitize(d, edges) - 1
    for k in range(-1, bins + 1):
        sel = np.flatnonzero(which == k)
        if sel.size:
            idx.append(rng.choice(sel, size=min(per_bin * (4 if k in (-1, bins) else 1), sel.size), replace=False))
    idx = np.concatenate(idx)
    return r[idx], rho[idx]


def band_distance(case):
    """Signed distance of every node to the nearest flat interface of a band
    case, positive inside the liquid band (height/2 - |z - c|)."""
    m = case.meta
    return 0.5 * m["height"] - np.abs(case.points[:, m["axis"]] - m["center"])


def band_samples(case, rho, rng, per_bin=48, bins=64):
    """As profile_samples, in the signed distance to the interface; returns
    (distance, rho)."""
    dist = band_distance(case)
    idx = []
    edges = np.linspace(-30.0, 30.0, bins + 1)
    which = np.digitize(dist, edges) - 1
    for k in range(-1, bins + 1):
        sel = np.flatnonzero(which == k)
        if sel.size:
            idx.append(rng.choice(sel, size=min(per_bin * (4 if k in (-1, bins) else 1), sel.size), replace=False))
    idx = np.concatenate(idx)
    return dist[idx], rho[idx]


def band(L, height, t_ratio, nx=8):
    """A D2Q9 liquid band across a periodic nx x L box (flat interfaces along x)."""
    return cases.band_case(abi.D2Q9, dims=(nx, L), axis=1, height=height, width=5.0, t_ratio=t_ratio)


def column_training_grid():
    """(L, height, T/Tc) of the training bands."""
    ts = np.linspace(T_RANGE[0], T_RANGE[1], 8)
    return [(L, H, float(t)) for L, H in [(128, 48.0), (256, 112.0)] for t in ts]


def build_column_training_set(grid=None, seed=1, log=None, **conv):
    """Converged bands -> samples (T/Tc, distance, rho); R = +inf marks the
    flat interface in the network's features."""
    rng = np.random.default_rng(seed)
    T, Dd, Y, meta = [], [], [], []
    for L, H, t in grid or column_training_grid():
        c = band(L, H, t)
        rho, steps, rate, wall = converge(c, **conv)
        if not np.isfinite(rate) or not np.all(np.isfinite(rho)):
            if log:
                log(f"column-set L={L} H={H} t={t:.3f}: diverged, skipped")
            continue
        d, y = band_samples(c, rho, rng)
        T.append(np.full(d.size, t))
        Dd.append(d)
        Y.append(y)
        meta.append(dict(L=L, height=H, t_ratio=t, steps=steps, rate=rate, wall_s=wall))
        if log:
            log(f"column-set L={L} H={H} t={t:.3f}: {steps} steps, {d.size} samples")
    d = np.concatenate(Dd)
    return np.concatenate(T), d, np.full(d.size, np.inf), np.concatenate(Y), meta


def bubble(lattice, L, R, t_ratio):
    if lattice == abi.D2Q9:
        return cases.bubble_case(abi.D2Q9, L=L, radius=R, width=5.0, t_ratio=t_ratio)
    return cases.bubble_case(abi.D3Q15, L=L, radius=R, width=5.0, t_ratio=t_ratio)


def run_eq(lat, max_steps, K, tol):
    """run_to_equilibrium that reports a diverged run (non-finite density) as
    (steps, inf) instead of raising."""
    try:
        return lat.run_to_equilibrium(max_steps, K, tol)
    except MplbError as e:
        if e.code != abi.E_NONFINITE:
            raise
        return max_steps, float("inf")


def converge(case, K=1000, tol=1e-9, max_steps=400000, precision=abi.FP64):
    """The plain solver to equilibrium: (rho, steps, rate, wall seconds);
    rate = inf if the run diverged."""
    with Lattice(case, path=abi.PATH_FUSED, precision=precision) as lat:
        lat.upload_case()
        lat.initialize()
        lat.sync()
        t0 = time.perf_counter()
        steps, rate = run_eq(lat, max_steps, K, tol)
        lat.sync()
        wall = time.perf_counter() - t0
        rho = lat.download()["rho"]
    return rho, steps, rate, wall


def training_grid(lattice):
    """(L, R, T/Tc) of the training bubbles."""
    ts = np.linspace(T_RANGE[0], T_RANGE[1], 8)
    if lattice == abi.D2Q9:
        LR = [(64, 8.0), (64, 16.0), (128, 32.0), (256, 64.0), (512, 128.0)]
    else:
        LR = [(64, 10.0), (80, 16.0), (112, 24.0), (128, 32.0), (144, 40.0)]
    return [(L, R, float(t)) for L, R in LR for t in ts]


def build_training_set(lattice, grid=None, seed=1, log=None, **conv):
    """Converged bubbles of the grid -> samples (T/Tc, r, R, rho) and a record per bubble."""
    rng = np.random.default_rng(seed)
    T, Rs, Rr, Y, meta = [], [], [], [], []
    for L, R, t in grid or training_grid(lattice):
        c = bubble(lattice, L, R, t)
        rho, steps, rate, wall = converge(c, **conv)
        if not np.isfinite(rate) or not np.all(np.isfinite(rho)):
            if log:
                log(f"train-set L={L} R={R} t={t:.3f}: diverged, skipped")
            continue
        r, y = profile_samples(c, rho, R, rng)
        T.append(np.full(r.size, t))
        Rs.append(r)
        Rr.append(np.full(r.size, R))
        Y.append(y)
        meta.append(dict(L=L, R=R, t_ratio=t, steps=steps, rate=rate, wall_s=wall))
        if log:
            log(f"train-set L={L} R={R} t={t:.3f}: {steps} steps, {r.size} samples")
    return np.concatenate(T), np.concatenate(Rs), np.concatenate(Rr), np.concatenate(Y), meta


def train(net, t, r, R, rho, steps=40000, batch=2048, lr=3e-3, lr_end=5e-5, chunks=12):
    """Adam with a stepwise geometric learning-rate decay; returns the loss history."""
    net.set_samples(t, CS_A, CS_B, r, R, rho)
    hist = []
    for k in range(chunks):
        rate = lr * (lr_end / lr) ** (k / max(chunks - 1, 1))
        hist.append(net.train(steps // chunks, batch, rate))
    return hist


def place(net, lat, t_ratio, centre_, R, T, mass):
    """The network's bubble on the lattice with the lattice holding `mass`
    (the mass of the state it replaces), so that the case relaxes to the same
    equilibrium as from its tanh/Maxwell state, only from closer
    (mplb_mlp_init_bubble_mass).  Returns the effective radius."""
    c, cp = _f64(np.asarray(centre_, dtype=np.float64).ravel().tolist() + [0.0] * (3 - len(centre_)))
    used = C.c_double()
    net._check(net.lib.mplb_mlp_init_bubble_mass(net.h, lat.h, t_ratio, cp, R, T, mass, C.byref(used)))
    return used.value


def place_column(net, lat, t_ratio, axis, center, height, T, mass):
    """The network's band on the lattice holding `mass` (mplb_mlp_init_column_mass);
    returns the effective height."""
    used = C.c_double()
    net._check(net.lib.mplb_mlp_init_column_mass(net.h, lat.h, t_ratio, axis, center, height, T, mass,
                                                 C.byref(used)))
    return used.value


def column_initializer(weights=None, device=-1):
    """As `initializer`, for band cases (cases.band_case) and the column network."""
    path = weights or COLUMN_WEIGHTS
    if not os.path.exists(path):
        return None
    net = Network.load(path, device)

    def init(lat, case):
        m = case.meta
        t_ratio = m["T"] / m["Tc"]
        if not (T_RANGE[0] - 1e-9 <= t_ratio <= T_RANGE[1] + 1e-9) or case.eos["type"] != abi.EOS_CS:
            return False
        mass = lat.mass_energy()[0]
        init.radius = place_column(net, lat, t_ratio, m["axis"], m["center"], m["height"], m["T"], mass)
        return True

    init.net = net
    init.radius = None
    return init


def initializer(lattice, weights=None, device=-1):
    """Function (lat, case) -> bool that overwrites a freshly uploaded bubble
    lattice with the network's profile (same mass as the uploaded state, see
    `place`), or returns False (the caller keeps the tanh/Maxwell state) when
    the case is outside the trained ranges.  None when no trained weights
    exist."""
    path = weights or DEFAULT_WEIGHTS[lattice]
    if not os.path.exists(path):
        return None
    net = Network.load(path, device)

    def init(lat, case):
        m = case.meta
        t_ratio = m["T"] / m["Tc"]
        if not (T_RANGE[0] - 1e-9 <= t_ratio <= T_RANGE[1] + 1e-9) or case.eos["type"] != abi.EOS_CS:
            return False
        mass = lat.mass_energy()[0]
        init.radius = place(net, lat, t_ratio, centre(case), m["radius"], m["T"], mass)
        return True

    init.net = net
    init.radius = None
    return init


# ---------------------------------------------------------------- evaluation
def evaluate(lattice, init, specs, K=1000, tol=1e-9, max_steps=400000, precision=abi.FP64, log=None):
    """Both initial states to equilibrium for every spec (L, R, T/Tc; or L,
    height, T/Tc for bands)."""
    rows = []
    for s in specs:
        c = band(s["L"], s["height"], s["t_ratio"]) if "height" in s else \
            bubble(lattice, s["L"], s["radius"], s["t_ratio"])
        rec = dict(s)
        for mode in ("plain", "warm"):
            with Lattice(c, path=abi.PATH_FUSED, precision=precision) as lat:
                lat.upload_case()
                used = mode == "warm" and init(lat, c)
                if mode == "warm" and not used:
                    rec["warm"] = None
                    continue
                lat.initialize()
                rho0 = lat.download()["rho"] if mode == "warm" else None
                lat.sync()
                t0 = time.perf_counter()
                steps, rate = run_eq(lat, max_steps, K, tol)
                lat.sync()
                wall = time.perf_counter() - t0
                rho = lat.download()["rho"]
            rec[mode] = dict(steps=steps, rate=rate, wall_s=wall, diverged=bool(not np.isfinite(rate)))
            if mode == "warm":
                rec["warm"]["radius_used"] = init.radius
            if mode == "plain":
                rho_eq = rho
                rec["tanh_err_max"] = float(np.abs(c.rho - rho_eq).max() / rho_eq.max())
            elif not rec["plain"]["diverged"] and not rec["warm"]["diverged"]:
                # the converged plain solver is the yardstick of the network's initial profile
                rec["init_err_max"] = float(np.abs(rho0 - rho_eq).max() / rho_eq.max())
                rec["final_rel_diff"] = float(np.abs(rho - rho_eq).max() / rho_eq.max())
                ctr = int(np.argmin(radial(c))) if "height" not in s else int(np.argmin(np.abs(band_distance(c))))
                rec["coexistence_rel_diff"] = float(max(abs(rho[ctr] - rho_eq[ctr]) / rho_eq[ctr],
                                                        abs(rho[0] - rho_eq[0]) / rho_eq[0]))
        rows.append(rec)
        if log:
            log(json.dumps(rec))
    return rows


def draw_3d(n, seed=7):
    rng = np.random.Generator(np.random.PCG64(seed))
    t = rng.uniform(0.6, 0.95, n)
    R = rng.uniform(12.0, 40.0, n)
    return [dict(L=128, radius=float(r), t_ratio=float(x)) for x, r in zip(t, R)]


def draw_columns(n, seed=11):
    rng = np.random.Generator(np.random.PCG64(seed))
    L = rng.choice(np.array([128, 192, 256, 384]), size=n)
    t = rng.uniform(0.6, 0.95, n)
    h = rng.uniform(0.2, 0.6, n) * L
    return [dict(L=int(a), height=float(b), t_ratio=float(x)) for a, b, x in zip(L, h, t)]


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=("train", "evaluate"))
    ap.add_argument("--geometry", choices=("bubble", "column"), default="bubble",
                    help="column: liquid bands with flat interfaces (D2Q9, the column network)")
    ap.add_argument("--lattice", choices=("d2q9", "d3q15"), default="d3q15")
    ap.add_argument("--weights", default=None)
    ap.add_argument("--out", default=None)
    ap.add_argument("--steps", type=int, default=40000)
    ap.add_argument("--cases", type=int, default=64)
    ap.add_argument("--tol", type=float, default=1e-9)
    ap.add_argument("--check", type=int, default=1000)
    ap.add_argument("--precision", choices=("fp64", "fp32dev"), default="fp64")
    a = ap.parse_args(argv)
    lat = abi.D2Q9 if a.lattice == "d2q9" else abi.D3Q15
    prec = abi.FP64 if a.precision == "fp64" else abi.FP32_DEV
    log = lambda m: print(m, file=sys.stderr, flush=True)  # noqa: E731
    column = a.geometry == "column"
    if column:
        lat = abi.D2Q9
    if a.cmd == "train":
        t0 = time.perf_counter()
        if column:
            t, r, R, rho, meta = build_column_training_set(log=log, K=a.check, tol=a.tol)
        else:
            t, r, R, rho, meta = build_training_set(lat, log=log, K=a.check, tol=a.tol)
        t1 = time.perf_counter()
        net = Network(seed=1)
        hist = train(net, t, r, R, rho, steps=a.steps)
        t2 = time.perf_counter()
        pred = net.predict(t, CS_A, CS_B, r, R)
        rep = dict(samples=int(r.size), cases=meta, loss=hist, data_s=t1 - t0, train_s=t2 - t1,
                   fit_max_abs=float(np.abs(pred - rho).max()), fit_rms=float(np.sqrt(np.mean((pred - rho) ** 2))),
                   fit_max_rel=float(np.abs(pred / rho - 1.0).max()))
        net.save(a.weights or (COLUMN_WEIGHTS if column else DEFAULT_WEIGHTS[lat]))
        txt = json.dumps(rep, indent=1)
    else:
        init = column_initializer(a.weights) if column else initializer(lat, a.weights)
        if init is None:
            raise SystemExit("no trained weights")
        specs = draw_3d(a.cases) if lat == abi.D3Q15 else (draw_columns(a.cases) if column else None)
        if specs is None:
            from .ensemble import draw
            specs = draw(a.cases)
        rows = evaluate(lat, init, specs, a.check, a.tol, precision=prec, log=log)
        ok = [r for r in rows if r.get("warm") and not r["warm"]["diverged"] and not r["plain"]["diverged"]]
        summ = dict(cases=len(rows), warm_used=sum(1 for r in rows if r.get("warm")),
                    plain_diverged=sum(1 for r in rows if r["plain"]["diverged"]),
                    warm_diverged=sum(1 for r in rows if r.get("warm") and r["warm"]["diverged"]),
                    compared=len(ok),
                    plain_steps=int(sum(r["plain"]["steps"] for r in ok)),
                    warm_steps=int(sum(r["warm"]["steps"] for r in ok)),
                    plain_wall_s=float(sum(r["plain"]["wall_s"] for r in ok)),
                    warm_wall_s=float(sum(r["warm"]["wall_s"] for r in ok)),
                    fewer_steps=sum(1 for r in ok if r["warm"]["steps"] < r["plain"]["steps"]),
                    more_steps=sum(1 for r in ok if r["warm"]["steps"] > r["plain"]["steps"]),
                    median_tanh_err=float(np.median([r["tanh_err_max"] for r in ok])) if ok else None,
                    median_init_err=float(np.median([r["init_err_max"] for r in ok])) if ok else None,
                    max_coexistence_rel_diff=max([r["coexistence_rel_diff"] for r in ok], default=None))
        txt = json.dumps(dict(summary=summ, rows=rows), indent=1)
        log(json.dumps(summ))
    if a.out:
        with open(a.out, "w") as fh:
            fh.write(txt + "\n")
    else:
        print(txt)
    return 0


if __name__ == "__main__":
    sys.exit(main())
