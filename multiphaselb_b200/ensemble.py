"""Time to equilibrium of static-bubble ensembles (D2Q9, Carnahan-Starling).

    python -m multiphaselb_b200.ensemble [--cases N] [--plain M] [--init tanh|mlp] ...

The ensemble: N independent fully periodic D2Q9 bubbles; lattice size L drawn
uniformly from {64, 96, 128, 192, 256, 384, 512} (L x L), T/Tc uniform in
[0.6, 0.95], bubble radius uniform in [8, 0.3 L]; CS EOS a = 1, b = 4, the
Li-MRT relaxation of the static-bubble workload, tanh width 5.  A case is at
equilibrium when max over nodes |drho/dt| < tol, measured over one check
interval of K steps.

Two ways to get there are timed:

* plain: each case alone, FP64, fused path, tanh/Maxwell initial profile,
  one case after the other (mplb_gpu_run_to_equilibrium), on the tile the
  autotuner keeps for its lattice (found on a throwaway handle outside the
  timed region, so the plain wall times hold no tuning);
* batched: all cases as FP32-deviation lattices advanced together
  (mplb_batch_run), initial profile from the tanh/Maxwell formula or from the
  learned warm start (multiphaselb_b200.warmstart).

The report gives per-case steps, the coexistence densities (rho at the bubble
centre and at the corner farthest from it) of both runs and their relative
difference, and the wall times.  Seeded; no dataset.
"""
import argparse
import json
import sys
import time

import numpy as np

from . import Batch, Lattice, abi, cases, warmstart

SIZES = (64, 96, 128, 192, 256, 384, 512)
SEED = 20240611
WIDTH = 5.0


def draw(n, seed=SEED):
    """n case specs (L, T/Tc, R), seeded."""
    rng = np.random.Generator(np.random.PCG64(seed))
    L = rng.choice(np.array(SIZES), size=n)
    t = rng.uniform(0.6, 0.95, size=n)
    R = rng.uniform(8.0, 0.3 * L)
    return [dict(L=int(a), t_ratio=float(b), radius=float(c)) for a, b, c in zip(L, t, R)]


def make_case(spec):
    return cases.bubble_case(abi.D2Q9, L=spec["L"], radius=spec["radius"], width=WIDTH, t_ratio=spec["t_ratio"],
                             name=f"bubble_d2q9_{spec['L']}_t{spec['t_ratio']:.3f}_r{spec['radius']:.1f}")


def coexistence(case, rho):
    """rho at the bubble centre (vapour) and at the corner farthest from it (liquid)."""
    nx, ny = case.dims
    cx, cy = nx // 2, ny // 2
    return float(rho[cx + nx * cy]), float(rho[0])


def tuned_tile(case):
    """The tile candidate the autotuner keeps for this lattice, as a
    Lattice tile_config (1-based), found on a throwaway handle."""
    with Lattice(case, path=abi.PATH_FUSED, precision=abi.FP64) as lat:
        lat.upload_case()
        lat.initialize()
        lat.step(1)
        return lat.info()["tile_config"] + 1


def run_plain(specs, K, tol, max_steps, log=None):
    out = []
    for i, s in enumerate(specs):
        c = make_case(s)
        tile = tuned_tile(c)
        with Lattice(c, path=abi.PATH_FUSED, precision=abi.FP64, tile_config=tile) as lat:
            lat.upload_case()
            lat.initialize()
            lat.sync()
            t0 = time.perf_counter()
            steps, rate = warmstart.run_eq(lat, max_steps, K, tol)
            lat.sync()
            wall = time.perf_counter() - t0
            rv, rl = coexistence(c, lat.download()["rho"])
        out.append(dict(steps=steps, rate=rate, wall_s=wall, rho_v=rv, rho_l=rl, diverged=bool(not np.isfinite(rate))))
        if log:
            log(f"plain {i} L={s['L']} t={s['t_ratio']:.3f} R={s['radius']:.1f}: {steps} steps {wall:.2f} s")
    return out


def crossing_steps(case):
    """Steps for sound in the liquid to cross the box: L / c_l with
    c_l^2 = dp/drho of the EOS at the Maxwell liquid density."""
    eos, T, rl = case.eos, case.meta["T"], case.meta["rho_l"]
    h = 1e-6 * rl
    c2 = (cases.p_eos(eos, rl + h, T) - cases.p_eos(eos, rl - h, T)) / (2 * h)
    return max(case.dims) / float(np.sqrt(c2))


def filter_windows(cs, scale):
    """Filter window of each case: scale x the sound crossing time, even."""
    return [int(2 * round(0.5 * scale * crossing_steps(c))) for c in cs]


def run_batched(specs, K, tol, max_steps, init=None, tile_config=0, filt=None):
    """All specs as one batch.  `init(lat, case)` (the learned warm start) may
    replace a lattice's tanh/Maxwell state on the device; it returns False to
    keep the fallback.  `filt` = (scale, first, every): time-averaging filter
    windows of `scale` sound crossing times (Batch.filter)."""
    t0 = time.perf_counter()
    cs = [make_case(s) for s in specs]
    t1 = time.perf_counter()
    lats, warm = [], 0
    for c in cs:
        lat = Lattice(c, path=abi.PATH_FUSED, precision=abi.FP32_DEV)
        lat.upload_case()
        if init is not None and init(lat, c):
            warm += 1
        lat.initialize()
        lats.append(lat)
    for lat in lats:
        lat.sync()
    t2 = time.perf_counter()
    host_s, setup = t1 - t0, t2 - t1
    with Batch(lats, check_interval=K, tol=tol, tile_config=tile_config) as b:
        if filt and filt[0] > 0:
            b.filter(filter_windows(cs, filt[0]), filt[1], filt[2])
        t0 = time.perf_counter()
        steps, rate, conv = b.run(max_steps)
        lats[0].sync()
        wall = time.perf_counter() - t0
        info = b.info()
    res = []
    for c, lat, st, r in zip(cs, lats, steps, rate):
        rv, rl = coexistence(c, lat.download()["rho"])
        res.append(dict(steps=int(st), rate=float(r), rho_v=rv, rho_l=rl, diverged=bool(not np.isfinite(r))))
        lat.close()
    out = dict(cases=res, wall_s=wall, setup_s=setup, host_build_s=host_s, warm_started=warm, converged=conv,
               info=info, nodes=int(sum(c.n for c in cs)), fallback_reran=0)
    # The tanh/Maxwell start is the warm start's fallback: a warm-started
    # lattice that diverged runs again from it (its time counts).
    bad = [i for i, r in enumerate(res) if r["diverged"]] if init is not None else []
    if bad:
        again = run_batched([specs[i] for i in bad], K, tol, max_steps, None, tile_config, filt)
        for i, r in zip(bad, again["cases"]):
            res[i] = dict(r, fallback=True)
        out["wall_s"] += again["wall_s"]
        out["setup_s"] += again["setup_s"]
        out["converged"] += again["converged"]
        out["fallback_reran"] = len(bad)
    return out


def compare(batched, plain):
    """Batched run against the plain runs of the same cases (by position)."""
    n = len(plain)
    sub = batched["cases"][:n]
    both = [(x, y) for x, y in zip(sub, plain) if not x["diverged"] and not y["diverged"]]
    rel = [max(abs(x["rho_v"] - y["rho_v"]) / y["rho_v"], abs(x["rho_l"] - y["rho_l"]) / y["rho_l"])
           for x, y in both]
    return dict(cases=n, plain_wall_s=sum(y["wall_s"] for y in plain), batched_wall_s=batched["wall_s"],
                speedup=sum(y["wall_s"] for y in plain) / batched["wall_s"],
                plain_steps=int(sum(y["steps"] for y in plain)), batched_steps=int(sum(x["steps"] for x in sub)),
                plain_diverged=sum(1 for y in plain if y["diverged"]),
                batched_diverged=sum(1 for x in sub if x["diverged"]),
                batched_converged=batched["converged"],
                max_rel_coexistence=max(rel, default=None),
                within_1e3=sum(1 for r in rel if r < 1e-3), compared=len(rel))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--cases", type=int, default=512)
    ap.add_argument("--plain", type=int, default=16, help="first M cases also run plain (FP64, one by one)")
    ap.add_argument("--seed", type=int, default=SEED)
    ap.add_argument("--tol", type=float, default=1e-9)
    ap.add_argument("--check", type=int, default=1000)
    ap.add_argument("--max-steps", type=int, default=400000)
    ap.add_argument("--init", choices=("tanh", "mlp", "both"), default="tanh")
    ap.add_argument("--weights", default=None, help="warm-start weights (.npz); default: the packaged D2Q9 network")
    ap.add_argument("--sizes", default=None, help="comma list: one case per size at T/Tc=0.8, R=0.2L")
    ap.add_argument("--filter", type=float, default=0.0,
                    help="time-averaging filter windows of this many sound crossing times (0: off)")
    ap.add_argument("--filter-first", type=int, default=2000)
    ap.add_argument("--filter-every", type=int, default=10000)
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    filt = (a.filter, a.filter_first, a.filter_every) if a.filter > 0 else None
    if a.sizes:
        specs = [dict(L=int(x), t_ratio=0.8, radius=0.2 * int(x)) for x in a.sizes.split(",")]
    else:
        specs = draw(a.cases, a.seed)
    log = lambda m: print(m, file=sys.stderr, flush=True)  # noqa: E731
    rep = dict(specs=specs, tol=a.tol, check_interval=a.check, max_steps=a.max_steps,
               filter=dict(scale=a.filter, first=a.filter_first, every=a.filter_every) if filt else None)
    m = min(a.plain, len(specs))
    if m:
        rep["plain"] = run_plain(specs[:m], a.check, a.tol, a.max_steps, log)
    for mode in (("tanh", "mlp") if a.init == "both" else (a.init,)):
        init = None
        if mode == "mlp":
            init = warmstart.initializer(abi.D2Q9, a.weights)
            if init is None:
                raise SystemExit("no trained warm-start weights")
        b = run_batched(specs, a.check, a.tol, a.max_steps, init, filt=filt)
        rep["batched_" + mode] = b
        log(f"batched ({mode}): {b['converged']}/{len(specs)} converged, {b['wall_s']:.2f} s")
        if m:
            # batched wall time is for all cases; compare per case on the
            # first m, and on the wall only when m covers every case
            sub = b if m == len(specs) else run_batched(specs[:m], a.check, a.tol, a.max_steps, init, filt=filt)
            rep["compare_" + mode] = compare(sub, rep["plain"])
            log(json.dumps(rep["compare_" + mode]))
    txt = json.dumps(rep, indent=1)
    if a.out:
        with open(a.out, "w") as fh:
            fh.write(txt + "\n")
    else:
        print(txt)
    return 0


if __name__ == "__main__":
    sys.exit(main())
