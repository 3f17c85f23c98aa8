"""Error of the FP32-deviation form against the FP64 path on the named workloads.

    python -m multiphaselb_b200.accuracy [--steps2d N] [--steps3d N] [--steps-column N] [--out report.json]

Both precisions run from the same initial state and the physical results
are compared.

Static bubbles (D2Q9 256^2, R = 40, T = 0.8 Tc, 20,000 steps; D3Q15 192^3,
R = 48, T = 0.75 Tc, 20,000 steps):

* coexistence densities: rho at the bubble centre (vapour) and at the corner
  farthest from it (liquid);
* the Laplace pressure jump dp = p(centre) - p(corner), with the reference's
  write-time pressure (macroPressure);
* the spurious-current magnitude max |u| over the lattice.

Thermal van der Waals column (D2Q9 128 x 512, liMRT + liTempMRT, fixedT
walls at 0.86 / 0.84 Tc, gravity; 50,000 steps, with the state also compared
at intermediate checkpoints):

* liquid and vapour densities: the mean of the row-averaged density over the
  bulk of each phase (rows 10-30 % and 60-90 % of the height);
* the temperature profile: the largest relative difference of the row means
  of T, and of T over all nodes;
* the interface height: where the row-averaged density crosses the mean of
  the two bulk densities (linear interpolation between rows);
* max |u| over the lattice, and the total energy sum T.

The FP64 path is bit-identical to the reference's CPU solver (tested on
smaller lattices), so it stands in for the reference at these sizes.
"""
import argparse
import json
import sys
import time

import numpy as np

from . import Lattice, abi, cases


def run(case, steps, precision):
    with Lattice(case, precision=precision) as lat:
        lat.upload_case()
        lat.initialize()
        t0 = time.perf_counter()
        lat.step(steps)
        lat.sync()
        wall = time.perf_counter() - t0
        out = lat.download()
        out["p"] = lat.macro_pressure()
        out["wall_s"] = wall
        return out


def observables(case, out):
    dims = case.dims
    ctr = tuple(d // 2 for d in dims)
    idx = lambda c: int(sum(c[i] * int(np.prod(dims[:i])) for i in range(len(dims))))  # noqa: E731
    ic, io = idx(ctr), idx(tuple(0 for _ in dims))
    umag = np.sqrt((out["U"] ** 2).sum(axis=1))
    return dict(rho_vapour=float(out["rho"][ic]), rho_liquid=float(out["rho"][io]),
                dp=float(out["p"][ic] - out["p"][io]), u_max=float(umag.max()), wall_s=out["wall_s"])


def compare(case, steps):
    a = observables(case, run(case, steps, abi.FP64))
    b = observables(case, run(case, steps, abi.FP32_DEV))
    rel = {k: abs(b[k] - a[k]) / max(abs(a[k]), 1e-300) for k in ("rho_vapour", "rho_liquid", "dp", "u_max")}
    return dict(case=case.name, steps=steps, nodes=case.n, fp64=a, fp32_dev=b, rel_err=rel,
                speedup=a["wall_s"] / b["wall_s"])


def column_observables(case, out):
    nx, ny = case.dims
    rho = out["rho"].reshape(ny, nx).mean(axis=1)
    T = out["T"].reshape(ny, nx)
    lo = rho[int(0.1 * ny):int(0.3 * ny)].mean()
    hi = rho[int(0.6 * ny):int(0.9 * ny)].mean()
    mid = 0.5 * (lo + hi)
    # first row (from the bottom) where the row mean falls below the midpoint
    j = int(np.argmax(rho < mid))
    h = (j - 1) + (rho[j - 1] - mid) / (rho[j - 1] - rho[j]) if j > 0 else float("nan")
    umag = np.sqrt((out["U"] ** 2).sum(axis=1))
    return dict(rho_liquid=float(lo), rho_vapour=float(hi), interface_y=float(h), u_max=float(umag.max()),
                energy=float(out["T"].sum()), T_rows=T.mean(axis=1), T=out["T"])


def compare_column(case, steps, checkpoints):
    """FP64 and FP32-deviation runs of the thermal column, compared at each checkpoint."""
    marks = sorted(set([c for c in checkpoints if 0 < c < steps] + [steps]))
    res = {}
    for prec in (abi.FP64, abi.FP32_DEV):
        with Lattice(case, precision=prec) as lat:
            lat.upload_case()
            lat.initialize()
            done, wall, obs = 0, 0.0, []
            for m in marks:
                t0 = time.perf_counter()
                lat.step(m - done)
                lat.sync()
                wall += time.perf_counter() - t0
                done = m
                obs.append(column_observables(case, lat.download()))
            res[prec] = (obs, wall)
    rows = []
    for i, m in enumerate(marks):
        a, b = res[abi.FP64][0][i], res[abi.FP32_DEV][0][i]
        rel = {k: abs(b[k] - a[k]) / max(abs(a[k]), 1e-300)
               for k in ("rho_liquid", "rho_vapour", "u_max", "energy")}
        rel["interface_y_abs"] = abs(b["interface_y"] - a["interface_y"])
        rel["T_rows"] = float(np.max(np.abs(b["T_rows"] - a["T_rows"]) / np.abs(a["T_rows"])))
        rel["T_nodes"] = float(np.max(np.abs(b["T"] - a["T"]) / np.abs(a["T"])))
        keep = lambda o: {k: v for k, v in o.items() if k not in ("T_rows", "T")}  # noqa: E731
        rows.append(dict(steps=m, fp64=keep(a), fp32_dev=keep(b), rel_err=rel))
    return dict(case=case.name, steps=steps, nodes=case.n, checkpoints=rows,
                wall_s={"fp64": res[abi.FP64][1], "fp32_dev": res[abi.FP32_DEV][1]},
                speedup=res[abi.FP64][1] / res[abi.FP32_DEV][1])


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps2d", type=int, default=20000)
    ap.add_argument("--steps3d", type=int, default=20000)
    ap.add_argument("--steps-column", type=int, default=50000)
    ap.add_argument("--only", default=None, choices=[None, "bubble2d", "bubble3d", "column"])
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    rep = []
    if a.only in (None, "bubble2d"):
        rep.append(compare(cases.bubble_case(abi.D2Q9, 256, 40.0, 5.0, 0.8), a.steps2d))
    if a.only in (None, "bubble3d"):
        rep.append(compare(cases.bubble_case(abi.D3Q15, 192, 48.0, 5.0, 0.75), a.steps3d))
    if a.only in (None, "column"):
        rep.append(compare_column(cases.column_case(128, 512), a.steps_column,
                                  [1000, 5000, 10000, 20000, 30000, 40000]))
    txt = json.dumps(rep, indent=1)
    print(txt)
    if a.out:
        with open(a.out, "w") as fh:
            fh.write(txt + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
