"""Error of the FP32-deviation form against the FP64 path on static bubbles.

    python -m multiphaselb_b200.accuracy [--steps N] [--out report.json]

For each bubble (D2Q9 256^2, R = 40, T = 0.8 Tc, 20,000 steps; D3Q15 192^3,
R = 48, T = 0.75 Tc, 2,000 steps by default) both precisions run from the
same initial state, and the physical results are compared:

* coexistence densities: rho at the bubble centre (vapour) and at the corner
  farthest from it (liquid);
* the Laplace pressure jump dp = p(centre) - p(corner), with the reference's
  write-time pressure (macroPressure);
* the spurious-current magnitude max |u| over the lattice.

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


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps2d", type=int, default=20000)
    ap.add_argument("--steps3d", type=int, default=2000)
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    rep = [compare(cases.bubble_case(abi.D2Q9, 256, 40.0, 5.0, 0.8), a.steps2d),
           compare(cases.bubble_case(abi.D3Q15, 192, 48.0, 5.0, 0.75), a.steps3d)]
    txt = json.dumps(rep, indent=1)
    print(txt)
    if a.out:
        with open(a.out, "w") as fh:
            fh.write(txt + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
