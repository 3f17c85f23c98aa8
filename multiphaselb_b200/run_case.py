"""Run one named workload for a few steps on cuda:0 (for profilers).

    python -m multiphaselb_b200.run_case WORKLOAD STEPS [--path auto|fused|operators]

WORKLOAD: column (thermal VdW column, D2Q9 128x512), column_big (the same
column at 512x2048, larger than L2, for ncu captures), bubble2d (D2Q9
256x256), bubble2d_big (D2Q9 1024x1024), bubble3d (D3Q15 192^3),
bubble3d_small (D3Q15 96^3, for full ncu captures), bubble3d_mid (D3Q15
128^3, 0.7 GB on the device: ncu captures where half the tiles are inner).
"""
import argparse
import sys

from . import PATH_AUTO, PATH_FUSED, PATH_OPERATORS, Lattice, abi, cases

WORKLOADS = {
    "column": lambda: cases.column_case(128, 512),
    "column_big": lambda: cases.column_case(512, 2048),
    "bubble2d": lambda: cases.bubble_case(abi.D2Q9, 256, 40.0, 5.0, 0.8),
    "bubble2d_big": lambda: cases.bubble_case(abi.D2Q9, 1024, 160.0, 5.0, 0.8),
    "bubble3d": lambda: cases.bubble_case(abi.D3Q15, 192, 48.0, 5.0, 0.75),
    "bubble3d_small": lambda: cases.bubble_case(abi.D3Q15, 96, 24.0, 5.0, 0.75),
    "bubble3d_mid": lambda: cases.bubble_case(abi.D3Q15, 128, 32.0, 5.0, 0.75),
}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("workload", choices=list(WORKLOADS))
    ap.add_argument("steps", type=int)
    ap.add_argument("--path", default="auto", choices=["auto", "fused", "operators"])
    ap.add_argument("--tile", type=int, default=0, help="0 = autotune, k > 0 = candidate k-1")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32dev"])
    a = ap.parse_args(argv)
    path = {"auto": PATH_AUTO, "fused": PATH_FUSED, "operators": PATH_OPERATORS}[a.path]
    case = WORKLOADS[a.workload]()
    prec = abi.FP64 if a.precision == "fp64" else abi.FP32_DEV
    with Lattice(case, path=path, device=0, tile_config=a.tile, precision=prec) as lat:
        lat.upload_case()
        lat.initialize()
        lat.step(a.steps)
        m, e = lat.mass_energy()
        print(a.workload, case.n, "nodes", a.steps, "steps", lat.info(), "mass", m, "energy", e)
    return 0


if __name__ == "__main__":
    sys.exit(main())
