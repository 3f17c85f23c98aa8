"""Generate the golden vectors in this directory from the REFERENCE build.

    python -m tests.golden.make_golden [case names]

Each .npz holds a self-contained small case (neighbour table, patches, EOS,
field constants, initial rho/U/T) and the reference's state after `steps`
time steps of its own solver loop, produced by oracle/_ref/libmplb_ref.so
(the reference's sources compiled in place by oracle/Makefile).  They pin the
CPU restatement and the GPU path on machines where the reference tree is not
available.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from multiphaselb_b200 import cases  # noqa: E402
from tests.helpers import FIELDS, run_checker, small_cases  # noqa: E402

STEPS = {"bubble_d2q9": 12, "column_d2q9": 12, "lid_d2q9": 9, "bubble_d3q15": 5, "walls_d3q15": 5,
         "st_d2q9": 10, "st_d3q15": 5, "my_column_d2q9": 9, "my_walls_d3q15": 5, "outflow_d2q9": 8,
         "outflow_corner_d2q9": 6, "outflow_d3q15": 5, "cylinder_d2q9": 8,
         "my_slab_d3q15": 6}
# Long runs (fixtures named long_<case>_<steps>steps.npz): a thermal column
# with bounce-back and fixedT walls, a walled D3Q15 box with gravity and an
# external force, and the surface-tension channel, each far past the first
# steps, where a divergence that starts late would show.
LONG_STEPS = {"column_d2q9": 1000, "walls_d3q15": 1000, "st_d2q9": 1000}


def save_case(path, case, steps, out):
    spec = dict(name=case.name, lattice=case.lattice, dims=list(case.dims), periodic=list(case.periodic),
                eos={k: (list(v) if isinstance(v, tuple) else v) for k, v in case.eos.items()},
                f=None if case.f is None else {k: (np.asarray(v).tolist() if k in ("bc_value", "Lambda", "bc_type") else v)
                                               for k, v in case.f.items()},
                g=None if case.g is None else {k: (np.asarray(v).tolist() if k in ("bc_value", "Lambda", "bc_type") else v)
                                               for k, v in case.g.items()},
                steps=steps, rank=int(case.meta.get("rank", 0)))
    arrs = {"in_" + k: getattr(case, k) for k in ("rho", "U", "T")}
    if not case.meta.get("box", True):
        # not a box: keep the mesh itself
        arrs.update(mesh_nb=case.nb, mesh_points=case.points,
                    mesh_patch_count=np.array([len(p) for p in case.patches], dtype=np.int64),
                    mesh_patch_nodes=np.concatenate([np.asarray(p, dtype=np.int64) for p in case.patches]))
        spec["patch_names"] = list(case.patch_names)
    arrs.update({"out_" + k: out[k] for k in FIELDS if not (k == "g" and case.g is None)})
    np.savez_compressed(path, spec=np.frombuffer(json.dumps(spec).encode(), dtype=np.uint8), **arrs)


def load_case(path):
    z = np.load(path)
    spec = json.loads(bytes(z["spec"]).decode())
    if "mesh_nb" in z.files:
        nb, points = z["mesh_nb"], z["mesh_points"]
        cuts = np.cumsum(z["mesh_patch_count"])[:-1]
        patches = [p.astype(np.uint32) for p in np.split(z["mesh_patch_nodes"], cuts)]
        names = spec["patch_names"]
    else:
        nb, points, patches, names = cases.box_mesh(spec["lattice"], tuple(spec["dims"]), tuple(spec["periodic"]))
    eos = {k: (tuple(v) if isinstance(v, list) else v) for k, v in spec["eos"].items()}
    c = cases.Case(spec["name"], spec["lattice"], tuple(spec["dims"]), tuple(spec["periodic"]), nb, points,
                   patches, names, eos, spec["f"], spec["g"], z["in_rho"], z["in_U"], z["in_T"],
                   meta=dict(rank=spec.get("rank", 0), box="mesh_nb" not in z.files))
    want = {k[4:]: z[k] for k in z.files if k.startswith("out_")}
    return c, spec["steps"], want


def main(names=None):
    """Write the fixtures of `names` (default: every small case)."""
    for name, case in small_cases().items():
        if names and name not in names:
            continue
        runs = [("", STEPS[name])] + ([("long_", LONG_STEPS[name])] if name in LONG_STEPS else [])
        for prefix, steps in runs:
            out = run_checker("ref", case, steps)
            path = os.path.join(HERE, f"{prefix}{name}_{steps}steps.npz")
            save_case(path, case, steps, out)
            print(path, os.path.getsize(path))


if __name__ == "__main__":
    main(sys.argv[1:])
