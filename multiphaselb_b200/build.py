"""Build the CUDA library in-tree with nvcc for sm_100a.

    python -m multiphaselb_b200.build

produces multiphaselb_b200/lib/libmplb_gpu.so.  The strict FP64 path is
compiled with -fmad=false so that no multiply-add is contracted: the
reference's x86-64 build never contracts either, and bit-identical results
depend on it.  Division and square root stay IEEE (nvcc's default
-prec-div=true -prec-sqrt=true).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libmplb_gpu.so")
# (source, multiply-add contraction): the bitwise FP64 path must not contract;
# the FP32-deviation path may.
SOURCES = [(os.path.join(HERE, "csrc", "mplb_gpu.cu"), False),
           (os.path.join(HERE, "csrc", "mplb_noalloc.cu"), False),
           (os.path.join(HERE, "csrc", "mplb_fp32.cu"), True),
           (os.path.join(HERE, "csrc", "mplb_mlp.cu"), False),
           (os.path.join(HERE, "csrc", "mplb_io.cu"), False)]
HEADERS = [os.path.join(HERE, "csrc", f) for f in ("lattice.cuh", "ops.cuh", "fused.cuh", "fused_host.cuh", "fused_tma.cuh", "tma_util.cuh", "umma.cuh", "fused32.cuh", "mplb_io.h")] + \
          [os.path.join(ROOT, "include", "mplb_gpu.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
    "-Xptxas", "-warn-spills",
]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(s) > t for s in [s for s, _ in SOURCES] + HEADERS)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)


def compile_objects(out_dir, verbose=False, extra=()):
    """Compile every translation unit to an object in out_dir (in parallel)."""
    import concurrent.futures as cf
    objs, jobs = [], []
    for src, fmad in SOURCES:
        obj = os.path.join(out_dir, os.path.basename(src) + ".o")
        cmd = [nvcc()] + NVCC_FLAGS + ["-fmad=" + ("true" if fmad else "false")] + list(extra) + \
              ["-I", os.path.join(ROOT, "include"), "-c", "-o", obj, src]
        jobs.append(cmd)
        objs.append(obj)
    with cf.ThreadPoolExecutor(max_workers=len(jobs)) as ex:
        list(ex.map(lambda c: _run(c, verbose), jobs))
    return objs


def build(force=False, verbose=False, extra=()):
    if not force and not needs_build():
        return LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    objs = compile_objects(LIB_DIR, verbose=verbose, extra=extra)
    _run([nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-Xcompiler", "-fPIC", "-o", LIB] + objs,
         verbose)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, extra=[a for a in sys.argv[1:] if a != "--force"])
