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
SOURCES = [os.path.join(HERE, "csrc", "mplb_gpu.cu"), os.path.join(HERE, "csrc", "mplb_noalloc.cu")]
HEADERS = [os.path.join(HERE, "csrc", f) for f in ("lattice.cuh", "ops.cuh", "fused.cuh")] + \
          [os.path.join(ROOT, "include", "mplb_gpu.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "-fmad=false",
    "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr",
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
    return any(os.path.getmtime(s) > t for s in SOURCES + HEADERS)


def build(force=False, verbose=False, extra=()):
    if not force and not needs_build():
        return LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    cmd = [nvcc()] + NVCC_FLAGS + list(extra) + ["-I", os.path.join(ROOT, "include"), "-o", LIB] + SOURCES
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, extra=[a for a in sys.argv[1:] if a != "--force"])
