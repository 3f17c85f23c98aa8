"""Generate tests/golden/writers.npz from the REFERENCE's field writers.

    python -m tests.golden.make_writer_golden

Each entry holds the bytes one reference writer (asciiRaw, binaryRaw or pvtu,
compiled in place into oracle/_ref/libmplb_ref.so) put in its file for the
values of golden_values(n, vsize): a few nodes whose values cover the cases
where "%g" text and the float cast are easy to get wrong.  For pvtu it is the
DataArray block the writer appends.  They pin the library's writers and the
Python restatement where the reference tree is not available.
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from multiphaselb_b200 import abi  # noqa: E402

# key -> (format, field name, nodes, components; 1 = scalar writer)
CASES = {
    "ascii_scalar": (abi.FMT_ASCII_RAW, "rho", 24, 1),
    "ascii_U": (abi.FMT_ASCII_RAW, "U", 8, 3),
    "ascii_f": (abi.FMT_ASCII_RAW, "f", 4, 9),
    "binary_scalar": (abi.FMT_BINARY_RAW, "T", 24, 1),
    "binary_g": (abi.FMT_BINARY_RAW, "g", 3, 15),
    "pvtu_scalar": (abi.FMT_PVTU, "p", 24, 1),
    "pvtu_U": (abi.FMT_PVTU, "U", 8, 3),
}


def golden_values(n, vs):
    """Zeros of both signs, infinities, subnormals, values whose six-digit
    text sits on a rounding tie, the ends of the float range, and lattice-like
    magnitudes; cycled to fill n x vs."""
    base = [0.0, -0.0, 1.0, -1.0, 0.5, 1e-300, -1e300, 5e-324, np.inf, -np.inf, 0.1234565, 1.0000005,
            999999.5, 9999995.0, 1e-5, 1e-4, 123456.5, 2.5e-5, 65504.0, 3.4028235e38, 1e39, 1e-46,
            0.38862114197, 3.1e-3, -2.2e-11, 1.0 / 3.0, 2.0 / 3.0, 0.0441, 7e-8, 1e6, 1e-6, 100000.0]
    a = np.array([base[i % len(base)] * (1.0 if i < len(base) else 1.0 + 1e-3 * (i // len(base)))
                  for i in range(n * vs)])
    return a.reshape(n, vs)


def main():
    from oracle import oracle
    out = {}
    cwd = os.getcwd()
    for key, (fmt, name, n, vs) in CASES.items():
        scalar = vs == 1
        a = golden_values(n, vs)
        field = a[:, 0] if scalar else a
        with tempfile.TemporaryDirectory() as d:
            os.makedirs(os.path.join(d, "processor0", "5"))
            try:
                os.chdir(d)
                oracle.ref_write_field(fmt, name, field, scalar, 0, 5)
            finally:
                os.chdir(cwd)
            fname = "fields.vtu" if fmt == abi.FMT_PVTU else name
            with open(os.path.join(d, "processor0", "5", fname), "rb") as fp:
                out[key] = np.frombuffer(fp.read(), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "writers.npz"), **out)
    print({k: v.size for k, v in out.items()})


if __name__ == "__main__":
    main()
