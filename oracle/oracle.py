"""ctypes access to the two CPU parity checkers.  TEST INFRASTRUCTURE ONLY.

* ``Checker("port")``  -> oracle/liboracle.so, the CPU restatement in
  oracle/mplb_oracle.c (plain C, no reference code).
* ``Checker("ref")``   -> oracle/_ref/libmplb_ref.so, the reference's own
  sources compiled by oracle/Makefile plus oracle/ref_harness.c.

Both expose the same handle API (create / upload / initialize / step / op /
download), keyed on the descriptors of include/mplb_gpu.h, so a test can run
the same case through either and through the GPU library.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  The product path (multiphaselb_b200) never does.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from multiphaselb_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIBS = {"port": os.path.join(HERE, "liboracle.so"),
        "ref": os.path.join(HERE, "_ref", "libmplb_ref.so")}
PREFIX = {"port": "orc_", "ref": "ref_"}

OP_EQUILIBRIUM, OP_COLLISION, OP_LBSTREAM, OP_BOUNDARIES, OP_DENSITY, OP_VELOCITY, \
    OP_TEMPERATURE, OP_INTERFORCE, OP_HEATSOURCE, OP_PRESSURE = range(10)

_loaded = {}


def build(kind="port"):
    """Compile a checker with oracle/Makefile if it is missing."""
    target = "oracle" if kind == "port" else "ref"
    subprocess.run(["make", "-s", "-C", HERE, target], check=True)


def available(kind):
    return os.path.exists(LIBS[kind])


def _lib(kind):
    if kind in _loaded:
        return _loaded[kind]
    if not available(kind):
        build(kind)
    lib = C.CDLL(LIBS[kind])
    p = PREFIX[kind]
    D = C.POINTER(C.c_double)
    fn = lambda n: getattr(lib, p + n)  # noqa: E731
    fn("create").restype = C.c_void_p
    fn("create").argtypes = [C.POINTER(abi.MeshDesc), C.POINTER(abi.EosDesc),
                             C.POINTER(abi.FieldDesc), C.POINTER(abi.FieldDesc), C.c_uint32]
    fn("destroy").argtypes = [C.c_void_p]
    fn("upload").argtypes = [C.c_void_p] + [D] * 8
    fn("download").argtypes = [C.c_void_p] + [D] * 8
    fn("initialize").argtypes = [C.c_void_p]
    fn("step").argtypes = [C.c_void_p, C.c_uint32]
    fn("op").argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_uint32, C.c_uint32]
    fn("set_time").argtypes = [C.c_void_p, C.c_uint32]
    fn("get_time").argtypes = [C.c_void_p]
    fn("get_time").restype = C.c_uint32
    fn("set_rho0").argtypes = [C.c_void_p, C.c_double]
    fn("average_rho0").argtypes = [C.c_void_p]
    fn("average_rho0").restype = C.c_double
    fn("get_p").argtypes = [C.c_void_p, D]
    for name in ("p_eos", "potential"):
        fn(name).argtypes = [C.c_void_p, C.c_double, C.c_double]
        fn(name).restype = C.c_double
    _loaded[kind] = lib
    return lib


class Checker:
    """One lattice held by a CPU checker."""

    def __init__(self, kind, case, start_time=0):
        self.kind, self.case = kind, case
        self.lib = _lib(kind)
        self.p = PREFIX[kind]
        self.desc = abi.Descriptors(case)
        self.h = self._f("create")(C.byref(self.desc.mesh), C.byref(self.desc.eos),
                                   C.byref(self.desc.f), C.byref(self.desc.g), start_time)
        if not self.h:
            raise RuntimeError(f"{kind} checker rejected case {case.name}")

    def _f(self, name):
        return getattr(self.lib, self.p + name)

    def close(self):
        if self.h:
            self._f("destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, rho=None, U=None, T=None, f=None, g=None, S=None, Fi=None, Ft=None):
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64)
                for a in (rho, U, T, f, g, S, Fi, Ft)]
        self._f("upload")(self.h, *[abi.dptr(a) for a in arrs])

    def upload_case(self):
        c = self.case
        self.upload(rho=c.rho, U=c.U, T=c.T)

    def download(self):
        n, Q = self.case.n, self.case.Q
        out = dict(rho=np.zeros(n), U=np.zeros((n, 3)), T=np.zeros(n), Fi=np.zeros((n, 3)),
                   Ft=np.zeros((n, 3)), S=np.zeros(n), f=np.zeros((n, Q)), g=np.zeros((n, Q)))
        self._f("download")(self.h, *[abi.dptr(out[k]) for k in
                                      ("rho", "U", "T", "Fi", "Ft", "S", "f", "g")])
        return out

    def initialize(self):
        self._f("initialize")(self.h)

    def step(self, n=1):
        self._f("step")(self.h, n)

    def op(self, op, field=abi.FIELD_F, start=0, end=None):
        self._f("op")(self.h, op, field, start, self.case.n if end is None else end)

    def set_time(self, t):
        self._f("set_time")(self.h, t)

    def get_time(self):
        return self._f("get_time")(self.h)

    def set_rho0(self, r):
        self._f("set_rho0")(self.h, r)

    def average_rho0(self):
        return self._f("average_rho0")(self.h)

    def pressure(self):
        """macroPressure, then the pressure field."""
        self.op(OP_PRESSURE)
        p = np.zeros(self.case.n)
        self._f("get_p")(self.h, abi.dptr(p))
        return p

    def p_eos(self, rho, T):
        return self._f("p_eos")(self.h, rho, T)

    def potential(self, rho, T):
        return self._f("potential")(self.h, rho, T)
