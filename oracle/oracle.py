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


# The reference tree that oracle/Makefile compiles the reference checker from
# (read in place, never copied): MPLB_REFERENCE, else the default location.
REF_ROOT = os.environ.get("MPLB_REFERENCE", "/root/reference")


def ref_tree_present():
    """Whether the reference sources are here to build the reference checkers."""
    return os.path.isdir(os.path.join(REF_ROOT, "src"))


def make(*targets):
    """Run oracle/Makefile for `targets` against REF_ROOT."""
    subprocess.run(["make", "-s", "-C", HERE, f"REF={REF_ROOT}", *targets], check=True)


def build(kind="port"):
    """Compile a checker with oracle/Makefile if it is missing."""
    make("oracle" if kind == "port" else "ref")


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
    fn("set_rank").argtypes = [C.c_void_p, C.c_int32]
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

    def __init__(self, kind, case, start_time=0, rank=None):
        self.kind, self.case = kind, case
        self.lib = _lib(kind)
        self.p = PREFIX[kind]
        self.desc = abi.Descriptors(case)
        self.h = self._f("create")(C.byref(self.desc.mesh), C.byref(self.desc.eos),
                                   C.byref(self.desc.f), C.byref(self.desc.g), start_time)
        if not self.h:
            raise RuntimeError(f"{kind} checker rejected case {case.name}")
        if rank is None:
            rank = (getattr(case, "meta", None) or {}).get("rank", 0)
        self._f("set_rank")(self.h, rank)

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


# ------------------------------------------------------------- field files
class RefRanks:
    """The ranks of a partitioned mesh (multiphaselb_b200.slabs Part objects,
    rank r = pid r) as reference cases with their mpiInfo, stepped together
    by the reference's own exchange code, one thread per rank
    (ref_harness.c::ref_ranks_run)."""

    def __init__(self, parts):
        import numpy as np
        self.lib = lib = _lib("ref")
        lib.ref_set_parallel.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32] + [C.c_void_p] * 4
        lib.ref_set_parallel.restype = C.c_int
        lib.ref_ranks_run.argtypes = [C.POINTER(C.c_void_p), C.c_uint32, C.c_int, C.c_uint32]
        lib.ref_ranks_run.restype = C.c_int
        self.parts = parts
        R = len(parts)
        self.k = [Checker("ref", p.case, rank=p.rank) for p in parts]
        cat = lambda a: np.ascontiguousarray(np.concatenate([np.asarray(x, dtype=np.uint32) for x in a]  # noqa: E731
                                                            + [np.zeros(1, np.uint32)]))
        for k, p in zip(self.k, parts):
            nrg = np.array([len(p.recv[s]) for s in range(R)], dtype=np.uint32)
            nsg = np.array([len(p.send[s]) for s in range(R)], dtype=np.uint32)
            recv, send = cat(p.recv), cat(p.send)
            rc = lib.ref_set_parallel(k.h, p.rank, R, len(p.own), nrg.ctypes.data, recv.ctypes.data,
                                      nsg.ctypes.data, send.ctypes.data)
            if rc != 0:
                raise ValueError(f"rank {p.rank}: ref_set_parallel refused the lists ({rc})")
            k.upload(rho=p.case.rho, U=p.case.U, T=p.case.T)
        self.harr = (C.c_void_p * R)(*[k.h for k in self.k])

    def run(self, init, nsteps=0):
        rc = self.lib.ref_ranks_run(self.harr, len(self.k), int(init), nsteps)
        if rc != 0:
            raise RuntimeError(f"reference ranks failed ({rc}: a message went missing)")

    def initialize(self):
        self.run(True)

    def step(self, n):
        self.run(False, n)

    def owned(self):
        return [(p, {n: v[:len(p.own)] for n, v in k.download().items()}) for p, k in zip(self.parts, self.k)]

    def average_rho0(self):
        """averageScalarField on every rank thread (its MPI_Allreduce across
        them); each rank's rho_0 is set to its result, which is returned."""
        self.lib.ref_ranks_average_rho0.argtypes = [C.POINTER(C.c_void_p), C.c_uint32, C.POINTER(C.c_double)]
        self.lib.ref_ranks_average_rho0.restype = C.c_int
        out = (C.c_double * len(self.k))()
        rc = self.lib.ref_ranks_average_rho0(self.harr, len(self.k), out)
        if rc != 0:
            raise RuntimeError(f"reference ranks failed ({rc})")
        return list(out)


def field_file_bytes(fmt, name, field, scalar):
    """The bytes the reference's writers put in one file, restated in Python.

    asciiRaw: "%g\\n" per node for a scalar (asciiRaw/writeScalarToAsciiRaw.c:36),
    "%g " per component and "\\n" per node for an array
    (asciiRaw/writeArrayToAsciiRaw.c:36-44).  binaryRaw: every value cast to
    float32, node order (binaryRaw/writeScalarToBinaryRaw.c:32-40,
    writeArrayToBinaryRaw.c:36-46).  pvtu: the DataArray block appended to
    fields.vtu (pvtu/writeScalarToPvtu.c:22-31, pvtu/writeArrayToPvtu.c:22-42).
    Python's '%g' is correctly rounded like the C library's, so the text is
    the same.
    """
    a = np.asarray(field, dtype=np.float64)
    if fmt == abi.FMT_BINARY_RAW:
        with np.errstate(over="ignore"):  # out-of-range values become +-inf, as the C cast does here
            return a.astype(np.float32).tobytes()
    rows = a.reshape(-1, 1) if scalar else a.reshape(a.shape[0], -1)
    lead = "          " if fmt == abi.FMT_PVTU else ""
    if scalar:
        body = "".join(f"{lead}{v:g}\n" for v in rows[:, 0].tolist())
    else:
        body = "".join(lead + "".join(f"{v:g} " for v in r) + "\n" for r in rows.tolist())
    if fmt == abi.FMT_PVTU:
        if scalar:
            head = f'        <DataArray type="Float32" Name="{name}" format="ascii">\n'
        else:
            head = f'        <DataArray type="Float32" Name="{name}"  NumberOfComponents="{rows.shape[1]}" format="ascii">\n'
        body = head + body + "        </DataArray>\n"
    return body.encode()


def ref_write_field(fmt, name, field, scalar, pid, time):
    """Run the reference's own writer (oracle/_ref) on ``field``; files go
    under the current folder, as in the reference."""
    lib = _lib("ref")
    lib.ref_write_field.argtypes = [C.c_int, C.c_int, C.c_char_p, C.POINTER(C.c_double), C.c_uint32, C.c_uint32,
                                    C.c_int, C.c_uint32]
    a = np.ascontiguousarray(field, dtype=np.float64)
    n = a.shape[0]
    vs = 1 if scalar else int(a.size // max(n, 1))
    rc = lib.ref_write_field(fmt, 1 if scalar else 0, name.encode(), abi.dptr(a.reshape(-1)), n, vs, pid, time)
    assert rc == 0
