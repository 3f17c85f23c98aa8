"""ctypes mirror of include/mplb_gpu.h.

The C header is the contract; these Structure classes must match it field
for field.  tests/test_abi.py checks the sizes against the compiled library.
"""
import ctypes as C

MAX_Q = 15
MAX_PATCHES = 64

D2Q9, D3Q15 = 0, 1
LIMRT, MYMRT, XUMRT, LITEMPMRT, NO_MODEL = 0, 1, 2, 3, -1
EOS_IDEAL, EOS_CS, EOS_PR, EOS_VDW = 0, 1, 2, 3
(BC_BOUNCEBACK, BC_FIXEDT, BC_FIXEDRANDOMT, BC_FIXEDGRADT, BC_FIXEDU, BC_UHF,
 BC_FIXEDEOSP, BC_OUTFLOW, BC_PERIODIC) = range(9)
FIELD_F, FIELD_G = 0, 1
FP64, FP32_DEV = 0, 1
PATH_AUTO, PATH_OPERATORS, PATH_FUSED = 0, 1, 2

OK, E_ARG, E_UNSUPPORTED, E_CUDA, E_STATE, E_NONFINITE, E_IO, E_TIMEOUT = 0, -1, -2, -3, -4, -5, -6, -7
FMT_ASCII_RAW, FMT_BINARY_RAW, FMT_PVTU, FMT_ENSIGHT = 0, 1, 2, 3
FORMATS = {"asciiRaw": FMT_ASCII_RAW, "binaryRaw": FMT_BINARY_RAW, "pvtu": FMT_PVTU, "ensight": FMT_ENSIGHT}
SNAP_PRESSURE, SNAP_PDFS = 1, 2
BATCH_MAX_WINDOW = 1048576  # MPLB_BATCH_MAX_WINDOW
# mplb_gpu_copy_nodes field bits, by the field names of download()
NODES = {"rho": 1, "U": 2, "T": 4, "Fi": 8, "Ft": 16, "S": 32, "f": 64, "g": 128}

Q_OF = {D2Q9: 9, D3Q15: 15}


class MeshDesc(C.Structure):
    _fields_ = [
        ("lattice", C.c_int32),
        ("n_points", C.c_uint32),
        ("nb", C.POINTER(C.c_int32)),
        ("points", C.POINTER(C.c_int32)),
        ("n_patches", C.c_uint32),
        ("patch_count", C.POINTER(C.c_uint32)),
        ("patch_nodes", C.POINTER(C.c_uint32)),
    ]


class EosDesc(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("a", C.c_double), ("b", C.c_double), ("w", C.c_double),
        ("R", C.c_double), ("G", C.c_double), ("M", C.c_double), ("Cv", C.c_double),
        ("g", C.c_double * 3),
        ("fext", C.c_double * 3),
        ("rho_0", C.c_double),
    ]


class FieldDesc(C.Structure):
    _fields_ = [
        ("model", C.c_int32),
        ("update", C.c_int32),
        ("Lambda", C.c_double * MAX_Q),
        ("sigma", C.c_double),
        ("surface_tension", C.c_int32),
        ("kappa_st", C.c_double),
        ("bc_type", C.POINTER(C.c_int32)),
        ("bc_value", C.POINTER(C.c_double)),
        ("alpha_1", C.c_double),
        ("alpha_2", C.c_double),
    ]


class Opts(C.Structure):
    _fields_ = [
        ("precision", C.c_int32),
        ("path", C.c_int32),
        ("device", C.c_int32),
        ("stream", C.c_void_p),
        ("start_time", C.c_uint32),
        ("tile_config", C.c_int32),
        ("rank", C.c_int32),
    ]


class Info(C.Structure):
    _fields_ = [
        ("path", C.c_int32),
        ("box_dims", C.c_int32 * 3),
        ("box_periodic", C.c_int32 * 3),
        ("bc_sequential", C.c_int32),
        ("current_time", C.c_uint32),
        ("device_bytes", C.c_uint64),
        ("kernel_launches", C.c_uint64),
        ("tile_config", C.c_int32),
        ("tile_ms", C.c_float * 16),
    ]


class BatchOpts(C.Structure):
    _fields_ = [
        ("tile_config", C.c_int32),
        ("check_interval", C.c_uint32),
        ("tol", C.c_double),
    ]


class GhostRun(C.Structure):
    """mplb_ghost_run: nodes [src_start, +count) of handle src fill nodes
    [dst_start, +count) of handle dst."""
    _fields_ = [
        ("dst", C.c_uint32),
        ("dst_start", C.c_uint32),
        ("src", C.c_uint32),
        ("src_start", C.c_uint32),
        ("count", C.c_uint32),
    ]


class BatchInfo(C.Structure):
    _fields_ = [
        ("n_lattices", C.c_uint32),
        ("nodes", C.c_uint64),
        ("tile_config", C.c_int32),
        ("n_candidates", C.c_int32),
        ("tile_x", C.c_int32 * 8),
        ("tile_y", C.c_int32 * 8),
        ("tile_ms", C.c_float * 8),
        ("grid", C.c_int32),
        ("kernel_launches", C.c_uint64),
        ("graph_launches", C.c_uint64),
    ]


def dptr(a):
    """double* of a contiguous float64 numpy array, or NULL for None."""
    if a is None:
        return None
    assert a.dtype.name == "float64" and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_double))


def iptr(a):
    if a is None:
        return None
    assert a.dtype.name == "int32" and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def uptr(a):
    if a is None:
        return None
    assert a.dtype.name == "uint32" and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


class Descriptors:
    """Owns the numpy buffers behind a (mesh, eos, f, g) descriptor set so the
    pointers stay valid while a library handle is being created."""

    def __init__(self, case):
        import numpy as np
        self.case = case
        self.nb = np.ascontiguousarray(case.nb, dtype=np.int32)
        self.points = np.ascontiguousarray(case.points, dtype=np.int32)
        self.patch_count = np.ascontiguousarray([len(p) for p in case.patches], dtype=np.uint32)
        if case.patches:
            self.patch_nodes = np.ascontiguousarray(np.concatenate(
                [np.asarray(p, dtype=np.uint32) for p in case.patches]), dtype=np.uint32)
        else:
            self.patch_nodes = np.zeros(1, dtype=np.uint32)
        self.mesh = MeshDesc(case.lattice, case.n, iptr(self.nb), iptr(self.points),
                             len(case.patches), uptr(self.patch_count), uptr(self.patch_nodes))
        e = case.eos
        self.eos = EosDesc(e["type"], e.get("a", 0.0), e.get("b", 0.0), e.get("w", 0.0),
                           e.get("R", 1.0), e.get("G", -1.0), e.get("M", 1.0), e.get("Cv", 1.0),
                           (C.c_double * 3)(*e.get("g", (0.0, 0.0, 0.0))),
                           (C.c_double * 3)(*e.get("fext", (0.0, 0.0, 0.0))),
                           e.get("rho_0", 0.0))
        self._keep = []
        self.f = self._field(case.f, len(case.patches))
        self.g = self._field(case.g, len(case.patches))

    def _field(self, fd, npatch):
        import numpy as np
        if fd is None:
            d = FieldDesc()
            d.model = NO_MODEL
            return d
        lam = list(fd["Lambda"]) + [0.0] * (MAX_Q - len(fd["Lambda"]))
        bct = np.ascontiguousarray(fd.get("bc_type", [BC_PERIODIC] * npatch), dtype=np.int32)
        bcv = np.ascontiguousarray(fd.get("bc_value", np.zeros((npatch, 3))), dtype=np.float64).reshape(-1)
        if bct.size == 0:
            bct = np.zeros(1, dtype=np.int32)
            bcv = np.zeros(3, dtype=np.float64)
        self._keep += [bct, bcv]
        return FieldDesc(fd["model"], int(fd.get("update", 1)), (C.c_double * MAX_Q)(*lam),
                         fd.get("sigma", 0.0), int(fd.get("surface_tension", 0)), fd.get("kappa_st", 0.0),
                         iptr(bct), dptr(bcv), fd.get("alpha_1", 0.0), fd.get("alpha_2", 0.0))
