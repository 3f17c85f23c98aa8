"""multiphaselb_b200 -- B200 (sm_100a) lattice update for multiphaseLB.

The product is the C-ABI library ``lib/libmplb_gpu.so`` (include/mplb_gpu.h).
This module is a thin ctypes mirror of it for Python callers, tests and the
benchmark.  ``Lattice`` mirrors the reference's operator sequence: the same
operator names as src/lbEquation/general (collision, lbstream,
update_boundaries, macro_density, macro_velocity, macro_temperature,
inter_force, heat_source, equilibrium) plus the solver-level calls
initialize / step / download.  ``Batch`` advances many such lattices
together (one launch per step for all of them).

There is no CPU fallback: if the library is missing or no CUDA device is
present, constructing a Lattice raises.
"""
import ctypes as C
import os

import numpy as np

from . import abi
from .abi import FIELD_F, FIELD_G, PATH_AUTO, PATH_FUSED, PATH_OPERATORS  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libmplb_gpu.so")

_lib = None


class MplbError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"mplb error {code}: {msg}")
        self.code = code


def load_library(path=LIB_PATH):
    """Load the C-ABI library and declare its signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python -m multiphaselb_b200.build`")
    lib = C.CDLL(path)
    H = C.c_void_p
    D = C.POINTER(C.c_double)
    sig = {
        "mplb_gpu_version": ([], C.c_char_p),
        "mplb_gpu_last_error": ([], C.c_char_p),
        "mplb_gpu_create": ([C.POINTER(abi.MeshDesc), C.POINTER(abi.EosDesc), C.POINTER(abi.FieldDesc),
                             C.POINTER(abi.FieldDesc), C.POINTER(abi.Opts), C.POINTER(H)], C.c_int),
        "mplb_gpu_destroy": ([H], C.c_int),
        "mplb_gpu_info": ([H, C.POINTER(abi.Info)], C.c_int),
        "mplb_gpu_upload": ([H] + [D] * 8, C.c_int),
        "mplb_gpu_download": ([H] + [D] * 8, C.c_int),
        "mplb_gpu_initialize": ([H], C.c_int),
        "mplb_gpu_step": ([H, C.c_uint32], C.c_int),
        "mplb_gpu_equilibrium": ([H, C.c_int32], C.c_int),
        "mplb_gpu_collision": ([H, C.c_int32], C.c_int),
        "mplb_gpu_lbstream": ([H, C.c_int32], C.c_int),
        "mplb_gpu_update_boundaries": ([H, C.c_int32], C.c_int),
        "mplb_gpu_macro_density": ([H, C.c_uint32, C.c_uint32], C.c_int),
        "mplb_gpu_macro_velocity": ([H, C.c_uint32, C.c_uint32], C.c_int),
        "mplb_gpu_macro_temperature": ([H, C.c_uint32, C.c_uint32], C.c_int),
        "mplb_gpu_inter_force": ([H], C.c_int),
        "mplb_gpu_heat_source": ([H], C.c_int),
        "mplb_gpu_macro_pressure": ([H], C.c_int),
        "mplb_gpu_download_pressure": ([H, D], C.c_int),
        "mplb_gpu_set_time": ([H, C.c_uint32], C.c_int),
        "mplb_gpu_set_rho0": ([H, C.c_double], C.c_int),
        "mplb_gpu_average_rho0": ([H, D], C.c_int),
        "mplb_gpu_mass_energy": ([H, D, D], C.c_int),
        "mplb_gpu_sync": ([H], C.c_int),
        "mplb_gpu_copy_nodes": ([H, C.c_uint32, H, C.c_uint32, C.c_uint32, C.c_int32], C.c_int),
        "mplb_gpu_copy_state": ([H, C.c_uint32, H, C.c_uint32, C.c_uint32], C.c_int),
        "mplb_gpu_set_owned": ([H, C.c_uint32, C.c_uint32], C.c_int),
        "mplb_gpu_add_mirror": ([H, C.c_uint32, C.c_uint32, H, C.c_uint32], C.c_int),
        "mplb_gpu_clear_mirrors": ([H], C.c_int),
        "mplb_ranks_initialize": ([C.POINTER(H), C.c_uint32, C.POINTER(abi.GhostRun), C.c_uint32], C.c_int),
        "mplb_ranks_step": ([C.POINTER(H), C.c_uint32, C.POINTER(abi.GhostRun), C.c_uint32, C.c_uint32], C.c_int),
        "mplb_gpu_snapshot": ([H, C.c_int32], C.c_int),
        "mplb_gpu_snapshot_wait": ([H, D, D, D, D], C.c_int),
        "mplb_gpu_snapshot_write": ([H, C.c_char_p, C.c_int32, C.c_int32], C.c_int),
        "mplb_gpu_snapshot_join": ([H], C.c_int),
        "mplb_write_scalar_field": ([C.c_char_p, C.c_int32, C.c_uint32, C.c_int32, C.c_char_p, D, C.c_uint64],
                                    C.c_int),
        "mplb_write_vector_field": ([C.c_char_p, C.c_int32, C.c_uint32, C.c_int32, C.c_char_p, D, C.c_uint64,
                                     C.c_uint32], C.c_int),
        "mplb_gpu_monitor": ([H, C.c_int32, D, D], C.c_int),
        "mplb_gpu_run_to_equilibrium": ([H, C.c_uint32, C.c_uint32, C.c_double, C.POINTER(C.c_uint32), D],
                                        C.c_int),
        "mplb_batch_create": ([C.POINTER(H), C.c_uint32, C.POINTER(abi.BatchOpts), C.POINTER(H)], C.c_int),
        "mplb_batch_destroy": ([H], C.c_int),
        "mplb_batch_info_get": ([H, C.POINTER(abi.BatchInfo)], C.c_int),
        "mplb_batch_step": ([H, C.c_uint32], C.c_int),
        "mplb_batch_run": ([H, C.c_uint32, C.POINTER(C.c_uint32), D, C.POINTER(C.c_uint32)], C.c_int),
        "mplb_batch_filter": ([H, C.POINTER(C.c_uint32), C.c_uint32, C.c_uint32], C.c_int),
        "mplb_batch_average": ([H, C.POINTER(C.c_uint32)], C.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def version():
    return load_library().mplb_gpu_version().decode()


def _format(fmt):
    return abi.FORMATS[fmt] if isinstance(fmt, str) else int(fmt)


def write_field(name, field, time, root="", pid=0, fmt="asciiRaw", scalar=None):
    """Write one field file in the reference's format (mplb_write_scalar_field
    / mplb_write_vector_field; host code, no GPU needed).  ``field`` is [n]
    (scalar) or [n][vsize]; ``scalar`` defaults to ``field.ndim == 1``."""
    lib = load_library()
    a = np.ascontiguousarray(field, dtype=np.float64)
    if scalar is None:
        scalar = a.ndim == 1
    root = os.fsencode(root)
    if scalar:
        rc = lib.mplb_write_scalar_field(root, pid, time, _format(fmt), name.encode(), abi.dptr(a.reshape(-1)),
                                         a.size)
    else:
        a2 = a.reshape(a.shape[0], -1) if a.ndim > 1 else a.reshape(-1, 1)
        rc = lib.mplb_write_vector_field(root, pid, time, _format(fmt), name.encode(), abi.dptr(a2.reshape(-1)),
                                         a2.shape[0], a2.shape[1])
    if rc != 0:
        raise MplbError(rc, lib.mplb_gpu_last_error().decode())


class Lattice:
    """One device-resident lattice (a C-ABI handle).

    ``case`` is a :class:`multiphaselb_b200.cases.Case` (or any object with
    the same attributes: lattice, n, nb, points, patches, eos, f, g).
    """

    def __init__(self, case, path=PATH_AUTO, device=-1, stream=None, start_time=0, tile_config=0,
                 precision=abi.FP64, rank=None):
        self.lib = load_library()
        self.case = case
        self.n, self.Q = case.n, case.Q
        self._desc = abi.Descriptors(case)
        if rank is None:
            rank = (getattr(case, "meta", None) or {}).get("rank", 0)
        opts = abi.Opts(precision, path, device, stream, start_time, tile_config, rank)
        h = C.c_void_p()
        self._check(self.lib.mplb_gpu_create(C.byref(self._desc.mesh), C.byref(self._desc.eos),
                                              C.byref(self._desc.f), C.byref(self._desc.g),
                                              C.byref(opts), C.byref(h)))
        self.h = h

    # ---------------------------------------------------------------- plumbing
    def _check(self, rc):
        if rc != 0:
            raise MplbError(rc, self.lib.mplb_gpu_last_error().decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.mplb_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def info(self):
        i = abi.Info()
        self._check(self.lib.mplb_gpu_info(self.h, C.byref(i)))
        return dict(path=i.path, box_dims=tuple(i.box_dims), box_periodic=tuple(i.box_periodic),
                    bc_sequential=i.bc_sequential, current_time=i.current_time,
                    device_bytes=i.device_bytes, kernel_launches=i.kernel_launches,
                    tile_config=i.tile_config, tile_ms=list(i.tile_ms))

    # -------------------------------------------------------------- host data
    def upload(self, rho=None, U=None, T=None, f=None, g=None, S=None, Fi=None, Ft=None):
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64)
                for a in (rho, U, T, f, g, S, Fi, Ft)]
        self._check(self.lib.mplb_gpu_upload(self.h, *[abi.dptr(a) for a in arrs]))

    def upload_case(self):
        c = self.case
        self.upload(rho=c.rho, U=c.U, T=c.T)

    def download(self, out=None):
        n, Q = self.n, self.Q
        if out is None:
            out = dict(rho=np.zeros(n), U=np.zeros((n, 3)), T=np.zeros(n), Fi=np.zeros((n, 3)),
                       Ft=np.zeros((n, 3)), S=np.zeros(n), f=np.zeros((n, Q)), g=np.zeros((n, Q)))
        self._check(self.lib.mplb_gpu_download(self.h, *[abi.dptr(out.get(k)) for k in
                                                          ("rho", "U", "T", "Fi", "Ft", "S", "f", "g")]))
        return out

    # ------------------------------------------------------------ solver level
    def initialize(self):
        self._check(self.lib.mplb_gpu_initialize(self.h))

    def step(self, n=1):
        self._check(self.lib.mplb_gpu_step(self.h, n))

    def sync(self):
        self._check(self.lib.mplb_gpu_sync(self.h))

    # ------------------------------------------------- reference operator names
    def equilibrium(self, field=FIELD_F):
        self._check(self.lib.mplb_gpu_equilibrium(self.h, field))

    def collision(self, field=FIELD_F):
        self._check(self.lib.mplb_gpu_collision(self.h, field))

    def lbstream(self, field=FIELD_F):
        self._check(self.lib.mplb_gpu_lbstream(self.h, field))

    def update_boundaries(self, field=FIELD_F):
        self._check(self.lib.mplb_gpu_update_boundaries(self.h, field))

    def macro_density(self, start=0, end=None):
        self._check(self.lib.mplb_gpu_macro_density(self.h, start, self.n if end is None else end))

    def macro_velocity(self, start=0, end=None):
        self._check(self.lib.mplb_gpu_macro_velocity(self.h, start, self.n if end is None else end))

    def macro_temperature(self, start=0, end=None):
        self._check(self.lib.mplb_gpu_macro_temperature(self.h, start, self.n if end is None else end))

    def inter_force(self):
        self._check(self.lib.mplb_gpu_inter_force(self.h))

    def heat_source(self):
        self._check(self.lib.mplb_gpu_heat_source(self.h))

    def macro_pressure(self):
        """macroPressure on the device; returns the pressure field."""
        self._check(self.lib.mplb_gpu_macro_pressure(self.h))
        p = np.zeros(self.n)
        self._check(self.lib.mplb_gpu_download_pressure(self.h, abi.dptr(p)))
        return p

    def set_time(self, t):
        self._check(self.lib.mplb_gpu_set_time(self.h, t))

    def copy_nodes(self, src, dst_start, src_start, count, fields=("f",)):
        """Copy nodes [src_start, src_start + count) of the Lattice `src` into
        nodes [dst_start, ...) of this one, device to device (peer to peer
        between GPUs), for the fields named as in download(); queued after
        both handles' earlier work, without blocking the host."""
        mask = 0
        for name in fields:
            mask |= abi.NODES[name]
        self._check(self.lib.mplb_gpu_copy_nodes(self.h, dst_start, src.h, src_start, count, mask))

    def copy_state(self, src, dst_start, src_start, count):
        """Copy the fused-path state (post-collision populations, T and U of the
        last step) of nodes [src_start, src_start + count) of `src` into nodes
        [dst_start, ...) of this Lattice, device to device: the halo exchange
        of slabs run on the fused path."""
        self._check(self.lib.mplb_gpu_copy_state(self.h, dst_start, src.h, src_start, count))

    def set_owned(self, start, count):
        """Fused steps store the outputs of nodes [start, start + count) only
        (the rest is the halo its neighbours write)."""
        self._check(self.lib.mplb_gpu_set_owned(self.h, start, count))

    def add_mirror(self, src_start, count, dst, dst_start):
        """Fused steps also store the outputs of owned nodes [src_start, ...)
        into nodes [dst_start, ...) of `dst`'s next-step input (its halo)."""
        self._check(self.lib.mplb_gpu_add_mirror(self.h, src_start, count, dst.h, dst_start))

    def clear_mirrors(self):
        self._check(self.lib.mplb_gpu_clear_mirrors(self.h))

    def set_rho0(self, r):
        self._check(self.lib.mplb_gpu_set_rho0(self.h, r))

    def average_rho0(self):
        r = C.c_double()
        self._check(self.lib.mplb_gpu_average_rho0(self.h, C.byref(r)))
        return r.value

    def monitor(self, reset=False):
        """(max |drho| since the previous call, total mass), from the current populations."""
        d, m = C.c_double(), C.c_double()
        self._check(self.lib.mplb_gpu_monitor(self.h, 1 if reset else 0, C.byref(d), C.byref(m)))
        return d.value, m.value

    def run_to_equilibrium(self, max_steps, check_interval=1000, tol=1e-9):
        """Step until max |drho/dt| < tol (whole check intervals); returns (steps, rate)."""
        st = C.c_uint32()
        r = C.c_double()
        self._check(self.lib.mplb_gpu_run_to_equilibrium(self.h, max_steps, check_interval, tol, C.byref(st),
                                                         C.byref(r)))
        return st.value, r.value

    def snapshot(self, pressure=False, pdfs=False):
        """Queue a write-step copy of rho, U, T (and p; and f, g with pdfs)
        and its transfer to the host; stepping may continue before
        snapshot_wait / snapshot_write."""
        flags = (abi.SNAP_PRESSURE if pressure else 0) | (abi.SNAP_PDFS if pdfs else 0)
        self._check(self.lib.mplb_gpu_snapshot(self.h, flags))
        self._snap_p = pressure

    def snapshot_write(self, root="", pid=0, fmt="asciiRaw"):
        """Write the last snapshot's fields (rho, T, p, U, f, g as taken) to
        <root>/processor<pid>/<time>/ on a host thread; returns at once."""
        self._check(self.lib.mplb_gpu_snapshot_write(self.h, os.fsencode(root), pid, _format(fmt)))

    def snapshot_join(self):
        """Wait for the snapshot writer; raises the first error of its writes."""
        self._check(self.lib.mplb_gpu_snapshot_join(self.h))

    def snapshot_wait(self):
        n = self.n
        out = dict(rho=np.zeros(n), U=np.zeros((n, 3)), T=np.zeros(n))
        if getattr(self, "_snap_p", False):
            out["p"] = np.zeros(n)
        self._check(self.lib.mplb_gpu_snapshot_wait(self.h, abi.dptr(out["rho"]), abi.dptr(out["U"]),
                                                    abi.dptr(out["T"]), abi.dptr(out.get("p"))))
        return out

    def mass_energy(self):
        m, e = C.c_double(), C.c_double()
        self._check(self.lib.mplb_gpu_mass_energy(self.h, C.byref(m), C.byref(e)))
        return m.value, e.value


class Batch:
    """Many independent lattices advanced together (mplb_batch_*).

    ``lattices`` are :class:`Lattice` objects (D2Q9, FP32-deviation, fused,
    fully periodic, isothermal); they stay usable between batch calls and
    must outlive the batch.
    """

    def __init__(self, lattices, check_interval=1000, tol=1e-9, tile_config=0):
        self.lib = load_library()
        self.lattices = list(lattices)
        arr = (C.c_void_p * len(self.lattices))(*[lat.h.value for lat in self.lattices])
        opts = abi.BatchOpts(tile_config, check_interval, tol)
        h = C.c_void_p()
        self._check(self.lib.mplb_batch_create(arr, len(self.lattices), C.byref(opts), C.byref(h)))
        self.h = h

    def _check(self, rc):
        if rc != 0:
            raise MplbError(rc, self.lib.mplb_gpu_last_error().decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.mplb_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def info(self):
        i = abi.BatchInfo()
        self._check(self.lib.mplb_batch_info_get(self.h, C.byref(i)))
        nc = i.n_candidates
        return dict(n_lattices=i.n_lattices, nodes=i.nodes, tile_config=i.tile_config,
                    tiles=[(i.tile_x[c], i.tile_y[c]) for c in range(nc)],
                    tile_ms=list(i.tile_ms)[:nc], grid=i.grid, kernel_launches=i.kernel_launches,
                    graph_launches=i.graph_launches)

    def step(self, n=1):
        self._check(self.lib.mplb_batch_step(self.h, n))

    def run(self, max_steps):
        """Run to convergence; returns (steps per lattice, last max |drho/dt|, converged count)."""
        m = len(self.lattices)
        steps = np.zeros(m, dtype=np.uint32)
        rate = np.zeros(m)
        conv = C.c_uint32()
        self._check(self.lib.mplb_batch_run(self.h, max_steps, abi.uptr(steps), abi.dptr(rate), C.byref(conv)))
        return steps, rate, conv.value

    def filter(self, window, first=0, every=0):
        """Time-averaging filter: lattice i's state replaced by its mean over
        its last window[i] steps (0: not filtered), in run() once `first`
        steps are done and `every` steps after each window (every = 0: only
        through average()).  window=None turns the filter off."""
        if window is None:
            self._check(self.lib.mplb_batch_filter(self.h, None, 0, 0))
            return
        w = np.ascontiguousarray(window, dtype=np.uint32)
        if w.shape != (len(self.lattices),):
            raise ValueError("one window per lattice")
        self._check(self.lib.mplb_batch_filter(self.h, abi.uptr(w), first, every))

    def average(self):
        """One filter window on every lattice now; returns its length in steps."""
        s = C.c_uint32()
        self._check(self.lib.mplb_batch_average(self.h, C.byref(s)))
        return s.value
