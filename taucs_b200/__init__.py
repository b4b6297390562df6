"""taucs_b200 -- B200 (sm_100a) multifrontal supernodal Cholesky behind the
TAUCS C interface.

The product is the C-ABI library ``libtaucs_b200.so`` built in this directory
(``make -C taucs_b200``); its interface is ``include/taucs_b200.h``.  This
module is a thin ctypes mirror of that interface for Python callers, tests and
benchmarks: the function names and return conventions are the reference's
(src/taucs_private.h:16-22, :222-257).  It loads the in-tree library and
fails loudly when it is missing -- there is no Python or CPU fallback.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libtaucs_b200.so")

TAUCS_SUCCESS = 0
TAUCS_ERROR = -1
TAUCS_ERROR_NOMEM = -2
TAUCS_ERROR_BADARGS = -3
TAUCS_ERROR_INDEFINITE = -4
TAUCS_ERROR_MAXDEPTH = -5
TAUCS_LOWER = 1
TAUCS_TRIANGULAR = 4
TAUCS_SYMMETRIC = 8
TAUCS_DOUBLE = 2048
SPD_FLAGS = TAUCS_DOUBLE | TAUCS_SYMMETRIC | TAUCS_LOWER

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


class _Values(C.Union):
    _fields_ = [("v", C.c_void_p), ("d", C.POINTER(C.c_double)), ("s", C.POINTER(C.c_float))]


class CCSStruct(C.Structure):
    """taucs_ccs_matrix, src/taucs.h:537-554."""
    _fields_ = [("n", C.c_int), ("m", C.c_int), ("flags", C.c_int),
                ("colptr", C.POINTER(C.c_int)), ("rowind", C.POINTER(C.c_int)),
                ("values", _Values)]


class Info(C.Structure):
    _fields_ = [("n", C.c_int), ("n_sn", C.c_int), ("n_live", C.c_int), ("n_levels", C.c_int),
                ("struct_len", C.c_long), ("l_values", C.c_long), ("flops", C.c_double),
                ("l_bytes", C.c_double), ("u_bytes", C.c_double), ("ea_bytes", C.c_double),
                ("solve_bytes", C.c_double), ("max_front", C.c_int), ("max_sn_size", C.c_int)]


class ServerInfo(C.Structure):
    _fields_ = [("patterns", C.c_int), ("instances", C.c_int), ("bytes_in_use", C.c_double),
                ("budget_bytes", C.c_double), ("factorizations", C.c_long), ("resident_solves", C.c_long),
                ("evictions", C.c_long), ("waits_for_memory", C.c_long), ("failed", C.c_long), ("queued", C.c_long)]


def build(quiet=True):
    """Compiles libtaucs_b200.so in place for sm_100a."""
    kw = dict(stdout=subprocess.DEVNULL, stderr=subprocess.STDOUT) if quiet else {}
    subprocess.run(["make", "-C", HERE, "-j8"], check=True, **kw)


_lib = None


def lib():
    """The loaded C-ABI library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBPATH):
        raise RuntimeError(f"{LIBPATH} is missing: build it with `make -C {HERE}`")
    L = C.CDLL(LIBPATH)
    vp = C.c_void_p
    pc = C.POINTER(CCSStruct)
    sig = {
        "taucs_ccs_create": (pc, [C.c_int, C.c_int, C.c_int, C.c_int]),
        "taucs_ccs_free": (None, [pc]),
        "taucs_ccs_generate_mesh2d": (pc, [C.c_int, C.c_char_p]),
        "taucs_ccs_generate_mesh3d": (pc, [C.c_int, C.c_int, C.c_int]),
        "taucs_b200_generate_lognormal": (pc, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                               C.c_double, C.c_double, C.c_ulonglong]),
        "taucs_ccs_permute_symmetrically": (pc, [pc, _i32p, _i32p]),
        "taucs_ccs_times_vec": (None, [pc, _f64p, _f64p]),
        "taucs_ccs_order": (None, [pc, C.POINTER(C.POINTER(C.c_int)), C.POINTER(C.POINTER(C.c_int)), C.c_char_p]),
        "taucs_ccs_factor_llt_mf": (vp, [pc]),
        "taucs_ccs_factor_llt_mf_maxdepth": (vp, [pc, C.c_int]),
        "taucs_ccs_factor_llt_symbolic": (vp, [pc]),
        "taucs_ccs_factor_llt_symbolic_maxdepth": (vp, [pc, C.c_int]),
        "taucs_ccs_factor_llt_numeric": (C.c_int, [pc, vp]),
        "taucs_supernodal_solve_llt": (C.c_int, [vp, _f64p, _f64p]),
        "taucs_supernodal_factor_free": (None, [vp]),
        "taucs_supernodal_factor_free_numeric": (None, [vp]),
        "taucs_supernodal_factor_to_ccs": (pc, [vp]),
        "taucs_supernodal_factor_get_diag": (vp, [vp]),
        "taucs_linsolve": (C.c_int, [pc, C.POINTER(vp), C.c_int, vp, vp, C.POINTER(C.c_char_p), C.POINTER(vp)]),
        "taucs_logfile": (None, [C.c_char_p]),
        "taucs_ccs_read_binary": (pc, [C.c_char_p]),
        "taucs_b200_ccs_write_binary": (C.c_int, [pc, C.c_char_p]),
        "taucs_vec_read_binary": (vp, [C.c_int, C.c_int, C.c_char_p]),
        "taucs_vec_write_binary": (C.c_int, [C.c_int, C.c_int, vp, C.c_char_p]),
        "taucs_b200_set_stream": (C.c_int, [vp]),
        "taucs_b200_factor_numeric_device": (C.c_int, [vp, vp]),
        "taucs_b200_factor_numeric_device_async": (C.c_int, [vp, vp]),
        "taucs_b200_factor_status": (C.c_int, [vp]),
        "taucs_b200_solve_device": (C.c_int, [vp, C.c_int, vp, vp, C.c_int]),
        "taucs_b200_solve_device_noalloc": (C.c_int, [vp, C.c_int, vp, vp, C.c_int]),
        "taucs_b200_solve_many": (C.c_int, [vp, C.c_int, _f64p, _f64p]),
        "taucs_b200_set_precision": (C.c_int, [vp, C.c_int]),
        "taucs_b200_solve_refine": (C.c_int, [vp, pc, C.c_int, _f64p, _f64p, C.c_double, C.c_int, _f64p]),
        "taucs_b200_solve_refine_device": (C.c_int, [vp, C.c_int, vp, vp, C.c_int, C.c_double, C.c_int, _f64p]),
        "taucs_b200_set_pcg": (C.c_int, [vp, C.c_int]),
        "taucs_b200_set_refinement": (C.c_int, [vp, C.c_int]),
        "taucs_b200_set_split_format": (C.c_int, [vp, C.c_int]),
        "taucs_conjugate_gradients": (C.c_int, [pc, vp, vp, _f64p, _f64p, C.c_int, C.c_double]),
        "taucs_b200_refine_report": (C.c_int, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "taucs_b200_batch_analyze": (vp, [C.c_int, C.POINTER(pc)]),
        "taucs_b200_batch_values": (C.c_int, [vp, C.POINTER(pc), _f64p]),
        "taucs_b200_batch_rhs": (C.c_int, [vp, C.POINTER(C.c_void_p), _f64p]),
        "taucs_b200_batch_split": (C.c_int, [vp, _f64p, C.POINTER(C.c_void_p)]),
        "taucs_b200_batch_factor": (C.c_int, [vp, C.POINTER(pc)]),
        "taucs_b200_batch_solve": (C.c_int, [vp, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_double,
                                             C.c_int, _f64p]),
        "taucs_b200_batch_info": (C.c_int, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_long)]),
        "taucs_b200_server_create": (vp, [C.c_int, C.c_double]),
        "taucs_b200_server_submit": (C.c_long, [vp, pc, C.c_int, vp, vp, C.c_double]),
        "taucs_b200_server_wait": (C.c_int, [vp, C.c_long, C.POINTER(C.c_double), C.POINTER(C.c_int),
                                             C.POINTER(C.c_double), C.POINTER(C.c_int)]),
        "taucs_b200_server_stats": (C.c_int, [vp, C.POINTER(ServerInfo)]),
        "taucs_b200_server_destroy": (None, [vp]),
        "taucs_b200_factor_info": (C.c_int, [vp, C.POINTER(Info)]),
        "taucs_b200_export_symbolic": (C.c_int, [vp, _i32p, _i32p, _i32p, _i32p, _i64p, _i32p]),
        "taucs_b200_export_values": (C.c_int, [vp, _i64p, _f64p]),
        "taucs_b200_etree": (C.c_int, [pc, _i32p]),
        "taucs_b200_export_layout": (C.c_int, [vp, vp, vp]),
        "taucs_b200_export_rows_maps": (C.c_int, [vp, vp, vp]),
        "taucs_b200_export_persistent": (C.c_int, [vp, vp, vp, vp]),
        "taucs_b200_export_solve_blocks": (C.c_int, [vp, C.c_int, vp, C.POINTER(C.c_int), C.POINTER(C.c_int), vp,
                                                     C.POINTER(C.c_int)]),
        "taucs_b200_launch_count": (C.c_long, [C.c_int]),
        "taucs_b200_autotune": (C.c_int, [vp, vp, _i32p]),
        "taucs_b200_set_gemm_choices": (C.c_int, [vp, C.c_int, C.c_int, _i32p]),
        "taucs_b200_get_gemm_choices": (C.c_int, [vp, C.c_int, _i32p]),
        "taucs_b200_tuning_save": (C.c_int, [C.c_char_p]),
        "taucs_b200_tuning_load": (C.c_int, [C.c_char_p]),
        "taucs_b200_tuning_entries": (C.c_int, []),
        "taucs_b200_tuning_clear": (None, []),
        "taucs_b200_solve_device_noalloc_status": (C.c_int, []),
        "taucs_b200_debug_waits": (C.c_int, [C.c_int, C.c_int]),
        "taucs_b200_allocation_induce_failure": (None, [C.c_int]),
        "taucs_b200_allocation_attempts": (C.c_int, []),
        "taucs_b200_allocation_mark_clean": (None, []),
        "taucs_b200_allocation_live": (C.c_int, [C.POINTER(C.c_double)]),
        "taucs_b200_profile": (C.c_int, [C.c_int]),
        "taucs_b200_profile_read": (C.c_int, [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_long),
                                              C.POINTER(C.c_double), C.POINTER(C.c_double)]),
        "taucs_b200_profile_log": (C.c_long, [vp, vp, C.c_long]),
        "taucs_b200_last_error": (C.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


class Matrix:
    """A taucs_ccs_matrix view over numpy arrays owned by this object."""

    def __init__(self, n, colptr, rowind, values, flags=SPD_FLAGS):
        self.n = int(n)
        self.colptr = np.ascontiguousarray(colptr, dtype=np.int32)
        self.rowind = np.ascontiguousarray(rowind, dtype=np.int32)
        self.values = np.ascontiguousarray(values, dtype=np.float64)
        self.flags = flags
        self.s = CCSStruct()
        self.s.n = self.n
        self.s.m = self.n
        self.s.flags = flags
        self.s.colptr = self.colptr.ctypes.data_as(C.POINTER(C.c_int))
        self.s.rowind = self.rowind.ctypes.data_as(C.POINTER(C.c_int))
        self.s.values.d = self.values.ctypes.data_as(C.POINTER(C.c_double))

    @property
    def ptr(self):
        return C.byref(self.s)

    @property
    def nnz(self):
        return int(self.colptr[-1])

    def arrays(self):
        return self.n, self.colptr, self.rowind, self.values

    @staticmethod
    def _adopt(p):
        """Copies a library-allocated matrix into numpy and frees it."""
        if not p:
            raise RuntimeError("taucs_b200: matrix allocation failed: " + last_error())
        s = p.contents
        n = s.n
        nnz = s.colptr[n]
        cp = np.ctypeslib.as_array(s.colptr, shape=(n + 1,)).copy()
        ri = np.ctypeslib.as_array(s.rowind, shape=(max(nnz, 1),))[:nnz].copy()
        va = np.ctypeslib.as_array(s.values.d, shape=(max(nnz, 1),))[:nnz].copy()
        flags = s.flags
        lib().taucs_ccs_free(p)
        return Matrix(n, cp, ri, va, flags)

    def matvec(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.n, np.float64)
        lib().taucs_ccs_times_vec(self.ptr, x, y)
        return y

    def permute(self, perm, invperm):
        return Matrix._adopt(lib().taucs_ccs_permute_symmetrically(
            self.ptr, np.ascontiguousarray(perm, np.int32), np.ascontiguousarray(invperm, np.int32)))

    def inf_norm(self):
        """||A||_inf of the full symmetric matrix."""
        a = np.abs(self.values)
        rs = np.zeros(self.n)
        cols = np.repeat(np.arange(self.n), np.diff(self.colptr))
        np.add.at(rs, self.rowind, a)
        off = self.rowind != cols
        np.add.at(rs, cols[off], a[off])
        return float(rs.max()) if self.n else 0.0


def last_error():
    return (lib().taucs_b200_last_error() or b"").decode()


def read_binary(path):
    """taucs_ccs_read_binary: a square double-valued matrix file as a Matrix
    (flags as stored in the file)."""
    p = lib().taucs_ccs_read_binary(os.fsencode(path))
    if not p:
        raise RuntimeError("read_binary failed: " + last_error())
    s = p.contents
    if s.m != s.n or not s.flags & TAUCS_DOUBLE:
        lib().taucs_ccs_free(p)
        raise ValueError("read_binary: only square double-valued matrices map to Matrix")
    return Matrix._adopt(p)


def write_binary(A, path):
    """taucs_b200_ccs_write_binary: the reference's binary CCS file format."""
    if lib().taucs_b200_ccs_write_binary(A.ptr, os.fsencode(path)) != 0:
        raise RuntimeError("write_binary failed: " + last_error())


def vec_read_binary(n, path):
    """taucs_vec_read_binary for n doubles."""
    p = lib().taucs_vec_read_binary(int(n), TAUCS_DOUBLE, os.fsencode(path))
    if not p:
        raise RuntimeError("vec_read_binary failed: " + last_error())
    v = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_double)), shape=(max(int(n), 1),))[:int(n)].copy()
    C.CDLL(None).free(C.c_void_p(p))
    return v


def vec_write_binary(v, path):
    """taucs_vec_write_binary for a double vector."""
    v = np.ascontiguousarray(v, dtype=np.float64)
    if lib().taucs_vec_write_binary(v.size, TAUCS_DOUBLE, v.ctypes.data, os.fsencode(path)) != 0:
        raise RuntimeError("vec_write_binary failed: " + last_error())


def mesh2d(k, which="dirichlet"):
    return Matrix._adopt(lib().taucs_ccs_generate_mesh2d(k, which.encode()))


def mesh3d(x, y=None, z=None):
    y = x if y is None else y
    z = x if z is None else z
    return Matrix._adopt(lib().taucs_ccs_generate_mesh3d(x, y, z))


def lognormal(x, y, z, sigma=2.0, aniso=(1.0, 1.0, 100.0), seed=0):
    """Seeded lognormal-coefficient 7-point (z > 0) or 5-point (z == 0) operator."""
    return Matrix._adopt(lib().taucs_b200_generate_lognormal(x, y, z, float(sigma), float(aniso[0]),
                                                             float(aniso[1]), float(aniso[2]), int(seed)))


def order(A, which="amd"):
    """taucs_ccs_order; returns (perm, invperm) or (None, None)."""
    p = C.POINTER(C.c_int)()
    ip = C.POINTER(C.c_int)()
    lib().taucs_ccs_order(A.ptr, C.byref(p), C.byref(ip), which.encode())
    if not p:
        return None, None
    perm = np.ctypeslib.as_array(p, shape=(A.n,)).copy()
    iperm = np.ctypeslib.as_array(ip, shape=(A.n,)).copy()
    libc = C.CDLL(None)
    libc.free(C.cast(p, C.c_void_p))
    libc.free(C.cast(ip, C.c_void_p))
    return perm, iperm


class Factor:
    """Owner of a factor handle (opaque void* whose first member is int flags)."""

    def __init__(self, handle):
        if not handle:
            raise RuntimeError("taucs_b200: factorization failed: " + last_error())
        self.h = C.c_void_p(handle)

    def __del__(self):
        try:
            self.free()
        except Exception:  # interpreter shutdown: the library may already be gone
            pass

    def free(self):
        if getattr(self, "h", None) and self.h.value:
            lib().taucs_supernodal_factor_free(self.h)
            self.h = C.c_void_p(None)

    def numeric(self, A):
        return lib().taucs_ccs_factor_llt_numeric(A.ptr, self.h)

    def numeric_device(self, d_values_ptr):
        return lib().taucs_b200_factor_numeric_device(self.h, C.c_void_p(d_values_ptr))

    def free_numeric(self):
        lib().taucs_supernodal_factor_free_numeric(self.h)

    def solve(self, b):
        b = np.ascontiguousarray(b, dtype=np.float64)
        if b.ndim == 1:
            x = np.empty_like(b)
            rc = lib().taucs_supernodal_solve_llt(self.h, x, b)
        else:
            nrhs = b.shape[1]
            bb = np.ascontiguousarray(b.T)   # column-major n x nrhs
            xx = np.empty_like(bb)
            rc = lib().taucs_b200_solve_many(self.h, nrhs, xx, bb)
            x = xx.T.copy()
        if rc != 0:
            raise RuntimeError("taucs_b200: solve failed: " + last_error())
        return x

    def solve_device(self, nrhs, d_x, d_b, ld):
        return lib().taucs_b200_solve_device(self.h, nrhs, C.c_void_p(d_x), C.c_void_p(d_b), ld)

    def info(self):
        inf = Info()
        lib().taucs_b200_factor_info(self.h, C.byref(inf))
        return inf

    def export_symbolic(self):
        inf = self.info()
        n_sn = inf.n_sn
        ss = np.empty(n_sn, np.int32)
        su = np.empty(n_sn, np.int32)
        fc = np.empty(n_sn + 1, np.int32)
        nc = np.empty(n_sn + 1, np.int32)
        sp = np.empty(n_sn + 1, np.int64)
        si = np.empty(max(inf.struct_len, 1), np.int32)
        lib().taucs_b200_export_symbolic(self.h, ss, su, fc, nc, sp, si)
        return dict(n=inf.n, n_sn=n_sn, sn_size=ss, sn_up_size=su, first_child=fc, next_child=nc,
                    struct_ptr=sp, struct_idx=si[:inf.struct_len])

    def export_values(self):
        inf = self.info()
        vp = np.empty(inf.n_sn + 1, np.int64)
        vv = np.empty(max(inf.l_values, 1), np.float64)
        if lib().taucs_b200_export_values(self.h, vp, vv) != 0:
            raise RuntimeError("export_values failed: " + last_error())
        return vp, vv[:inf.l_values]

    def to_ccs(self):
        return Matrix._adopt(lib().taucs_supernodal_factor_to_ccs(self.h))

    def diag(self):
        p = lib().taucs_supernodal_factor_get_diag(self.h)
        if not p:
            raise RuntimeError("get_diag failed: " + last_error())
        n = self.info().n
        d = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_double)), shape=(n,)).copy()
        C.CDLL(None).free(C.c_void_p(p))
        return d

    def autotune(self, d_values_ptr):
        """Per-level GEMM variants chosen from measured times (see
        taucs_b200_autotune); returns the choices, 2 per level."""
        ch = np.zeros(2 * max(self.info().n_levels, 1), np.int32)
        if lib().taucs_b200_autotune(self.h, C.c_void_p(d_values_ptr), ch) != 0:
            raise RuntimeError("autotune failed: " + last_error())
        return ch

    def set_precision(self, p):
        return lib().taucs_b200_set_precision(self.h, p)

    def gemm_choices(self, precision):
        ch = np.zeros(2 * max(self.info().n_levels, 1), np.int32)
        lib().taucs_b200_get_gemm_choices(self.h, precision, ch)
        return ch

    def set_gemm_choices(self, precision, choices):
        """GEMM variant per level and product (taucs_b200_set_gemm_choices);
        an empty sequence restores the defaults."""
        ch = np.ascontiguousarray(choices, dtype=np.int32)
        if lib().taucs_b200_set_gemm_choices(self.h, precision, ch.size, ch if ch.size else np.zeros(1, np.int32)):
            raise RuntimeError("set_gemm_choices failed: " + last_error())

    def layout(self):
        """(fronts, totals): the plan's per-front device layout as an
        (n_fronts, 14) int64 array and its arena totals
        (taucs_b200_export_layout)."""
        nf = self.info().n_live
        fr = np.zeros((nf, 14), np.int64)
        tot = np.zeros(8, np.int64)
        lib().taucs_b200_export_layout(self.h, fr.ctypes.data, tot.ctypes.data)
        return fr, tot

    def rows_maps(self):
        """(rows, maps): the plan's per-front global row lists and
        child-to-parent maps (offsets in layout() columns 12 and 13)."""
        _, tot = self.layout()
        rows = np.zeros(max(int(tot[6]), 1), np.int32)
        maps = np.zeros(max(int(tot[7]), 1), np.int32)
        lib().taucs_b200_export_rows_maps(self.h, rows.ctypes.data, maps.ctypes.data)
        return rows[:int(tot[6])], maps[:int(tot[7])]

    def solve_blocks(self, h):
        """(fwd, n_diag, bwd): level h's solve block lists, (front, block)
        rows in launch order (taucs_b200_export_solve_blocks)."""
        nf, nd, nb = C.c_int(), C.c_int(), C.c_int()
        lib().taucs_b200_export_solve_blocks(self.h, h, None, C.byref(nf), C.byref(nd), None, C.byref(nb))
        fwd = np.zeros((nf.value, 2), np.int32)
        bwd = np.zeros((nb.value, 2), np.int32)
        lib().taucs_b200_export_solve_blocks(self.h, h, fwd.ctypes.data, C.byref(nf), C.byref(nd), bwd.ctypes.data,
                                             C.byref(nb))
        return fwd, nd.value, bwd

    def set_pcg(self, maxits):
        """PCG iterations allowed when FP32 refinement stalls (0: go straight
        to the FP64 refactorization)."""
        return lib().taucs_b200_set_pcg(self.h, int(maxits))

    def refine_report(self):
        """(fallback, pcg_iterations) of the last refinement: fallback 0 FP32
        steps only, 1 PCG on the FP32 factor, 2 FP64 refactorization."""
        fb, its = C.c_int(), C.c_int()
        lib().taucs_b200_refine_report(self.h, C.byref(fb), C.byref(its))
        return fb.value, its.value

    def solve_refine(self, A, b, tol=1e-12, maxits=10):
        b = np.ascontiguousarray(b, dtype=np.float64)
        one = b.ndim == 1
        bb = b.reshape(-1, 1) if one else b
        nrhs = bb.shape[1]
        bc = np.ascontiguousarray(bb.T)
        xc = np.empty_like(bc)
        res = np.empty(nrhs, np.float64)
        its = lib().taucs_b200_solve_refine(self.h, A.ptr, nrhs, xc, bc, tol, maxits, res)
        x = xc.T.copy()
        return (x[:, 0] if one else x), its, res

    def solve_refine_device(self, nrhs, d_x, d_b, ld, tol=1e-12, maxits=10):
        """Refinement on device vectors (column-major, leading dimension ld);
        returns (steps, final scaled residuals)."""
        nseg = getattr(self, "count", 1)          # batches: one residual per system and column
        res = np.empty(max(nrhs, 1) * nseg, np.float64)
        its = lib().taucs_b200_solve_refine_device(self.h, nrhs, C.c_void_p(d_x), C.c_void_p(d_b), ld, tol,
                                                   maxits, res)
        return its, res[:nrhs * nseg]


def factor_mf(A, max_depth=0):
    """taucs_ccs_factor_llt_mf[_maxdepth]: None on failure (as the reference's NULL)."""
    h = lib().taucs_ccs_factor_llt_mf_maxdepth(A.ptr, max_depth)
    return Factor(h) if h else None


def factor_symbolic(A, max_depth=0):
    h = lib().taucs_ccs_factor_llt_symbolic_maxdepth(A.ptr, max_depth)
    return Factor(h) if h else None


def etree(A):
    par = np.empty(A.n, np.int32)
    lib().taucs_b200_etree(A.ptr, par)
    return par


class Batch(Factor):
    """Many independent SPD systems (unpermuted lower triangles) analysed,
    factored and solved as one (taucs_b200_batch_*).  Inherits the factor
    methods (set_precision, numeric_device, solve_device,
    solve_refine_device) for device-resident use in the combined order."""

    def __init__(self, systems):
        self.systems = list(systems)
        arr = (C.POINTER(CCSStruct) * len(self.systems))(*[C.pointer(A.s) for A in self.systems])
        h = lib().taucs_b200_batch_analyze(len(self.systems), arr)
        if not h:
            raise RuntimeError("batch_analyze failed: " + last_error())
        self.h = C.c_void_p(h)
        cnt, rows, nnz = C.c_int(), C.c_int(), C.c_long()
        lib().taucs_b200_batch_info(self.h, C.byref(cnt), C.byref(rows), C.byref(nnz))
        self.count, self.n, self.nnz = cnt.value, rows.value, nnz.value

    def _ptrs(self, systems):
        return (C.POINTER(CCSStruct) * len(systems))(*[C.pointer(A.s) for A in systems])

    def combined_values(self, systems=None):
        v = np.empty(self.nnz, np.float64)
        if lib().taucs_b200_batch_values(self.h, self._ptrs(systems or self.systems), v) != 0:
            raise RuntimeError(last_error())
        return v

    def combined_rhs(self, bs):
        bs = [np.ascontiguousarray(b, dtype=np.float64) for b in bs]
        v = np.empty(self.n, np.float64)
        lib().taucs_b200_batch_rhs(self.h, (C.c_void_p * len(bs))(*[b.ctypes.data for b in bs]), v)
        return v

    def split(self, combined):
        xs = [np.empty(A.n, np.float64) for A in self.systems]
        lib().taucs_b200_batch_split(self.h, np.ascontiguousarray(combined, dtype=np.float64),
                                     (C.c_void_p * len(xs))(*[x.ctypes.data for x in xs]))
        return xs

    def factor(self, systems=None):
        return lib().taucs_b200_batch_factor(self.h, self._ptrs(systems or self.systems))

    def solve_all(self, bs, tol=1e-12, maxits=10):
        """(steps, [x_s], per-system scaled residuals)"""
        bs = [np.ascontiguousarray(b, dtype=np.float64) for b in bs]
        xs = [np.empty_like(b) for b in bs]
        res = np.empty(len(bs), np.float64)
        steps = lib().taucs_b200_batch_solve(self.h, (C.c_void_p * len(xs))(*[x.ctypes.data for x in xs]),
                                             (C.c_void_p * len(bs))(*[b.ctypes.data for b in bs]), tol, maxits, res)
        return steps, xs, res


class Server:
    """Request server (taucs_b200_server_*): worker threads with their own CUDA
    streams take factor/solve requests from one queue, so requests overlap on
    the GPU; patterns, orderings and factors are cached; device memory held by
    factor instances stays under `budget_bytes`."""

    def __init__(self, workers=8, budget_bytes=64e9):
        self.h = lib().taucs_b200_server_create(int(workers), float(budget_bytes))
        if not self.h:
            raise RuntimeError("server_create failed: " + last_error())
        self._live = {}

    def submit(self, A, B, tol=1e-12):
        """A: unpermuted lower-triangle Matrix; B: (n,) or (n, nrhs).  Returns a
        request id; the solution is returned by wait()."""
        B = np.asarray(B, dtype=np.float64)
        Bc = np.ascontiguousarray((B.reshape(-1, 1) if B.ndim == 1 else B).T)   # nrhs x n = column-major n x nrhs
        Xc = np.empty_like(Bc)
        rid = lib().taucs_b200_server_submit(self.h, A.ptr, Bc.shape[0], Bc.ctypes.data, Xc.ctypes.data, float(tol))
        if rid <= 0:
            raise RuntimeError("server_submit failed")
        self._live[rid] = (A, Bc, Xc, B.ndim == 1)
        return rid

    def wait(self, rid):
        """(status, X, latency_s, refinement steps, worst scaled residual, factored)"""
        lat, st, res, fac = C.c_double(), C.c_int(), C.c_double(), C.c_int()
        rc = lib().taucs_b200_server_wait(self.h, rid, C.byref(lat), C.byref(st), C.byref(res), C.byref(fac))
        A, Bc, Xc, one = self._live.pop(rid)
        X = Xc.T.copy()
        return rc, (X[:, 0] if one else X), lat.value, st.value, res.value, bool(fac.value)

    def stats(self):
        inf = ServerInfo()
        lib().taucs_b200_server_stats(self.h, C.byref(inf))
        return {k: getattr(inf, k) for k, _ in ServerInfo._fields_}

    def close(self):
        if self.h:
            lib().taucs_b200_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def set_stream(stream_handle):
    return lib().taucs_b200_set_stream(C.c_void_p(stream_handle))


def launch_count(reset=False):
    return int(lib().taucs_b200_launch_count(1 if reset else 0))


def logfile(name):
    lib().taucs_logfile(name.encode() if name else None)


def linsolve(A, F, nrhs, X, B, options, opt_arg=None):
    """taucs_linsolve.  F is a one-element list holding the factor handle
    (or None); X and B are column-major n x nrhs float64 arrays (Fortran
    order) or None."""
    opts = (C.c_char_p * (len(options) + 1))(*[o.encode() for o in options], None)
    args = None
    if opt_arg:
        args = (C.c_void_p * (len(opt_arg) + 1))(*opt_arg, None)
    h = C.c_void_p(F[0]) if F and F[0] else C.c_void_p(None)
    xp = X.ctypes.data_as(C.c_void_p) if X is not None else None
    bp = B.ctypes.data_as(C.c_void_p) if B is not None else None
    rc = lib().taucs_linsolve(A.ptr if A is not None else None, C.byref(h), nrhs, xp, bp, opts, args)
    if F is not None:
        F[0] = h.value
    return rc
