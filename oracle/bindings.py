"""ctypes bindings to the two ORACLE libraries built by oracle/Makefile.

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the taucs_b200 package.

* ``Ref`` wraps ``oracle/_ref/libtaucs_ref.so``: the reference's own sources
  compiled unmodified (AMD ordering, symmetric permutation, multifrontal
  factor/solve through OpenBLAS) plus ``ref_driver.c``, which dumps the
  reference's private factor structure (src/taucs_sn_llt.c:603-623).
* ``Port`` wraps ``oracle/_ref/liboracle.so``: the plain-C restatement in
  ``oracle/taucs_oracle.c`` (no BLAS), pinned against ``Ref``.

Matrices cross the boundary as (n, colptr, rowind, values) numpy arrays in the
reference's lower-triangle CCS convention (src/taucs.h:537-554).
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")

TAUCS_LOWER = 1
TAUCS_SYMMETRIC = 8
TAUCS_DOUBLE = 2048
SPD_FLAGS = TAUCS_DOUBLE | TAUCS_SYMMETRIC | TAUCS_LOWER

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def build(quiet=True):
    """Runs oracle/Makefile (libtaucs_ref.so only where the reference exists)."""
    kw = dict(stdout=subprocess.DEVNULL, stderr=subprocess.STDOUT) if quiet else {}
    subprocess.run(["make", "-C", HERE, "-j8"], check=True, **kw)


def ref_available():
    return os.path.exists(os.path.join(OUT, "libtaucs_ref.so"))


def port_available():
    return os.path.exists(os.path.join(OUT, "liboracle.so"))


class Symbolic:
    """Supernodal structure in the reference's own arrays (n_sn slots)."""

    def __init__(self, n, n_sn, sn_size, sn_up_size, first_child, next_child,
                 struct_ptr, struct_idx):
        self.n = n
        self.n_sn = n_sn
        self.sn_size = sn_size
        self.sn_up_size = sn_up_size
        self.first_child = first_child
        self.next_child = next_child
        self.struct_ptr = struct_ptr
        self.struct_idx = struct_idx

    def sn_struct(self, sn):
        return self.struct_idx[self.struct_ptr[sn]:self.struct_ptr[sn + 1]]

    def flops(self):
        """The reference's relaxed flop count, src/taucs_sn_llt.c:3957-3965."""
        s = self.sn_size.astype(np.float64)
        f = self.sn_up_size.astype(np.float64)

        def sq(x):   # sum of c^2 for c = 1..x
            return x * (x + 1.0) * (2.0 * x + 1.0) / 6.0
        # sum over the s columns of 1 + c^2, c = f, f-1, ..., f-s+1
        return float(np.sum(s + sq(f) - sq(f - s)))


def dense_lower_entries(sym, val_ptr, vals):
    """Maps a panel dump (f x s per supernode, rows in sn_struct order) to a
    dict-free representation: arrays (row, col, value) of the lower factor."""
    rows, cols, vv = [], [], []
    for sn in range(sym.n_sn):
        s = int(sym.sn_size[sn])
        if s == 0:
            continue
        f = int(sym.sn_up_size[sn])
        st = sym.sn_struct(sn)
        panel = vals[val_ptr[sn]:val_ptr[sn] + f * s].reshape(s, f).T  # f x s
        for j in range(s):
            r = st[j:]
            rows.append(r)
            cols.append(np.full(len(r), st[j], dtype=np.int32))
            vv.append(panel[j:, j])
    return np.concatenate(rows), np.concatenate(cols), np.concatenate(vv)


class Ref:
    """The reference library (unmodified sources + dump shim)."""

    def __init__(self, threads=None):
        if threads is not None:
            os.environ["OPENBLAS_NUM_THREADS"] = str(threads)
        self.lib = C.CDLL(os.path.join(OUT, "libtaucs_ref.so"))
        L = self.lib
        L.taucs_ccs_generate_mesh2d.restype = C.c_void_p
        L.taucs_ccs_generate_mesh2d.argtypes = [C.c_int, C.c_char_p]
        L.taucs_ccs_generate_mesh3d.restype = C.c_void_p
        L.taucs_ccs_generate_mesh3d.argtypes = [C.c_int, C.c_int, C.c_int]
        L.taucs_ccs_free.argtypes = [C.c_void_p]
        L.ref_ccs_dims.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.ref_ccs_copy.argtypes = [C.c_void_p, _i32p, _i32p, _f64p]
        L.ref_ccs_wrap.restype = C.c_void_p
        L.ref_ccs_wrap.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _f64p]
        L.ref_ccs_unwrap.argtypes = [C.c_void_p]
        L.ref_order.argtypes = [C.c_void_p, C.c_char_p, _i32p, _i32p]
        L.taucs_ccs_permute_symmetrically.restype = C.c_void_p
        L.taucs_ccs_permute_symmetrically.argtypes = [C.c_void_p, _i32p, _i32p]
        L.ref_etree.argtypes = [C.c_void_p, _i32p]
        for fn in ("taucs_ccs_factor_llt_mf", "taucs_ccs_factor_llt_symbolic"):
            getattr(L, fn).restype = C.c_void_p
            getattr(L, fn).argtypes = [C.c_void_p]
        for fn in ("taucs_ccs_factor_llt_mf_maxdepth", "taucs_ccs_factor_llt_symbolic_maxdepth"):
            getattr(L, fn).restype = C.c_void_p
            getattr(L, fn).argtypes = [C.c_void_p, C.c_int]
        L.taucs_ccs_factor_llt_numeric.argtypes = [C.c_void_p, C.c_void_p]
        L.taucs_supernodal_solve_llt.argtypes = [C.c_void_p, _f64p, _f64p]
        L.taucs_supernodal_factor_free.argtypes = [C.c_void_p]
        L.taucs_supernodal_factor_free_numeric.argtypes = [C.c_void_p]
        L.ref_factor_dims.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.ref_factor_struct_len.restype = C.c_long
        L.ref_factor_struct_len.argtypes = [C.c_void_p]
        L.ref_factor_values_len.restype = C.c_long
        L.ref_factor_values_len.argtypes = [C.c_void_p]
        L.ref_factor_symbolic.argtypes = [C.c_void_p, _i32p, _i32p, _i32p, _i32p, _i64p, _i32p]
        L.ref_factor_values.argtypes = [C.c_void_p, _i64p, _f64p]
        L.taucs_logfile.argtypes = [C.c_char_p]
        L.taucs_ccs_read_binary.restype = C.c_void_p
        L.taucs_ccs_read_binary.argtypes = [C.c_char_p]
        L.taucs_vec_read_binary.restype = C.c_void_p
        L.taucs_vec_read_binary.argtypes = [C.c_int, C.c_int, C.c_char_p]
        L.taucs_vec_write_binary.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_char_p]
        L.ref_free.argtypes = [C.c_void_p]
        try:
            self._set_threads = self.lib.openblas_set_num_threads
        except AttributeError:
            self._set_threads = None

    def set_threads(self, t):
        if self._set_threads is not None:
            self._set_threads(C.c_int(int(t)))

    # ---- matrices
    def _copy_out(self, p):
        n, nnz, fl = C.c_int(), C.c_int(), C.c_int()
        self.lib.ref_ccs_dims(p, C.byref(n), C.byref(nnz), C.byref(fl))
        cp = np.empty(n.value + 1, np.int32)
        ri = np.empty(nnz.value, np.int32)
        va = np.empty(nnz.value, np.float64)
        self.lib.ref_ccs_copy(p, cp, ri, va)
        return n.value, cp, ri, va

    def mesh2d(self, k, which="dirichlet"):
        p = self.lib.taucs_ccs_generate_mesh2d(k, which.encode())
        out = self._copy_out(p)
        self.lib.taucs_ccs_free(p)
        return out

    def mesh3d(self, x, y, z):
        p = self.lib.taucs_ccs_generate_mesh3d(x, y, z)
        out = self._copy_out(p)
        self.lib.taucs_ccs_free(p)
        return out

    def read_binary(self, path):
        """the reference's taucs_ccs_read_binary: (n, colptr, rowind, values, flags)"""
        p = self.lib.taucs_ccs_read_binary(os.fsencode(path))
        n, nnz, fl = C.c_int(), C.c_int(), C.c_int()
        self.lib.ref_ccs_dims(p, C.byref(n), C.byref(nnz), C.byref(fl))
        cp = np.empty(n.value + 1, np.int32)
        ri = np.empty(nnz.value, np.int32)
        va = np.empty(nnz.value, np.float64)
        self.lib.ref_ccs_copy(p, cp, ri, va)
        self.lib.taucs_ccs_free(p)
        return n.value, cp, ri, va, fl.value

    def vec_read_binary(self, n, path):
        p = self.lib.taucs_vec_read_binary(n, 2048, os.fsencode(path))
        v = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_double)), shape=(n,)).copy()
        self.lib.ref_free(p)
        return v

    def vec_write_binary(self, v, path):
        v = np.ascontiguousarray(v, dtype=np.float64)
        return self.lib.taucs_vec_write_binary(v.size, 2048, v.ctypes.data, os.fsencode(path))

    def wrap(self, n, cp, ri, va):
        return self.lib.ref_ccs_wrap(n, SPD_FLAGS, cp, ri, va)

    def order(self, n, cp, ri, va, which="amd"):
        A = self.wrap(n, cp, ri, va)
        perm = np.empty(n, np.int32)
        iperm = np.empty(n, np.int32)
        rc = self.lib.ref_order(A, which.encode(), perm, iperm)
        self.lib.ref_ccs_unwrap(A)
        if rc:
            return None, None
        return perm, iperm

    def permute(self, n, cp, ri, va, perm, iperm):
        A = self.wrap(n, cp, ri, va)
        P = self.lib.taucs_ccs_permute_symmetrically(A, perm, iperm)
        out = self._copy_out(P)
        self.lib.taucs_ccs_free(P)
        self.lib.ref_ccs_unwrap(A)
        return out

    def etree(self, n, cp, ri, va):
        A = self.wrap(n, cp, ri, va)
        par = np.empty(n, np.int32)
        self.lib.ref_etree(A, par)
        self.lib.ref_ccs_unwrap(A)
        return par

    # ---- factor handles (the matrix arrays must outlive the handle's use)
    def factor_mf(self, n, cp, ri, va, max_depth=0):
        A = self.wrap(n, cp, ri, va)
        L = self.lib.taucs_ccs_factor_llt_mf_maxdepth(A, max_depth)
        self.lib.ref_ccs_unwrap(A)
        return L

    def symbolic(self, n, cp, ri, va, max_depth=0):
        A = self.wrap(n, cp, ri, va)
        L = self.lib.taucs_ccs_factor_llt_symbolic_maxdepth(A, max_depth)
        self.lib.ref_ccs_unwrap(A)
        return L

    def numeric(self, L, n, cp, ri, va):
        A = self.wrap(n, cp, ri, va)
        rc = self.lib.taucs_ccs_factor_llt_numeric(A, L)
        self.lib.ref_ccs_unwrap(A)
        return rc

    def free_numeric(self, L):
        self.lib.taucs_supernodal_factor_free_numeric(L)

    def solve(self, L, b):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.empty_like(b)
        rc = self.lib.taucs_supernodal_solve_llt(L, x, b)
        assert rc == 0
        return x

    def free(self, L):
        if L:
            self.lib.taucs_supernodal_factor_free(L)

    def dump_symbolic(self, L):
        n, n_sn = C.c_int(), C.c_int()
        self.lib.ref_factor_dims(L, C.byref(n), C.byref(n_sn))
        n, n_sn = n.value, n_sn.value
        tl = self.lib.ref_factor_struct_len(L)
        ss = np.empty(n_sn, np.int32)
        su = np.empty(n_sn, np.int32)
        fc = np.empty(n_sn + 1, np.int32)
        nc = np.empty(n_sn + 1, np.int32)
        sp = np.empty(n_sn + 1, np.int64)
        si = np.empty(max(tl, 1), np.int32)
        self.lib.ref_factor_symbolic(L, ss, su, fc, nc, sp, si)
        return Symbolic(n, n_sn, ss, su, fc, nc, sp, si[:tl])

    def dump_values(self, L):
        n, n_sn = C.c_int(), C.c_int()
        self.lib.ref_factor_dims(L, C.byref(n), C.byref(n_sn))
        vl = self.lib.ref_factor_values_len(L)
        vp = np.empty(n_sn.value + 1, np.int64)
        vv = np.empty(max(vl, 1), np.float64)
        rc = self.lib.ref_factor_values(L, vp, vv)
        assert rc == 0
        return vp, vv[:vl]


class Port:
    """The plain-C restatement (oracle/taucs_oracle.c)."""

    def __init__(self):
        self.lib = C.CDLL(os.path.join(OUT, "liboracle.so"))
        L = self.lib
        L.orc_etree.argtypes = [C.c_int, _i32p, _i32p, _i32p]
        L.orc_analyze.restype = C.c_void_p
        L.orc_analyze.argtypes = [C.c_int, _i32p, _i32p, C.c_int]
        L.orc_free.argtypes = [C.c_void_p]
        L.orc_dims.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                               C.POINTER(C.c_long), C.POINTER(C.c_long)]
        L.orc_symbolic_copy.argtypes = [C.c_void_p, _i32p, _i32p, _i32p, _i32p, _i64p, _i32p]
        L.orc_numeric.argtypes = [C.c_void_p, _i32p, _i32p, _f64p]
        L.orc_values.argtypes = [C.c_void_p, _i64p, _f64p]
        L.orc_solve.argtypes = [C.c_void_p, _f64p, _f64p]
        L.orc_spmv_sym_lower.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p]
        L.orc_generate_lognormal.restype = C.c_long
        L.orc_generate_lognormal.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                             C.c_double, C.c_ulonglong, _i32p, _i32p, _f64p]

    def etree(self, n, cp, ri):
        par = np.empty(n, np.int32)
        assert self.lib.orc_etree(n, cp, ri, par) == 0
        return par

    def analyze(self, n, cp, ri, max_depth=0):
        return self.lib.orc_analyze(n, cp, ri, max_depth)

    def free(self, h):
        if h:
            self.lib.orc_free(h)

    def dims(self, h):
        n, n_sn, tl, vl = C.c_int(), C.c_int(), C.c_long(), C.c_long()
        self.lib.orc_dims(h, C.byref(n), C.byref(n_sn), C.byref(tl), C.byref(vl))
        return n.value, n_sn.value, tl.value, vl.value

    def dump_symbolic(self, h):
        n, n_sn, tl, _ = self.dims(h)
        ss = np.empty(n_sn, np.int32)
        su = np.empty(n_sn, np.int32)
        fc = np.empty(n_sn + 1, np.int32)
        nc = np.empty(n_sn + 1, np.int32)
        sp = np.empty(n_sn + 1, np.int64)
        si = np.empty(max(tl, 1), np.int32)
        self.lib.orc_symbolic_copy(h, ss, su, fc, nc, sp, si)
        return Symbolic(n, n_sn, ss, su, fc, nc, sp, si[:tl])

    def numeric(self, h, cp, ri, va):
        return self.lib.orc_numeric(h, cp, ri, va)

    def dump_values(self, h):
        _, n_sn, _, vl = self.dims(h)
        vp = np.empty(n_sn + 1, np.int64)
        vv = np.empty(max(vl, 1), np.float64)
        assert self.lib.orc_values(h, vp, vv) == 0
        return vp, vv[:vl]

    def solve(self, h, b):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.empty_like(b)
        assert self.lib.orc_solve(h, x, b) == 0
        return x

    def spmv(self, n, cp, ri, va, x):
        y = np.empty(n, np.float64)
        self.lib.orc_spmv_sym_lower(n, cp, ri, va, np.ascontiguousarray(x, np.float64), y)
        return y

    def lognormal(self, X, Y, Z, sigma, aniso, seed):
        """The benchmarks' lognormal-coefficient operator, stated independently
        of the product library: (n, colptr, rowind, values) of the lower CCS."""
        N = X * Y * max(Z, 1)
        per = 3 if Z == 0 else 4
        cp = np.empty(N + 1, np.int32)
        ri = np.empty(per * N, np.int32)
        va = np.empty(per * N, np.float64)
        nnz = self.lib.orc_generate_lognormal(X, Y, Z, float(sigma), float(aniso[0]), float(aniso[1]),
                                              float(aniso[2]), int(seed), cp, ri, va)
        if nnz < 0:
            raise ValueError("bad grid")
        return N, cp, ri[:nnz].copy(), va[:nnz].copy()
