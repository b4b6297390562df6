"""The C-ABI library loads, exports every function include/taucs_b200.h
declares, and its host helpers behave like the reference's (generators,
symmetric permutation, SpMV, vector permutes).  CPU only: no compute call
needs a GPU here."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "taucs_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = set(re.findall(r"\b(taucs_\w+)\s*\(", src))
    return sorted(names)


def test_every_declared_symbol_is_exported(tb):
    lib = C.CDLL(tb.LIBPATH)
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing
    assert len(_declared()) > 40


@pytest.mark.parametrize("args", [(10, "dirichlet"), (7, "neumann"), (9, "anisotropic_x"), (6, "anisotropic_y")])
def test_mesh2d_identical(tb, ref, args):
    a = tb.mesh2d(*args)
    b = ref.mesh2d(*args)
    for x, y in zip(a.arrays(), b):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("dims", [(1, 1, 1), (4, 3, 2), (9, 9, 9)])
def test_mesh3d_identical(tb, ref, dims):
    a = tb.mesh3d(*dims)
    b = ref.mesh3d(*dims)
    for x, y in zip(a.arrays(), b):
        assert np.array_equal(x, y)


def test_permute_and_spmv(tb, ref, port):
    A = tb.mesh3d(6, 5, 4)
    perm, iperm = tb.order(A, "random")
    P = A.permute(perm, iperm)
    pr = ref.permute(*A.arrays(), perm, iperm)
    for x, y in zip(P.arrays(), pr):
        assert np.array_equal(x, y)
    x = np.random.default_rng(1).standard_normal(A.n)
    assert np.allclose(P.matvec(x), port.spmv(*P.arrays(), x), rtol=0, atol=1e-13)


def test_lognormal_generator_properties(tb):
    A = tb.lognormal(7, 6, 5, 2.0, (1, 1, 100), 42)
    B = tb.lognormal(7, 6, 5, 2.0, (1, 1, 100), 42)
    C_ = tb.lognormal(7, 6, 5, 2.0, (1, 1, 100), 43)
    M = tb.mesh3d(7, 6, 5)
    assert np.array_equal(A.values, B.values)              # seeded
    assert not np.array_equal(A.values, C_.values)
    assert np.array_equal(A.rowind, M.rowind) and np.array_equal(A.colptr, M.colptr)
    # strictly diagonally dominant (boundary faces) and symmetric M-matrix
    cols = np.repeat(np.arange(A.n), np.diff(A.colptr))
    off = A.rowind != cols
    assert np.all(A.values[off] < 0)
    rs = np.zeros(A.n)
    np.add.at(rs, A.rowind[off], A.values[off])
    np.add.at(rs, cols[off], A.values[off])
    d = A.values[~off]
    # interior rows sum to zero (up to rounding); boundary rows carry the
    # Dirichlet face conductances and are strictly dominant
    assert np.all(d + rs >= -1e-12 * d)
    x, y, z = np.arange(A.n) % 7, (np.arange(A.n) // 7) % 6, np.arange(A.n) // 42
    bnd = (x == 0) | (x == 6) | (y == 0) | (y == 5) | (z == 0) | (z == 4)
    assert np.all(d[bnd] + rs[bnd] > 1e-6 * d[bnd])
    # anisotropy: z edges are 100x heavier on average (in log space)
    zedge = (A.rowind - cols) == 7 * 6
    xedge = (A.rowind - cols) == 1
    ratio = np.exp(np.mean(np.log(-A.values[zedge])) - np.mean(np.log(-A.values[xedge])))
    assert 30 < ratio < 300


def test_2d_lognormal_pattern(tb):
    A = tb.lognormal(9, 8, 0, 1.0, (1, 1, 1), 1)
    M = tb.mesh2d(9)
    assert A.n == 72 and A.nnz == 72 + 8 * 8 + 9 * 7


def test_symbolic_works_without_gpu(tb):
    A = tb.mesh2d(12)
    perm, iperm = tb.order(A, "amd")
    F = tb.factor_symbolic(A.permute(perm, iperm))
    inf = F.info()
    assert inf.n == 144 and inf.n_live > 0 and inf.flops > 0


def test_vec_permute_roundtrip(tb):
    lib = tb.lib()
    n = 50
    rng = np.random.default_rng(2)
    p = rng.permutation(n).astype(np.int32)
    v = rng.standard_normal(n)
    pv = np.empty(n)
    w = np.empty(n)
    f = C.c_void_p
    lib.taucs_vec_permute.argtypes = [C.c_int, C.c_int, f, f, f]
    lib.taucs_vec_ipermute.argtypes = [C.c_int, C.c_int, f, f, f]
    lib.taucs_vec_permute(n, tb.TAUCS_DOUBLE, v.ctypes.data, pv.ctypes.data, p.ctypes.data)
    assert np.array_equal(pv, v[p])
    lib.taucs_vec_ipermute(n, tb.TAUCS_DOUBLE, pv.ctypes.data, w.ctypes.data, p.ctypes.data)
    assert np.array_equal(w, v)
