"""taucs_conjugate_gradients (src/taucs_iter.c:66-223) and its taucs_linsolve
wiring (taucs.solve.cg, src/taucs_linsolve.c:555-567).

Without a preconditioner the routine is host code: it is compared with the
reference's own taucs_conjugate_gradients on the same inputs (same iteration,
same summation order: the iterates agree to 1e-12 relative).  With the
factor's solve as preconditioner (GPU), the linsolve bar of
progs/test_linsolve.c:45 applies: relative 2-norm residual <= 1e-8."""
import ctypes as C

import numpy as np
import pytest

LLT = "taucs.factor.LLT=true"


def _cg_ours(tb, A, b, x0, itermax, tol):
    x = x0.copy()
    rc = tb.lib().taucs_conjugate_gradients(A.ptr, None, None, x, np.ascontiguousarray(b), itermax, tol)
    return rc, x


def _cg_ref(ref, A, b, x0, itermax, tol):
    L = ref.lib
    L.taucs_conjugate_gradients.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                            C.c_double]
    h = ref.wrap(*A.arrays())
    x = x0.copy()
    bb = np.ascontiguousarray(b)
    rc = L.taucs_conjugate_gradients(h, None, None, x.ctypes.data, bb.ctypes.data, itermax, tol)
    L.ref_ccs_unwrap(h)
    return rc, x


@pytest.mark.parametrize("itermax,tol", [(300, 1e-10), (7, 1e-14)])
def test_unpreconditioned_cg_matches_reference(tb, ref, itermax, tol):
    A = tb.mesh2d(12)
    rng = np.random.default_rng(0)
    b = rng.uniform(-1, 1, A.n)
    x0 = np.zeros(A.n)
    rc1, x1 = _cg_ours(tb, A, b, x0, itermax, tol)
    rc2, x2 = _cg_ref(ref, A, b, x0, itermax, tol)
    assert rc1 == 0 and rc2 == 0
    assert np.max(np.abs(x1 - x2)) <= 1e-12 * np.max(np.abs(x2))
    if tol == 1e-10:
        r = b - A.matvec(x1)
        assert np.linalg.norm(r) <= 1e-9 * np.linalg.norm(b)


def test_cg_rejects_non_double(tb):
    A = tb.mesh2d(4)
    A.s.flags = 0
    x = np.zeros(A.n)
    assert tb.lib().taucs_conjugate_gradients(A.ptr, None, None, x, np.ones(A.n), 10, 1e-6) != 0


@pytest.mark.gpu
def test_linsolve_cg_preconditioned_by_the_factor(tb):
    A = tb.mesh3d(20)
    rng = np.random.default_rng(0)
    Xt = rng.random((A.n, 2))
    B = np.asfortranarray(np.column_stack([A.matvec(Xt[:, q]) for q in range(2)]))
    Y = np.zeros((A.n, 2), order="F")
    rc = tb.linsolve(A, None, 2, Y, B, [LLT, "taucs.factor.mf=true", "taucs.solve.cg=true",
                                        "taucs.solve.convergetol=1e-12", "taucs.solve.maxits=20"])
    assert rc == tb.TAUCS_SUCCESS
    for q in range(2):
        assert np.linalg.norm(A.matvec(Y[:, q]) - B[:, q]) <= 1e-8 * np.linalg.norm(B[:, q])
