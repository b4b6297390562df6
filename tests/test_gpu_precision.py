"""FP32 fronts + FP64 iterative refinement (the mixed-precision path).

Bars: scaled residual ||Ax-b||_inf / (||A||_inf ||x||_inf + ||b||_inf) <= 1e-12
(the stated target), forward error against the FP64 GPU solution, and the
fallbacks: a nonpositive FP32 pivot refactors in FP64; a stalled refinement
finishes with an FP64 factor.
"""
import numpy as np
import pytest

from tests.helpers import scaled_residual

pytestmark = pytest.mark.gpu


def _permuted(tb, A):
    perm, iperm = tb.order(A, "amd")
    return A.permute(perm, iperm)


@pytest.mark.parametrize("case", ["lognormal_sigma2_aniso100", "mesh3d_neumann", "lognormal2d"])
def test_mixed_refines_to_target(tb, case):
    if case == "lognormal_sigma2_aniso100":
        A = tb.lognormal(18, 17, 16, 2.0, (1.0, 1.0, 100.0), 7)
    elif case == "mesh3d_neumann":
        A = tb.mesh3d(16)
    else:
        A = tb.lognormal(90, 80, 0, 1.0, (1, 1, 1), 3)
    P = _permuted(tb, A)
    F = tb.factor_symbolic(P)
    assert F.set_precision(1) == 0
    assert F.numeric(P) == 0, tb.last_error()
    rng = np.random.default_rng(1)
    B = rng.uniform(-1, 1, (P.n, 8))
    X, its, res = F.solve_refine(P, B, tol=1e-12, maxits=10)
    assert its >= 0, (its, res)
    G = tb.factor_mf(P)
    X64 = G.solve(B)
    for q in range(B.shape[1]):
        r = scaled_residual(P, X[:, q], B[:, q])
        assert r <= 1e-12, (case, q, r)
        assert abs(r - res[q]) <= 1e-13 + 0.5 * r
        fe = np.max(np.abs(X[:, q] - X64[:, q])) / np.max(np.abs(X64[:, q]))
        assert fe <= 1e-6, fe


def test_plain_solve_on_mixed_factor_is_refined(tb):
    A = tb.lognormal(14, 13, 12, 1.0, (1, 1, 1), 2)
    P = _permuted(tb, A)
    F = tb.factor_symbolic(P)
    F.set_precision(1)
    assert F.numeric(P) == 0
    b = P.matvec(np.random.default_rng(3).uniform(-1, 1, P.n))
    x = F.solve(b)
    assert scaled_residual(P, x, b) <= 1e-12


def test_fp32_pivot_failure_falls_back_to_fp64(tb):
    # SPD in FP64 (smallest eigenvalue 1e-9) but singular once rounded to FP32
    d = 1e-9
    A = tb.Matrix(2, np.array([0, 2, 3], np.int32), np.array([0, 1, 1], np.int32), np.array([1.0, 1.0 - d, 1.0]))
    F = tb.factor_symbolic(A)
    F.set_precision(1)
    assert F.numeric(A) == 0, tb.last_error()
    b = np.array([1.0, 2.0])
    x = F.solve(b)
    xe = np.linalg.solve(np.array([[1.0, 1.0 - d], [1.0 - d, 1.0]]), b)
    assert np.max(np.abs(x - xe)) / np.max(np.abs(xe)) <= 1e-6


def test_stalled_refinement_finishes_in_fp64(tb):
    A = tb.lognormal(16, 15, 14, 2.0, (1.0, 1.0, 100.0), 9)
    P = _permuted(tb, A)
    F = tb.factor_symbolic(P)
    F.set_precision(1)
    assert F.numeric(P) == 0
    B = np.random.default_rng(4).uniform(-1, 1, (P.n, 2))
    # maxits = 0 and no PCG: after one FP32 step the driver switches to an
    # FP64 factor
    F.set_pcg(0)
    X, its, res = F.solve_refine(P, B, tol=1e-14, maxits=0)
    assert its >= 1
    assert F.refine_report()[0] == 2
    for q in range(2):
        assert scaled_residual(P, X[:, q], B[:, q]) <= 1e-14


def test_fp64_factor_refinement(tb):
    A = tb.mesh3d(15)
    P = _permuted(tb, A)
    F = tb.factor_mf(P)
    b = P.matvec(np.ones(P.n))
    x, its, res = F.solve_refine(P, b, tol=1e-15, maxits=3)
    assert scaled_residual(P, x, b) <= 1e-15 or its == -1


def test_linsolve_mixed_option(tb):
    A = tb.lognormal(12, 12, 12, 1.0, (1.0, 1.0, 10.0), 5)
    n = A.n
    rng = np.random.default_rng(6)
    Xt = rng.uniform(-1, 1, (n, 3))
    B = np.column_stack([A.matvec(Xt[:, q]) for q in range(3)])
    Bf = np.asfortranarray(B)
    Xf = np.asfortranarray(np.zeros_like(B))
    F = [None]
    rc = tb.linsolve(A, F, 3, Xf, Bf, ["taucs.factor.LLT=true", "taucs.factor.mf=true",
                                       "taucs.factor.ordering=amd", "taucs.gpu.precision=mixed"])
    assert rc == 0, tb.last_error()
    for q in range(3):
        assert scaled_residual(A, Xf[:, q], B[:, q]) <= 1e-12
    assert tb.linsolve(None, F, 0, None, None, []) == 0
