"""taucs_linsolve, after the reference's progs/test_linsolve.c: the same
mesh3d(20) system, b = A x for four random x, the same option sets and the
same expectations (relative 2-norm residual <= 1e-8, progs/test_linsolve.c:45;
failures where the reference expects them, :83-86, :116-121, :141-148).
The failure cases are decided on the host and run without a GPU."""
import numpy as np
import pytest

LLT = "taucs.factor.LLT=true"


@pytest.fixture(scope="module")
def system(tb):
    A = tb.mesh3d(20)
    rng = np.random.default_rng(0)
    X = np.asfortranarray(rng.random((A.n, 4)))
    B = np.asfortranarray(np.column_stack([A.matvec(X[:, q]) for q in range(4)]))
    return A, X, B


def rnorm(A, y, b):
    return np.linalg.norm(A.matvec(y) - b) / np.linalg.norm(b)


def test_solve_without_factor_fails(tb, system):
    A, _, B = system
    Y = np.zeros((A.n, 1), order="F")
    b = np.asfortranarray(B[:, :1])
    assert tb.linsolve(A, None, 1, Y, b, ["taucs.factor=false"]) != tb.TAUCS_SUCCESS
    F = [None]
    assert tb.linsolve(A, F, 1, Y, b, ["taucs.factor=false"]) != tb.TAUCS_SUCCESS
    assert F[0] is None


def test_colamd_fails_on_spd(tb, system):
    A, _, B = system
    Y = np.zeros((A.n, 1), order="F")
    rc = tb.linsolve(A, None, 1, Y, np.asfortranarray(B[:, :1]), [LLT, "taucs.factor.ordering=colamd"])
    assert rc != tb.TAUCS_SUCCESS


@pytest.mark.parametrize("method", ["taucs.factor.mf=true", "taucs.factor.ll=true"])
def test_low_maxdepth_fails(tb, system, method):
    A, _, B = system
    Y = np.zeros((A.n, 1), order="F")
    rc = tb.linsolve(A, None, 1, Y, np.asfortranarray(B[:, :1]), [LLT, method, "taucs.maxdepth=5"])
    assert rc != tb.TAUCS_SUCCESS


@pytest.mark.gpu
def test_factor_solve_free_sequences(tb, system):
    A, _, B = system
    b = np.asfortranarray(B[:, :1])
    Y = np.zeros((A.n, 1), order="F")
    F = [None]
    # factor, solve, free in one call each
    assert tb.linsolve(A, F, 1, Y, b, [LLT]) == tb.TAUCS_SUCCESS
    assert rnorm(A, Y[:, 0], b[:, 0]) <= 1e-8
    assert tb.linsolve(None, F, 0, None, None, [LLT]) == tb.TAUCS_SUCCESS
    # factor only, then solve with the kept factor, then free
    F = [None]
    Y[:] = 0
    assert tb.linsolve(A, F, 0, None, None, [LLT]) == tb.TAUCS_SUCCESS
    assert F[0] is not None
    assert tb.linsolve(A, F, 1, Y, b, ["taucs.factor=false"]) == tb.TAUCS_SUCCESS
    assert rnorm(A, Y[:, 0], b[:, 0]) <= 1e-8
    assert tb.linsolve(None, F, 0, None, None, [LLT]) == tb.TAUCS_SUCCESS


@pytest.mark.gpu
def test_four_rhs(tb, system):
    A, _, B = system
    Y = np.zeros((A.n, 4), order="F")
    F = [None]
    assert tb.linsolve(A, F, 4, Y, B, [LLT]) == tb.TAUCS_SUCCESS
    for q in range(4):
        assert rnorm(A, Y[:, q], B[:, q]) <= 1e-8
    assert tb.linsolve(None, F, 0, None, None, [LLT]) == tb.TAUCS_SUCCESS


@pytest.mark.gpu
@pytest.mark.parametrize("opts", [[LLT, "taucs.factor.mf=true"], [LLT, "taucs.factor.ll=true"],
                                  [LLT, "taucs.factor.ordering=amd"], [LLT, "taucs.factor.ordering=genmmd"]])
def test_spd_factorizations(tb, system, opts):
    A, X, B = system
    Y = np.zeros((A.n, 1), order="F")
    assert tb.linsolve(A, None, 1, Y, np.asfortranarray(B[:, :1]), opts) == tb.TAUCS_SUCCESS
    assert rnorm(A, Y[:, 0], B[:, 0]) <= 1e-8
    assert np.max(np.abs(Y[:, 0] - X[:, 0])) <= 1e-8 * np.max(np.abs(X[:, 0]))
