"""Induced device-allocation failures, the device-memory counterpart of the
reference's allocation test (progs/xtest_allocations.c:62-87 over
taucs_allocation_induce_failure, src/taucs_malloc.c:127): a factor + solve
sequence is run once to count its device and pinned-host allocations, then
once per allocation with exactly that one made to fail.  Every such run must
report failure (NULL / -1, never a wrong answer with success) and, once its
handle is freed, leave no allocation of the library behind.  FP64 fronts
with a direct solve, and FP32 fronts with FP64 refinement."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _system(tb):
    A = tb.lognormal(14, 13, 12, 1.0, (1.0, 1.0, 10.0), 2)
    perm, iperm = tb.order(A, "amd")
    P = A.permute(perm, iperm)
    b = P.matvec(np.random.default_rng(0).uniform(-1, 1, P.n))
    return P, b


def _run(tb, P, b, precision):
    """True when factor + solve succeeded (and the solution is right)."""
    F = tb.factor_symbolic(P)
    if F is None:
        return False
    try:
        F.set_precision(precision)
        if F.numeric(P) != 0:
            return False
        if precision == 0:
            try:
                x = F.solve(b)
            except RuntimeError:
                return False
        else:
            x, its, _ = F.solve_refine(P, b)
            if its < 0:
                return False
        r = np.max(np.abs(P.matvec(x) - b)) / np.max(np.abs(b))
        assert r < 1e-10, "a run that reported success returned a wrong solution"
        return True
    finally:
        F.free()


@pytest.mark.parametrize("precision", [0, 1])
def test_every_allocation_failure_fails_cleanly(tb, precision):
    P, b = _system(tb)
    lib = tb.lib()
    base = lib.taucs_b200_allocation_live(None)
    lib.taucs_b200_allocation_mark_clean()
    assert _run(tb, P, b, precision)
    attempts = lib.taucs_b200_allocation_attempts()
    assert attempts > 10
    assert lib.taucs_b200_allocation_live(None) == base
    for i in range(attempts):
        lib.taucs_b200_allocation_mark_clean()
        lib.taucs_b200_allocation_induce_failure(i)
        assert not _run(tb, P, b, precision), i
        assert lib.taucs_b200_allocation_live(None) == base, i
    lib.taucs_b200_allocation_mark_clean()
    assert _run(tb, P, b, precision)
