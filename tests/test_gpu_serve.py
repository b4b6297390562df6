"""Request server: every result is the same alone and in a mix of concurrent
requests, meets the requested scaled residual, and the caches and the
device-memory admission behave as documented.

Tolerances: scaled residual ||Ax-b||_inf / (||A||_inf ||x||_inf + ||b||_inf)
<= 1e-12 (the refinement target); mix vs alone: max |x_mix - x_alone| /
max |x_alone| <= 1e-13 (each request runs the same deterministic kernels on
its own stream, so the results are expected to agree to the last bit)."""
import numpy as np
import pytest

from tests.helpers import scaled_residual

TOL = 1e-12
MIX_TOL = 1e-13


def _requests(tb):
    """A small serving mix: 2D and 3D lognormal systems, a pattern seen again
    with new coefficients, and a matrix seen again with new right-hand sides."""
    rng = np.random.default_rng(7)
    mats = {
        "2d_a": tb.lognormal(24, 24, 0, 1.0, (1, 1, 1), 1),
        "2d_b": tb.lognormal(45, 31, 0, 1.0, (1, 1, 1), 2),
        "3d_a": tb.lognormal(9, 9, 9, 1.0, (1, 1, 1), 3),
        "3d_b": tb.lognormal(14, 14, 14, 1.0, (1, 1, 1), 4),
        "2d_a_newvals": tb.lognormal(24, 24, 0, 1.0, (1, 1, 1), 11),
        "3d_b_newvals": tb.lognormal(14, 14, 14, 1.0, (1, 1, 1), 12),
    }
    order = ["2d_a", "3d_b", "2d_b", "3d_a", "2d_a_newvals", "3d_b", "2d_a", "3d_b_newvals", "2d_b", "3d_a"]
    reqs = []
    for name in order:
        A = mats[name]
        nrhs = int(rng.integers(1, 5))
        reqs.append((name, A, rng.uniform(-1, 1, (A.n, nrhs))))
    return reqs


def _run(tb, reqs, workers, concurrent, budget=16e9):
    S = tb.Server(workers=workers, budget_bytes=budget)
    out = []
    if concurrent:
        ids = [S.submit(A, B, TOL) for _, A, B in reqs]
        out = [S.wait(i) for i in ids]
    else:
        for _, A, B in reqs:
            out.append(S.wait(S.submit(A, B, TOL)))
    st = S.stats()
    S.close()
    return out, st


@pytest.mark.gpu
def test_mix_equals_alone(tb):
    reqs = _requests(tb)
    alone, st_alone = _run(tb, reqs, workers=1, concurrent=False)
    mixed, st_mix = _run(tb, reqs, workers=4, concurrent=True)
    for (name, A, B), a, m in zip(reqs, alone, mixed):
        assert a[0] == 0 and m[0] == 0, name
        for q in range(B.shape[1]):
            assert scaled_residual(A, a[1][:, q], B[:, q]) <= TOL, name
            assert scaled_residual(A, m[1][:, q], B[:, q]) <= TOL, name
        assert np.max(np.abs(m[1] - a[1])) <= MIX_TOL * np.max(np.abs(a[1])), name
    assert st_alone["failed"] == 0 and st_mix["failed"] == 0
    # four patterns; the repeated matrices were solved on resident factors
    assert st_alone["patterns"] == 4 and st_mix["patterns"] == 4
    assert st_alone["resident_solves"] >= 3
    assert st_alone["factorizations"] + st_alone["resident_solves"] == len(reqs)


@pytest.mark.gpu
def test_resident_factor_skips_numeric(tb):
    A = tb.lognormal(30, 30, 0, 1.0, (1, 1, 1), 5)
    rng = np.random.default_rng(1)
    S = tb.Server(workers=2, budget_bytes=8e9)
    r1 = S.wait(S.submit(A, rng.uniform(-1, 1, A.n)))
    r2 = S.wait(S.submit(A, rng.uniform(-1, 1, (A.n, 3))))
    st = S.stats()
    S.close()
    assert r1[0] == 0 and r1[5] is True
    assert r2[0] == 0 and r2[5] is False
    assert st["resident_solves"] == 1 and st["factorizations"] == 1


@pytest.mark.gpu
def test_memory_budget_evicts_and_waits(tb):
    """A budget that holds about one instance of the largest pattern forces
    evictions (and waits while instances are busy); results stay correct."""
    reqs = _requests(tb)
    big = tb.lognormal(14, 14, 14, 1.0, (1, 1, 1), 4)
    probe = tb.Server(workers=1, budget_bytes=64e9)
    probe.wait(probe.submit(big, np.ones(big.n)))
    one = probe.stats()["bytes_in_use"]
    probe.close()
    out, st = _run(tb, reqs, workers=3, concurrent=True, budget=1.6 * one)
    for (name, A, B), r in zip(reqs, out):
        assert r[0] == 0, name
        for q in range(B.shape[1]):
            assert scaled_residual(A, r[1][:, q], B[:, q]) <= TOL, name
    assert st["evictions"] > 0
    assert st["bytes_in_use"] <= 1.6 * one


@pytest.mark.gpu
def test_oversized_request_fails_cleanly(tb):
    A = tb.lognormal(12, 12, 12, 1.0, (1, 1, 1), 6)
    S = tb.Server(workers=1, budget_bytes=1e5)
    r = S.wait(S.submit(A, np.ones(A.n)))
    assert r[0] == -1
    assert S.stats()["failed"] == 1
    S.close()
