"""Failure paths of the bounded device waits, made to run out on purpose
without a fault or a hang: taucs_b200_debug_waits shifts the value every
handshake wait between thread blocks waits for, so no wait can succeed and
each gives up after a short polling limit.  The solve must then report the
timeout (-1 and a message), never a wrong answer with success, and the
device must stay usable: with the controls restored, the same solve gives
the same result as before."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DEFAULT_LIMIT = 1 << 22


def _factor(tb):
    # fronts of order up to ~1000: the big-front solve kernels and their flags
    A = tb.lognormal(24, 24, 24, 1.0, (1.0, 1.0, 10.0), 3)
    perm, iperm = tb.order(A, "amd")
    P = A.permute(perm, iperm)
    F = tb.factor_mf(P)
    assert F is not None, tb.last_error()
    return P, F


def test_solve_timeout_is_reported_and_device_recovers(tb):
    P, F = _factor(tb)
    lib = tb.lib()
    b = P.matvec(np.random.default_rng(0).uniform(-1, 1, P.n))
    x_ok = F.solve(b)
    assert lib.taucs_b200_debug_waits(2000, 1) == 0
    try:
        with pytest.raises(RuntimeError, match="timed out"):
            F.solve(b)
    finally:
        assert lib.taucs_b200_debug_waits(DEFAULT_LIMIT, 0) == 0
    assert np.array_equal(F.solve(b), x_ok)
    F.free()


def test_noalloc_status_reports_timeout(tb):
    import torch
    P, F = _factor(tb)
    lib = tb.lib()
    b = torch.from_numpy(P.matvec(np.ones(P.n))).cuda()
    x = torch.empty_like(b)
    assert lib.taucs_b200_debug_waits(2000, 1) == 0
    try:
        assert lib.taucs_b200_solve_device_noalloc(F.h, 1, C.c_void_p(x.data_ptr()), C.c_void_p(b.data_ptr()),
                                                   P.n) == 0
        assert lib.taucs_b200_solve_device_noalloc_status() == -1
        assert "timed out" in tb.last_error()
    finally:
        assert lib.taucs_b200_debug_waits(DEFAULT_LIMIT, 0) == 0
    assert lib.taucs_b200_solve_device_noalloc(F.h, 1, C.c_void_p(x.data_ptr()), C.c_void_p(b.data_ptr()), P.n) == 0
    assert lib.taucs_b200_solve_device_noalloc_status() == 0
    xr = F.solve(b.cpu().numpy())
    assert np.max(np.abs(x.cpu().numpy() - xr)) <= 1e-12 * np.max(np.abs(xr))
    F.free()
