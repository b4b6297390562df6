"""The allocation-free device solve (taucs_b200_solve_device_noalloc).

Callers that work inside a fixed, pre-reserved device-memory budget, or may
not call cudaMalloc at all, cannot let the solve allocate its work vectors;
this entry point serves them from a static device array.  Checked through
the C ABI against the regular device solve on the same factor and
right-hand sides, twice in a row (the static array keeps the previous
call's contents, so the second call also checks that whatever must start at
zero is cleared), with the status query after each call, plus the size
limit.  This file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from tests.helpers import scaled_residual

pytestmark = pytest.mark.gpu


def _factor(tb):
    A = tb.lognormal(22, 19, 17, 1.0, (1.0, 1.0, 10.0), 5)
    perm, iperm = tb.order(A, "amd")
    P = A.permute(perm, iperm)
    F = tb.factor_mf(P)
    assert F is not None, tb.last_error()
    return P, F


def test_noalloc_solve_matches_device_solve_twice(tb):
    import torch
    P, F = _factor(tb)
    n, nrhs = P.n, 3
    B = np.random.default_rng(11).uniform(-1.0, 1.0, (nrhs, n))   # row q = column q (ld n)
    dB = torch.from_numpy(B).cuda()
    ref = torch.empty_like(dB)
    out1 = torch.full_like(dB, float("nan"))
    out2 = torch.full_like(dB, float("nan"))
    lib = tb.lib()
    assert F.solve_device(nrhs, ref.data_ptr(), dB.data_ptr(), n) == 0, tb.last_error()
    for out in (out1, out2):
        rc = lib.taucs_b200_solve_device_noalloc(F.h, nrhs, C.c_void_p(out.data_ptr()), C.c_void_p(dB.data_ptr()), n)
        assert rc == 0, tb.last_error()
        assert lib.taucs_b200_solve_device_noalloc_status() == 0, tb.last_error()
    torch.cuda.synchronize()
    xr, x1, x2 = ref.cpu().numpy(), out1.cpu().numpy(), out2.cpu().numpy()
    for x in (x1, x2):
        assert np.all(np.isfinite(x))
        err = np.linalg.norm(x - xr) / np.linalg.norm(xr)
        assert err <= 1e-12, err
    for q in range(nrhs):
        assert scaled_residual(P, x2[q], B[q]) <= 1e-13


def test_noalloc_solve_rejects_factor_over_the_limit(tb):
    # a 3D grid whose solve needs more than 4 Mi doubles of work vectors;
    # the size check happens before any device work
    A = tb.mesh3d(110)
    perm, iperm = tb.order(A, "amd")
    F = tb.factor_symbolic(A.permute(perm, iperm))
    assert F is not None
    x = C.c_void_p(16)
    rc = tb.lib().taucs_b200_solve_device_noalloc(F.h, 1, x, x, A.n)
    assert rc == -1
    msg = tb.last_error()
    assert "static scratch" in msg and "4194304" in msg, msg
