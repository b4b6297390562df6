"""Fallback of the refinement: preconditioned conjugate gradients on the FP32
factor (after src/taucs_iter.c:66-223) before an FP64 refactorization; and the
leading-dimension contract of the device refinement entry.

Tolerances: scaled residual ||Ax-b||_inf / (||A||_inf ||x||_inf + ||b||_inf)
<= 1e-12 (the refinement target); PCG and FP64-refactor solutions agree to
1e-9 relative; reruns are bit-identical (the dot products are fixed-order
reductions); ld > n gives the same bits as ld = n."""
import ctypes as C

import numpy as np
import pytest

from tests.helpers import scaled_residual

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _factored(tb, A, split_format=None):
    perm, iperm = tb.order(A, "amd")
    P = A.permute(perm, iperm)
    F = tb.factor_symbolic(P)
    F.set_precision(1)
    if split_format is not None:
        assert tb.lib().taucs_b200_set_split_format(F.h, split_format) == 0
    assert F.numeric(P) == 0, tb.last_error()
    return P, F


def test_step_limit_hands_over_to_pcg(tb):
    P, F = _factored(tb, tb.lognormal(20, 19, 18, 1.5, (1, 1, 10), 3))
    B = np.random.default_rng(0).uniform(-1, 1, (P.n, 3))
    # one FP32 step is not enough for 1e-12; the step limit hands over to PCG
    X, its, res = F.solve_refine(P, B, tol=TOL, maxits=1)
    fb, pcg_its = F.refine_report()
    assert its >= 1 and fb == 1 and pcg_its >= 1, (its, fb, pcg_its)
    for q in range(3):
        assert scaled_residual(P, X[:, q], B[:, q]) <= TOL
        assert res[q] <= TOL
    X2, _, _ = F.solve_refine(P, B, tol=TOL, maxits=1)
    assert np.array_equal(X, X2)
    # the same with PCG off: an FP64 refactorization finishes
    F.set_pcg(0)
    X3, its3, _ = F.solve_refine(P, B, tol=TOL, maxits=1)
    assert its3 >= 1 and F.refine_report()[0] == 2
    assert np.max(np.abs(X3 - X)) <= 1e-9 * np.max(np.abs(X3))
    F.free()


def test_converging_refinement_needs_no_fallback(tb):
    P, F = _factored(tb, tb.lognormal(16, 16, 16, 1.0, (1, 1, 1), 4))
    b = np.random.default_rng(1).uniform(-1, 1, P.n)
    x, its, res = F.solve_refine(P, b, tol=TOL, maxits=10)
    assert its >= 1 and F.refine_report() == (0, 0)
    assert scaled_residual(P, x, b) <= TOL
    F.free()


def test_device_refinement_with_padded_leading_dimension(tb):
    """8 columns with ld = n + 37 (the internal residual keeps its own leading
    dimension n) give the same bits as ld = n."""
    import torch
    P, F = _factored(tb, tb.lognormal(14, 13, 12, 1.0, (1, 1, 1), 5))
    n, nrhs, ld = P.n, 8, P.n + 37
    B = np.random.default_rng(2).uniform(-1, 1, (nrhs, n))
    dv = torch.from_numpy(P.values).cuda()
    assert F.numeric_device(dv.data_ptr()) == 0
    out = []
    for lda in (n, ld):
        hb = np.zeros((nrhs, lda))
        hb[:, :n] = B
        db = torch.from_numpy(hb.ravel()).cuda()
        dx = torch.zeros_like(db)
        its, res = F.solve_refine_device(nrhs, dx.data_ptr(), db.data_ptr(), lda, TOL, 10)
        torch.cuda.synchronize()
        assert its >= 1 and np.all(res <= TOL), (its, res)
        out.append(dx.cpu().numpy().reshape(nrhs, lda)[:, :n])
    assert np.array_equal(out[0], out[1])
    for q in range(nrhs):
        assert scaled_residual(P, out[1][q], B[q]) <= TOL
    F.free()


def _shifted_neumann(tb, k, eps):
    """mesh3d(k) with every diagonal set to (1 + eps) x its off-diagonal row
    sum: a Neumann Laplacian shifted to condition number ~ 2 / eps."""
    A = tb.mesh3d(k)
    cp, ri, va = A.colptr, A.rowind, A.values.copy()
    cols = np.repeat(np.arange(A.n), np.diff(cp))
    off = ri != cols
    rs = np.zeros(A.n)
    np.add.at(rs, ri[off], np.abs(va[off]))
    np.add.at(rs, cols[off], np.abs(va[off]))
    diag = np.where(~off)[0]
    va[diag] = rs[cols[diag]] * (1.0 + eps)
    return tb.Matrix(A.n, cp, ri, va)


def test_stalled_refinement_rescued_by_pcg(tb):
    """Condition ~2e8: FP32 refinement stalls; PCG on the same FP32 factor
    reaches the target without an FP64 refactorization.  The stall is
    reproduced with the TF32x3 products (split format 0); with the FP16x3
    default this matrix refines to the target in one step."""
    P, F = _factored(tb, _shifted_neumann(tb, 24, 1e-8), split_format=0)
    b = np.random.default_rng(0).uniform(-1, 1, P.n)
    x, its, res = F.solve_refine(P, b, tol=TOL, maxits=10)
    fb, pcg_its = F.refine_report()
    assert its >= 1 and fb == 1 and 1 <= pcg_its <= 20, (its, fb, pcg_its)
    assert scaled_residual(P, x, b) <= TOL
    F.free()
