"""Autotuner: the chosen GEMM variants change only which kernel computes a
tile, so the factor's results stay within rounding of the default variants
(solutions: max relative difference <= 1e-12 for FP64 fronts; for FP32 fronts
both refine to a scaled residual <= 1e-12)."""
import numpy as np
import pytest

from tests.helpers import scaled_residual


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [0, 1])
def test_autotune_keeps_results(tb, prec):
    import torch
    A = tb.lognormal(28, 28, 28, 1.0, (1.0, 1.0, 10.0), 3)
    p, ip = tb.order(A, "amd")
    P = A.permute(p, ip)
    b = np.random.default_rng(0).uniform(-1, 1, P.n)
    F = tb.factor_symbolic(P)
    F.set_precision(prec)
    dv = torch.from_numpy(P.values).cuda()
    db = torch.from_numpy(b).cuda()
    dx = torch.empty_like(db)

    def solve():
        assert F.numeric_device(dv.data_ptr()) == 0
        if prec == 0:
            assert F.solve_device(1, dx.data_ptr(), db.data_ptr(), P.n) == 0
        else:
            its, res = F.solve_refine_device(1, dx.data_ptr(), db.data_ptr(), P.n, 1e-12, 10)
            assert its >= 0 and res[0] <= 1e-12
        torch.cuda.synchronize()
        return dx.cpu().numpy().copy()

    x0 = solve()
    ch = F.autotune(dv.data_ptr())
    assert ch.shape == (2 * F.info().n_levels,) and set(np.unique(ch)) <= {0, 1}
    x1 = solve()
    assert scaled_residual(P, x1, b) <= 1e-12
    if prec == 0:
        assert np.max(np.abs(x1 - x0)) <= 1e-12 * np.max(np.abs(x0))
