"""Parity at the benchmark sizes, against the reference compiled here
(oracle/_ref, its own multifrontal factor and solve through OpenBLAS, run on
all host threads):

* C2, the reference's mesh3d 64^3 (n = 262,144, 35,565 supernodes), FP64, one
  right-hand side b = A x_true;
* C3, the 80^3 lognormal operator (sigma = 2, anisotropy 1:1:100, n = 512,000,
  70,679 supernodes), FP64 and FP32 fronts + FP64 refinement, 8 right-hand
  sides ~ U(-1, 1).

Bars: supernodal structure bit-exact; the FP64 L within 1e-10 relative
Frobenius of the reference's; every solution's scaled residual
||Ax-b||_inf / (||A||_inf ||x||_inf + ||b||_inf) <= 1e-12 and its relative
forward error against the reference's FP64 solution (max-norm) <= 1e-8, the
residual bar of the reference's own test (progs/test_linsolve.c:45).  The
reference takes about a minute at C3; the arrays are compared in chunks so
the host holds the two L arrays and nothing larger.
"""
import os

import numpy as np
import pytest

from tests.helpers import scaled_residual, same_symbolic

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


def _rel_frob_chunked(a, b, chunk=1 << 24):
    num = den = 0.0
    for i in range(0, a.size, chunk):
        d = a[i:i + chunk] - b[i:i + chunk]
        num += float(d @ d)
        den += float(b[i:i + chunk] @ b[i:i + chunk])
    return (num / den) ** 0.5


def _fwd(X, Xr):
    return max(float(np.max(np.abs(X[:, q] - Xr[:, q])) / np.max(np.abs(Xr[:, q]))) for q in range(X.shape[1]))


@pytest.mark.parametrize("which", ["mesh3d_64", "lognormal_80"])
def test_benchmark_system_matches_reference(tb, which):
    from oracle.bindings import Ref, ref_available
    if not ref_available():
        pytest.skip("oracle/_ref/libtaucs_ref.so not built")
    R = Ref()
    R.set_threads(os.cpu_count() or 1)
    if which == "mesh3d_64":
        A = tb.mesh3d(64)
    else:
        A = tb.lognormal(80, 80, 80, 2.0, (1, 1, 100), 0)
    perm, iperm = R.order(*A.arrays(), "amd")
    P = A.permute(perm, iperm)
    n, cp, ri, va = P.arrays()
    rng = np.random.default_rng(0)
    if which == "mesh3d_64":
        B = P.matvec(rng.uniform(-1, 1, n)).reshape(-1, 1)
    else:
        B = rng.uniform(-1, 1, (n, 8))

    Lr = R.factor_mf(n, cp, ri, va)
    assert Lr
    Xr = np.column_stack([R.solve(Lr, np.ascontiguousarray(B[:, q])) for q in range(B.shape[1])])
    sym = R.dump_symbolic(Lr)
    vp_r, v_r = R.dump_values(Lr)
    R.free(Lr)

    F = tb.factor_mf(P)
    assert F is not None, tb.last_error()
    assert same_symbolic(F.export_symbolic(), sym)
    vp_g, v_g = F.export_values()
    assert np.array_equal(vp_g, vp_r)
    err_l = _rel_frob_chunked(v_g, v_r)
    del v_g, v_r
    assert err_l <= 1e-10, err_l

    X = F.solve(B)
    for q in range(B.shape[1]):
        assert scaled_residual(P, X[:, q], B[:, q]) <= 1e-12
    fe64 = _fwd(X, Xr)
    assert fe64 <= 1e-8, fe64
    F.free()

    if which == "lognormal_80":
        G = tb.factor_symbolic(P)
        G.set_precision(1)
        assert G.numeric(P) == 0, tb.last_error()
        Xm, its, _ = G.solve_refine(P, B)
        assert its >= 0, tb.last_error()
        for q in range(B.shape[1]):
            assert scaled_residual(P, Xm[:, q], B[:, q]) <= 1e-12
        fe32 = _fwd(Xm, Xr)
        assert fe32 <= 1e-8, fe32
        G.free()
    print(f"{which}: L rel err {err_l:.2e}, FP64 forward error {fe64:.2e}")
