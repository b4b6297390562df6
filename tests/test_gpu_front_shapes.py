"""The dense front kernels on awkward shapes, against the reference's FP64
factor.  Each matrix is two dense diagonal blocks (s1 and s2 columns) coupled
to a dense separator of m rows, which is coupled to a dense top block of g
rows, given in that order (no reordering).  The top block keeps the
reference's relaxed amalgamation (src/taucs_sn_llt.c:1715-1725) from merging
the blocks into the separator, so the factor has fronts (s1, m) and (s2, m)
with s and m chosen by the test -- m not a multiple of the 128 / 64 / 16 / 8
tiles, m below 16, K = s with tails, a single diagonal tile -- and a root
front of order m + g.  Every front has order > 96, so the tiled path runs
(k_build, k_potrf_diag, k_trsm, the panel GEMM and the update-matrix GEMM).

* FP64 fronts (DMMA GEMM, both tile shapes): L within 1e-10 relative
  Frobenius of the reference (src/taucs_sn_llt.c:1084-1194).
* FP32 fronts (the tcgen05 GEMMs: split-fed TF32x3 and FP16x3, and the
  producer-split one): the FP32 factor of the scaled matrix D A D
  (D = diag(A)^-1/2) within 1e-4 relative Frobenius of the reference's FP64
  factor of the same scaled matrix, per supernode (an FP32 Cholesky of a
  supernode of s columns is accurate to about s * 2^-24, 3e-5 at s = 513; a
  tile or mask error is O(1)).
"""
import numpy as np
import pytest

from tests.helpers import rel_frob, same_symbolic


SHAPES = [(97, 130, 5), (200, 64, 129), (64, 257, 300), (150, 99, 1), (33, 300, 127), (513, 40, 200),
          (100, 100, 16), (129, 65, 8)]


def blocks_and_separator(tb, s1, s2, m, seed, g=64):
    """Lower CCS of the two blocks, the separator and the top block, every
    block dense, off-diagonal entries -U(0.05, 1), dominant diagonal (SPD)."""
    rng = np.random.default_rng(seed)
    n = s1 + s2 + m + g
    sep = np.arange(s1 + s2, s1 + s2 + m)
    top = np.arange(s1 + s2 + m, n)
    cols, rows = [], []
    for lo, hi in ((0, s1), (s1, s1 + s2)):
        for j in range(lo, hi):
            r = np.concatenate([np.arange(j, hi), sep])
            rows.append(r)
            cols.append(np.full(r.size, j))
    for j in sep:
        r = np.concatenate([np.arange(j, s1 + s2 + m), top])
        rows.append(r)
        cols.append(np.full(r.size, j))
    for j in top:
        r = np.arange(j, n)
        rows.append(r)
        cols.append(np.full(r.size, j))
    rows = np.concatenate(rows)
    cols = np.concatenate(cols)
    vals = -rng.uniform(0.05, 1.0, rows.size)
    off = rows != cols
    d = np.ones(n)
    np.add.at(d, rows[off], -vals[off])
    np.add.at(d, cols[off], -vals[off])
    vals[~off] = d[rows[~off]]
    cp = np.zeros(n + 1, np.int64)
    np.add.at(cp, cols + 1, 1)
    cp = np.cumsum(cp)
    return tb.Matrix(n, cp.astype(np.int32), rows.astype(np.int32), vals)


def test_shapes_give_the_intended_fronts(tb):
    """Host check: the fronts are (s1, m), (s2, m) and (m + g, 0)."""
    for s1, s2, m in SHAPES:
        F = tb.factor_symbolic(blocks_and_separator(tb, s1, s2, m, seed=1))
        assert _fronts(F) == sorted({(s1, m), (s2, m), (m + 64, 0)}), (s1, s2, m)
        F.free()


def _scaled(A):
    n, cp, ri, va = A.arrays()
    col = np.repeat(np.arange(n), np.diff(cp))
    diag = va[ri == col]
    dsc = np.zeros(n)
    dsc[col[ri == col]] = 1.0 / np.sqrt(diag)
    return va * dsc[ri] * dsc[col]


def _per_supernode_err(sym, vp, vg, vr):
    worst = 0.0
    for sn in range(sym.n_sn):
        a, b = vp[sn], vp[sn + 1]
        if b > a:
            worst = max(worst, rel_frob(vg[a:b], vr[a:b]))
    return worst


def _fronts(F):
    fr, _ = F.layout()
    return sorted({(int(s), int(f) - int(s)) for s, f in zip(fr[:, 2], fr[:, 3])})


@pytest.mark.parametrize("shape", SHAPES, ids=[f"{a}_{b}_{c}" for a, b, c in SHAPES])
@pytest.mark.gpu
@pytest.mark.parametrize("variant", [0, 1])
def test_fp64_fronts_match_reference(tb, ref, shape, variant):
    A = blocks_and_separator(tb, *shape, seed=sum(shape))
    n, cp, ri, va = A.arrays()
    F = tb.factor_symbolic(A)
    F.set_gemm_choices(0, [variant] * (2 * F.info().n_levels))
    assert F.numeric(A) == 0, tb.last_error()
    Lr = ref.factor_mf(n, cp, ri, va)
    sym = ref.dump_symbolic(Lr)
    assert same_symbolic(F.export_symbolic(), sym)
    vp_r, v_r = ref.dump_values(Lr)
    vp_g, v_g = F.export_values()
    assert np.array_equal(vp_r, vp_g)
    err = rel_frob(v_g, v_r)
    assert err <= 1e-10, (shape, _fronts(F), err)
    ref.free(Lr)
    F.free()


@pytest.mark.parametrize("shape", SHAPES, ids=[f"{a}_{b}_{c}" for a, b, c in SHAPES])
@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["split_tf32", "split_fp16", "producer_split"])
def test_fp32_fronts_match_reference_scaled(tb, ref, shape, variant):
    A = blocks_and_separator(tb, *shape, seed=sum(shape))
    n, cp, ri, va = A.arrays()
    F = tb.factor_symbolic(A)
    F.set_precision(1)
    tb.lib().taucs_b200_set_split_format(F.h, 1 if variant == "split_fp16" else 0)
    F.set_gemm_choices(1, [1 if variant == "producer_split" else 0] * (2 * F.info().n_levels))
    assert F.numeric(A) == 0, tb.last_error()
    Lr = ref.factor_mf(n, cp, ri, _scaled(A))
    sym = ref.dump_symbolic(Lr)
    vp_r, v_r = ref.dump_values(Lr)
    vp_g, v_g = F.export_values()
    assert np.array_equal(vp_r, vp_g)
    err = _per_supernode_err(sym, vp_r, v_g, v_r)
    assert err <= 1e-4, (shape, _fronts(F), err)
    ref.free(Lr)
    F.free()
