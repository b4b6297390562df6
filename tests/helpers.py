"""Shared test helpers: inputs, orderings and comparisons."""
import numpy as np

import taucs_b200 as tb


def amd_permuted(A, ref=None):
    """P A P^T with the AMD order (the reference's when available, else the
    product's own), and the permutation."""
    if ref is not None:
        perm, iperm = ref.order(*A.arrays(), "amd")
    else:
        perm, iperm = tb.order(A, "amd")
        if perm is None:
            perm = np.arange(A.n, dtype=np.int32)
            iperm = perm.copy()
    return A.permute(perm, iperm), perm, iperm


def random_spd_pattern(n, density, seed, forest=False):
    """Random symmetric pattern with a dominant diagonal (SPD), lower CCS,
    rows in each column unsorted and with a few duplicated entries."""
    rng = np.random.default_rng(seed)
    cols, rows, vals = [], [], []
    m = max(1, int(density * n * n / 2))
    i = rng.integers(0, n, m)
    j = rng.integers(0, n, m)
    lo = np.minimum(i, j)
    hi = np.maximum(i, j)
    keep = lo != hi
    if forest:
        keep &= (lo < n // 2) == (hi < n // 2)
    lo, hi = lo[keep], hi[keep]
    v = -rng.uniform(0.1, 1.0, lo.size)
    diag = np.full(n, 1.0)
    np.add.at(diag, lo, -v)
    np.add.at(diag, hi, -v)
    rows = np.concatenate([hi, np.arange(n)])
    cols = np.concatenate([lo, np.arange(n)])
    vals = np.concatenate([v, diag])
    order = rng.permutation(rows.size)
    rows, cols, vals = rows[order], cols[order], vals[order]
    srt = np.argsort(cols, kind="stable")
    rows, cols, vals = rows[srt], cols[srt], vals[srt]
    cp = np.zeros(n + 1, np.int64)
    np.add.at(cp, cols + 1, 1)
    cp = np.cumsum(cp)
    return tb.Matrix(n, cp.astype(np.int32), rows.astype(np.int32), vals)


def scaled_residual(A, x, b):
    r = A.matvec(x) - b
    return float(np.max(np.abs(r)) / (A.inf_norm() * np.max(np.abs(x)) + np.max(np.abs(b))))


def same_symbolic(d, s):
    """d: product export dict; s: oracle Symbolic."""
    return all(np.array_equal(d[k], getattr(s, k)) for k in
               ("sn_size", "sn_up_size", "first_child", "next_child", "struct_ptr", "struct_idx"))


def rel_frob(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))
