"""Host phase of the product, bit-exact against the reference: the AMD
permutation, the symmetric permutation, the elimination tree and the whole
supernodal structure (slots, sizes, sn_struct row order, child lists) --
checked on the golden fixtures and, where the reference library is built,
directly on more patterns.  CPU only."""
import glob
import os

import numpy as np
import pytest

from tests.helpers import random_spd_pattern, same_symbolic

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_symbolic_matches_golden(tb, path):
    g = np.load(path)
    A = tb.Matrix(int(g["n"]), g["colptr"], g["rowind"], g["values"])
    perm, iperm = tb.order(A, "genmmd")
    assert np.array_equal(perm, g["perm_genmmd"]) and np.array_equal(iperm, g["iperm_genmmd"])
    perm, iperm = tb.order(A, "amd")
    assert np.array_equal(perm, g["perm"]) and np.array_equal(iperm, g["iperm"])
    P = A.permute(perm, iperm)
    assert np.array_equal(tb.etree(P), g["parent"])
    F = tb.factor_symbolic(P)
    d = F.export_symbolic()
    assert d["n_sn"] == int(g["n_sn"])
    for k in ("sn_size", "sn_up_size", "first_child", "next_child", "struct_ptr", "struct_idx"):
        assert np.array_equal(d[k], g[k]), k
    inf = F.info()
    assert abs(inf.flops - float(g["flops"])) <= 1e-9 * float(g["flops"])


def _cases(tb):
    out = [
        ("mesh2d_1", tb.mesh2d(1)),
        ("mesh2d_2", tb.mesh2d(2)),
        ("mesh2d_64_aniso_x", tb.mesh2d(64, "anisotropic_x")),
        ("mesh2d_50_aniso_y", tb.mesh2d(50, "anisotropic_y")),
        ("mesh3d_1x1x1", tb.mesh3d(1, 1, 1)),
        ("mesh3d_40x3x2", tb.mesh3d(40, 3, 2)),
        ("mesh3d_17x9x13", tb.mesh3d(17, 9, 13)),
        ("lognormal_3d", tb.lognormal(14, 12, 10, 2.0, (1, 1, 100), 3)),
        ("lognormal_2d", tb.lognormal(40, 35, 0, 1.0, (1, 1, 1), 9)),
    ]
    for s in range(8):
        out.append((f"random_{s}", random_spd_pattern(60 + 53 * s, 0.004 + 0.01 * s, 200 + s, forest=s % 3 == 0)))
    return out


@pytest.mark.parametrize("idx", range(17))
def test_host_phase_matches_reference(tb, ref, idx):
    name, A = _cases(tb)[idx]
    # generators and ordering
    perm_r, iperm_r = ref.order(*A.arrays(), "amd")
    perm, iperm = tb.order(A, "amd")
    assert np.array_equal(perm, perm_r) and np.array_equal(iperm, iperm_r), name
    P = A.permute(perm, iperm)
    pr = ref.permute(*A.arrays(), perm, iperm)
    for a, b in zip(P.arrays()[1:], pr[1:]):
        assert np.array_equal(a, b), name
    assert np.array_equal(tb.etree(P), ref.etree(*P.arrays())), name
    Lr = ref.symbolic(*P.arrays())
    F = tb.factor_symbolic(P)
    assert same_symbolic(F.export_symbolic(), ref.dump_symbolic(Lr)), name
    ref.free(Lr)


@pytest.mark.parametrize("idx", range(17))
def test_genmmd_matches_reference(tb, ref, idx):
    """GENMMD (src/taucs_ccs_order.c:262-442, external/src/genmmd.c) bit for
    bit, and the supernodal structure of the matrix it orders."""
    name, A = _cases(tb)[idx]
    perm_r, iperm_r = ref.order(*A.arrays(), "genmmd")
    perm, iperm = tb.order(A, "genmmd")
    assert np.array_equal(perm, perm_r) and np.array_equal(iperm, iperm_r), name
    P = A.permute(perm, iperm)
    Lr = ref.symbolic(*P.arrays())
    F = tb.factor_symbolic(P)
    assert same_symbolic(F.export_symbolic(), ref.dump_symbolic(Lr)), name
    ref.free(Lr)


@pytest.mark.parametrize("which", ["mesh3d_64", "lognormal_80"])
def test_genmmd_matches_reference_at_benchmark_sizes(tb, ref, which):
    A = tb.mesh3d(64) if which == "mesh3d_64" else tb.lognormal(80, 80, 80, 2.0, (1, 1, 100), 0)
    perm_r, iperm_r = ref.order(*A.arrays(), "genmmd")
    perm, iperm = tb.order(A, "genmmd")
    assert np.array_equal(perm, perm_r) and np.array_equal(iperm, iperm_r)


def test_genmmd_diagonal_and_empty(tb, ref):
    """Every node isolated (diagonal matrix), and a 1x1 matrix."""
    for n in (1, 50):
        A = tb.Matrix(n, np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32), np.ones(n))
        perm_r, _ = ref.order(*A.arrays(), "genmmd")
        perm, _ = tb.order(A, "genmmd")
        assert np.array_equal(perm, perm_r)


@pytest.mark.parametrize("order", ["identity", "random"])
def test_symbolic_other_orders(tb, ref, order):
    A = tb.mesh3d(9, 8, 7)
    perm, iperm = tb.order(A, order)
    assert sorted(perm.tolist()) == list(range(A.n))
    assert np.array_equal(iperm[perm], np.arange(A.n))
    P = A.permute(perm, iperm)
    Lr = ref.symbolic(*P.arrays())
    F = tb.factor_symbolic(P)
    assert same_symbolic(F.export_symbolic(), ref.dump_symbolic(Lr))
    ref.free(Lr)


def test_path_graph_deep_etree(tb, ref):
    """An etree that is one path of length n (recursion depth n in the
    reference's recursive formulation; explicit stacks here)."""
    n = 20000
    cp = np.arange(0, 2 * n, 2, dtype=np.int32)
    cp = np.append(cp, 2 * n - 1).astype(np.int32)
    ri = np.empty(2 * n - 1, np.int32)
    va = np.empty(2 * n - 1)
    for j in range(n):
        ri[cp[j]] = j
        va[cp[j]] = 4.0
        if j < n - 1:
            ri[cp[j] + 1] = j + 1
            va[cp[j] + 1] = -1.0
    A = tb.Matrix(n, cp, ri, va)
    F = tb.factor_symbolic(A)
    Lr = ref.symbolic(*A.arrays())
    assert same_symbolic(F.export_symbolic(), ref.dump_symbolic(Lr))
    ref.free(Lr)


def test_maxdepth_symbolic(tb):
    A = tb.mesh3d(12)
    perm, iperm = tb.order(A, "amd")
    P = A.permute(perm, iperm)
    assert tb.factor_symbolic(P, max_depth=5) is None
    assert tb.factor_symbolic(P, max_depth=0) is not None


def test_unknown_ordering_fails(tb):
    A = tb.mesh2d(5)
    assert tb.order(A, "colamd") == (None, None)


@pytest.mark.parametrize("which", ["mesh3d_64", "lognormal_80"])
def test_host_phase_matches_reference_at_benchmark_sizes(tb, ref, which):
    """The two benchmark systems (64^3 mesh3d, 35,565 live supernodes; 80^3
    lognormal, 70,679): AMD permutation, etree and the whole supernodal
    structure bit-exact against the reference at full size."""
    A = tb.mesh3d(64) if which == "mesh3d_64" else tb.lognormal(80, 80, 80, 2.0, (1, 1, 100), 0)
    perm_r, iperm_r = ref.order(*A.arrays(), "amd")
    perm, iperm = tb.order(A, "amd")
    assert np.array_equal(perm, perm_r) and np.array_equal(iperm, iperm_r)
    P = A.permute(perm, iperm)
    assert np.array_equal(tb.etree(P), ref.etree(*P.arrays()))
    Lr = ref.symbolic(*P.arrays())
    F = tb.factor_symbolic(P)
    sr = ref.dump_symbolic(Lr)
    assert same_symbolic(F.export_symbolic(), sr)
    assert int(np.count_nonzero(sr.sn_size)) == F.info().n_live
    assert abs(F.info().flops - sr.flops()) <= 1e-9 * sr.flops()
    ref.free(Lr)
    F.free()
