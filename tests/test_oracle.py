"""The oracle, pinned: the plain-C restatement (oracle/taucs_oracle.c) against
the golden fixtures generated from the reference itself, and against the
reference library directly where it is built."""
import glob
import os

import numpy as np
import pytest

from tests.helpers import random_spd_pattern, rel_frob

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def _permuted(g, port):
    import taucs_b200 as tb
    A = tb.Matrix(int(g["n"]), g["colptr"], g["rowind"], g["values"])
    return A.permute(g["perm"], g["iperm"])


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_port_matches_golden(path, port):
    g = np.load(path)
    P = _permuted(g, port)
    n, cp, ri, va = P.arrays()
    assert np.array_equal(port.etree(n, cp, ri), g["parent"])
    h = port.analyze(n, cp, ri)
    s = port.dump_symbolic(h)
    for k in ("sn_size", "sn_up_size", "first_child", "next_child", "struct_ptr", "struct_idx"):
        assert np.array_equal(getattr(s, k), g[k]), k
    assert s.n_sn == int(g["n_sn"])
    assert abs(s.flops() - float(g["flops"])) <= 1e-9 * float(g["flops"])
    assert port.numeric(h, cp, ri, va) == 0
    vp, vv = port.dump_values(h)
    assert np.array_equal(vp, g["val_ptr"])
    if "l_values" in g:
        assert rel_frob(vv, g["l_values"]) <= 1e-12
    assert abs(np.sum(vv * vv) - float(g["l_sumsq"])) <= 1e-10 * float(g["l_sumsq"])
    x = port.solve(h, g["b"])
    assert rel_frob(x, g["x"]) <= 1e-10
    port.free(h)


def test_port_spmv_matches_reference_convention(port):
    g = np.load(GOLDEN[0])
    P = _permuted(g, port)
    y = port.spmv(*P.arrays(), g["x_true"])
    assert rel_frob(y, g["b"]) <= 1e-14


@pytest.mark.parametrize("seed", range(6))
def test_port_matches_reference_random(seed, ref, port):
    A = random_spd_pattern(120 + 40 * seed, 0.03, 100 + seed, forest=seed % 2 == 1)
    perm, iperm = ref.order(*A.arrays(), "amd")
    P = A.permute(perm, iperm)
    n, cp, ri, va = P.arrays()
    L = ref.factor_mf(n, cp, ri, va)
    h = port.analyze(n, cp, ri)
    sr, sp = ref.dump_symbolic(L), port.dump_symbolic(h)
    for k in ("sn_size", "sn_up_size", "first_child", "next_child", "struct_ptr", "struct_idx"):
        assert np.array_equal(getattr(sr, k), getattr(sp, k)), k
    assert port.numeric(h, cp, ri, va) == 0
    assert rel_frob(port.dump_values(h)[1], ref.dump_values(L)[1]) <= 1e-12
    ref.free(L)
    port.free(h)


def test_port_maxdepth(port):
    g = np.load(GOLDEN[0])
    P = _permuted(g, port)
    n, cp, ri, va = P.arrays()
    assert port.analyze(n, cp, ri, 5) is None
    h = port.analyze(n, cp, ri, 10000)
    assert h
    port.free(h)


@pytest.mark.parametrize("args", [(80, 80, 80, 2.0, (1, 1, 100), 0), (7, 5, 3, 1.0, (1, 2, 3), 9),
                                  (30, 20, 0, 1.5, (1, 1, 1), 4), (1, 1, 1, 1.0, (1, 1, 1), 2)])
def test_port_lognormal_generator_is_the_products(args, port):
    """The oracle's own statement of the lognormal operator (used by the
    reference timing arm, which must not load the product library) gives the
    product generator's matrix bit for bit."""
    import taucs_b200 as tb
    A = tb.lognormal(*args)
    n, cp, ri, va = port.lognormal(*args)
    assert n == A.n
    assert np.array_equal(cp, A.colptr) and np.array_equal(ri, A.rowind)
    assert np.array_equal(va, A.values)
