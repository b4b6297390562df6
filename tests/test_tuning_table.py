"""The GEMM tuning table (host logic, no GPU): measurements saved to a file
and loaded in another table decide the per-level variants of every handle
analysed afterwards, by the shape class of each level's largest product."""
import os

import numpy as np


def _handle(tb):
    A = tb.mesh3d(24)
    perm, iperm = tb.order(A, "amd")
    return tb.factor_symbolic(A.permute(perm, iperm))


def test_tuning_file_round_trip_decides_new_handles(tb, tmp_path):
    lib = tb.lib()
    lib.taucs_b200_tuning_clear()
    F0 = _handle(tb)
    assert not np.any(F0.gemm_choices(0)) and not np.any(F0.gemm_choices(1))
    F0.free()
    # a table that finds variant 1 faster for every shape class and product
    path = os.path.join(tmp_path, "tune.txt")
    with open(path, "w") as fh:
        fh.write("# precision product row_class k_class ms0 n0 ms1 n1\n")
        for prec in (0, 1):
            for kind in (0, 1):
                for r in range(0, 20):
                    for k in range(0, 20):
                        fh.write(f"{prec} {kind} {r} {k} 2.0 1 1.0 1\n")
    assert lib.taucs_b200_tuning_load(path.encode()) == 2 * 2 * 20 * 20
    F = _handle(tb)
    inf = F.info()
    fr, _ = F.layout()
    big_levels = sorted({int(l) for l, f in zip(fr[:, 0], fr[:, 3]) if f > 96})
    assert big_levels
    for prec in (0, 1):
        ch = F.gemm_choices(prec)
        for h in big_levels:
            assert ch[2 * h] == 1, (prec, h)
    out = os.path.join(tmp_path, "saved.txt")
    assert lib.taucs_b200_tuning_save(out.encode()) == 0
    lib.taucs_b200_tuning_clear()
    assert lib.taucs_b200_tuning_entries() == 0
    assert lib.taucs_b200_tuning_load(out.encode()) == 2 * 2 * 20 * 20
    lib.taucs_b200_tuning_clear()
    F.free()
    assert inf.n_levels > 0
