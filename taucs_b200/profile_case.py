"""Fixed workloads for kernel profiling (ncu launch lists and single-launch
captures): each runs one piece of the solver's work on cuda:0 and prints what
a capture command needs to know.

    python -m taucs_b200.profile_case factor-refine G   one FP32-front numeric factorization of the
                                                       G^3 lognormal system and its refinement
                                                       (8 right-hand sides): one bench step
    python -m taucs_b200.profile_case update-gemm G     two FP32-front factorizations of the G^3
                                                       system (the first unprofiled); prints the
                                                       launch index, among the tcgen05 GEMM
                                                       launches of the process, of the second
                                                       one's largest update-matrix product (for
                                                       ncu -k/-s)
    python -m taucs_b200.profile_case leaf G            the same two factorizations; prints the
                                                       index, among the panel-leaf launches of the
                                                       process, of the second one's first leaf of
                                                       the root front's level (the root front's
                                                       supernode is the largest)
    python -m taucs_b200.profile_case batch K           one FP32-front factorization and refinement
                                                       (1 right-hand side each) of a batch of K
                                                       systems: half 2D 5-point grids of side
                                                       U{8..96}, half 3D 7-point grids of side
                                                       U{4..24}, lognormal(0, 1) conductances
                                                       (system i: generator seed i); the launch
                                                       order starts with the two persistent
                                                       small-front launches (one warp per front,
                                                       then one CTA per front)

The lognormal systems are the bench's (sigma 2, anisotropy 1:1:100, seed 0,
AMD ordering).  Profiling mode (per-launch CUDA events) is used only where an
index is printed; captures replay the same command with it off.
"""
import ctypes as C
import sys

import numpy as np


def _system(tb, g):
    A = tb.lognormal(g, g, g, 2.0, (1, 1, 100), 0)
    p, ip = tb.order(A, "amd")
    return A.permute(p, ip)


def _batch(tb, count, seed=0):
    rng = np.random.default_rng(seed)
    systems = []
    for i in range(count):
        if i < count // 2:
            k = int(rng.integers(8, 97))
            systems.append(tb.lognormal(k, k, 0, 1.0, (1, 1, 1), i))
        else:
            k = int(rng.integers(4, 25))
            systems.append(tb.lognormal(k, k, k, 1.0, (1, 1, 1), i))
    bs = [rng.uniform(-1, 1, A.n) for A in systems]
    return systems, bs


def _factor(tb, torch, P, profile):
    F = tb.factor_symbolic(P)
    F.set_precision(1)
    dv = torch.from_numpy(P.values).cuda()
    lib = tb.lib()
    if profile:
        # one factorization first, unprofiled: the first launch of each
        # kernel carries one-time costs that would skew the per-launch times
        assert lib.taucs_b200_factor_numeric_device(F.h, C.c_void_p(dv.data_ptr())) == 0, tb.last_error()
        torch.cuda.synchronize()
        lib.taucs_b200_profile(1)
    assert lib.taucs_b200_factor_numeric_device(F.h, C.c_void_p(dv.data_ptr())) == 0, tb.last_error()
    torch.cuda.synchronize()
    log = None
    if profile:
        n = lib.taucs_b200_profile_log(None, None, 0)
        kc = np.zeros(n, np.int32)
        ms = np.zeros(n, np.float32)
        lib.taucs_b200_profile_log(kc.ctypes.data_as(C.c_void_p), ms.ctypes.data_as(C.c_void_p), n)
        lib.taucs_b200_profile(0)
        log = (kc, ms)
    return F, dv, log


def main(argv):
    import torch
    import taucs_b200 as tb
    case, g = argv[1], int(argv[2])
    if case == "batch":
        systems, bs = _batch(tb, g)
        B = tb.Batch(systems)
        B.set_precision(1)
        dv = torch.from_numpy(B.combined_values()).cuda()
        db = torch.from_numpy(B.combined_rhs(bs)).cuda()
        dx = torch.zeros_like(db)
        assert tb.lib().taucs_b200_factor_numeric_device(B.h, C.c_void_p(dv.data_ptr())) == 0, tb.last_error()
        its, res = B.solve_refine_device(1, dx.data_ptr(), db.data_ptr(), B.n)
        torch.cuda.synchronize()
        print("systems", B.count, "rows", B.n, "refinement steps", its, "worst scaled residual", max(res))
        return
    P = _system(tb, g)
    if case == "factor-refine":
        F, _, _ = _factor(tb, torch, P, False)
        n, nrhs = P.n, 8
        db = torch.from_numpy(np.random.default_rng(0).uniform(-1, 1, n * nrhs)).cuda()
        dx = torch.zeros_like(db)
        its, res = F.solve_refine_device(nrhs, dx.data_ptr(), db.data_ptr(), n)
        torch.cuda.synchronize()
        print("refinement steps", its, "worst scaled residual", max(res))
    elif case == "update-gemm":
        _, _, (kc, ms) = _factor(tb, torch, P, True)
        g = [(int(k), float(t)) for k, t in zip(kc, ms) if k in (4, 5)]   # panel and update products
        best = max(range(len(g)), key=lambda j: g[j][1] if g[j][0] == 5 else -1.0)
        # the index counts the unprofiled factorization's launches too
        print("tcgen05 GEMM launches", len(g), "largest update-matrix launch: index", len(g) + best, "ms", g[best][1])
    elif case == "leaf":
        F, _, (kc, ms) = _factor(tb, torch, P, True)
        leaves = [float(t) for k, t in zip(kc, ms) if k == 2]
        # the root's level runs last: its first leaf (the largest grid) is
        # the first of the final run of leaf launches of the root's width
        s_root = int(F.info().max_sn_size)
        first = max(0, len(leaves) - (s_root + 63) // 64)
        print("leaf launches", len(leaves), "first leaf of the root level: index", len(leaves) + first,
              "ms", leaves[first] if leaves else 0.0)
    else:
        raise SystemExit(__doc__)


if __name__ == "__main__":
    main(sys.argv)
