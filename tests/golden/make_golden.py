"""Generates the golden fixtures in this directory by running the reference
itself (oracle/_ref/libtaucs_ref.so, built from the unmodified sources by
oracle/Makefile).  The reference ships no golden vectors of its own, so these
pin the oracle and the product to the reference's actual outputs:
AMD and GENMMD permutations, elimination tree, supernodal structure (slots, sizes,
sn_struct rows, child lists), the L panels (small cases) or their checksums,
and the solution of A x = b for x_true ~ U(-1,1) with seed 0.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.bindings import Ref  # noqa: E402

CASES = [
    # name, generator, args, store full L values
    ("mesh2d_20_dirichlet", "mesh2d", (20, "dirichlet"), True),
    ("mesh2d_100_dirichlet", "mesh2d", (100, "dirichlet"), False),
    ("mesh2d_33_neumann", "mesh2d", (33, "neumann"), True),
    ("mesh3d_8", "mesh3d", (8, 8, 8), True),
    ("mesh3d_20", "mesh3d", (20, 20, 20), False),
]


def main():
    R = Ref(threads=1)
    for name, gen, args, full in CASES:
        n, cp, ri, va = getattr(R, gen)(*args)
        perm, iperm = R.order(n, cp, ri, va, "amd")
        perm_g, iperm_g = R.order(n, cp, ri, va, "genmmd")
        _, pc, pr, pv = R.permute(n, cp, ri, va, perm, iperm)
        parent = R.etree(n, pc, pr, pv)
        L = R.factor_mf(n, pc, pr, pv)
        sym = R.dump_symbolic(L)
        vp, vv = R.dump_values(L)
        xt = np.random.default_rng(0).uniform(-1, 1, n)
        # b = A x_true on the permuted matrix (lower triangle, symmetric)
        b = np.zeros(n)
        cols = np.repeat(np.arange(n), np.diff(pc))
        np.add.at(b, pr, pv * xt[cols])
        off = pr != cols
        np.add.at(b, cols[off], pv[off] * xt[pr[off]])
        x = R.solve(L, b)
        out = dict(n=n, colptr=cp, rowind=ri, values=va, perm=perm, iperm=iperm, parent=parent,
                   perm_genmmd=perm_g, iperm_genmmd=iperm_g,
                   n_sn=sym.n_sn, sn_size=sym.sn_size, sn_up_size=sym.sn_up_size,
                   first_child=sym.first_child, next_child=sym.next_child,
                   struct_ptr=sym.struct_ptr, struct_idx=sym.struct_idx, val_ptr=vp,
                   l_sum=np.sum(vv), l_sumsq=np.sum(vv * vv), l_abs=np.sum(np.abs(vv)),
                   b=b, x=x, x_true=xt, flops=sym.flops())
        if full:
            out["l_values"] = vv
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        R.free(L)
        print(name, n, sym.n_sn, os.path.getsize(os.path.join(HERE, name + ".npz")))


if __name__ == "__main__":
    main()
