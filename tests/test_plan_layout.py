"""Device layout of the level plan (plan.cpp), checked on the host for every
front: L panels, solve work vectors, diagonal-block inverses and handshake
flags never overlap and stay inside their arenas; update matrices that are
live at the same time never overlap; backward partial sums of one level
never overlap.  Lifetimes of update matrices: the small fronts with only
small fronts below them are factored by one persistent launch before the
level launches, in no fixed order among unrelated subtrees, so their update
matrices are live from that launch until it ends (consumer in the same set)
or until the consumer's level; every other update matrix is live from its
front's level through its parent's level.  An overlap would corrupt a
factorization or a solve only for some inputs, so the plan is checked
directly.  Host code only."""
import numpy as np
import pytest

from tests.helpers import amd_permuted, random_spd_pattern

BR = 64           # rows of a diagonal block / solve block
SOLVE_NRHS = 8    # right-hand sides per solve pass (partial-sum stride)


def _disjoint(name, starts, lens, total):
    if starts.size == 0:
        return
    order = np.argsort(starts, kind="stable")
    s = starts[order]
    e = s + lens[order]
    assert s[0] >= 0 and e.max() <= total, (name, int(s[0]), int(e.max()), int(total))
    bad = np.nonzero(s[1:] < e[:-1])[0]
    assert bad.size == 0, (name, int(s[bad[0] + 1]), int(e[bad[0]]))


def check_layout(F):
    fr, tot = F.layout()
    level, parent, s, f = fr[:, 0], fr[:, 1], fr[:, 2], fr[:, 3]
    l_off, u_off, v_off, dinv_off, blk_off, part_off, nchunk = (fr[:, k] for k in range(4, 11))
    m = f - s
    assert np.all(s >= 1) and np.all(m >= 0)
    _disjoint("L panels", l_off, f * s, tot[0])
    _disjoint("work vectors", v_off, f, tot[2])
    big = dinv_off >= 0
    nbs = (s + BR - 1) // BR
    assert np.array_equal(big, blk_off >= 0)
    _disjoint("inverses", dinv_off[big], nbs[big] * BR * BR, tot[3])
    _disjoint("flags", blk_off[big], nbs[big], tot[5])
    hu = u_off >= 0
    assert np.array_equal(hu, m > 0)
    assert np.all(parent[m > 0] >= 0), "a front with update rows has a parent"
    plev = np.where(parent >= 0, level[np.maximum(parent, 0)], level)
    assert np.all(plev[hu] > level[hu])
    # the persistent set: f <= 96 and every child in it (children have lower levels)
    pure = f <= 96
    for i in np.argsort(level, kind="stable"):
        if parent[i] >= 0 and not pure[i]:
            pure[parent[i]] = False
    # live intervals on the time axis -1 (the persistent launch), 0, 1, ...
    start = np.where(pure, -1, level)
    end = np.where(pure & pure[np.maximum(parent, 0)] & (parent >= 0), -1, plev)
    for t in range(-1, int(level.max()) + 1):
        live = hu & (start <= t) & (end >= t)
        _disjoint("update matrices at time %d" % t, u_off[live], m[live] ** 2, tot[1])
    for L in range(int(level.max()) + 1):
        sel = (part_off >= 0) & (level == L)
        _disjoint("partial sums at level %d" % L, part_off[sel], nchunk[sel] * s[sel] * SOLVE_NRHS, tot[4])
    return fr, tot


@pytest.mark.parametrize("case", ["lognormal64", "mesh2d", "random"])
def test_single_system_layout(tb, case):
    if case == "lognormal64":
        A = tb.lognormal(64, 64, 64, 1.0, (1, 1, 1), 1)
    elif case == "mesh2d":
        A = tb.mesh2d(90)
    else:
        A = random_spd_pattern(3000, 0.002, 5)
    P, _, _ = amd_permuted(A)
    F = tb.factor_symbolic(P)
    fr, tot = check_layout(F)
    assert (fr[:, 7] >= 0).any() or case == "random"   # big fronts exist on the grids
    F.free()


def test_batch_layout(tb):
    rng = np.random.default_rng(3)
    systems = []
    for i in range(200):
        if i % 2:
            k = int(rng.integers(4, 16))
            systems.append(tb.lognormal(k, k, k, 1.0, (1, 1, 1), 100 + i))
        else:
            k = int(rng.integers(8, 60))
            systems.append(tb.lognormal(k, k, 0, 1.0, (1, 1, 1), 100 + i))
    B = tb.Batch(systems)
    check_layout(B)
    B.free()


def check_solve_order(F):
    """Every solve block comes after the blocks of its front that it waits
    for, in the launch order of its level (a CTA must never wait for a CTA
    that is launched after it): forward, the diagonal blocks of all big
    fronts first, each front's in increasing order, then the update-row
    blocks; backward, each front's column blocks in decreasing order.  Each
    level's lists cover its big fronts' blocks exactly once."""
    fr, _ = F.layout()
    level, s, f, dinv_off = fr[:, 0], fr[:, 2], fr[:, 3], fr[:, 7]
    nbs = (s + BR - 1) // BR
    nrb = (f + BR - 1) // BR
    for h in range(F.info().n_levels):
        fwd, nd, bwd = F.solve_blocks(h)
        big = np.nonzero((level == h) & (dinv_off >= 0))[0]
        if big.size == 0:
            assert fwd.shape[0] == 0 and bwd.shape[0] == 0
            continue
        assert np.all(level[fwd[:, 0]] == h) and np.all(dinv_off[fwd[:, 0]] >= 0)
        diag, upd = fwd[:nd], fwd[nd:]
        assert np.all(diag[:, 1] < nbs[diag[:, 0]]), "diagonal blocks first"
        assert np.all(upd[:, 1] >= nbs[upd[:, 0]])
        assert np.all(upd[:, 1] < nrb[upd[:, 0]])
        for fi in big:
            rows = diag[diag[:, 0] == fi, 1]
            assert np.array_equal(rows, np.arange(nbs[fi])), ("forward diagonal order", int(fi))
            assert np.array_equal(np.sort(upd[upd[:, 0] == fi, 1]), np.arange(nbs[fi], nrb[fi]))
            cols = bwd[bwd[:, 0] == fi, 1]
            assert np.array_equal(cols, np.arange(nbs[fi])[::-1]), ("backward order", int(fi))
        assert set(np.unique(bwd[:, 0])) == set(big.tolist())


@pytest.mark.parametrize("case", ["lognormal48_aniso", "mesh2d", "batch"])
def test_solve_block_order(tb, case):
    if case == "batch":
        systems = [tb.lognormal(k, k, k, 1.0, (1, 1, 1), k) for k in range(10, 26)]
        F = tb.Batch(systems)
    else:
        A = tb.lognormal(48, 48, 48, 2.0, (1, 1, 100), 0) if case == "lognormal48_aniso" else tb.mesh2d(120)
        P, _, _ = amd_permuted(A)
        F = tb.factor_symbolic(P)
    check_solve_order(F)
    F.free()


def check_rows_maps(F, n):
    """Row lists ascend and lie in [0, n); the pivot rows of all fronts cover
    every row exactly once; each child-to-parent map ascends strictly and
    points at the same global rows in the parent's list (what extend-add and
    the solve gathers rely on)."""
    fr, _ = F.layout()
    rows, maps = F.rows_maps()
    parent, s, f, roff, moff = fr[:, 1], fr[:, 2], fr[:, 3], fr[:, 12], fr[:, 13]
    seen = np.zeros(n, np.int32)
    for i in range(fr.shape[0]):
        R = rows[roff[i]:roff[i] + f[i]]
        assert R.size == f[i] and np.all(np.diff(R) > 0) and R[0] >= 0 and R[-1] < n, i
        seen[R[:s[i]]] += 1
        m = f[i] - s[i]
        if m > 0:
            p = parent[i]
            Rp = rows[roff[p]:roff[p] + f[p]]
            mp = maps[moff[i]:moff[i] + m]
            assert np.all(np.diff(mp) > 0) and mp[0] >= 0 and mp[-1] < f[p], i
            assert np.array_equal(Rp[mp], R[s[i]:]), i
    assert np.all(seen == 1)


@pytest.mark.parametrize("case", ["lognormal40", "random", "batch"])
def test_rows_and_maps(tb, case):
    if case == "batch":
        systems = [tb.lognormal(k, k, 0, 1.0, (1, 1, 1), k) for k in range(6, 70, 3)]
        F = tb.Batch(systems)
        n = F.n
    else:
        A = tb.lognormal(40, 40, 40, 1.0, (1, 1, 1), 2) if case == "lognormal40" else random_spd_pattern(2500, 0.003, 9)
        P, _, _ = amd_permuted(A)
        F = tb.factor_symbolic(P)
        n = P.n
    check_rows_maps(F, n)
    F.free()


def check_persistent(F):
    """The persistent set and its device-side queues: every task is a small
    front (f <= 96) whose children are all tasks, queued after them (so a
    task is only taken after everything it waits for was taken); the fronts
    whose subtree has only fronts of order <= 32 come first (the one-warp
    launch), each part in level order; every small front whose subtree is
    small is in the set; parent links and child counts agree with the tree."""
    import ctypes as C
    lib = __import__("taucs_b200").lib()
    fr, _ = F.layout()
    level, parent, f = fr[:, 0], fr[:, 1], fr[:, 3]
    n = lib.taucs_b200_export_persistent(F.h, None, None, None)
    tasks = np.zeros(max(n, 1), np.int32)
    ptask = np.zeros(max(n, 1), np.int32)
    pend = np.zeros(max(n, 1), np.int32)
    lib.taucs_b200_export_persistent(F.h, tasks.ctypes.data, ptask.ctypes.data, pend.ctypes.data)
    tasks, ptask, pend = tasks[:n], ptask[:n], pend[:n]
    task_of = np.full(fr.shape[0], -1)
    task_of[tasks] = np.arange(n)
    nchild = np.bincount(parent[parent >= 0], minlength=fr.shape[0])
    assert np.all(f[tasks] <= 96)
    smax = f.copy()
    for i in np.argsort(level, kind="stable"):
        if parent[i] >= 0:
            smax[parent[i]] = max(smax[parent[i]], smax[i])
    nw = int(np.sum(smax[tasks] <= 32))
    assert np.all(smax[tasks[:nw]] <= 32) and np.all(smax[tasks[nw:]] > 32), "one-warp part first"
    assert np.all(np.diff(level[tasks[:nw]]) >= 0) and np.all(np.diff(level[tasks[nw:]]) >= 0), \
        "each part in level order"
    for t, i in enumerate(tasks):
        assert pend[t] == nchild[i]
        kids = np.nonzero(parent == i)[0]
        assert np.all(task_of[kids] >= 0) and np.all(task_of[kids] < t), "children are queued before the parent"
        p = parent[i]
        assert ptask[t] == (task_of[p] if p >= 0 else -1)
    # completeness: a small front is a task exactly when its whole subtree is small
    pure = f <= 96
    for i in np.argsort(level, kind="stable"):
        if parent[i] >= 0 and not pure[i]:
            pure[parent[i]] = False
    assert np.array_equal(task_of >= 0, pure)
    return n


@pytest.mark.parametrize("case", ["lognormal40", "mesh2d", "batch"])
def test_persistent_queue(tb, case):
    if case == "batch":
        systems = [tb.lognormal(k, k, 0, 1.0, (1, 1, 1), k) for k in range(6, 70, 3)]
        F = tb.Batch(systems)
    else:
        A = tb.lognormal(40, 40, 40, 1.0, (1, 1, 1), 2) if case == "lognormal40" else tb.mesh2d(120)
        P, _, _ = amd_permuted(A)
        F = tb.factor_symbolic(P)
    assert check_persistent(F) > 0
    F.free()
