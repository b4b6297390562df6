"""Batches: many independent systems analysed, factored and solved as one.

CPU: the batch keeps every system's own supernodal structure (the
reference's symbolic phase per system, joined under one virtual root), and
the value / right-hand-side maps are exact.  GPU: FP64 batch results equal
the systems factored one at a time (same kernels, same per-front
arithmetic: max relative difference <= 1e-13); FP32+refinement meets the
scaled residual 1e-12 for every system on its own."""
import numpy as np
import pytest

from tests.helpers import scaled_residual


def _systems(tb, k=10, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(k):
        if i % 2 == 0:
            s = int(rng.integers(8, 40))
            out.append(tb.lognormal(s, int(rng.integers(8, 40)), 0, 1.0, (1, 1, 1), 100 + i))
        else:
            s = int(rng.integers(4, 12))
            out.append(tb.lognormal(s, s, s, 1.0, (1, 1, 1), 100 + i))
    return out


def test_batch_keeps_each_systems_structure(tb):
    systems = _systems(tb)
    B = tb.Batch(systems)
    d = B.export_symbolic()
    off_sn = 0
    flops = 0.0
    for A in systems:
        p, ip = tb.order(A, "amd")
        F = tb.factor_symbolic(A.permute(p, ip))
        di = F.export_symbolic()
        k = di["n_sn"]
        assert np.array_equal(d["sn_size"][off_sn:off_sn + k], di["sn_size"])
        assert np.array_equal(d["sn_up_size"][off_sn:off_sn + k], di["sn_up_size"])
        flops += F.info().flops
        off_sn += k
    assert off_sn == d["n_sn"]
    assert abs(B.info().flops - flops) <= 1e-9 * flops
    assert B.count == len(systems) and B.n == sum(A.n for A in systems)


def test_batch_maps_round_trip(tb):
    systems = _systems(tb, k=6, seed=3)
    B = tb.Batch(systems)
    rng = np.random.default_rng(0)
    bs = [rng.uniform(-1, 1, A.n) for A in systems]
    assert all(np.array_equal(x, b) for x, b in zip(B.split(B.combined_rhs(bs)), bs))
    v = B.combined_values()
    assert v.shape == (B.nnz,)
    assert np.isclose(v.sum(), sum(A.values.sum() for A in systems))


@pytest.mark.gpu
def test_batch_fp64_equals_one_at_a_time(tb):
    systems = _systems(tb, k=12, seed=5)
    rng = np.random.default_rng(1)
    bs = [rng.uniform(-1, 1, A.n) for A in systems]
    B = tb.Batch(systems)
    B.set_precision(0)
    assert B.factor() == 0
    steps, xs, res = B.solve_all(bs, tol=1e-12)
    assert steps >= 1 and np.all(res <= 1e-12)
    for A, b, x in zip(systems, bs, xs):
        p, ip = tb.order(A, "amd")
        P = A.permute(p, ip)
        F = tb.factor_mf(P)
        xi = np.empty(A.n)
        xi[p] = F.solve(np.ascontiguousarray(b[p]))
        assert scaled_residual(A, x, b) <= 1e-12
        assert np.max(np.abs(x - xi)) <= 1e-10 * np.max(np.abs(xi))


@pytest.mark.gpu
def test_batch_mixed_meets_target_per_system(tb):
    systems = _systems(tb, k=16, seed=9)
    rng = np.random.default_rng(2)
    bs = [rng.uniform(-1, 1, A.n) * (10.0 ** rng.integers(-3, 4)) for A in systems]   # uneven scales
    B = tb.Batch(systems)
    B.set_precision(1)
    assert B.factor() == 0
    steps, xs, res = B.solve_all(bs, tol=1e-12)
    assert steps >= 1
    for A, b, x, r in zip(systems, bs, xs, res):
        assert r <= 1e-12
        assert scaled_residual(A, x, b) <= 1e-12


@pytest.mark.gpu
def test_batch_device_path(tb):
    import torch
    systems = _systems(tb, k=8, seed=11)
    rng = np.random.default_rng(3)
    bs = [rng.uniform(-1, 1, A.n) for A in systems]
    B = tb.Batch(systems)
    B.set_precision(1)
    dv = torch.from_numpy(B.combined_values()).cuda()
    db = torch.from_numpy(B.combined_rhs(bs)).cuda()
    dx = torch.empty_like(db)
    assert B.numeric_device(dv.data_ptr()) == 0
    its, res = B.solve_refine_device(1, dx.data_ptr(), db.data_ptr(), B.n, 1e-12, 10)
    assert its >= 1
    torch.cuda.synchronize()
    xs = B.split(dx.cpu().numpy())
    for A, b, x in zip(systems, bs, xs):
        assert scaled_residual(A, x, b) <= 1e-12
