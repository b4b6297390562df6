"""Binary CCS matrix and vector files (src/taucs_ccs_io.c:31-113, :966-1052;
the matrix layout of matlab/taucs_ccs_write_binary.m): files written here are
read by the reference's own reader with identical arrays and flags, files in
the MATLAB writer's layout are read identically by both, and malformed files
are rejected (the reference asserts or reads garbage on those, so they are
not given to it).  Host code only."""
import os

import numpy as np
import pytest

TAUCS_DOUBLE = 2048


def matlab_layout(path, n, colptr, rowind, values):
    """The byte stream matlab/taucs_ccs_write_binary.m writes for a real
    matrix: nrows, ncols, flags = 2048, colptr, 0-based rows, doubles."""
    with open(path, "wb") as f:
        np.array([n, n, TAUCS_DOUBLE], np.int32).tofile(f)
        np.asarray(colptr, np.int32).tofile(f)
        np.asarray(rowind, np.int32).tofile(f)
        np.asarray(values, np.float64).tofile(f)


def same(A, n, cp, ri, va, flags):
    return (A.n == n and A.flags == flags and np.array_equal(A.colptr, cp) and np.array_equal(A.rowind, ri)
            and np.array_equal(A.values, va))


def test_round_trip_and_reference_reads_ours(tb, ref, tmp_path):
    A = tb.lognormal(9, 7, 5, 1.5, (1, 1, 10), 3)
    path = str(tmp_path / "a.bin")
    tb.write_binary(A, path)
    assert os.path.getsize(path) == 12 + 4 * (A.n + 1) + 12 * A.nnz
    B = tb.read_binary(path)
    assert same(B, A.n, A.colptr, A.rowind, A.values, A.flags)
    assert same(B, *ref.read_binary(path))


def test_matlab_layout_read_by_both(tb, ref, tmp_path):
    M = tb.mesh3d(6)
    path = str(tmp_path / "m.bin")
    matlab_layout(path, M.n, M.colptr, M.rowind, M.values)
    A = tb.read_binary(path)
    n, cp, ri, va, fl = ref.read_binary(path)
    assert fl == TAUCS_DOUBLE and same(A, n, cp, ri, va, fl)
    assert same(A, M.n, M.colptr, M.rowind, M.values, TAUCS_DOUBLE)


def test_vectors_both_ways(tb, ref, tmp_path):
    v = np.random.default_rng(0).standard_normal(1001)
    p1, p2 = str(tmp_path / "ours.bin"), str(tmp_path / "refs.bin")
    tb.vec_write_binary(v, p1)
    assert ref.vec_write_binary(v, p2) == 0
    assert open(p1, "rb").read() == open(p2, "rb").read()
    assert np.array_equal(ref.vec_read_binary(v.size, p1), v)
    assert np.array_equal(tb.vec_read_binary(v.size, p2), v)


def test_malformed_files_rejected(tb, tmp_path):
    M = tb.mesh2d(5)
    good = str(tmp_path / "good.bin")
    tb.write_binary(M, good)
    raw = open(good, "rb").read()
    cases = {
        "truncated values": raw[:-8],
        "truncated header": raw[:8],
        "colptr not from 0": raw[:12] + np.int32(1).tobytes() + raw[16:],
        "row out of range": raw[:12 + 4 * (M.n + 1)] + np.int32(M.n).tobytes() + raw[16 + 4 * (M.n + 1):],
        "complex values": raw[:8] + np.int32(8192).tobytes() + raw[12:],
        "negative size": np.int32(-1).tobytes() + raw[4:],
    }
    for why, data in cases.items():
        path = str(tmp_path / "bad.bin")
        open(path, "wb").write(data)
        with pytest.raises(RuntimeError):
            tb.read_binary(path)
    with pytest.raises(RuntimeError):
        tb.read_binary(str(tmp_path / "missing.bin"))
    short = str(tmp_path / "short.bin")
    tb.vec_write_binary(np.ones(10), short)
    with pytest.raises(RuntimeError):
        tb.vec_read_binary(11, short)


def test_served_request_replays_from_files(tb, tmp_path):
    """A request saved as matrix + right-hand-side files reads back to the
    same system (the serving wire format)."""
    A = tb.lognormal(12, 12, 0, 1.0, (1, 1, 1), 9)
    b = np.random.default_rng(2).uniform(-1, 1, A.n)
    tb.write_binary(A, str(tmp_path / "req.A"))
    tb.vec_write_binary(b, str(tmp_path / "req.b"))
    A2 = tb.read_binary(str(tmp_path / "req.A"))
    b2 = tb.vec_read_binary(A2.n, str(tmp_path / "req.b"))
    assert np.array_equal(A2.matvec(b2), A.matvec(b))
