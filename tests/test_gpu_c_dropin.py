"""The C-level drop-in check: the reference's own acceptance program
(progs/test_linsolve.c), compiled unmodified against this library's drop-in
header (include/taucs.h) and linked against libtaucs_b200.so by
oracle/Makefile, runs to its own success message -- factor/solve sequences
through taucs_linsolve, the GENMMD and AMD orderings, colamd failing on an
SPD matrix, maxdepth=5 failing, every residual below 1e-8."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "test_linsolve_b200")


def test_reference_test_program_passes_against_this_library(tmp_path):
    if not os.path.exists(BIN):
        pytest.skip("oracle/_ref/test_linsolve_b200 was not built (needs the reference sources)")
    r = subprocess.run([BIN], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert "test succeeded" in r.stdout
    assert "TESING SPD FACTORIZATIONS SUCCEDDED" in r.stdout
