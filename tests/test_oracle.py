"""The oracle itself, pinned (CPU): our C restatement of the reference's
sweeps (oracle/oracle.c) against the golden outputs of the reference's own C
kernels, and the reference kernels (oracle/_ref, when built here) against the
same goldens."""
import numpy as np
import pytest

import golden_cases as G
from helpers import assert_blocks_close
from oracle import oracle, ref

NUM = G.names(numeric_only=True)


@pytest.mark.parametrize("name", NUM)
def test_restated_cholesky_matches_reference_golden(name):
    d, A, s = G.load(name)
    x = d["blkval"].copy()
    assert oracle.cholesky(s, x) == 0
    assert_blocks_close(s, x, d["ref_cholesky"])


@pytest.mark.skipif(not ref.available(), reason="reference kernels not built here")
@pytest.mark.parametrize("name", NUM)
def test_reference_build_reproduces_goldens(name):
    d, A, s = G.load(name)
    x = d["blkval"].copy()
    assert ref.cholesky(s, x) == 0
    assert np.array_equal(x, d["ref_cholesky"])
    y = x.copy()
    assert ref.projected_inverse(s, y) == 0
    assert np.array_equal(y, d["ref_projected_inverse"])


def test_restated_cholesky_reports_failure():
    d, A, s = G.load("quick7")
    x = -d["blkval"].copy()          # negative definite: first pivot fails
    assert oracle.cholesky(s, x) > 0
