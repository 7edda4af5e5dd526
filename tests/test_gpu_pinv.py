"""GPU parity of the projected-inverse sweep (the log-det gradient) against
the reference's own C kernels, plus the reference test suite's round-trip
identity <Y, A> = n (tests/test_numeric.py:40-46 of the reference)."""
import numpy as np
import pytest
import torch

import chompack_b200 as cp
from helpers import problem, assert_blocks_close
from oracle import ref

pytestmark = pytest.mark.gpu

CASES = [
    ("grid2d", (30,), (16, 16)),
    ("grid2d", (12,), None),
    ("random", (200, 0.02), (16, 4)),
    ("grid3d", (12,), (32, 32)),
    ("grid3d", (20,), (32, 32)),
    ("random", (300, 0.05), (16, 16)),
]


@pytest.fixture(scope="module", autouse=True)
def _need_cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")


@pytest.mark.parametrize("kind,args,merge", CASES)
def test_projected_inverse_matches_reference(kind, args, merge):
    A, s = problem(kind, *args, merge=merge, seed=4)
    X = cp.cspmatrix(s) + A
    r = X.blkval.cpu().numpy().copy()
    assert ref.cholesky(s, r) == 0
    assert ref.projected_inverse(s, r) == 0
    cp.cholesky(X)
    cp.projected_inverse(X)
    assert X.is_factor is False
    y = X.blkval.cpu().numpy()
    assert_blocks_close(s, y, r)
    # the strict upper part of every diagonal block is zero, as in the reference
    assert np.array_equal(y == 0.0, r == 0.0) or np.max(np.abs(y[r == 0.0])) == 0.0


def test_projected_inverse_trace_identity():
    A, s = problem("grid3d", 10, merge=(16, 16), seed=5)
    X = cp.cspmatrix(s) + A
    Am = X.spmatrix(reordered=False, symmetric=True)
    cp.cholesky(X)
    cp.projected_inverse(X)
    Ym = X.spmatrix(reordered=False, symmetric=True)
    # <Y, A> over the pattern = trace(A^{-1} A) = n
    a = Am.todense()
    y = Ym.todense()
    assert abs(float(np.sum(a * y)) - s.n) < 1e-9 * s.n


def test_projected_inverse_requires_factor():
    A, s = problem("grid2d", 6, seed=0)
    X = cp.cspmatrix(s) + A
    with pytest.raises(ValueError):
        cp.projected_inverse(X)
