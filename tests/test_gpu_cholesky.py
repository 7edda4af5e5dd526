"""GPU parity of the multifrontal Cholesky sweep against the reference's own
C kernels (oracle/_ref), on the same symbolic factorisation and values."""
import numpy as np
import pytest
import torch

import chompack_b200 as cp
from helpers import problem, assert_blocks_close
from oracle import ref

pytestmark = pytest.mark.gpu

CASES = [
    ("grid2d", (30,), (16, 16)),          # 2D 30x30, merge(16,16)
    ("grid2d", (12,), None),              # small, no merging
    ("random", (200, 0.02), (16, 4)),     # irregular pattern
    ("grid3d", (12,), (32, 32)),
    ("grid3d", (20,), (32, 32)),          # multi-tile fronts
    ("random", (300, 0.05), (16, 16)),    # dense-ish root front
]


@pytest.fixture(scope="module", autouse=True)
def _need_cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")


@pytest.mark.parametrize("kind,args,merge", CASES)
def test_cholesky_matches_reference(kind, args, merge):
    A, s = problem(kind, *args, merge=merge, seed=3)
    X = cp.cspmatrix(s) + A
    r = X.blkval.cpu().numpy().copy()
    assert ref.cholesky(s, r) == 0
    cp.cholesky(X)
    assert X.is_factor is True
    assert_blocks_close(s, X.blkval.cpu().numpy(), r)


def test_cholesky_repeat_is_deterministic():
    A, s = problem("grid3d", 16, merge=(32, 32), seed=1)
    X1 = cp.cspmatrix(s) + A
    X2 = X1.copy()
    cp.cholesky(X1)
    cp.cholesky(X2)
    assert torch.equal(X1.blkval, X2.blkval)


def test_cholesky_not_spd_raises():
    A, s = problem("grid2d", 10, merge=None, seed=2)
    X = cp.cspmatrix(s) + A
    X.blkval.mul_(-1.0)
    with pytest.raises(ArithmeticError):
        cp.cholesky(X)
    assert X.is_factor is True   # the reference flips the flag first (cbase.c:278)


def test_cholesky_rejects_factor():
    A, s = problem("grid2d", 6, seed=0)
    X = cp.cspmatrix(s) + A
    cp.cholesky(X)
    with pytest.raises(ValueError):
        cp.cholesky(X)


@pytest.mark.parametrize("kind,args,merge", [("grid3d", (12,), (128, 128)), ("grid3d", (20,), (128, 128))])
def test_cholesky_split_schur_matches_reference(kind, args, merge, monkeypatch):
    """Schur-complement tiles split along K (CHB_CHOL_KSPLIT=128, read when
    the plan builds the program): same results as the reference within the
    FP64 tolerance, and bit-identical across runs."""
    monkeypatch.setenv("CHB_CHOL_KSPLIT", "128")
    A, s = problem(kind, *args, merge=merge, seed=4)
    X = cp.cspmatrix(s) + A
    r = X.blkval.cpu().numpy().copy()
    assert ref.cholesky(s, r) == 0
    got = []
    for _ in range(2):
        Y = cp.cspmatrix(s, blkval=X.blkval.clone(), factor=False)
        cp.cholesky(Y)
        got.append(Y.blkval.cpu().numpy())
    assert_blocks_close(s, got[0], r)
    assert np.array_equal(got[0], got[1])
