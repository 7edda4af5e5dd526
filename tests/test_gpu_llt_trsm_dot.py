"""GPU parity of llt, trsm and dot against the reference's own C kernels,
plus the reference test suite's round trips (tests/test_numeric.py:20-38,
:92-124 of the reference)."""
import numpy as np
import pytest
import torch

import chompack_b200 as cp
from helpers import problem, assert_blocks_close, RTOL
from oracle import ref

pytestmark = pytest.mark.gpu

CASES = [
    ("grid2d", (30,), (16, 16)),
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
def test_llt_matches_reference(kind, args, merge):
    A, s = problem(kind, *args, merge=merge, seed=6)
    X = cp.cspmatrix(s) + A
    L = X.blkval.cpu().numpy().copy()
    assert ref.cholesky(s, L) == 0
    r = L.copy()
    ref.llt(s, r)
    Xg = cp.cspmatrix(s, blkval=torch.from_numpy(L.copy()).cuda(), factor=True)
    cp.llt(Xg)
    assert Xg.is_factor is False
    assert_blocks_close(s, Xg.blkval.cpu().numpy(), r)


@pytest.mark.parametrize("kind,args,merge", CASES)
@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("nrhs", [1, 8, 70])
def test_trsm_matches_reference(kind, args, merge, trans, nrhs):
    A, s = problem(kind, *args, merge=merge, seed=7)
    X = cp.cspmatrix(s) + A
    L = X.blkval.cpu().numpy().copy()
    assert ref.cholesky(s, L) == 0
    rng = np.random.default_rng(nrhs)
    B0 = np.asfortranarray(rng.standard_normal((s.n, nrhs)))
    rb = B0.copy(order="F")
    ref.trsm(s, L, rb, alpha=0.75, trans=trans)
    Lg = cp.cspmatrix(s, blkval=torch.from_numpy(L).cuda(), factor=True)
    Bg = torch.from_numpy(B0.T.copy()).cuda().t()  # column-major view
    cp.trsm(Lg, Bg, alpha=0.75, trans=trans)
    got = Bg.cpu().numpy()
    assert np.max(np.abs(got - rb)) <= RTOL * max(1.0, np.max(np.abs(rb))) * 10


def test_trsm_host_array_and_solve_identity():
    A, s = problem("grid3d", 10, merge=(16, 16), seed=8)
    L = cp.cspmatrix(s) + A
    cp.cholesky(L)
    rng = np.random.default_rng(1)
    b = np.asfortranarray(rng.standard_normal((s.n, 4)))
    x = b.copy(order="F")
    cp.trsm(L, x)
    cp.trsm(L, x, trans='T')
    Ad = A.todense()
    Ad = np.tril(Ad) + np.tril(Ad, -1).T
    assert np.max(np.abs(Ad @ x - b)) < 1e-10 * np.max(np.abs(b))


def test_cholesky_llt_round_trip():
    A, s = problem("random", 200, 0.03, merge=(8, 8), seed=9)
    X = cp.cspmatrix(s) + A
    X0 = X.blkval.clone()
    cp.cholesky(X)
    cp.llt(X)
    assert torch.max(torch.abs(X.blkval - X0)).item() < 1e-12 * torch.max(torch.abs(X0)).item()


@pytest.mark.parametrize("kind,args,merge", CASES)
def test_dot_matches_reference(kind, args, merge):
    A, s = problem(kind, *args, merge=merge, seed=10)
    X = cp.cspmatrix(s) + A
    Y = cp.cspmatrix(s) + A * (-0.5)
    r = ref.dot(s, X.blkval.cpu().numpy().copy(), Y.blkval.cpu().numpy().copy())
    got = cp.dot(X, Y)
    assert abs(got - r) <= 1e-12 * abs(r)


def test_dot_other_symbolic_returns_none():
    A, s = problem("grid2d", 5, seed=0)
    _, s2 = problem("grid2d", 5, seed=0)
    assert cp.dot(cp.cspmatrix(s) + A, cp.cspmatrix(s2) + A) is None
