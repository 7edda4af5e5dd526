"""GPU parity of completion (both update modes) and hessian (all adj/inv
modes, both update modes, lists of U) against the committed golden outputs
of the reference's C kernels and against those kernels run live on larger
problems, plus the reference test suite's round trips
(tests/test_numeric.py:48-96 of the reference)."""
import numpy as np
import pytest
import torch

import chompack_b200 as cp
import golden_cases
from helpers import problem, assert_blocks_close
from oracle import ref

pytestmark = pytest.mark.gpu

CASES = [
    ("grid2d", (30,), (16, 16)),
    ("random", (200, 0.02), (16, 4)),
    ("grid3d", (12,), (32, 32)),
    ("grid3d", (20,), (32, 32)),
    ("random", (300, 0.05), (16, 16)),
]
MODES = [(a, i) for a in (False, True) for i in (False, True)]


@pytest.fixture(scope="module", autouse=True)
def _need_cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")


def _dev(s, v, factor):
    return cp.cspmatrix(s, blkval=torch.from_numpy(np.array(v, dtype=np.float64)).cuda(), factor=factor)


@pytest.mark.parametrize("name", golden_cases.names(numeric_only=True))
@pytest.mark.parametrize("fu", [False, True])
def test_completion_golden(name, fu):
    d, A, s = golden_cases.load(name)
    X = _dev(s, d["ref_projected_inverse"], False)
    cp.completion(X, factored_updates=fu)
    assert X.is_factor is True
    assert_blocks_close(s, X.blkval.cpu().numpy(), d["ref_completion_fu%d" % int(fu)])


@pytest.mark.parametrize("name", golden_cases.names(numeric_only=True))
@pytest.mark.parametrize("fu", [False, True])
@pytest.mark.parametrize("adj,inv", MODES + [(None, False)])
def test_hessian_golden(name, fu, adj, inv):
    d, A, s = golden_cases.load(name)
    L = _dev(s, d["ref_cholesky"], True)
    Y = _dev(s, d["ref_projected_inverse"], False)
    U = _dev(s, d["ref_hessian_U0"], False)
    cp.hessian(L, Y, U, adj=adj, inv=inv, factored_updates=fu)
    key = ("ref_hessian_full_fu%d" % int(fu)) if adj is None else \
        ("ref_hessian_a%d_i%d_fu%d" % (int(adj), int(inv), int(fu)))
    assert_blocks_close(s, U.blkval.cpu().numpy(), d[key])


@pytest.mark.parametrize("kind,args,merge", CASES)
@pytest.mark.parametrize("fu", [False, True])
def test_completion_matches_reference(kind, args, merge, fu):
    A, s = problem(kind, *args, merge=merge, seed=8)
    X = cp.cspmatrix(s, device="cpu") + A
    L = X.blkval.numpy().copy()
    assert ref.cholesky(s, L) == 0
    Y = L.copy()
    assert ref.projected_inverse(s, Y) == 0
    r = Y.copy()
    assert ref.completion(s, r, factored_updates=fu) == 0
    Xg = _dev(s, Y, False)
    cp.completion(Xg, factored_updates=fu)
    assert_blocks_close(s, Xg.blkval.cpu().numpy(), r)
    # and the completion of P(L^-T L^-1) is L itself
    assert_blocks_close(s, Xg.blkval.cpu().numpy(), L, rtol=1e-9)


@pytest.mark.parametrize("kind,args,merge", CASES)
@pytest.mark.parametrize("fu", [False, True])
@pytest.mark.parametrize("adj,inv", MODES + [(None, False), (None, True)])
def test_hessian_matches_reference(kind, args, merge, fu, adj, inv):
    A, s = problem(kind, *args, merge=merge, seed=9)
    X = cp.cspmatrix(s, device="cpu") + A
    blk0 = X.blkval.numpy().copy()
    L = blk0.copy()
    assert ref.cholesky(s, L) == 0
    Y = L.copy()
    assert ref.projected_inverse(s, Y) == 0
    rng = np.random.default_rng(len(args) + int(fu))
    U0 = [blk0 * rng.standard_normal(blk0.size) for _ in range(3)]
    R = [u.copy() for u in U0]
    ref.hessian(s, L, Y, R, adj=adj, inv=inv, factored_updates=fu)
    Lg, Yg = _dev(s, L, True), _dev(s, Y, False)
    Ug = [_dev(s, u, False) for u in U0]
    cp.hessian(Lg, Yg, Ug, adj=adj, inv=inv, factored_updates=fu)
    for u, r in zip(Ug, R):
        assert_blocks_close(s, u.blkval.cpu().numpy(), r)


@pytest.mark.parametrize("fu", [False, True])
def test_completion_round_trip(fu):
    # tests/test_numeric.py:48-64 of the reference
    A, s = problem("random", 31, 0.15, seed=1)
    L = cp.cspmatrix(s) + A
    cp.cholesky(L)
    L2 = L.copy()
    cp.projected_inverse(L2)
    cp.completion(L2, factored_updates=fu)
    d = (L.spmatrix() - L2.spmatrix())
    assert np.max(np.abs(np.asarray(d.V))) < 1e-7


@pytest.mark.parametrize("fu", [False, True])
def test_hessian_round_trip(fu):
    # tests/test_numeric.py:66-96 of the reference: G, G^adj, then their
    # inverses, give back U
    A, s = problem("grid3d", 8, merge=(16, 16), seed=2)
    L = cp.cspmatrix(s) + A
    cp.cholesky(L)
    Y = L.copy()
    cp.projected_inverse(Y)
    U = cp.cspmatrix(s) + A
    U *= 0.1
    U0 = U.blkval.cpu().numpy().copy()
    cp.hessian(L, Y, U, adj=False, inv=False, factored_updates=fu)
    cp.hessian(L, Y, U, adj=True, inv=False, factored_updates=fu)
    cp.hessian(L, Y, U, adj=True, inv=True, factored_updates=fu)
    cp.hessian(L, Y, U, adj=False, inv=True, factored_updates=fu)
    assert_blocks_close(s, U.blkval.cpu().numpy(), U0, rtol=1e-9)


def test_hessian_many_u_split():
    # more U matrices than one C call takes (59): the wrapper splits the list
    A, s = problem("grid2d", 10, merge=(8, 8), seed=3)
    X = cp.cspmatrix(s, device="cpu") + A
    blk0 = X.blkval.numpy().copy()
    L = blk0.copy()
    assert ref.cholesky(s, L) == 0
    Y = L.copy()
    assert ref.projected_inverse(s, Y) == 0
    rng = np.random.default_rng(11)
    U0 = [blk0 * rng.standard_normal(blk0.size) for _ in range(61)]
    R = [u.copy() for u in U0]
    ref.hessian(s, L, Y, R, adj=None, inv=False, factored_updates=True)
    Ug = [_dev(s, u, False) for u in U0]
    cp.hessian(_dev(s, L, True), _dev(s, Y, False), Ug, adj=None)
    for u, r in zip(Ug, R):
        assert_blocks_close(s, u.blkval.cpu().numpy(), r)


def test_hessian_argument_errors():
    A, s = problem("grid2d", 6, seed=0)
    A2, s2 = problem("grid2d", 6, seed=1)
    L = cp.cspmatrix(s) + A
    cp.cholesky(L)
    Y = L.copy()
    cp.projected_inverse(Y)
    with pytest.raises(ValueError, match="symbolic factorizations must be the same"):
        cp.hessian(L, Y, cp.cspmatrix(s2) + A2)
    with pytest.raises(ValueError, match="L must be a cspmatrix factor"):
        cp.hessian(Y, Y, Y.copy())
    with pytest.raises(ValueError, match="Y must be a cspmatrix"):
        cp.hessian(L, L, Y.copy())
    with pytest.raises(ValueError, match="X must be a cspmatrix"):
        cp.completion(L)
