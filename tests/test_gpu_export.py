"""cspmatrix exports and element-wise updates on the device: spmatrix()
(chb_factor_conventional + chb_lower_ccs), diag() (chb_diag),
add_projection (chb_add_projection) and syr2 (chb_syr2), against the
reference's own tests (tests/test_cspmatrix.py:16-46 of the reference), the
oracle's dense factor (oracle/trmm.py, pinned by the reference's trmm test)
and numpy restatements of base.py:28-67 and symbolic.py:1176-1210
(oracle/blocks.py).  Values on the device and in host memory (the device
mirror) both."""
import numpy as np
import pytest
import torch

import chompack_b200 as cp
import golden_cases as G
from helpers import problem, block_errors
from oracle import blocks as OB
from oracle import ref
from oracle import trmm as OT

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")


@pytest.mark.parametrize("device", ["cuda", "cpu"])
def test_round_trips(device):                    # reference tests/test_cspmatrix.py:16-46
    d, A, _ = G.load("chordal17")
    s = cp.symbolic(A, p=cp.amd.order)
    Ac = cp.cspmatrix(s, device=device) + A
    assert Ac.is_factor is False and Ac.size == (17, 17)
    dense = A.todense()
    sym = np.tril(dense) + np.tril(dense, -1).T
    assert np.allclose(Ac.spmatrix(reordered=False, symmetric=False).todense(), np.tril(dense))
    assert np.allclose(Ac.spmatrix(reordered=False, symmetric=True).todense(), sym)
    assert np.allclose(Ac.spmatrix(reordered=True, symmetric=True).todense(), sym[np.ix_(s.p, s.p)])
    assert np.allclose(Ac.spmatrix(reordered=True, symmetric=False).todense(), np.tril(sym[np.ix_(s.p, s.p)]))
    assert np.allclose((2 * Ac).spmatrix(reordered=False).todense(), 2 * np.tril(dense))
    assert np.allclose((Ac + Ac).spmatrix(reordered=False).todense(), 2 * np.tril(dense))
    Ac2 = Ac.copy()
    Ac2 += Ac
    assert np.allclose(Ac2.spmatrix(reordered=False).todense(), 2 * np.tril(dense))
    assert np.allclose(Ac.diag(reordered=False), np.diag(dense))
    assert np.allclose(Ac.diag(reordered=True), np.diag(sym[np.ix_(s.p, s.p)]))


@pytest.mark.parametrize("name", ["nc23_amd", "numeric31", "rand200_m164"])
@pytest.mark.parametrize("device", ["cuda", "cpu"])
def test_factor_export_is_the_dense_factor(name, device):
    """spmatrix() of a factor (symbolic.py:1032-1111: off-diagonal blocks
    multiplied back by L_kk) equals the oracle's dense factor, the matrix
    trmm(L, I)[p, p] gives in the reference's own test."""
    d, A, s = G.load(name)
    L = d["ref_cholesky"]
    X = cp.cspmatrix(s, blkval=torch.from_numpy(L.copy()).to(device), factor=True)
    S = X.spmatrix(reordered=True)
    D = np.zeros((s.n, s.n))
    D[np.asarray(S._I), np.asarray(S._J)] = np.asarray(S._V)
    Ld = OT.dense_factor(s, L)
    assert np.max(np.abs(D - Ld)) <= 1e-13 * np.max(np.abs(Ld))
    # the factor itself is left as it was
    assert np.array_equal(X.blkval.cpu().numpy(), L)


def test_factor_export_at_40_cubed_reproduces_the_matrix():
    """Full size (n = 64,000): L L^T x = P A P^T x for random x, with L the
    exported conventional factor (a sparse product on the host)."""
    import scipy.sparse as sp
    A, s = problem("grid3d", 40, merge=(32, 32), seed=0)
    X = cp.cspmatrix(s) + A
    Sx = X.spmatrix(reordered=True, symmetric=True)
    cp.cholesky(X)
    S = X.spmatrix(reordered=True)
    n = s.n
    Lm = sp.csc_matrix((np.asarray(S._V), (np.asarray(S._I), np.asarray(S._J))), shape=(n, n))
    Am = sp.csc_matrix((np.asarray(Sx._V), (np.asarray(Sx._I), np.asarray(Sx._J))), shape=(n, n))
    x = np.random.default_rng(3).standard_normal(n)
    lhs = Lm @ (Lm.T @ x)
    rhs = Am @ x
    assert np.max(np.abs(lhs - rhs)) <= 1e-11 * np.max(np.abs(rhs))
    # one stored entry per position of the blocks' lower trapezoids
    nn = np.diff(np.asarray(s.snptr))
    nj = np.diff(np.asarray(s.sncolptr))
    assert len(np.asarray(S._V)) == int(np.sum(nj * nn - nn * (nn - 1) // 2))


@pytest.mark.parametrize("reordered", [False, True])
def test_add_projection_matches_restatement(reordered):
    d, A, s = G.load("numeric31")
    rng = np.random.default_rng(4)
    M = rng.standard_normal((s.n, s.n))
    x0 = rng.standard_normal(int(s.blkptr[-1]))
    want = OB.add_projection(s, x0.copy(), M, alpha=0.7, beta=-1.3, reordered=reordered)
    X = cp.cspmatrix(s, blkval=torch.from_numpy(x0.copy()).cuda())
    X.add_projection(M, alpha=0.7, beta=-1.3, reordered=reordered)
    got = X.blkval.cpu().numpy()
    assert np.max(np.abs(got - want)) <= 1e-14 * np.max(np.abs(want))


def test_add_projection_of_the_matrix_gives_its_values():
    d, A, s = G.load("numeric31")
    X = cp.cspmatrix(s)
    dense = A.todense()
    sym = np.tril(dense) + np.tril(dense, -1).T
    X.add_projection(sym)
    Y = cp.cspmatrix(s, device="cpu") + A
    # add_projection fills whole blocks (symbolic.py:1208), + A only the lower
    # trapezoid; they agree on the lower trapezoid
    assert block_errors(s, X.blkval.cpu().numpy(), Y.blkval.numpy()) < 1e-15


@pytest.mark.parametrize("name", ["numeric31", "rand200_m164", "grid3d_12_m32"])
@pytest.mark.parametrize("reordered", [False, True])
@pytest.mark.parametrize("device", ["cuda", "cpu"])
def test_syr2_matches_restatement(name, reordered, device):
    d, A, s = G.load(name)
    rng = np.random.default_rng(len(name))
    u = rng.standard_normal(s.n)
    v = rng.standard_normal(s.n)
    x0 = (cp.cspmatrix(s, device="cpu") + A).blkval.numpy().copy()
    want = OB.syr2(s, x0.copy(), u, v, alpha=0.5, beta=2.0, reordered=reordered)
    X = cp.cspmatrix(s, blkval=torch.from_numpy(x0.copy()).to(device))
    cp.syr2(X, u, v, alpha=0.5, beta=2.0, reordered=reordered)
    assert block_errors(s, X.blkval.cpu().numpy(), want) <= 1e-14
    # the strict upper part of the diagonal blocks is untouched
    got = X.blkval.cpu().numpy()
    for k in range(s.Nsn):
        nn = int(s.snptr[k + 1] - s.snptr[k])
        nj = int(s.sncolptr[k + 1] - s.sncolptr[k])
        b = slice(int(s.blkptr[k]), int(s.blkptr[k + 1]))
        up = np.triu(np.ones((nj, nn), dtype=bool), 1)
        assert np.array_equal(got[b].reshape((nj, nn), order="F")[up], x0[b].reshape((nj, nn), order="F")[up])


def test_syr2_is_the_projected_rank_two_update():
    """P(u v^T + v u^T) through the dense matrix: the exported values equal
    the pattern's entries of the dense update."""
    d, A, s = G.load("numeric31")
    rng = np.random.default_rng(9)
    u = rng.standard_normal(s.n)
    v = rng.standard_normal(s.n)
    X = cp.cspmatrix(s)
    cp.syr2(X, u, v)
    S = X.spmatrix(reordered=False, symmetric=True)
    D = np.zeros((s.n, s.n))
    D[np.asarray(S._I), np.asarray(S._J)] = np.asarray(S._V)
    M = np.outer(u, v) + np.outer(v, u)
    mask = D != 0
    assert np.max(np.abs(D[mask] - M[mask])) <= 1e-14 * np.max(np.abs(M))
    # the dot product with the pattern's matrix matches: <X, P(M)> = <X, M>
    Y = cp.cspmatrix(s) + A
    assert abs(cp.dot(Y, X) - np.sum(np.asarray(A.todense() + np.tril(A.todense(), -1).T) * M)) <= \
        1e-10 * np.abs(M).sum()
