"""Positive semidefinite completions on the GPU (chompack_b200.completions):
psdcompletion against a numpy restatement of the reference
(oracle/completions.py, psdcompletion.py:4-71) and against the maximum
determinant completion of the `completion` sweep; mrcompletion through the
reference's own test (tests/test_mrcompletion.py of the reference:
P(Y Y^T) = A, for a PSD matrix and for a rank-2 matrix made by syr2)."""
import numpy as np
import pytest
import torch

import chompack_b200 as cp
import golden_cases as G
from helpers import problem
from oracle import completions as OC

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")


def _dense_sym(X):
    S = X.spmatrix(reordered=True, symmetric=True)
    D = np.zeros((X.symb.n, X.symb.n))
    D[np.asarray(S._I), np.asarray(S._J)] = np.asarray(S._V)
    return D


def _pattern_mask(s):
    M = np.zeros((s.n, s.n), dtype=bool)
    for k in range(s.Nsn):
        beta = np.asarray(s.snrowidx[s.sncolptr[k]:s.sncolptr[k + 1]])
        M[np.ix_(beta, beta)] = True
    return M


@pytest.mark.parametrize("kind,args,merge", [("grid2d", (12,), (8, 8)), ("grid3d", (6,), None),
                                             ("random", (120, 0.04), (4, 4))])
def test_psdcompletion_matches_restatement_and_is_the_maxdet_completion(kind, args, merge):
    A, s = problem(kind, *args, merge=merge, seed=3)
    X = cp.cspmatrix(s) + A
    D0 = _dense_sym(X)
    got = cp.psdcompletion(X).cpu().numpy()
    want = OC.psdcompletion(s, D0)
    assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(want))
    # P(X) = A and X^{-1} vanishes outside the pattern (maximum determinant)
    mask = _pattern_mask(s)
    assert np.max(np.abs(got[mask] - D0[mask])) <= 1e-13 * np.max(np.abs(D0))
    Xi = np.linalg.inv(got)
    assert np.max(np.abs(Xi[~mask])) <= 1e-10 * np.max(np.abs(Xi))
    # the same completion through the GPU completion sweep: L L^T = X^{-1}
    Y = cp.cspmatrix(s) + A
    cp.completion(Y)
    L = Y.spmatrix(reordered=True)
    Ld = np.zeros((s.n, s.n))
    Ld[np.asarray(L._I), np.asarray(L._J)] = np.asarray(L._V)
    assert np.max(np.abs(Ld @ Ld.T - Xi)) <= 1e-10 * np.max(np.abs(Xi))
    # original numbering
    back = cp.psdcompletion(X, reordered=False).cpu().numpy()
    assert np.array_equal(back, got[np.ix_(s.ip, s.ip)])


def _reference_test_matrix():
    """The 17 x 17 pattern of the reference's test_mrcompletion (all ones,
    two diagonal entries raised by one), with AMD."""
    I = list(range(17)) + [2, 2, 3, 3, 4, 14, 4, 14, 8, 14, 15, 8, 15, 7, 8, 14, 8, 14, 14, 15, 10, 12, 13, 16, 12, 13,
                           16, 12, 13, 15, 16, 13, 15, 16, 15, 16, 15, 16, 16]
    J = list(range(17)) + [0, 1, 1, 2, 2, 2, 3, 3, 4, 4, 4, 5, 5, 6, 6, 6, 7, 7, 8, 8, 9, 9, 9, 9, 10, 10, 10, 11, 11,
                           11, 11, 12, 12, 12, 13, 13, 14, 14, 15]
    V = np.ones(len(I))
    V[0] += 1.0
    V[1] += 1.0
    A = cp.spmatrix(V, I, J, (17, 17))
    return A, cp.symbolic(A, p=cp.amd.order)


def _check_factor(Ac, Y, reordered=True):
    """P(Y Y^T) = A through add_projection, as the reference's test does."""
    Yh = Y.cpu().numpy()
    Ap = cp.cspmatrix(Ac.symb)
    Ap.add_projection(Yh @ Yh.T, beta=0.0, reordered=reordered)
    a = Ac.spmatrix().todense()
    b = Ap.spmatrix().todense()
    assert np.max(np.abs(a - b)) <= 1e-10 * max(1.0, np.max(np.abs(a)))


def test_mrcompletion_reference_suite_case():
    A, s = _reference_test_matrix()
    Ac = cp.cspmatrix(s) + A
    Y = cp.mrcompletion(Ac)
    _check_factor(Ac, Y)
    assert Y.shape[1] == max(OC.clique_ranks(s, _dense_sym(Ac)))
    # a rank-2 matrix made by syr2 with beta = 0, as the reference's test
    U = np.random.default_rng(1).standard_normal((17, 2))
    cp.syr2(Ac, U[:, 0], U[:, 0], alpha=0.5, beta=0.0)
    cp.syr2(Ac, U[:, 1], U[:, 1], alpha=0.5, beta=1.0)
    Y = cp.mrcompletion(Ac)
    assert Y.shape[1] == 2
    _check_factor(Ac, Y)
    Ap = cp.cspmatrix(s)
    Ap.add_projection(U @ U.T, beta=0.0, reordered=False)
    assert np.max(np.abs(Ac.spmatrix().todense() - Ap.spmatrix().todense())) <= 1e-12
    # original numbering: Y[ip] of the reordered factor
    Yo = cp.mrcompletion(Ac, reordered=False).cpu().numpy()
    Ap2 = cp.cspmatrix(s)
    Ap2.add_projection(Yo @ Yo.T, beta=0.0, reordered=False)
    assert np.max(np.abs(Ac.spmatrix().todense() - Ap2.spmatrix().todense())) <= 1e-10


@pytest.mark.parametrize("rank", [1, 3, 6])
def test_mrcompletion_low_rank_on_a_grid(rank):
    """P(U U^T) of a rank-r U on a 3-D grid pattern: the completion has rank
    r and reproduces every stored entry."""
    A, s = problem("grid3d", 8, merge=(16, 16), seed=2)
    U = np.random.default_rng(rank).standard_normal((s.n, rank))
    Ac = cp.cspmatrix(s)
    Ac.add_projection(U @ U.T, beta=0.0, reordered=False)
    Y = cp.mrcompletion(Ac)
    assert Y.shape[1] == rank
    _check_factor(Ac, Y)
