"""cspmatrix assembly / export on the host (CPU tensors): bit-exact against
the reference's own _iadd_spmatrix, and the round trips of the reference's
tests/test_cspmatrix.py."""
import numpy as np
import pytest

import chompack_b200 as cp
import golden_cases as G
from helpers import block_errors  # noqa: F401


@pytest.mark.parametrize("name", G.names())
def test_assembly_matches_reference(name):
    d, A, s = G.load(name)
    X = cp.cspmatrix(s, device="cpu") + A
    assert np.array_equal(X.blkval.numpy(), d["blkval"])


def test_round_trips():                    # reference tests/test_cspmatrix.py:16-46
    d, A, _ = G.load("chordal17")
    s = cp.symbolic(A, p=cp.amd.order)
    Ac = cp.cspmatrix(s, device="cpu") + A
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


def test_add_projection_and_factor_export():
    d, A, s = G.load("numeric31")
    X = cp.cspmatrix(s, device="cpu")
    dense = A.todense()
    sym = np.tril(dense) + np.tril(dense, -1).T
    X.add_projection(sym)
    Y = cp.cspmatrix(s, device="cpu") + A
    # add_projection fills whole blocks (symbolic.py:1208), + A only the lower
    # trapezoid; they agree on the lower trapezoid
    from helpers import block_errors
    assert block_errors(s, X.blkval.numpy(), Y.blkval.numpy()) < 1e-15
    # export of a factor multiplies the off-diagonal blocks back by L_kk
    L = cp.cspmatrix(s, blkval=d["ref_cholesky"], factor=True, device="cpu")
    Lm = L.spmatrix(reordered=True).todense()
    P = sym[np.ix_(s.p, s.p)]
    assert np.max(np.abs(Lm @ Lm.T - P)) < 1e-12 * np.max(np.abs(P))


def test_pattern_mismatch_raises():
    d, A, s = G.load("quick7")
    bad = cp.spmatrix([1.0], [6], [0], (7, 7))
    X = cp.cspmatrix(s, device="cpu")
    # (6, 0) of the original order is outside the chordal pattern
    with pytest.raises(ValueError):
        X += bad
