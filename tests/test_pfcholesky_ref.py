"""The checker for the product-form Cholesky factor (the next sweep after
trmm; the reference's src/C/pfcholesky.c, compiled unchanged into
oracle/_ref, and src/python/pfcholesky.py:113-211), on the CPU: composed as
the reference's pfcholesky class composes it (L0 from cholesky, V := L0^{-1}
V, the product form of I + V diag(a) V^T), it satisfies the reference's own
test identities (tests/test_numeric.py:120-159):

    L^T then L applied to W gives (A + V diag(a) V^T) W,
    the two triangular solves undo it."""
import numpy as np
import pytest

from oracle import ref
from oracle import trmm as OT
import golden_cases as G

pytestmark = pytest.mark.skipif(not ref.available(), reason="reference kernels not built")


def _dense(d):
    n = int(d["size"][0])
    A = np.zeros((n, n))
    np.add.at(A, (d["I"].astype(int), d["J"].astype(int)), d["V"])
    return np.tril(A) + np.tril(A, -1).T


class _PF(object):
    """pfcholesky.py:140-211 over the checker's kernels."""

    def __init__(self, s, L0, V, a):
        self.s, self.L0 = s, L0
        self.V = np.asfortranarray(V.copy())
        ref.trsm(s, L0, self.V)                       # V := L0^{-1} V  (:151-153)
        self.L, self.B, info = ref.pfchol(a, self.V)  # (:168-171)
        assert info == 0

    def trmm(self, W, trans):
        if trans == 'N':                              # (:195-197)
            ref.pftrmm(self.V, self.L, self.B, W, 'N')
            OT.trmm(self.s, self.L0, W, trans='N')
        else:                                         # (:198-200)
            OT.trmm(self.s, self.L0, W, trans='T')
            ref.pftrmm(self.V, self.L, self.B, W, 'T')

    def trsm(self, W, trans):
        if trans == 'N':                              # (:175-177)
            ref.trsm(self.s, self.L0, W, trans='N')
            ref.pftrsm(self.V, self.L, self.B, W, 'N')
        else:                                         # (:178-180)
            ref.pftrsm(self.V, self.L, self.B, W, 'T')
            ref.trsm(self.s, self.L0, W, trans='T')


@pytest.mark.parametrize("name", ["nc23_amd", "numeric31", "rand200_m164"])
@pytest.mark.parametrize("m", [1, 4])
def test_product_form_identities(name, m):
    d, A, s = G.load(name)
    rng = np.random.default_rng(m)
    V = np.asfortranarray(rng.standard_normal((s.n, m)))
    a = rng.uniform(0.5, 2.0, m)
    pf = _PF(s, d["ref_cholesky"], V, a)
    M = _dense(d) + V @ np.diag(a) @ V.T
    W = np.asfortranarray(V.copy())
    pf.trmm(W, 'T')
    pf.trmm(W, 'N')
    want = M @ V
    assert np.max(np.abs(W - want)) <= 1e-11 * np.max(np.abs(want))
    pf.trsm(W, 'N')
    pf.trsm(W, 'T')
    assert np.max(np.abs(W - V)) <= 1e-10 * np.max(np.abs(V))
