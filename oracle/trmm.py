"""numpy restatement of the reference's multiplication with the supernodal
factor (src/python/pybase/trmm.py:4-116, Python only in the reference).
TEST INFRASTRUCTURE ONLY: the checker used by tests/, never by the product.

`symb` carries the reference's symbolic attributes (snpost, snptr, snode,
relptr, relidx, chptr, chidx, blkptr, p, n); `blkval` is the factor as the
reference's cholesky leaves it (per supernode the nj x nn block, column
major: the diagonal block L_kk, then blk21 = L21 L_kk^{-1}).

Parity is pinned by the reference's own test (tests/test_numeric.py:92-104):
trmm(L, I)[p, p] is the factor in the permuted order, and its transpose for
trans 'T' (see dense_factor).
"""
import numpy as np


def _block(symb, blkval, k):
    nn = int(symb.snptr[k + 1] - symb.snptr[k])
    na = int(symb.relptr[k + 1] - symb.relptr[k])
    nj = nn + na
    b0 = int(symb.blkptr[k])
    return nn, na, np.asarray(blkval[b0:b0 + nj * nn]).reshape(nn, nj).T  # nj x nn, column major


def trmm(symb, blkval, B, alpha=1.0, trans='N'):
    """B (n x nrhs, any layout) := alpha L B (trans 'N') or alpha L^T B
    (trans 'T'), in place; returns B."""
    assert trans in ('N', 'T')
    B2 = B.reshape(B.shape[0], -1)
    snpost = [int(k) for k in np.asarray(symb.snpost)]
    snptr, snode, p = np.asarray(symb.snptr), np.asarray(symb.snode), np.asarray(symb.p)
    relptr, relidx = np.asarray(symb.relptr), np.asarray(symb.relidx)
    chptr, chidx = np.asarray(symb.chptr), np.asarray(symb.chidx)
    if trans == 'N':
        # postorder (trmm.py:55-83); stacked updates by front
        upd = {}
        for k in snpost:
            nn, na, F = _block(symb, blkval, k)
            rows = p[snode[snptr[k]:snptr[k + 1]]]
            U = np.zeros((nn + na, B2.shape[1]))
            U[:nn] = alpha * B2[rows]
            U[:nn] = np.tril(F[:nn]) @ U[:nn]                    # trmm.py:63
            if na > 0:
                U[nn:] = F[nn:] @ U[:nn]                         # :65-68
            for ii in range(chptr[k + 1] - 1, chptr[k] - 1, -1):  # stack order (:70-74)
                c = int(chidx[ii])
                U[relidx[relptr[c]:relptr[c + 1]]] += upd.pop(c)
            if na > 0:
                upd[k] = U[nn:].copy()
            B2[rows] = U[:nn]                                    # :80-82
    else:
        # reverse postorder (trmm.py:87-114)
        down = {}
        for k in reversed(snpost):
            nn, na, F = _block(symb, blkval, k)
            rows = p[snode[snptr[k]:snptr[k + 1]]]
            U = np.zeros((nn + na, B2.shape[1]))
            U[:nn] = alpha * B2[rows]
            if na > 0:
                U[nn:] = down.pop(k)                             # :96-97
            for ii in range(chptr[k], chptr[k + 1]):             # :99-102
                c = int(chidx[ii])
                down[c] = U[relidx[relptr[c]:relptr[c + 1]]].copy()
            if na > 0:
                U[:nn] += F[nn:].T @ U[nn:]                      # :104-106
            U[:nn] = np.tril(F[:nn]).T @ U[:nn]                  # :109
            B2[rows] = U[:nn]
    return B


def dense_factor(symb, blkval):
    """The factor as a dense n x n lower-triangular matrix in the permuted
    order (what the reference's L.spmatrix(reordered=True) holds for a
    factor, symbolic.py:1032-1111): column block k has L_kk on rows snptr[k]..
    and L21 = blk21 L_kk on the clique's remaining rows snrowidx."""
    n = int(symb.n)
    L = np.zeros((n, n))
    snptr, sncolptr, snrowidx = np.asarray(symb.snptr), np.asarray(symb.sncolptr), np.asarray(symb.snrowidx)
    for k in range(int(symb.Nsn)):
        nn, na, F = _block(symb, blkval, k)
        cols = np.arange(snptr[k], snptr[k + 1])
        rows = snrowidx[sncolptr[k]:sncolptr[k + 1]]
        L11 = np.tril(F[:nn])
        L[np.ix_(rows[:nn], cols)] = L11
        if na > 0:
            L[np.ix_(rows[nn:], cols)] = F[nn:] @ L11
    return L
