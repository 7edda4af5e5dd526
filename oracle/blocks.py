"""numpy restatements of the reference's element-wise cspmatrix updates
(Python loops over supernodes in the reference).  TEST INFRASTRUCTURE ONLY:
the checker used by tests/, never by the product.

`symb` carries the reference's symbolic attributes; `blkval` is a float64
numpy array in the reference's block layout, updated in place.
"""
import numpy as np


def syr2(symb, blkval, u, v, alpha=1.0, beta=1.0, reordered=False):
    """X := alpha P(u v^T + v u^T) + beta X (src/python/base.py:28-67): per
    supernode the lower trapezoid (blas.scal of each column from its
    diagonal, blas.syr2 on the lower triangle of the diagonal block,
    blas.ger twice on the rows below it)."""
    p = np.asarray(symb.p)
    up = u[p] if not reordered else u
    vp = v[p] if not reordered else v
    for k in range(int(symb.Nsn)):
        nn = int(symb.snptr[k + 1] - symb.snptr[k])
        na = int(symb.relptr[k + 1] - symb.relptr[k])
        nj = nn + na
        rows = np.asarray(symb.snrowidx[symb.sncolptr[k]:symb.sncolptr[k + 1]])
        uk, vk = up[rows], vp[rows]
        b = blkval[int(symb.blkptr[k]):int(symb.blkptr[k + 1])].reshape((nn, nj)).T   # nj x nn view
        for i in range(nn):
            b[i:, i] = beta * b[i:, i] + alpha * (uk[i:] * vk[i] + vk[i:] * uk[i])
    return blkval


def add_projection(symb, blkval, A, alpha=1.0, beta=1.0, reordered=False):
    """X := alpha proj(A) + beta X for a dense A (src/python/symbolic.py:
    1176-1210): with reordered=False the symmetric matrix of A's lower
    triangle is permuted by p first; every entry of each block is set."""
    A = np.asarray(A, dtype=np.float64)
    if not reordered:
        At = np.tril(A)
        At = At + At.T
        At[np.diag_indices_from(At)] *= 0.5
        p = np.asarray(symb.p)
        A = At[np.ix_(p, p)]
    for k in range(int(symb.Nsn)):
        rows = np.asarray(symb.snrowidx[symb.sncolptr[k]:symb.sncolptr[k + 1]])
        cols = np.asarray(symb.snode[symb.snptr[k]:symb.snptr[k + 1]])
        sl = slice(int(symb.blkptr[k]), int(symb.blkptr[k + 1]))
        blkval[sl] = beta * blkval[sl] + alpha * A[np.ix_(rows, cols)].reshape(-1, order="F")
    return blkval
