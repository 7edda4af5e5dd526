"""numpy restatements of the reference's positive semidefinite completions
(Python-only in the reference).  TEST INFRASTRUCTURE ONLY: the checker used
by tests/, never by the product.

`symb` carries the reference's symbolic attributes; `X0` is the dense
symmetric matrix of the cspmatrix in the reordered numbering.
"""
import numpy as np


def psdcompletion(symb, X0, tol=1e-15):
    """Maximum-determinant PSD completion (src/python/pybase/psdcompletion.py:
    4-71): supernodes from last to first, X[eta, nu] = X[eta, alpha]
    X[alpha, alpha]^{-1} X[alpha, nu] via a Cholesky factor of X[alpha,
    alpha] (the pseudo-inverse from an eigendecomposition if it fails)."""
    X = np.array(X0, dtype=np.float64)
    n = int(symb.n)
    snptr, sncolptr, snrowidx = (np.asarray(a) for a in (symb.snptr, symb.sncolptr, symb.snrowidx))
    for k in range(int(symb.Nsn) - 1, -1, -1):
        nn = int(snptr[k + 1] - snptr[k])
        beta = snrowidx[sncolptr[k]:sncolptr[k + 1]]
        nj = len(beta)
        if nj - nn == 0:
            continue
        alpha, nu = beta[nn:], beta[:nn]
        eta = np.concatenate([np.arange(beta[kk] + 1, beta[kk + 1]) for kk in range(nj - 1)] +
                             [np.arange(beta[-1] + 1, n)]).astype(np.int64)
        Xaa = X[np.ix_(alpha, alpha)]
        try:
            L = np.linalg.cholesky(Xaa)
            Xan = np.linalg.solve(L, X[np.ix_(alpha, nu)])
            XeaT = np.linalg.solve(L, X[np.ix_(eta, alpha)].T)
            tmp = XeaT.T @ Xan
        except np.linalg.LinAlgError:
            w, Z = np.linalg.eigh(Xaa)
            lam = w.max()
            winv = np.array([1.0 / wi if wi > lam * tol else 0.0 for wi in w])
            tmp = X[np.ix_(eta, alpha)] @ (Z * winv) @ Z.T @ X[np.ix_(alpha, nu)]
        X[np.ix_(eta, nu)] = tmp
        X[np.ix_(nu, eta)] = tmp.T
    return X


def clique_ranks(symb, X0):
    """Numerical rank of each clique's principal submatrix of a PSD matrix
    (eigenvalues above 1e-14 of the largest): mrcompletion's r is their
    maximum (mrcompletion.py:75-76)."""
    X = np.asarray(X0)
    out = []
    for k in range(int(symb.Nsn)):
        beta = np.asarray(symb.snrowidx[symb.sncolptr[k]:symb.sncolptr[k + 1]])
        w = np.linalg.eigvalsh(X[np.ix_(beta, beta)])
        out.append(int(np.sum(w > 1e-14 * w[-1])))
    return out
