"""Positive semidefinite completions of a cspmatrix, on its device
(reference: src/python/pybase/psdcompletion.py:4-71 and
src/python/pybase/mrcompletion.py:6-108; both are Python-only in the
reference, one LAPACK call per clique).

* psdcompletion(A): the maximum-determinant positive semidefinite
  completion X (dense, n x n) with P(X) = A, built from the last supernode
  to the first: the entries between the supernode's columns nu and the
  later indices eta outside its clique are X[eta, nu] = X[eta, alpha]
  X[alpha, alpha]^{-1} X[alpha, nu] (alpha: the separator), through a
  Cholesky factor of X[alpha, alpha], or its pseudo-inverse from an
  eigendecomposition when that factorisation fails.
* mrcompletion(A): a factor Y (n x r) of a minimum-rank positive
  semidefinite completion, P(Y Y^T) = A, r = the largest clique rank: per
  clique, in reverse topological order, an eigendecomposition of the front
  [A_{J,N}, V_k] (V_k from the parent's front), the rank-revealing part
  scaled into Y, and two SVDs that rotate the supernode's rows of Y to agree
  with its separator rows fixed by the ancestors.

The dense per-clique factorisations (Cholesky, triangular solves,
eigendecompositions, SVDs) run on the device through torch.linalg; the
sweep, its index sets and the data stay on the device, and only the
symbolic index arrays are read on the host.  Eigen- and singular vectors
are defined up to signs and rotations, so Y matches the reference's only
through P(Y Y^T) = A and its rank.
"""
import numpy as np
import torch

from . import cbase
from .cspmatrix import cspmatrix

__all__ = ["psdcompletion", "mrcompletion"]


def _dense_symmetric(A):
    """The symmetric matrix of A (reordered numbering) as a dense device
    tensor, from the device gather of the blocks' lower trapezoids."""
    v = cbase._values(A)
    dev = v.device
    cp_, I, V = A._ccs(v)
    n = A.symb.n
    J = np.repeat(np.arange(n, dtype=np.int64), np.diff(cp_))
    It = torch.from_numpy(np.asarray(I, dtype=np.int64)).to(dev)
    Jt = torch.from_numpy(J).to(dev)
    Vt = torch.from_numpy(np.asarray(V)).to(dev)
    X = torch.zeros((n, n), dtype=torch.float64, device=dev)
    X[Jt, It] = Vt
    X[It, Jt] = Vt
    return X


def psdcompletion(A, reordered=True, **kwargs):
    """Maximum determinant positive semidefinite completion X of the
    cspmatrix A (P(X) = A), as a dense device tensor (psdcompletion.py:4-71).
    tol (default 1e-15): relative threshold of the pseudo-inverse used when
    a separator block is not positive definite."""
    assert isinstance(A, cspmatrix) and A.is_factor is False, "A must be a cspmatrix"
    tol = kwargs.get('tol', 1e-15)
    X = _dense_symmetric(A)
    dev = X.device
    symb = A.symb
    n = symb.n
    snptr = np.asarray(symb.snptr)
    sncolptr = np.asarray(symb.sncolptr)
    snrowidx = np.asarray(symb.snrowidx)
    outside = np.ones(n, dtype=bool)
    for k in range(symb.Nsn - 1, -1, -1):
        nn = int(snptr[k + 1] - snptr[k])
        beta = snrowidx[sncolptr[k]:sncolptr[k + 1]]
        nj = len(beta)
        if nj - nn == 0:
            continue
        # eta: the indices after beta[0] that are not in the clique
        outside[:] = True
        outside[:beta[0] + 1] = False
        outside[beta] = False
        eta = torch.from_numpy(np.nonzero(outside)[0]).to(dev)
        alpha = torch.from_numpy(beta[nn:].astype(np.int64)).to(dev)
        nu = torch.from_numpy(beta[:nn].astype(np.int64)).to(dev)
        Xaa = X[alpha][:, alpha]
        Xan = X[alpha][:, nu]
        Xea = X[eta][:, alpha]
        L, info = torch.linalg.cholesky_ex(Xaa)
        if int(info) == 0:
            Wan = torch.linalg.solve_triangular(L, Xan, upper=False)
            Wea = torch.linalg.solve_triangular(L, Xea.T, upper=False)
            tmp = Wea.T @ Wan
        else:
            w, Z = torch.linalg.eigh(Xaa)
            lam = w.max()
            winv = torch.where(w > lam * tol, 1.0 / w, torch.zeros_like(w))
            tmp = Xea @ ((Z * winv) @ Z.T) @ Xan
        X[eta[:, None], nu[None, :]] = tmp
        X[nu[:, None], eta[None, :]] = tmp.T
    if reordered:
        return X
    ip = torch.from_numpy(np.asarray(symb.ip, dtype=np.int64)).to(dev)
    return X[ip][:, ip]


def mrcompletion(A, reordered=True):
    """Factor Y (n x r, a device tensor) of a minimum-rank positive
    semidefinite completion of the cspmatrix A: P(Y Y^T) = A, r the largest
    rank of a clique's front (mrcompletion.py:6-108)."""
    assert isinstance(A, cspmatrix) and A.is_factor is False, "A must be a cspmatrix"
    symb = A.symb
    v = cbase._values(A)
    dev = v.device
    n = symb.n
    snptr = np.asarray(symb.snptr)
    relptr = np.asarray(symb.relptr)
    relidx = np.asarray(symb.relidx)
    chptr = np.asarray(symb.chptr)
    chidx = np.asarray(symb.chidx)
    blkptr = np.asarray(symb.blkptr)
    sncolptr = np.asarray(symb.sncolptr)
    snrowidx = np.asarray(symb.snrowidx)
    maxr = int(symb.clique_number)
    Y = torch.zeros((n, maxr), dtype=torch.float64, device=dev)
    stack = []
    r = 0
    for k in range(symb.Nsn - 1, -1, -1):
        nn = int(snptr[k + 1] - snptr[k])
        na = int(relptr[k + 1] - relptr[k])
        nj = nn + na
        # F: the lower trapezoid of the block, then V_k's lower triangle
        blk = v[int(blkptr[k]):int(blkptr[k + 1])].reshape(nn, nj).T
        F = torch.zeros((nj, nj), dtype=torch.float64, device=dev)
        F[:, :nn] = torch.tril(blk)
        if na > 0:
            F[nn:, nn:] = torch.tril(stack.pop())
        for ii in range(int(chptr[k]), int(chptr[k + 1])):
            c = int(chidx[ii])
            rr = torch.from_numpy(relidx[relptr[c]:relptr[c + 1]].astype(np.int64)).to(dev)
            stack.append(F[rr][:, rr])
        w, Z = torch.linalg.eigh(F, UPLO='L')
        rk = int((w > 1e-14 * w[nj - 1]).sum())
        r = max(rk, r)
        Zs = Z[:, nj - rk:] * torch.sqrt(w[nj - rk:])
        In = torch.from_numpy(snrowidx[sncolptr[k]:sncolptr[k] + nn].astype(np.int64)).to(dev)
        Y[In, :rk] = Zs[:nn]
        if na > 0:
            Ia = torch.from_numpy(snrowidx[sncolptr[k] + nn:sncolptr[k + 1]].astype(np.int64)).to(dev)
            Ya = Y[Ia, :r]
            Vm = torch.zeros((na, r), dtype=torch.float64, device=dev)
            Vm[:, :rk] = Zs[nn:nj]
            P, _, Q1t = torch.linalg.svd(Vm, full_matrices=True)
            _, S, Q2t = torch.linalg.svd(Ya, full_matrices=True)
            Q2t = Q2t.clone()
            m = min(na, rk)
            if m > 0 and S.numel() > 0:
                keep = S[:m] > 1e-14 * S[0]
                rows = (P[:, :m].T @ Ya) / torch.where(keep, S[:m], torch.ones_like(S[:m]))[:, None]
                Q2t[:m] = torch.where(keep[:, None], rows, Q2t[:m])
            Y[In, :r] = Y[In, :r] @ Q1t[:r, :r].T @ Q2t[:r, :r]
    if reordered:
        return Y[:, :r]
    ip = torch.from_numpy(np.asarray(symb.ip, dtype=np.int64)).to(dev)
    return Y[ip, :r]
