"""Supernodal multifrontal product-form Cholesky factorisation
(src/python/pfcholesky.py:113-211 of the reference):

    X + V diag(a) V^T = L_m ... L_1 L_0 L_0^T L_1^T ... L_m^T

where X = L_0 L_0^T is the chordal factor (chompack_b200.cholesky) and the
L_i are the product-form factors of I + (L_0^{-1} V) diag(a) (L_0^{-1} V)^T
(cbase.pfchol, the GPU kernels of csrc/pf.cu).  V is n x m, dense: a CUDA
float64 tensor or a numpy array; the factors live on the device of X.
"""
import numpy as np
import torch

from . import cbase
from .cspmatrix import cspmatrix
from .sparse import spmatrix
from .symbolic import symbolic

__all__ = ["pfcholesky"]


def _column_major(M, dev):
    """A new column-major CUDA float64 copy of a dense n x m matrix."""
    if isinstance(M, torch.Tensor):
        t = M.to(device=dev, dtype=torch.float64)
    else:
        t = torch.from_numpy(np.asarray(M, dtype=np.float64)).to(dev)
    if t.dim() == 1:
        t = t[:, None]
    return t.t().contiguous().t()


class pfcholesky(object):
    """Product-form Cholesky factor of X + V diag(a) V^T.

    :param X: cspmatrix (values or factor) or spmatrix
    :param V: n-by-m dense matrix
    :param a: m-vector (optional, default all ones)
    :param p: permutation for the symbolic analysis of an spmatrix X
    """

    def __init__(self, X, V, a=None, p=None):
        self._n = X.size[0]
        assert X.size[0] == X.size[1], 'X must be a square matrix'
        assert X.size[0] == V.shape[0], 'V must have have the same number of rows as X'
        if isinstance(X, cspmatrix) and X.is_factor is False:
            self._L0 = X.copy()
            cbase.cholesky(self._L0)
        elif isinstance(X, cspmatrix) and X.is_factor is True:
            self._L0 = X
        elif isinstance(X, spmatrix):
            symb = symbolic(X, p=p)
            self._L0 = cspmatrix(symb) + X
            cbase.cholesky(self._L0)
        elif isinstance(X, (np.ndarray, torch.Tensor)):
            raise NotImplementedError
        else:
            raise TypeError
        dev = cbase._values(self._L0, "L").device
        self._V = _column_major(V, dev)
        cbase.trsm(self._L0, self._V)
        if a is None:
            a = np.ones(self._V.shape[1])
        self._L = torch.zeros_like(self._V)
        self._B = torch.zeros_like(self._V)
        cbase.pfchol(a, self._V, self._L, self._B)

    def __repr__(self):
        return "<%ix%i product-form Cholesky factor, r=%i, tc='d'>" % (self._n, self._n, self._V.shape[1])

    def _apply(self, B, steps):
        """Run steps on B: a column-major CUDA tensor in place, or a numpy
        array (Fortran order) through a device copy."""
        if isinstance(B, torch.Tensor):
            for step in steps:
                step(B)
            return
        host = np.asarray(B)
        if host.dtype != np.float64 or (host.ndim == 2 and not host.flags["F_CONTIGUOUS"]):
            raise ValueError("B must be a column-major float64 array")
        flat = torch.from_numpy(host.reshape(-1, order="F")).to(self._V.device)
        Bt = flat if host.ndim == 1 else flat.reshape(host.shape[1], host.shape[0]).t()
        for step in steps:
            step(Bt)
        host.reshape(-1, order="F")[:] = flat.cpu().numpy()

    def trsm(self, B, trans='N'):
        """B := L^{-1} B ('N') or L^{-T} B ('T'), in place."""
        if trans == 'N':
            self._apply(B, [lambda t: cbase.trsm(self._L0, t),
                            lambda t: cbase.pftrsm(self._V, self._L, self._B, t, trans='N')])
        elif trans == 'T':
            self._apply(B, [lambda t: cbase.pftrsm(self._V, self._L, self._B, t, trans='T'),
                            lambda t: cbase.trsm(self._L0, t, trans='T')])
        elif type(trans) is str:
            raise ValueError("trans must be 'N' or 'T'")
        else:
            raise TypeError("trans must be 'N' or 'T'")

    def trmm(self, B, trans='N'):
        """B := L B ('N') or L^T B ('T'), in place."""
        if trans == 'N':
            self._apply(B, [lambda t: cbase.pftrmm(self._V, self._L, self._B, t, trans='N'),
                            lambda t: cbase.trmm(self._L0, t)])
        elif trans == 'T':
            self._apply(B, [lambda t: cbase.trmm(self._L0, t, trans='T'),
                            lambda t: cbase.pftrmm(self._V, self._L, self._B, t, trans='T')])
        elif type(trans) is str:
            raise ValueError("trans must be 'N' or 'T'")
        else:
            raise TypeError("trans must be 'N' or 'T'")
