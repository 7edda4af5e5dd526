"""Approximate minimum degree ordering (`amd.order`), the ordering the
reference uses through `cvxopt.amd.order` (symbolic.py:541-542).

`order(A)` accepts any sparse matrix, uses its lower triangle (like
cvxopt's default uplo='L') and returns the permutation as an int64 array;
pass it, or the function itself, as `p=` to `symbolic`.
"""
import numpy as np

from . import _native as N
from .sparse import as_spmatrix

__all__ = ["order"]


def order(A, uplo='L'):
    A = as_spmatrix(A)
    n = A.size[0]
    assert A.size[1] == n, "A must be square"
    I, J = A._I, A._J
    if uplo == 'L':
        k = I >= J
        I, J = I[k], J[k]
    else:
        k = I <= J
        I, J = J[k], I[k]
    key = J * max(n, 1) + I
    order_ = np.argsort(key, kind="stable")
    I, J = I[order_], J[order_]
    cp = np.zeros(n + 1, dtype=np.int64)
    np.add.at(cp, J + 1, 1)
    cp = np.ascontiguousarray(np.cumsum(cp))
    ri = np.ascontiguousarray(I.astype(np.int64))
    perm = np.empty(n, dtype=np.int64)
    N.check(N.amd_order(n, N.ptr(cp), N.ptr(ri), N.ptr(perm)), "amd.order")
    return perm
