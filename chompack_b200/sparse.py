"""Sparse input container with the cvxopt `spmatrix` semantics the reference
API relies on (entries kept in compressed-column order, duplicates summed,
explicit zeros kept as structure), plus the helpers of chompack
`src/python/misc.py` (tril, triu, symmetrize, perm, eye).

Callers holding a real `cvxopt.spmatrix` or a `scipy.sparse` matrix can pass
it directly: every entry point converts with `as_spmatrix`.
"""
import numpy as np

__all__ = ["spmatrix", "as_spmatrix", "tril", "triu", "symmetrize", "perm", "eye"]


class spmatrix(object):
    """Sparse matrix with cvxopt-compatible constructor `spmatrix(V, I, J, size)`.

    `V` may be a scalar or a sequence; `I`, `J` are row/column indices.
    Attributes `I`, `J`, `V` (numpy arrays, compressed-column order), `size`,
    and `CCS` -> (colptr, rowidx, values).
    """

    __slots__ = ("_I", "_J", "_V", "_size")

    def __init__(self, V, I, J, size=None):
        I = np.asarray(_seq(I), dtype=np.int64).reshape(-1)
        J = np.asarray(_seq(J), dtype=np.int64).reshape(-1)
        if np.isscalar(V):
            V = np.full(I.size, float(V))
        else:
            V = np.asarray(_seq(V), dtype=np.float64).reshape(-1)
        if V.size != I.size or J.size != I.size:
            raise ValueError("V, I and J must have equal lengths")
        if size is None:
            size = (int(I.max()) + 1 if I.size else 0, int(J.max()) + 1 if J.size else 0)
        m, n = int(size[0]), int(size[1])
        if I.size and (I.min() < 0 or I.max() >= m or J.min() < 0 or J.max() >= n):
            raise ValueError("index out of range")
        self._size = (m, n)
        key = J * max(m, 1) + I
        order = np.argsort(key, kind="stable")
        key = key[order]
        V = V[order]
        if key.size:
            uniq, start = np.unique(key, return_index=True)
            V = np.add.reduceat(V, start)
        else:
            uniq = key
        mm = max(m, 1)
        self._I = (uniq % mm).astype(np.int64)
        self._J = (uniq // mm).astype(np.int64)
        self._V = V.astype(np.float64)

    @classmethod
    def _raw(cls, I, J, V, size):
        """Construct from already sorted, duplicate-free arrays."""
        obj = cls.__new__(cls)
        obj._I, obj._J, obj._V, obj._size = I, J, V, (int(size[0]), int(size[1]))
        return obj

    @property
    def size(self):
        return self._size

    @property
    def I(self):
        return self._I.copy()

    @property
    def J(self):
        return self._J.copy()

    @property
    def V(self):
        return self._V.copy()

    def __len__(self):
        return int(self._V.size)

    @property
    def CCS(self):
        n = self._size[1]
        cp = np.zeros(n + 1, dtype=np.int64)
        np.add.at(cp, self._J + 1, 1)
        return np.cumsum(cp), self._I.copy(), self._V.copy()

    @property
    def T(self):
        return spmatrix(self._V, self._J, self._I, (self._size[1], self._size[0]))

    def __add__(self, other):
        other = as_spmatrix(other)
        if other.size != self.size:
            raise ValueError("dimension mismatch")
        return spmatrix(np.concatenate([self._V, other._V]), np.concatenate([self._I, other._I]),
                        np.concatenate([self._J, other._J]), self._size)

    def __sub__(self, other):
        other = as_spmatrix(other)
        return self + other * (-1.0)

    def __mul__(self, a):
        if np.isscalar(a):
            return spmatrix._raw(self._I.copy(), self._J.copy(), self._V * float(a), self._size)
        raise TypeError("only scalar multiplication is supported")

    __rmul__ = __mul__

    def __neg__(self):
        return self * (-1.0)

    def __getitem__(self, key):
        r, c = key
        r = np.asarray(_seq(r), dtype=np.int64).reshape(-1)
        c = np.asarray(_seq(c), dtype=np.int64).reshape(-1)
        rinv = np.full(self._size[0], -1, dtype=np.int64)
        rinv[r] = np.arange(r.size)
        cinv = np.full(self._size[1], -1, dtype=np.int64)
        cinv[c] = np.arange(c.size)
        ni, nj = rinv[self._I], cinv[self._J]
        keep = (ni >= 0) & (nj >= 0)
        return spmatrix(self._V[keep], ni[keep], nj[keep], (r.size, c.size))

    def todense(self):
        a = np.zeros(self._size)
        a[self._I, self._J] = self._V
        return a

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csc_matrix((self._V, (self._I, self._J)), shape=self._size)

    def __repr__(self):
        return "<%ix%i sparse matrix, nnz=%i>" % (self._size[0], self._size[1], len(self))


def _seq(x):
    if isinstance(x, (range, list, tuple, np.ndarray)):
        return x
    if hasattr(x, "__iter__"):
        return list(x)
    return [x]


def as_spmatrix(A):
    """Convert a cvxopt spmatrix, scipy.sparse matrix or `spmatrix` to `spmatrix`."""
    if isinstance(A, spmatrix):
        return A
    if hasattr(A, "tocoo") and hasattr(A, "shape"):
        C = A.tocoo()
        return spmatrix(C.data, C.row, C.col, C.shape)
    if hasattr(A, "I") and hasattr(A, "J") and hasattr(A, "V") and hasattr(A, "size"):
        return spmatrix(np.asarray(list(A.V), dtype=np.float64), list(A.I), list(A.J), tuple(A.size))
    raise TypeError("expected a sparse matrix")


def tril(A):
    """Lower triangular part of A (misc.py:4-16)."""
    A = as_spmatrix(A)
    k = A._I >= A._J
    return spmatrix._raw(A._I[k], A._J[k], A._V[k], A.size)


def triu(A):
    """Upper triangular part of A (misc.py:18-30)."""
    A = as_spmatrix(A)
    k = A._I <= A._J
    return spmatrix._raw(A._I[k], A._J[k], A._V[k], A.size)


def symmetrize(A):
    """Symmetric matrix from the lower triangle of A (misc.py:32-40)."""
    A = as_spmatrix(A)
    if A.size[0] != A.size[1]:
        raise ValueError("argument must be a square matrix")
    lo = A._I >= A._J
    st = A._I > A._J
    return spmatrix(np.concatenate([A._V[lo], A._V[st]]), np.concatenate([A._I[lo], A._J[st]]),
                    np.concatenate([A._J[lo], A._I[st]]), A.size)


def perm(A, p):
    """Symmetric permutation A[p, p] (misc.py:42-53)."""
    A = as_spmatrix(A)
    p = np.asarray(_seq(p), dtype=np.int64).reshape(-1)
    if A.size[0] != A.size[1] or A.size[0] != p.size:
        raise ValueError("length of p must be equal to the order of A")
    return A[p, p]


def eye(n):
    """Dense identity matrix of order n (misc.py:55-61), as a numpy array."""
    return np.eye(n)
