"""Minimal numpy-backed stand-in for the parts of cvxopt that the reference
chompack's pure-Python modules (`symbolic.py`, `misc.py`) touch.

TEST INFRASTRUCTURE ONLY.  cvxopt is not installable in this environment, so
`tests/golden/make_golden.py` puts this directory on `sys.path` to import the
reference's own `symbolic.py` unmodified and record its outputs as golden
fixtures.  Nothing in the product imports this module.

Semantics mirrored (cvxopt 1.2 behaviour, as used by the reference):
  * `matrix` is a column-major dense matrix of typecode 'i' (int64) or 'd'
    (float64); a flat list argument gives a column vector, a list of matrices
    is stacked vertically; integer / slice / index-list / index-matrix
    indexing is linear (column-major) for one subscript and (row, col) for
    two; unary `+` copies.
  * `spmatrix(V, I, J, size)` keeps entries in compressed-column order with
    duplicates summed; `A.I`, `A.J`, `A.V` and `A.CCS` follow that order;
    `A[p, q]` is the submatrix B[i, j] = A[p[i], q[j]] (pattern kept, explicit
    zeros kept); `len(A)` is the number of stored entries.
"""
import numpy as _np

__all__ = ["matrix", "spmatrix", "sparse", "normal", "blas", "lapack", "printing", "amd"]


def _tc_of(arr):
    return 'd' if arr.dtype.kind == 'f' else 'i'


def _as_index(key, n):
    """Linear index specification -> numpy int array (or slice/int)."""
    if isinstance(key, (int, _np.integer)):
        return int(key)
    if isinstance(key, slice):
        return key
    if isinstance(key, matrix):
        return key._a.reshape(-1, order='F').astype(_np.int64)
    if isinstance(key, range):
        return _np.asarray(list(key), dtype=_np.int64)
    return _np.asarray(list(key), dtype=_np.int64)


class matrix(object):
    def __init__(self, x=None, size=None, tc=None):
        if isinstance(x, matrix):
            a = x._a.copy()
        elif isinstance(x, _np.ndarray):
            a = x.copy()
            if a.ndim == 1:
                a = a.reshape(-1, 1)
        elif isinstance(x, (int, float, _np.integer, _np.floating)) and not isinstance(x, bool):
            if size is None:
                size = (1, 1)
            dt = _np.float64 if (isinstance(x, (float, _np.floating)) or tc == 'd') else _np.int64
            a = _np.full(size, x, dtype=dt)
            size = None
        elif isinstance(x, range):
            a = _np.asarray(list(x), dtype=_np.int64).reshape(-1, 1)
        elif isinstance(x, (list, tuple)):
            if len(x) > 0 and all(isinstance(e, matrix) for e in x):
                a = _np.concatenate([e._a.reshape(-1, 1, order='F') for e in x], axis=0)
            elif len(x) > 0 and isinstance(x[0], (list, tuple)):
                cols = [_np.asarray(c).reshape(-1, 1) for c in x]
                a = _np.concatenate(cols, axis=1)
            else:
                vals = list(x)
                if any(isinstance(v, (float, _np.floating)) for v in vals):
                    a = _np.asarray(vals, dtype=_np.float64).reshape(-1, 1)
                else:
                    a = _np.asarray(vals, dtype=_np.int64).reshape(-1, 1)
        elif x is None:
            a = _np.zeros((0, 1), dtype=_np.int64)
        else:
            raise TypeError("unsupported matrix argument %r" % (type(x),))
        if size is not None:
            a = a.reshape(-1, order='F').reshape(size, order='F')
        if tc == 'd':
            a = a.astype(_np.float64)
        elif tc == 'i':
            a = a.astype(_np.int64)
        if a.ndim == 1:
            a = a.reshape(-1, 1)
        self._a = a

    # -- basic protocol ---------------------------------------------------
    @property
    def size(self):
        return tuple(self._a.shape)

    @property
    def typecode(self):
        return _tc_of(self._a)

    def __len__(self):
        return self._a.size

    def _flat(self):
        return self._a.reshape(-1, order='F')

    def __iter__(self):
        for v in self._flat():
            yield v.item()

    def __pos__(self):
        return matrix(self._a.copy())

    def __neg__(self):
        return matrix(-self._a)

    @property
    def T(self):
        return matrix(self._a.T.copy())

    def __repr__(self):
        return "<shim matrix %s %r>" % (self.typecode, self._a.shape)

    # -- indexing ---------------------------------------------------------
    def __getitem__(self, key):
        if isinstance(key, tuple):
            r, c = key
            rr = self._sub_index(r, self._a.shape[0])
            cc = self._sub_index(c, self._a.shape[1])
            if isinstance(rr, int) and isinstance(cc, int):
                return self._a[rr, cc].item()
            if isinstance(rr, int):
                rr = [rr]
            if isinstance(cc, int):
                cc = [cc]
            return matrix(self._a[_np.ix_(_np.arange(self._a.shape[0])[rr] if isinstance(rr, slice) else _np.asarray(rr),
                                          _np.arange(self._a.shape[1])[cc] if isinstance(cc, slice) else _np.asarray(cc))].copy())
        flat = self._flat()
        k = _as_index(key, flat.size)
        if isinstance(k, int):
            return flat[k].item()
        return matrix(flat[k].reshape(-1, 1).copy())

    @staticmethod
    def _sub_index(k, n):
        if isinstance(k, (int, _np.integer)):
            return int(k) % n if k < 0 else int(k)
        if isinstance(k, slice):
            return k
        return [int(v) for v in (k._flat() if isinstance(k, matrix) else k)]

    def __setitem__(self, key, value):
        if isinstance(key, tuple):
            r, c = key
            rr = self._sub_index(r, self._a.shape[0])
            cc = self._sub_index(c, self._a.shape[1])
            rows = _np.arange(self._a.shape[0])[rr] if not isinstance(rr, list) else _np.asarray(rr)
            cols = _np.arange(self._a.shape[1])[cc] if not isinstance(cc, list) else _np.asarray(cc)
            rows = _np.atleast_1d(rows)
            cols = _np.atleast_1d(cols)
            v = value._a if isinstance(value, matrix) else value
            if isinstance(v, _np.ndarray):
                v = v.reshape(-1, order='F').reshape((rows.size, cols.size), order='F')
            self._a[_np.ix_(rows, cols)] = v
            return
        flat = self._a.reshape(-1, order='F').copy()
        k = _as_index(key, flat.size)
        if isinstance(value, matrix):
            v = value._flat()
        elif isinstance(value, (list, tuple, range)):
            v = _np.asarray(list(value))
        else:
            v = value
        if isinstance(k, int):
            flat[k] = v if not isinstance(v, _np.ndarray) else v.reshape(-1)[0]
        else:
            flat[k] = v
        self._a = flat.reshape(self._a.shape, order='F')

    # -- arithmetic (elementwise / scalar) --------------------------------
    def _other(self, o):
        return o._a if isinstance(o, matrix) else o

    def __add__(self, o):
        return matrix(self._a + self._other(o))
    __radd__ = __add__

    def __sub__(self, o):
        return matrix(self._a - self._other(o))

    def __rsub__(self, o):
        return matrix(self._other(o) - self._a)

    def __mul__(self, o):
        if isinstance(o, matrix):
            if o._a.shape == (1, 1):
                return matrix(self._a * o._a[0, 0])
            if self._a.shape == (1, 1):
                return matrix(self._a[0, 0] * o._a)
            return matrix(self._a @ o._a)
        return matrix(self._a * o)

    def __rmul__(self, o):
        return matrix(o * self._a)

    def __truediv__(self, o):
        return matrix(self._a / self._other(o))

    def __mod__(self, o):
        return matrix(self._a % self._other(o))

    def __iadd__(self, o):
        self._a = self._a + self._other(o)
        return self

    def __isub__(self, o):
        self._a = self._a - self._other(o)
        return self

    def __imul__(self, o):
        self._a = self._a * self._other(o)
        return self

    def numpy(self):
        return self._flat().copy()


class spmatrix(object):
    def __init__(self, V, I, J, size=None, tc=None):
        I = _np.asarray(list(I) if not isinstance(I, matrix) else I._flat(), dtype=_np.int64)
        J = _np.asarray(list(J) if not isinstance(J, matrix) else J._flat(), dtype=_np.int64)
        if isinstance(V, matrix):
            V = V._flat().astype(_np.float64)
        elif isinstance(V, (int, float, _np.integer, _np.floating)):
            V = _np.full(I.size, float(V))
        else:
            V = _np.asarray(list(V), dtype=_np.float64)
        if size is None:
            size = (int(I.max()) + 1 if I.size else 0, int(J.max()) + 1 if J.size else 0)
        self._size = (int(size[0]), int(size[1]))
        m = self._size[0]
        key = J * max(m, 1) + I
        order = _np.argsort(key, kind='stable')
        key = key[order]
        V = V[order]
        if key.size:
            uniq, start = _np.unique(key, return_index=True)
            Vs = _np.add.reduceat(V, start)
        else:
            uniq = key
            Vs = V
        self._I = (uniq % max(m, 1)).astype(_np.int64)
        self._J = (uniq // max(m, 1)).astype(_np.int64)
        self._V = Vs.astype(_np.float64)

    @property
    def size(self):
        return self._size

    def __len__(self):
        return self._V.size

    @property
    def I(self):
        return matrix(self._I.reshape(-1, 1).copy())

    @property
    def J(self):
        return matrix(self._J.reshape(-1, 1).copy())

    @property
    def V(self):
        return matrix(self._V.reshape(-1, 1).copy())

    @property
    def CCS(self):
        n = self._size[1]
        cp = _np.zeros(n + 1, dtype=_np.int64)
        _np.add.at(cp, self._J + 1, 1)
        cp = _np.cumsum(cp)
        return matrix(cp.reshape(-1, 1)), matrix(self._I.reshape(-1, 1).copy()), matrix(self._V.reshape(-1, 1).copy())

    @property
    def T(self):
        return spmatrix(self._V, self._J, self._I, (self._size[1], self._size[0]))

    def __add__(self, o):
        if isinstance(o, spmatrix):
            return spmatrix(_np.concatenate([self._V, o._V]), _np.concatenate([self._I, o._I]),
                            _np.concatenate([self._J, o._J]), self._size)
        raise TypeError

    def __sub__(self, o):
        if isinstance(o, spmatrix):
            return spmatrix(_np.concatenate([self._V, -o._V]), _np.concatenate([self._I, o._I]),
                            _np.concatenate([self._J, o._J]), self._size)
        raise TypeError

    def __mul__(self, a):
        if isinstance(a, (int, float)):
            return spmatrix(self._V * a, self._I, self._J, self._size)
        raise TypeError

    __rmul__ = __mul__

    def __getitem__(self, key):
        r, c = key
        r = _np.asarray(list(r) if not isinstance(r, matrix) else r._flat(), dtype=_np.int64)
        c = _np.asarray(list(c) if not isinstance(c, matrix) else c._flat(), dtype=_np.int64)
        rinv = -_np.ones(self._size[0], dtype=_np.int64)
        rinv[r] = _np.arange(r.size)
        cinv = -_np.ones(self._size[1], dtype=_np.int64)
        cinv[c] = _np.arange(c.size)
        ni = rinv[self._I]
        nj = cinv[self._J]
        keep = (ni >= 0) & (nj >= 0)
        return spmatrix(self._V[keep], ni[keep], nj[keep], (r.size, c.size))

    def todense(self):
        a = _np.zeros(self._size)
        a[self._I, self._J] = self._V
        return a


def sparse(x):
    raise NotImplementedError


def normal(m, n=1, mean=0.0, std=1.0):
    raise NotImplementedError


class _Printing(object):
    options = {'iformat': '% i', 'dformat': '% .2e', 'width': 7, 'height': -1}


printing = _Printing()


class _Blas(object):
    """The few BLAS-1/3 calls cspmatrix.spmatrix()/copy() make (offsets are
    linear column-major positions, as in cvxopt)."""

    @staticmethod
    def copy(x, y, n=None, offsetx=0, offsety=0):
        xf = x._flat()
        yf = y._a.reshape(-1, order='F').copy()
        if n is None:
            n = xf.size - offsetx
        yf[offsety:offsety + n] = xf[offsetx:offsetx + n]
        y._a = yf.reshape(y._a.shape, order='F')

    @staticmethod
    def scal(alpha, x, n=None, offset=0):
        xf = x._a.reshape(-1, order='F').copy()
        if n is None:
            n = xf.size - offset
        xf[offset:offset + n] *= alpha
        x._a = xf.reshape(x._a.shape, order='F')

    @staticmethod
    def axpy(x, y, alpha=1.0):
        y._a = y._a + alpha * x._a

    @staticmethod
    def dot(x, y):
        return float(_np.dot(x._flat(), y._flat()))

    @staticmethod
    def trmm(A, B, side='L', uplo='L', transA='N', diag='N', alpha=1.0, m=None, n=None,
             ldA=0, ldB=0, offsetA=0, offsetB=0):
        assert side == 'R' and uplo == 'L' and transA == 'N' and diag == 'N'
        af = A._flat()
        bf = B._a.reshape(-1, order='F').copy()
        Lk = _np.zeros((n, n))
        for j in range(n):
            for i in range(j, n):
                Lk[i, j] = af[offsetA + j * ldA + i]
        Bk = _np.zeros((m, n))
        for j in range(n):
            Bk[:, j] = bf[offsetB + j * ldB: offsetB + j * ldB + m]
        R = alpha * (Bk @ Lk)
        for j in range(n):
            bf[offsetB + j * ldB: offsetB + j * ldB + m] = R[:, j]
        B._a = bf.reshape(B._a.shape, order='F')


blas = _Blas()


class _Lapack(object):
    @staticmethod
    def lacpy(A, B, uplo='N'):
        a = A._a
        if uplo == 'L':
            B._a = _np.tril(a).copy()
        elif uplo == 'U':
            B._a = _np.triu(a).copy()
        else:
            B._a = a.copy()


lapack = _Lapack()


class _Amd(object):
    @staticmethod
    def order(A):
        raise NotImplementedError("cvxopt.amd is not available; pass an explicit permutation")


amd = _Amd()
