"""Chordal sparse matrix in the reference's block storage, with the values in
a torch float64 tensor (normally on the GPU).

Layout (symbolic.py:1087-1094): supernode k owns
`blkval[blkptr[k] : blkptr[k] + nj*nn]`, an nj x nn column-major block
(leading dimension nj) whose rows are the clique
`snrowidx[sncolptr[k]:sncolptr[k+1]]`, supernode rows first; only the lower
trapezoid is meaningful.  After `cholesky` the diagonal block holds L_kk and
the off-diagonal block holds L_{Ak,Nk} L_kk^{-1} (cholesky.c:72).
"""
import numpy as np
import torch

from .sparse import as_spmatrix, spmatrix, symmetrize, tril

__all__ = ["cspmatrix"]


def _symbolic_arrays(symb, dev):
    """sncolptr / snrowidx of a symbolic factorisation on a device (cached)."""
    cache = symb.__dict__.setdefault("_sym_dev", {})
    key = str(dev)
    if key not in cache:
        cache[key] = (torch.as_tensor(np.asarray(symb.sncolptr), dtype=torch.int64).to(dev),
                      torch.as_tensor(np.asarray(symb.snrowidx), dtype=torch.int64).to(dev))
    return cache[key]


def _default_device():
    return torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else torch.device("cpu")


class cspmatrix(object):
    """Chordal sparse matrix (symbolic.py:892-943).

    :param symb:   symbolic factorisation
    :param blkval: optional values: a float (fill), or a 1-D float64 tensor /
                   array of length symb.blkptr[-1] (tensors are used, not copied)
    :param factor: True if the values represent a Cholesky factor
    :param device: torch device for a newly created value array
    """

    def __init__(self, symb, blkval=None, factor=False, device=None):
        from .symbolic import symbolic
        assert isinstance(symb, symbolic), "symb must be an instance of symbolic"
        self._is_factor = factor
        self.symb = symb
        L = int(symb.blkptr[-1])
        dev = torch.device(device) if device is not None else _default_device()
        if blkval is None:
            self.blkval = torch.zeros(L, dtype=torch.float64, device=dev)
        elif isinstance(blkval, float):
            self.blkval = torch.full((L,), blkval, dtype=torch.float64, device=dev)
        elif isinstance(blkval, torch.Tensor):
            assert blkval.numel() == L, "dimension mismatch: length of blkval is incorrect"
            assert blkval.dtype == torch.float64, "blkval must be float64"
            self.blkval = blkval
        else:
            arr = np.asarray(blkval, dtype=np.float64).reshape(-1)
            assert arr.size == L, "dimension mismatch: length of blkval is incorrect"
            self.blkval = torch.from_numpy(arr.copy()).to(dev)

    # ------------------------------------------------------------- basics
    def __repr__(self):
        kind = "chordal sparse matrix (factor)" if self.is_factor else "chordal sparse matrix"
        return "<%ix%i %s, tc='d', nnz=%i, nsn=%i>" % (self.symb.n, self.symb.n, kind, self.symb.nnz,
                                                       self.symb.Nsn)

    def __str__(self):
        return str(self.spmatrix(reordered=True, symmetric=False).todense())

    @property
    def is_factor(self):
        return self._is_factor

    @is_factor.setter
    def is_factor(self, value):
        self._is_factor = value

    @property
    def size(self):
        return (self.symb.n, self.symb.n)

    @property
    def device(self):
        return self.blkval.device

    def copy(self):
        """New cspmatrix on the same symbolic object with a copy of the values."""
        return cspmatrix(self.symb, blkval=self.blkval.clone(), factor=self.is_factor)

    def to(self, device):
        return cspmatrix(self.symb, blkval=self.blkval.to(device), factor=self.is_factor)

    # --------------------------------------------------------- arithmetic
    def __iadd__(self, B):
        assert self.is_factor is False, "Addition of cspmatrix factors not supported"
        if isinstance(B, cspmatrix):
            assert self.symb is B.symb, "Symbolic factorization mismatch"
            assert B.is_factor is False, "Addition of cspmatrix factors not supported"
            self.blkval.add_(B.blkval.to(self.blkval.device))
        else:
            self._iadd_spmatrix(B)
        return self

    def __isub__(self, B):
        assert self.is_factor is False, "Addition of cspmatrix factors not supported"
        if isinstance(B, cspmatrix):
            assert self.symb is B.symb, "Symbolic factorization mismatch"
            assert B.is_factor is False, "Addition of cspmatrix factors not supported"
            self.blkval.sub_(B.blkval.to(self.blkval.device))
        else:
            self._iadd_spmatrix(B, alpha=-1.0)
        return self

    def __add__(self, B):
        C = self.copy()
        C += B
        return C

    def __sub__(self, B):
        C = self.copy()
        C -= B
        return C

    def __imul__(self, a):
        if isinstance(a, (int, float)):
            self.blkval.mul_(float(a))
        else:
            raise NotImplementedError("only scalar multiplication has been implemented")
        return self

    def __mul__(self, a):
        ret = self.copy()
        ret *= a
        return ret

    def __rmul__(self, a):
        return self.__mul__(a)

    # ------------------------------------------------------ host indexing
    def _entry_index(self, I, J):
        """Positions in blkval of reordered lower entries (I >= J)."""
        s = self.symb
        n = s.n
        sn_of = np.repeat(np.arange(s.Nsn, dtype=np.int64), np.diff(s.snptr))
        k = sn_of[J]
        seg_owner = np.repeat(np.arange(s.Nsn, dtype=np.int64), np.diff(s.sncolptr))
        comb = seg_owner * (n + 1) + s.snrowidx
        q = np.searchsorted(comb, k * (n + 1) + I)
        ok = (q < comb.size)
        ok &= comb[np.minimum(q, comb.size - 1)] == k * (n + 1) + I
        if not np.all(ok):
            raise ValueError("sparse matrix entry outside the chordal pattern")
        pos = q - s.sncolptr[k]
        nj = s.sncolptr[k + 1] - s.sncolptr[k]
        return s.blkptr[k] + nj * (J - s.snptr[k]) + pos

    def _iadd_spmatrix(self, X, alpha=1.0):
        """Add a sparse matrix (lower triangle used) to the values
        (symbolic.py:1138-1174)."""
        assert self.is_factor is False, "cannot add spmatrix to a cspmatrix factor"
        X = as_spmatrix(X)
        if X.size[0] != self.symb.n or X.size[1] != self.symb.n:
            raise ValueError("sparse matrix must be of order n")
        if self.blkval.device.type == "cuda":
            return self._iadd_spmatrix_device(X, alpha)
        Xs = symmetrize(X)
        ip = self.symb.ip
        I, J, V = ip[Xs._I], ip[Xs._J], Xs._V
        lo = I >= J
        I, J, V = I[lo], J[lo], V[lo]
        idx = self._entry_index(I, J)
        # one entry per position (spmatrix sums duplicates; of (i, j) and
        # (j, i) only one is in the permuted lower triangle), added in place
        # where the values live: no copy of blkval through the host
        dev = self.blkval.device
        self.blkval.index_add_(0, torch.from_numpy(np.ascontiguousarray(idx, dtype=np.int64)).to(dev),
                               torch.from_numpy(np.ascontiguousarray(alpha * V, dtype=np.float64)).to(dev))

    def _iadd_spmatrix_device(self, X, alpha):
        """The same addition on the device (chb_add_sparse): the triplets of
        X's lower triangle are copied over and placed by one thread each."""
        from . import _native as N
        s = self.symb
        dev = self.blkval.device
        lo = X._I >= X._J
        I = torch.from_numpy(np.ascontiguousarray(X._I[lo], dtype=np.int64)).to(dev)
        J = torch.from_numpy(np.ascontiguousarray(X._J[lo], dtype=np.int64)).to(dev)
        V = torch.from_numpy(np.ascontiguousarray(X._V[lo], dtype=np.float64)).to(dev)
        colptr, rowidx = _symbolic_arrays(s, dev)
        bad = torch.zeros(1, dtype=torch.int64, device=dev)
        plan = s.plan(dev.index)
        rc = N.add_sparse(plan.handle, self.blkval.data_ptr(), colptr.data_ptr(), rowidx.data_ptr(), int(I.numel()),
                          I.data_ptr(), J.data_ptr(), V.data_ptr(), float(alpha), 0, bad.data_ptr(),
                          torch.cuda.current_stream(dev).cuda_stream)
        if rc < 0:
            raise RuntimeError("add_sparse failed: %s" % N.last_error().decode())
        if int(bad.item()) != 0:
            raise ValueError("sparse matrix entry outside the chordal pattern")

    def add_projection(self, A, alpha=1.0, beta=1.0, reordered=False):
        """X := alpha*proj(A) + beta*X for a dense symmetric A
        (symbolic.py:1176-1210), on the values' device (chb_add_projection):
        every entry of every block is updated; with reordered=False the
        symmetric matrix of A's lower triangle is read through p."""
        assert self.is_factor is False, "cannot project matrix onto a cspmatrix factor"
        from . import _native as N
        from . import cbase
        s = self.symb
        v = cbase._values(self)
        dev = v.device
        At = A if isinstance(A, torch.Tensor) else torch.from_numpy(np.asarray(A, dtype=np.float64))
        At = At.to(device=dev, dtype=torch.float64)
        if At.dim() != 2 or tuple(At.shape) != (s.n, s.n):
            raise ValueError("A must be a dense %d x %d matrix" % (s.n, s.n))
        Acm = At.t().contiguous()                      # column-major storage of A
        colptr, rowidx = _symbolic_arrays(s, dev)
        plan = s.plan(dev.index)
        rc = N.add_projection(plan.handle, v.data_ptr(), colptr.data_ptr(), rowidx.data_ptr(), Acm.data_ptr(), s.n,
                              float(alpha), float(beta), 0 if reordered else 1, torch.cuda.current_stream(dev).cuda_stream)
        if rc < 0:
            raise RuntimeError("add_projection failed: %s" % N.last_error().decode())
        cbase._write_back(self)

    def _ccs(self, values):
        """(colptr, row indices, values) of the lower trapezoid of the blocks
        in compressed-column order (reordered numbering), gathered on the
        device (chb_lower_ccs); the symbolic parts are cached on symb."""
        from . import _native as N
        s = self.symb
        dev = values.device
        cache = s.__dict__.setdefault("_ccs_cache", {})
        key = str(dev)
        nn = np.diff(np.asarray(s.snptr))
        nj = np.diff(np.asarray(s.sncolptr))
        if key not in cache:
            # column j = snptr[k] + i holds nj_k - i entries
            cc = np.repeat(nj, nn) - (np.arange(s.n) - np.repeat(np.asarray(s.snptr)[:-1], nn))
            cp = np.concatenate([[0], np.cumsum(cc)]).astype(np.int64)
            cache[key] = [torch.from_numpy(cp).to(dev), cp, None]
        cp_d, cp, rows = cache[key]
        sncolptr, snrowidx = _symbolic_arrays(s, dev)
        vals = torch.empty(int(cp[-1]), dtype=torch.float64, device=dev)
        ri = torch.empty(int(cp[-1]), dtype=torch.int64, device=dev) if rows is None else None
        plan = s.plan(dev.index)
        rc = N.lower_ccs(plan.handle, values.data_ptr(), sncolptr.data_ptr(), snrowidx.data_ptr(), cp_d.data_ptr(),
                         vals.data_ptr(), None if ri is None else ri.data_ptr(), torch.cuda.current_stream(dev).cuda_stream)
        if rc < 0:
            raise RuntimeError("lower_ccs failed: %s" % N.last_error().decode())
        if rows is None:
            rows = ri.cpu().numpy()
            cache[key][2] = rows
        return cp, rows, vals.cpu().numpy()

    def spmatrix(self, reordered=True, symmetric=False):
        """Convert to a sparse matrix (symbolic.py:1032-1111).  For a factor
        the off-diagonal blocks are multiplied back by L_kk on the device
        (chb_factor_conventional) to give the conventional lower-triangular
        factor; only the default options are allowed then.  The lower
        trapezoid is gathered on the device (chb_lower_ccs) and only the
        nonzeros cross to the host."""
        from . import _native as N
        from . import cbase
        s = self.symb
        if self.is_factor:
            if symmetric:
                raise ValueError("'symmetric = True' not implemented for Cholesky factors")
            if not reordered:
                raise ValueError("'reordered = False' not implemented for Cholesky factors")
        v = cbase._values(self, "L" if self.is_factor else "X")
        if self.is_factor:
            v = v.clone()
            plan = s.plan(v.device.index)
            cbase._run_and_status(plan, N.OP_CONVENTIONAL,
                                  lambda ws, nb, st: N.factor_conventional(plan.handle, v.data_ptr(), ws, nb, st))
        cp, I, V = self._ccs(v)
        J = np.repeat(np.arange(s.n, dtype=np.int64), np.diff(cp))
        tmp = spmatrix(V, I, J, (s.n, s.n))
        if reordered:
            return symmetrize(tmp) if symmetric else tmp
        p = s.p
        full = symmetrize(tmp)
        out = spmatrix(full._V, p[full._I], p[full._J], (s.n, s.n))
        return out if symmetric else tril(out)

    def diag(self, reordered=True):
        """Diagonal entries (symbolic.py:1113-1128), gathered on the device
        (chb_diag), as a numpy array."""
        from . import _native as N
        from . import cbase
        s = self.symb
        v = cbase._values(self, "L" if self.is_factor else "X")
        dev = v.device
        d = torch.empty(s.n, dtype=torch.float64, device=dev)
        rc = N.diag(s.plan(dev.index).handle, v.data_ptr(), d.data_ptr(), torch.cuda.current_stream(dev).cuda_stream)
        if rc < 0:
            raise RuntimeError("diag failed: %s" % N.last_error().decode())
        D = d.cpu().numpy()
        return D if reordered else D[s.ip]
