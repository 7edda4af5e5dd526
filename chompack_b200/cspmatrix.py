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

    def add_projection(self, A, alpha=1.0, beta=1.0, reordered=False):
        """X := alpha*proj(A) + beta*X for a dense symmetric A
        (symbolic.py:1176-1210)."""
        assert self.is_factor is False, "cannot project matrix onto a cspmatrix factor"
        s = self.symb
        A = np.asarray(A.cpu().numpy() if isinstance(A, torch.Tensor) else A, dtype=np.float64)
        if not reordered:
            At = np.tril(A)
            At = At + At.T
            At[np.diag_indices_from(At)] *= 0.5
            A = At[np.ix_(s.p, s.p)]
        host = self.blkval.detach().to("cpu").numpy().copy()
        for k in range(s.Nsn):
            rows = s.snrowidx[s.sncolptr[k]:s.sncolptr[k + 1]]
            cols = s.snode[s.snptr[k]:s.snptr[k + 1]]
            blk = A[np.ix_(rows, cols)].reshape(-1, order="F")
            host[s.blkptr[k]:s.blkptr[k + 1]] = beta * host[s.blkptr[k]:s.blkptr[k + 1]] + alpha * blk
        self.blkval.copy_(torch.from_numpy(host))

    def _lower_entries(self, blk):
        """(I, J, V) of the reordered lower triangle stored in blk (host)."""
        s = self.symb
        Is, Js, Vs = [], [], []
        nn = np.diff(s.snptr)
        for k in range(s.Nsn):
            nj = int(s.sncolptr[k + 1] - s.sncolptr[k])
            rows = s.snrowidx[s.sncolptr[k]:s.sncolptr[k + 1]]
            b = blk[s.blkptr[k]:s.blkptr[k + 1]].reshape((nj, int(nn[k])), order="F")
            for i in range(int(nn[k])):
                Is.append(rows[i:])
                Js.append(np.full(nj - i, s.snptr[k] + i, dtype=np.int64))
                Vs.append(b[i:, i])
        if not Is:
            z = np.zeros(0, dtype=np.int64)
            return z, z, np.zeros(0)
        return np.concatenate(Is), np.concatenate(Js), np.concatenate(Vs)

    def spmatrix(self, reordered=True, symmetric=False):
        """Convert to a sparse matrix (symbolic.py:1032-1111).  For a factor
        the off-diagonal blocks are multiplied back by L_kk to give the
        conventional lower-triangular factor; only the default options are
        allowed then."""
        s = self.symb
        blk = self.blkval.detach().to("cpu").numpy().copy()
        if self.is_factor:
            if symmetric:
                raise ValueError("'symmetric = True' not implemented for Cholesky factors")
            if not reordered:
                raise ValueError("'reordered = False' not implemented for Cholesky factors")
            for k in range(s.Nsn):
                nn = int(s.snptr[k + 1] - s.snptr[k])
                na = int(s.relptr[k + 1] - s.relptr[k])
                if na == 0:
                    continue
                nj = nn + na
                b = blk[s.blkptr[k]:s.blkptr[k + 1]].reshape((nj, nn), order="F").copy()
                Lkk = np.tril(b[:nn, :nn])
                b[nn:, :] = b[nn:, :] @ Lkk
                blk[s.blkptr[k]:s.blkptr[k + 1]] = b.reshape(-1, order="F")
        I, J, V = self._lower_entries(blk)
        tmp = spmatrix(V, I, J, (s.n, s.n))
        if reordered:
            return symmetrize(tmp) if symmetric else tmp
        p = s.p
        full = symmetrize(tmp)
        out = spmatrix(full._V, p[full._I], p[full._J], (s.n, s.n))
        return out if symmetric else tril(out)

    def diag(self, reordered=True):
        """Diagonal entries (symbolic.py:1113-1128), as a numpy array."""
        s = self.symb
        blk = self.blkval.detach().to("cpu").numpy()
        D = np.zeros(s.n)
        for k in range(s.Nsn):
            nn = int(s.snptr[k + 1] - s.snptr[k])
            w = int(s.sncolptr[k + 1] - s.sncolptr[k])
            for i in range(nn):
                D[s.snode[s.snptr[k] + i]] = blk[s.blkptr[k] + i * w + i]
        return D if reordered else D[s.ip]
