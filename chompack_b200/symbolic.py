"""Symbolic factorisation of a sparse symmetric pattern: the host side of the
multifrontal sweeps.

`symbolic(A, p=None, merge_function=None)` reproduces the reference's
`chompack.symbolic` (src/python/symbolic.py:499-890) array for array: the
same permutation composition, supernode partition, amalgamation, postorder
renumbering, relative indices, child lists, block pointers and workspace
sizes.  The per-step loops run in native code (chb_sym_* in
include/chompack_b200.h); index arrays are int64 numpy arrays.
"""
import numpy as np

from . import _native as N
from .sparse import as_spmatrix, symmetrize, spmatrix

__all__ = ["symbolic", "merge_size_fill", "peo"]


def _ccs_of(I, J, n):
    """CCS (colptr, rowidx) with rows sorted within columns."""
    key = J * n + I
    order = np.argsort(key, kind="stable")
    I = I[order]
    J = J[order]
    cp = np.zeros(n + 1, dtype=np.int64)
    np.add.at(cp, J + 1, 1)
    return np.ascontiguousarray(np.cumsum(cp)), np.ascontiguousarray(I.astype(np.int64))


def merge_size_fill(tsize=8, tfill=8):
    """Supernodal merge heuristic (symbolic.py:455-497).

    Returns a function that returns True if either (i) supernode k and its
    parent are both of size at most `tsize`, or (ii) merging them induces at
    most `tfill` lower-triangular nonzeros.
    """
    assert tsize >= 0, "tsize must be nonnegative"
    assert tfill >= 0, "tfill must be nonnegative"

    def fmerge(ccp, cck, np_, nk):
        fill = (ccp - (cck - nk)) * nk
        return fill <= tfill or (nk <= tsize and np_ <= tsize)

    fmerge.tsize = int(tsize)
    fmerge.tfill = int(tfill)
    fmerge.__doc__ = ("Supernodal merge heuristic: merge if both supernodes have order <= %i "
                      "or the merge induces at most %i edges." % (tsize, tfill))
    return fmerge


def peo(A, p):
    """True if p is a perfect elimination order of the pattern of A
    (symbolic.py:413-449)."""
    A = as_spmatrix(A)
    n = A.size[0]
    assert A.size[1] == n, "A must be a square matrix"
    p = np.asarray(list(p), dtype=np.int64)
    assert p.size == n, "length of p must be equal to the order of A"
    As = symmetrize(A)
    cp, ri, _ = As.CCS
    ip = np.empty(n, dtype=np.int64)
    ip[p] = np.arange(n)
    for k in range(n):
        v = p[k]
        r = set(int(rj) for rj in ri[cp[v]:cp[v + 1]] if ip[rj] > k)
        for rj in r:
            if not r.issubset(set(ri[cp[rj]:cp[rj + 1]].tolist())):
                return False
    return True


class symbolic(object):
    """Symbolic factorisation object (symbolic.py:499-890).

    :param A: sparse matrix (lower triangle used; diagonal must be present)
    :param p: permutation vector or ordering routine (optional)
    :param merge_function: merge heuristic f(|J_par|, |J_k|, |N_par|, |N_k|)
    """

    def __init__(self, A, p=None, merge_function=None, **kwargs):
        A = as_spmatrix(A)
        assert A.size[0] == A.size[1], "A must be a square matrix"
        supernodal = kwargs.get('supernodal', True)
        n = A.size[0]

        Ap = symmetrize(A)
        nnz_Ap = (len(Ap) + n) // 2
        assert int(np.count_nonzero(Ap._I == Ap._J)) == n, \
            "the sparsity pattern of A must include diagonal elements"

        if p is not None:
            if callable(p):
                p = p(Ap)
            p = np.asarray(list(p) if not isinstance(p, np.ndarray) else p, dtype=np.int64).reshape(-1)
            assert p.size == n, "length of permutation vector must be equal to the order of A"
            ip0 = np.empty(n, dtype=np.int64)
            ip0[p] = np.arange(n)
            I, J = ip0[Ap._I], ip0[Ap._J]
        else:
            I, J = Ap._I.copy(), Ap._J.copy()
        cp, ri = _ccs_of(I, J, n)

        par = np.empty(n, dtype=np.int64)
        N.check(N.sym_etree(n, N.ptr(cp), N.ptr(ri), N.ptr(par)), "etree")
        post = np.empty(n, dtype=np.int64)
        N.check(N.sym_post_order(n, N.ptr(par), N.ptr(post)), "post_order")
        colcount = np.empty(n, dtype=np.int64)
        N.check(N.sym_counts(n, N.ptr(cp), N.ptr(ri), N.ptr(par), N.ptr(post), N.ptr(colcount)), "counts")
        nnz_Ae = int(colcount.sum())

        if supernodal:
            snode = np.empty(n, dtype=np.int64)
            snptr = np.empty(n + 1, dtype=np.int64)
            snpar = np.empty(n, dtype=np.int64)
            nsn = np.zeros(1, dtype=np.int64)
            N.check(N.sym_supernodes(n, N.ptr(par), N.ptr(post), N.ptr(colcount), N.ptr(snode),
                                     N.ptr(snptr), N.ptr(snpar), N.ptr(nsn)), "supernodes")
            Ns = int(nsn[0])
            snptr = np.ascontiguousarray(snptr[:Ns + 1])
            snpar = np.ascontiguousarray(snpar[:Ns])
            snpost = np.empty(Ns, dtype=np.int64)
            N.check(N.sym_post_order(Ns, N.ptr(snpar), N.ptr(snpost)), "post_order")
        else:
            snpar, snpost = par, post
            snode = np.arange(n, dtype=np.int64)
            snptr = np.arange(n + 1, dtype=np.int64)
            Ns = n

        if merge_function:
            tsize = getattr(merge_function, "tsize", None)
            tfill = getattr(merge_function, "tfill", None)
            cb_keep = None
            if tsize is not None and tfill is not None:
                cb = N.MERGE_FN()
            else:
                def _cb(ccp, cck, np_, nk, _f=merge_function):
                    return 1 if _f(int(ccp), int(cck), int(np_), int(nk)) else 0
                cb = cb_keep = N.MERGE_FN(_cb)
                tsize, tfill = 0, 0
            nsn = np.array([Ns], dtype=np.int64)
            snpar = np.ascontiguousarray(snpar.copy())
            snpost_new = np.empty(Ns, dtype=np.int64)
            N.check(N.sym_amalgamate(n, N.ptr(colcount), N.ptr(snode), N.ptr(snptr), N.ptr(snpar),
                                     N.ptr(np.ascontiguousarray(snpost)), N.ptr(snpost_new), N.ptr(nsn),
                                     int(tsize), int(tfill), cb), "amalgamate")
            del cb_keep
            Ns = int(nsn[0])
            snptr = np.ascontiguousarray(snptr[:Ns + 1])
            snpar = np.ascontiguousarray(snpar[:Ns])
            snpost = np.ascontiguousarray(snpost_new[:Ns])

        # postorder renumbering: supernodes consecutive and in postorder
        # (symbolic.py:564-575)
        sizes = snptr[snpost + 1] - snptr[snpost]
        pp = np.concatenate([snode[snptr[k]:snptr[k + 1]] for k in snpost]) if Ns else np.zeros(0, np.int64)
        snptr2 = np.zeros(Ns + 1, dtype=np.int64)
        snptr2[1:] = np.cumsum(sizes)
        colcount = colcount[pp]
        snposti = np.empty(Ns, dtype=np.int64)
        snposti[snpost] = np.arange(Ns)
        snpar = snposti[snpar[snpost]]
        snode = np.arange(n, dtype=np.int64)
        snpost = np.arange(Ns, dtype=np.int64)
        snptr = snptr2

        # effective permutation and its inverse (symbolic.py:577-584)
        self._p = pp.copy() if p is None else p[pp]
        self._ip = np.empty(n, dtype=np.int64)
        self._ip[self._p] = np.arange(n)

        # permuted pattern, lower triangle, for the embedding
        ipp = np.empty(n, dtype=np.int64)
        ipp[pp] = np.arange(n)
        I2, J2 = ipp[I], ipp[J]
        lo = I2 >= J2
        cpl, ril = _ccs_of(I2[lo], J2[lo], n)

        sncolptr = np.empty(Ns + 1, dtype=np.int64)
        N.check(N.sym_embed(n, N.ptr(cpl), N.ptr(ril), N.ptr(colcount), N.ptr(snode), N.ptr(snptr),
                            N.ptr(snpar), N.ptr(snpost), Ns, N.ptr(sncolptr), None), "embed")
        snrowidx = np.empty(int(sncolptr[-1]), dtype=np.int64)
        N.check(N.sym_embed(n, N.ptr(cpl), N.ptr(ril), N.ptr(colcount), N.ptr(snode), N.ptr(snptr),
                            N.ptr(snpar), N.ptr(snpost), Ns, N.ptr(sncolptr), N.ptr(snrowidx)), "embed")
        relptr = np.empty(Ns + 1, dtype=np.int64)
        relidx = np.empty(int(sncolptr[-1]), dtype=np.int64)
        N.check(N.sym_relative_idx(Ns, N.ptr(sncolptr), N.ptr(snrowidx), N.ptr(snptr), N.ptr(snpar),
                                   N.ptr(relptr), N.ptr(relidx)), "relative_idx")
        relidx = np.ascontiguousarray(relidx[:relptr[-1]])

        # child lists (symbolic.py:587-604): children of each supernode in
        # increasing (postorder) index
        nonroot = snpar != np.arange(Ns)
        chcnt = np.bincount(snpar[nonroot], minlength=Ns)
        chptr = np.zeros(Ns + 1, dtype=np.int64)
        chptr[1:] = np.cumsum(chcnt)
        kids = np.nonzero(nonroot)[0]
        order = np.argsort(snpar[kids], kind="stable")
        chidx = kids[order].astype(np.int64)

        nn = snptr[1:] - snptr[:-1]
        na = relptr[1:] - relptr[:-1]
        nj = nn + na

        # stack statistics (symbolic.py:606-627 and :634-675)
        stack = []
        stack_mem_cur = 0
        stack_max = 0
        stack_size = 0
        frontal_max = 0
        stack_depth = 0
        stack_mem = 0
        stack_solve = 0
        stack_stmp = 0
        cln = 0
        for k in range(Ns):
            nnk, nak, njk = int(nn[k]), int(na[k]), int(nj[k])
            frontal_max = max(frontal_max, njk ** 2)
            cln = max(cln, njk)
            for _ in range(int(chptr[k + 1] - chptr[k])):
                v = stack.pop()
                stack_mem_cur -= v ** 2
                stack_stmp -= v
            if nak > 0:
                stack.append(nak)
                stack_mem_cur += nak ** 2
                stack_max = max(stack_max, stack_mem_cur)
                stack_size = max(stack_size, len(stack))
                stack_stmp += nak
                stack_solve = max(stack_solve, stack_stmp)
            stack_depth = max(stack_depth, len(stack))
        stack_mem = stack_max
        self.frontal_len = frontal_max
        self.stack_len = stack_max
        self.stack_size = stack_size

        blkptr = np.zeros(Ns + 1, dtype=np.int64)
        blkptr[1:] = np.cumsum(nn * (sncolptr[1:] - sncolptr[:-1]))

        self._clique_number = int(cln)
        self._n = n
        self._Nsn = Ns
        self._snode = snode
        self._snptr = snptr
        self._chptr = chptr
        self._chidx = chidx
        self._snpar = snpar
        self._snpost = snpost
        self._relptr = relptr
        self._relidx = relidx
        self._sncolptr = sncolptr
        self._snrowidx = snrowidx
        self._blkptr = blkptr
        self._nnz = int(np.sum(nn * (nn + 1) // 2 + nn * na))
        self._fill = (nnz_Ae - nnz_Ap, self._nnz - nnz_Ae)
        self._memory = {'stack_depth': stack_depth, 'stack_mem': stack_mem,
                        'frontal_mem': cln ** 2, 'stack_solve': stack_solve}
        self._plan = None

    # ---------------------------------------------------------------- repr
    def __repr__(self):
        return "<symbolic factorization, n=%i, nnz=%i, nsn=%i>" % (self.n, self.nnz, self.Nsn)

    def __str__(self):
        P = self.sparsity_pattern(reordered=True, symmetric=True).todense()
        return "\n".join("[" + " ".join("X" if v else " " for v in row) + "]" for row in P)

    def sparsity_pattern(self, reordered=True, symmetric=True):
        """Sparse matrix with the filled pattern (symbolic.py:703-714)."""
        from .cspmatrix import cspmatrix
        return cspmatrix(self, 1.0).spmatrix(reordered=reordered, symmetric=symmetric)

    # ---------------------------------------------------------- properties
    n = property(lambda self: self._n, doc="Number of nodes (matrix order)")
    Nsn = property(lambda self: self._Nsn, doc="Number of supernodes")
    snode = property(lambda self: self._snode, doc="Supernode array")
    snptr = property(lambda self: self._snptr, doc="Supernode pointer array")
    chptr = property(lambda self: self._chptr, doc="Pointer array associated with chidx")
    chidx = property(lambda self: self._chidx, doc="Children of each supernode")
    snpar = property(lambda self: self._snpar, doc="Supernode parent array (roots: snpar[k] == k)")
    snpost = property(lambda self: self._snpost, doc="Supernode post-ordering")
    relptr = property(lambda self: self._relptr, doc="Pointer array associated with relidx")
    relidx = property(lambda self: self._relidx, doc="Relative indices of update matrices in parent fronts")
    sncolptr = property(lambda self: self._sncolptr, doc="Pointer array associated with snrowidx")
    snrowidx = property(lambda self: self._snrowidx, doc="Row indices of the representative columns (cliques)")
    blkptr = property(lambda self: self._blkptr, doc="Pointer array for block storage")
    fill = property(lambda self: self._fill, doc="(fill from symbolic factorization, fill from amalgamation)")
    nnz = property(lambda self: self._nnz, doc="Number of lower-triangular nonzeros")
    p = property(lambda self: self._p, doc="Permutation vector")
    ip = property(lambda self: self._ip, doc="Inverse permutation vector")
    memory = property(lambda self: self._memory)
    clique_number = property(lambda self: self._clique_number, doc="Order of the largest clique")

    def cliques(self, reordered=True):
        rows = self._snrowidx if reordered else self._p[self._snrowidx]
        return [rows[self._sncolptr[k]:self._sncolptr[k + 1]].tolist() for k in range(self._Nsn)]

    def separators(self, reordered=True):
        rows = self._snrowidx if reordered else self._p[self._snrowidx]
        return [rows[self._sncolptr[k] + self._snptr[k + 1] - self._snptr[k]:self._sncolptr[k + 1]].tolist()
                for k in range(self._Nsn)]

    def supernodes(self, reordered=True):
        nodes = self._snode if reordered else self._p[self._snode]
        return [nodes[self._snptr[k]:self._snptr[k + 1]].tolist() for k in range(self._Nsn)]

    def parent(self):
        return self._snpar.tolist()

    # ------------------------------------------------------------ device
    def plan(self, device=None):
        """Device plan for this factorisation (uploaded once, then cached)."""
        from .plan import Plan
        if self._plan is None or (device is not None and self._plan.device != device):
            self._plan = Plan(self, device)
        return self._plan
