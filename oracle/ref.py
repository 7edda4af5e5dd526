"""ctypes driver of the reference's own numeric C kernels, compiled unchanged
into oracle/_ref/libchompack_ref.so by oracle/Makefile.

TEST INFRASTRUCTURE (the checker): only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference legs use this module.  It marshals the
symbolic arrays and workspaces exactly as the reference's CPython wrapper
does (src/C/cbase.c: cchol :187-284, cllt :298-390, cprojected_inverse
:404-500, ccompletion :521-621, chessian :675-857, ctrsm :965-1077, cdot
:106-174): int_t is Py_ssize_t (int64), workspaces are sized from
symb.memory, and the U list of hessian is NULL-terminated.

All arrays are numpy; `symb` is any object with the reference's symbolic
attributes (chompack_b200.symbolic qualifies: its arrays are bit-identical).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libchompack_ref.so")

_lib = None


def available():
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("reference kernels not built (make -C oracle ref)")
        _lib = ctypes.CDLL(LIB)
        P = ctypes.POINTER
        i64, dbl = ctypes.c_int64, ctypes.c_double
        pi, pd = P(i64), P(dbl)
        sweep = [i64, i64, pi, pi, pi, pi, pi, pi, pi, pd, pd, pd, pi]
        _lib.cholesky.argtypes = sweep
        _lib.cholesky.restype = ctypes.c_int
        _lib.llt.argtypes = sweep
        _lib.llt.restype = None
        _lib.projected_inverse.argtypes = sweep
        _lib.projected_inverse.restype = ctypes.c_int
        _lib.completion.argtypes = sweep + [ctypes.c_int]
        _lib.completion.restype = ctypes.c_int
        _lib.hessian.argtypes = [i64, i64, pi, pi, pi, pi, pi, pi, pi, pd, pd, P(pd), pd, pd, pi,
                                 ctypes.c_int, ctypes.c_int, ctypes.c_int]
        _lib.hessian.restype = ctypes.c_int
        _lib.trsm.argtypes = [ctypes.c_char, ctypes.c_int, dbl, i64, i64, pi, pi, pi, pi, pi, pi, pi, pi, pi, pd,
                              pd, P(ctypes.c_int), pd, pd, pi]
        _lib.trsm.restype = None
        _lib.dot.argtypes = [pi, pi, pi, pi, pd, pd]
        _lib.dot.restype = dbl
        ci = P(ctypes.c_int)
        _lib.dpftrf.argtypes = [ci, ci, pd, pd, ci, pd, ci, pd, ci]
        _lib.dpftrf.restype = ctypes.c_int
        for f in (_lib.dpfsv, _lib.dpfmv):
            f.argtypes = [ci, ci, ctypes.c_char_p, pd, ci, pd, ci, pd, ci, pd]
            f.restype = None
    return _lib


def _i(a):
    a = np.ascontiguousarray(a, dtype=np.int64)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))


def _d(a):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class _Sym(object):
    """int64 views of the symbolic arrays, kept alive for the call."""

    def __init__(self, symb):
        self.n = int(symb.n)
        self.nsn = int(symb.Nsn)
        self.keep = []
        for name in ("snpost", "snptr", "relptr", "relidx", "chptr", "chidx", "blkptr", "snode", "p", "sncolptr"):
            arr, ptr = _i(np.asarray(getattr(symb, name)))
            self.keep.append(arr)
            setattr(self, name, ptr)
        mem = symb.memory
        self.stack_depth = int(mem["stack_depth"])
        self.stack_mem = int(mem["stack_mem"])
        self.frontal_mem = int(mem["frontal_mem"])
        self.stack_solve = int(mem["stack_solve"])
        self.clique_number = int(symb.clique_number)

    def ws(self):
        upd = np.zeros(max(self.stack_mem, 1))
        fws = np.zeros(max(self.frontal_mem, 1))
        usz = np.zeros(max(self.stack_depth, 1), dtype=np.int64)
        self.keep += [upd, fws, usz]
        return _d(fws), _d(upd), usz.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))

    def common(self):
        return (self.n, self.nsn, self.snpost, self.snptr, self.relptr, self.relidx, self.chptr, self.chidx,
                self.blkptr)


def cholesky(symb, blkval):
    """In-place reference cholesky on a float64 numpy blkval; returns info."""
    s = _Sym(symb)
    fws, upd, usz = s.ws()
    return lib().cholesky(*s.common(), _d(blkval), fws, upd, usz)


def llt(symb, blkval):
    s = _Sym(symb)
    fws, upd, usz = s.ws()
    lib().llt(*s.common(), _d(blkval), fws, upd, usz)
    return 0


def projected_inverse(symb, blkval):
    s = _Sym(symb)
    fws, upd, usz = s.ws()
    return lib().projected_inverse(*s.common(), _d(blkval), fws, upd, usz)


def completion(symb, blkval, factored_updates=True):
    s = _Sym(symb)
    fws, upd, usz = s.ws()
    return lib().completion(*s.common(), _d(blkval), fws, upd, usz, 1 if factored_updates else 0)


def hessian(symb, lblkval, yblkval, ublkvals, adj=False, inv=False, factored_updates=True):
    """Reference hessian on a list of U blkvals (each updated in place).
    adj=None applies the full Hessian: two passes with adj toggled, as
    cbase.c:833-841 does."""
    s = _Sym(symb)
    fws, upd, usz = s.ws()
    ptrs = (ctypes.POINTER(ctypes.c_double) * (len(ublkvals) + 1))()
    for i, u in enumerate(ublkvals):
        ptrs[i] = _d(u)
    ptrs[len(ublkvals)] = ctypes.POINTER(ctypes.c_double)()
    inv_i = 1 if inv else 0
    adj_i = inv_i if adj is None else (1 if adj else 0)
    fu = 1 if factored_updates else 0
    info = lib().hessian(*s.common(), _d(lblkval), _d(yblkval), ptrs, fws, upd, usz, inv_i, adj_i, fu)
    if adj is None:
        info = lib().hessian(*s.common(), _d(lblkval), _d(yblkval), ptrs, fws, upd, usz, inv_i, 1 ^ adj_i, fu)
    return info


def trsm(symb, blkval, B, alpha=1.0, trans='N', nrhs=None, offsetB=0, ldB=None):
    """Reference trsm on a column-major numpy B (flattened, Fortran order)."""
    s = _Sym(symb)
    Bf = B if B.ndim == 1 else None
    if Bf is None:
        assert B.flags["F_CONTIGUOUS"]
        rows, cols = B.shape
        Bf = B.reshape(-1, order="F")
    else:
        rows, cols = B.size, 1
    if nrhs is None:
        nrhs = cols
    if ldB is None:
        ldB = rows
    upd = np.zeros(max(s.stack_solve * nrhs, 1))
    fws = np.zeros(max(s.clique_number * nrhs, 1))
    usz = np.zeros(max(s.stack_depth, 1), dtype=np.int64)
    lda = ctypes.c_int(ldB)
    base = Bf.ctypes.data + 8 * offsetB
    lib().trsm(trans.encode(), nrhs, alpha, s.n, s.nsn, s.snpost, s.snptr, s.snode, s.relptr, s.relidx,
               s.chptr, s.chidx, s.blkptr, s.p, _d(blkval), ctypes.cast(base, ctypes.POINTER(ctypes.c_double)),
               ctypes.byref(lda), _d(fws), _d(upd), usz.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
    return B


def dot(symb, x, y):
    s = _Sym(symb)
    nsn = ctypes.c_int64(s.nsn)
    return lib().dot(ctypes.byref(nsn), s.snptr, s.sncolptr, s.blkptr, _d(x), _d(y))


def set_threads(n):
    """Thread count of the OpenBLAS the reference kernels are linked against."""
    lib()
    import glob
    import scipy
    d = os.path.realpath(os.path.join(os.path.dirname(scipy.__file__), "..", "scipy.libs"))
    for f in glob.glob(os.path.join(d, "libscipy_openblas*.so")):
        ob = ctypes.CDLL(f)
        if hasattr(ob, "scipy_openblas_set_num_threads"):
            ob.scipy_openblas_set_num_threads(int(n))
            return True
    return False


# Product-form factor of I + V diag(a) V^T (pfcholesky.c:52-136, called by
# pfcholesky.py:113-211 as pfchol / pftrsm / pftrmm).  V, L, B are n x k
# Fortran-ordered float64 arrays; V is overwritten as dpftrf does.

def _ci(v):
    return ctypes.byref(ctypes.c_int(int(v)))


def _dF(a):
    assert a.dtype == np.float64 and a.flags["F_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def pfchol(a, V):
    """Returns (L, B, info) of dpftrf on V (modified in place)."""
    assert V.flags["F_CONTIGUOUS"] and V.dtype == np.float64
    n, k = V.shape
    L = np.zeros((n, k), order="F")
    B = np.zeros((n, k), order="F")
    a = np.ascontiguousarray(a, dtype=np.float64)
    info = lib().dpftrf(_ci(n), _ci(k), _d(a), _dF(V), _ci(n), _dF(L), _ci(n), _dF(B), _ci(n))
    return L, B, info


def _pf_columns(fn, V, L, B, U, trans):
    assert U.flags["F_CONTIGUOUS"] and U.dtype == np.float64
    n, k = V.shape
    U2 = U.reshape(n, -1, order="F")
    for j in range(U2.shape[1]):
        col = np.ascontiguousarray(U2[:, j])
        fn(_ci(n), _ci(k), trans.encode(), _dF(V), _ci(n), _dF(L), _ci(n), _dF(B), _ci(n), _d(col))
        U2[:, j] = col
    return U


def pftrsm(V, L, B, U, trans='N'):
    """U := (L_1 ... L_k)^{-1} U ('N') or (L_k^T ... L_1^T)^{-1} U ('T')."""
    return _pf_columns(lib().dpfsv, V, L, B, U, trans)


def pftrmm(V, L, B, U, trans='N'):
    """U := L_1 ... L_k U ('N') or L_k^T ... L_1^T U ('T')."""
    return _pf_columns(lib().dpfmv, V, L, B, U, trans)
