"""ctypes driver of oracle/liboracle.so, our plain-C restatement of the
reference's numeric sweeps (oracle/oracle.c).  TEST INFRASTRUCTURE ONLY: the
checker used by tests/, never by the product.  Same calling convention as
oracle/ref.py (numpy arrays; `symb` with the reference's attributes)."""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
_lib = None


def available():
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(LIB)
        P = ctypes.POINTER
        i64, pi, pd = ctypes.c_int64, P(ctypes.c_int64), P(ctypes.c_double)
        sweep = [i64, i64, pi, pi, pi, pi, pi, pi, pi, pd, pd, pd, pi]
        _lib.orc_cholesky.argtypes = sweep
        _lib.orc_cholesky.restype = ctypes.c_int
        _lib.orc_llt.argtypes = sweep
        _lib.orc_llt.restype = None
        _lib.orc_projected_inverse.argtypes = sweep
        _lib.orc_projected_inverse.restype = ctypes.c_int
        _lib.orc_completion.argtypes = sweep + [ctypes.c_int]
        _lib.orc_completion.restype = ctypes.c_int
        _lib.orc_hessian.argtypes = [i64, i64, pi, pi, pi, pi, pi, pi, pi, pd, pd, P(pd), i64, pd, pd, pi,
                                     ctypes.c_int, ctypes.c_int, ctypes.c_int]
        _lib.orc_hessian.restype = ctypes.c_int
        _lib.orc_trsm.argtypes = [ctypes.c_char, ctypes.c_int, ctypes.c_double, i64, i64, pi, pi, pi, pi, pi, pi,
                                  pi, pi, pi, pd, pd, ctypes.c_int, pd, pd, pi]
        _lib.orc_trsm.restype = None
        _lib.orc_dot.argtypes = [i64, pi, pi, pi, pd, pd]
        _lib.orc_dot.restype = ctypes.c_double
    return _lib


def _i(a):
    a = np.ascontiguousarray(a, dtype=np.int64)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))


def _d(a):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _common(symb, keep):
    out = [int(symb.n), int(symb.Nsn)]
    for name in ("snpost", "snptr", "relptr", "relidx", "chptr", "chidx", "blkptr"):
        arr, ptr = _i(np.asarray(getattr(symb, name)))
        keep.append(arr)
        out.append(ptr)
    return out


def _ws(symb, keep):
    mem = symb.memory
    upd = np.zeros(max(int(mem["stack_mem"]), 1))
    fws = np.zeros(max(int(mem["frontal_mem"]), 1))
    usz = np.zeros(max(int(mem["stack_depth"]), 1), dtype=np.int64)
    keep += [upd, fws, usz]
    return _d(fws), _d(upd), usz.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))


def cholesky(symb, blkval):
    keep = []
    return lib().orc_cholesky(*_common(symb, keep), _d(blkval), *_ws(symb, keep))


def llt(symb, blkval):
    keep = []
    lib().orc_llt(*_common(symb, keep), _d(blkval), *_ws(symb, keep))
    return 0


def projected_inverse(symb, blkval):
    keep = []
    return lib().orc_projected_inverse(*_common(symb, keep), _d(blkval), *_ws(symb, keep))


def completion(symb, blkval, factored_updates=True):
    keep = []
    return lib().orc_completion(*_common(symb, keep), _d(blkval), *_ws(symb, keep), 1 if factored_updates else 0)


def hessian(symb, lblkval, yblkval, ublkvals, adj=False, inv=False, factored_updates=True):
    """U := the Hessian factor selected by adj/inv, on a list of blkvals in
    place; adj=None applies both (adj = inv first, then toggled), as the
    reference's wrapper does (cbase.c:706-713, :833-841)."""
    keep = []
    ptrs = (ctypes.POINTER(ctypes.c_double) * max(len(ublkvals), 1))()
    for i, u in enumerate(ublkvals):
        ptrs[i] = _d(u)
    inv_i = 1 if inv else 0
    adj_i = inv_i if adj is None else (1 if adj else 0)
    fu = 1 if factored_updates else 0
    passes = [adj_i, 1 ^ adj_i] if adj is None else [adj_i]
    info = 0
    for a in passes:
        ws = _ws(symb, keep)
        info |= lib().orc_hessian(*_common(symb, keep), _d(lblkval), _d(yblkval), ptrs, len(ublkvals), *ws,
                                  inv_i, a, fu)
    return info


def trsm(symb, blkval, B, alpha=1.0, trans='N'):
    """B (Fortran-ordered n x nrhs numpy array) := alpha L^{-1} B or alpha L^{-T} B."""
    keep = []
    assert B.flags["F_CONTIGUOUS"] and B.dtype == np.float64
    rows, nrhs = (B.shape[0], 1) if B.ndim == 1 else B.shape
    Bf = B.reshape(-1, order="F")
    com = _common(symb, keep)
    snode, psnode = _i(np.asarray(symb.snode))
    p, pp = _i(np.asarray(symb.p))
    keep += [snode, p]
    mem = symb.memory
    fws = np.zeros(max(int(symb.clique_number) * nrhs, 1))
    upd = np.zeros(max(int(mem["stack_solve"]) * nrhs, 1))
    usz = np.zeros(max(int(mem["stack_depth"]), 1), dtype=np.int64)
    keep += [fws, upd, usz]
    lib().orc_trsm(trans.encode(), int(nrhs), float(alpha), com[0], com[1], com[2], com[3], psnode, com[4], com[5],
                   com[6], com[7], com[8], pp, _d(np.ascontiguousarray(blkval)), Bf.ctypes.data_as(
                       ctypes.POINTER(ctypes.c_double)), int(rows), _d(fws), _d(upd),
                   usz.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))


def dot(symb, x, y):
    keep = []
    a = [_i(np.asarray(getattr(symb, nm))) for nm in ("snptr", "sncolptr", "blkptr")]
    keep += [t[0] for t in a]
    return lib().orc_dot(int(symb.Nsn), a[0][1], a[1][1], a[2][1], _d(x), _d(y))
