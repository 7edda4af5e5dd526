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
        _lib.orc_cholesky.argtypes = [i64, i64, pi, pi, pi, pi, pi, pi, pi, pd, pd, pd, pi]
        _lib.orc_cholesky.restype = ctypes.c_int
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
