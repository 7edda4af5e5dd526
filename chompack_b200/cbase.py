"""Drop-in numeric sweeps with the signatures, defaults and exceptions of the
reference's `chompack.cbase` (src/C/cbase.c), running on the GPU through the
C ABI of include/chompack_b200.h.

Each call uploads nothing but what changed: the symbolic factorisation is
uploaded once per `symbolic` object (its Plan), the task program of each
sweep is compiled once, and the workspace is reused.  Values stay in the
cspmatrix's CUDA float64 tensor, transformed in place.  Calls are
synchronous like the reference's (they read the device status to raise
ArithmeticError); the `*_async` variants in `chompack_b200.engine` skip that.
"""
import torch

from . import _native as N

__all__ = ["cholesky", "llt", "projected_inverse", "completion", "hessian", "trsm", "dot"]


def _values(X, name="X"):
    v = X.blkval
    if not isinstance(v, torch.Tensor) or v.device.type != "cuda":
        raise RuntimeError("%s.blkval must be a CUDA tensor: the sweeps run on the GPU only" % name)
    if v.dtype != torch.float64 or not v.is_contiguous():
        raise ValueError("%s.blkval must be a contiguous float64 tensor" % name)
    return v


def _stream(dev):
    return torch.cuda.current_stream(dev).cuda_stream


def _check(rc, what):
    if rc < 0:
        raise RuntimeError("%s failed: %s" % (what, N.last_error().decode()))


def _run_and_status(plan, op, launch, k=0, flags=0):
    dev = torch.device("cuda", plan.device)
    ws, nbytes = plan.workspace(op, k, flags)
    s = _stream(dev)
    _check(launch(ws, nbytes, s), "launch")
    info = N.info(plan.handle, ws, s)
    _check(info, "sweep")
    return info


def cholesky(X):
    """Supernodal multifrontal Cholesky factorisation X = L L^T, in place
    (cbase.c:176-284).  On exit X holds the factor and X.is_factor is True."""
    if X.is_factor is not False:
        raise ValueError("X must be a cspmatrix")
    v = _values(X)
    plan = X.symb.plan(v.device.index)
    info = _run_and_status(plan, N.OP_CHOLESKY,
                           lambda ws, nb, s: N.cholesky(plan.handle, v.data_ptr(), ws, nb, s))
    X.is_factor = True
    if info:
        raise ArithmeticError("factorization failed")


def projected_inverse(L):
    """Supernodal multifrontal projected inverse Y = P(L^{-T} L^{-1}), in place
    (cbase.c:393-500).  On exit L holds Y and L.is_factor is False."""
    if L.is_factor is not True:
        raise ValueError("X must be a cspmatrix")
    v = _values(L)
    plan = L.symb.plan(v.device.index)
    info = _run_and_status(plan, N.OP_PROJECTED_INVERSE,
                           lambda ws, nb, s: N.projected_inverse(plan.handle, v.data_ptr(), ws, nb, s))
    L.is_factor = False
    if info:
        raise ArithmeticError("partial inverse failed")


def _missing(name):
    def f(*args, **kwargs):
        raise NotImplementedError("%s is not available in this build" % name)
    f.__name__ = name
    return f


llt = _missing("llt")
completion = _missing("completion")
hessian = _missing("hessian")
trsm = _missing("trsm")
dot = _missing("dot")
