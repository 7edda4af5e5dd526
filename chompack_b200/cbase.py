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


def llt(L):
    """Supernodal multifrontal Cholesky product X = L L^T, in place
    (cbase.c:287-390).  On exit L holds X and L.is_factor is False."""
    if L.is_factor is not True:
        raise ValueError("X must be a cspmatrix")
    v = _values(L)
    plan = L.symb.plan(v.device.index)
    _run_and_status(plan, N.OP_LLT, lambda ws, nb, s: N.llt(plan.handle, v.data_ptr(), ws, nb, s))
    L.is_factor = False


def trsm(L, B, alpha=1.0, trans='N', nrhs=None, offsetB=0, ldB=None):
    """Triangular solve with a cspmatrix factor (cbase.c:944-1077):
    B := alpha L^{-1} B (trans 'N') or alpha L^{-T} B (trans 'T'), in place.

    B holds the right-hand sides column by column (column-major), rows in
    the original order: a CUDA float64 tensor whose element (i, j) is at
    storage offset i + j*ld (a 1-D tensor, or a 2-D tensor with stride(0) ==
    1), or a Fortran-ordered numpy array (copied to the GPU and back)."""
    if L.is_factor is not True:
        raise ValueError("L must be a cspmatrix factor")
    if trans not in ('N', 'T'):
        raise ValueError("trans must be 'N' or 'T'")
    v = _values(L, "L")
    dev = v.device
    host = None
    if isinstance(B, torch.Tensor):
        if B.device != dev or B.dtype != torch.float64:
            raise ValueError("B must be a float64 tensor on the device of L")
        if B.dim() == 1:
            rows, cols, ld0 = B.shape[0], 1, B.shape[0]
        elif B.stride(0) == 1:
            rows, cols, ld0 = B.shape[0], B.shape[1], B.stride(1)
        else:
            raise ValueError("B must be column-major (stride(0) == 1)")
        Bt = B
    else:
        import numpy as np
        host = np.asarray(B)
        if host.dtype != np.float64:
            raise ValueError("B must be float64")
        if host.ndim == 1:
            rows, cols, ld0 = host.shape[0], 1, host.shape[0]
        else:
            if not host.flags["F_CONTIGUOUS"]:
                raise ValueError("B must be column-major (Fortran order)")
            rows, cols, ld0 = host.shape[0], host.shape[1], host.shape[0]
        Bt = torch.from_numpy(host.reshape(-1, order="F")).to(dev)
    if nrhs is None:
        nrhs = cols
    if ldB is None:
        ldB = ld0 if host is None else rows
    plan = L.symb.plan(dev.index)
    flags = 1 if trans == 'T' else 0
    ptr = Bt.data_ptr() + 8 * int(offsetB)
    _run_and_status(plan, N.OP_TRSM,
                    lambda ws, nb, s: N.trsm(plan.handle, trans.encode(), int(nrhs), float(alpha), v.data_ptr(), ptr,
                                             int(ldB), ws, nb, s), k=int(nrhs), flags=flags)
    if host is not None:
        out = Bt.cpu().numpy()
        host.reshape(-1, order="F")[:] = out if host.ndim == 1 else out
        if host.ndim > 1:
            host[:, :] = out.reshape(host.shape, order="F")


def dot(X, Y):
    """Trace inner product <X, Y> of two chordal matrices on the same
    symbolic factorisation (cbase.c:106-174); None if the factorisations
    differ, as in the reference."""
    if X.is_factor is not False:
        raise ValueError("X must be a cspmatrix")
    if Y.is_factor is not False:
        raise ValueError("Y must be a cspmatrix")
    if X.symb is not Y.symb:
        return None
    x = _values(X)
    y = _values(Y, "Y")
    plan = X.symb.plan(x.device.index)
    ws, nb = plan.workspace(N.OP_DOT)
    out = torch.empty(1, dtype=torch.float64, device=x.device)
    s = _stream(x.device)
    _check(N.dot(plan.handle, x.data_ptr(), y.data_ptr(), out.data_ptr(), ws, nb, s), "dot")
    return float(out.item())


def _missing(name):
    def f(*args, **kwargs):
        raise NotImplementedError("%s is not available in this build" % name)
    f.__name__ = name
    return f


completion = _missing("completion")
hessian = _missing("hessian")
