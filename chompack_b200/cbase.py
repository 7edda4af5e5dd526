"""Drop-in numeric sweeps with the signatures, defaults and exceptions of the
reference's `chompack.cbase` (src/C/cbase.c), running on the GPU through the
C ABI of include/chompack_b200.h.

Each call uploads nothing but what changed: the symbolic factorisation is
uploaded once per `symbolic` object (its Plan), the task program of each
sweep is compiled once, and the workspace is reused.  Calls are synchronous
like the reference's (they read the device status to raise ArithmeticError).

Values live either in a CUDA float64 tensor (transformed in place on the
device) or, as in the reference, in host memory (a CPU float64 tensor,
pinned for the copies to overlap).  Host values keep a device mirror on the
cspmatrix: cholesky, projected_inverse and llt stream the values in while
the sweep runs (unless the mirror already holds them) and each finished
chunk of the result back out; the other sweeps copy in, run, copy out.
"""
import ctypes

import torch

from . import _native as N

__all__ = ["cholesky", "llt", "projected_inverse", "completion", "hessian", "trsm", "trmm", "dot", "pfchol",
           "pftrsm", "pftrmm"]


def _on_host(X):
    v = X.blkval
    return isinstance(v, torch.Tensor) and v.device.type == "cpu"


def _values(X, name="X"):
    """Device values of X: its CUDA tensor, or for host values the device
    mirror, brought up to date with a copy if the host values changed."""
    v = X.blkval
    if not isinstance(v, torch.Tensor) or v.device.type not in ("cuda", "cpu"):
        raise RuntimeError("%s.blkval must be a float64 tensor" % name)
    if v.dtype != torch.float64 or not v.is_contiguous():
        raise ValueError("%s.blkval must be a contiguous float64 tensor" % name)
    if v.device.type == "cuda":
        return v
    m = _mirror(X, X.symb.plan())
    if not _synced(X):
        m.copy_(v)
        _mark_synced(X)
    return m


def _mirror(X, plan):
    dev = torch.device("cuda", plan.device)
    m = X.__dict__.get("_dev")
    if m is None or m.device != dev or m.numel() != X.blkval.numel():
        m = torch.empty(X.blkval.numel(), dtype=torch.float64, device=dev)
        X._dev = m
        X._dev_tag = None
    return m


def _synced(X):
    v = X.blkval
    return X.__dict__.get("_dev_tag") == (v.data_ptr(), v._version)


def _mark_synced(X):
    v = X.blkval
    X._dev_tag = (v.data_ptr(), v._version)


def _write_back(X):
    """After an in-place sweep on the device mirror of host values."""
    if _on_host(X):
        X.blkval.copy_(X._dev)
        _mark_synced(X)


def _precision(precision):
    if precision not in N.PREC:
        raise ValueError("precision must be one of %s" % ", ".join(sorted(N.PREC)))
    return N.PREC[precision]


def _streamed(X, op, launch, name="X", prec=0):
    """A streamed sweep on host values: chunks go in (unless the mirror
    holds them) while the sweep runs, and come back out as they finish."""
    v = X.blkval
    if v.dtype != torch.float64 or not v.is_contiguous():
        raise ValueError("%s.blkval must be a contiguous float64 tensor" % name)
    plan = X.symb.plan()
    m = _mirror(X, plan)
    host_in = None if _synced(X) else v.data_ptr()
    flags = N.io_flags(host_in is not None, 1) | N.precision_flags(prec)
    dev = torch.device("cuda", plan.device)
    ws, nbytes = plan.workspace(op, 0, flags)
    s = _stream(dev)
    _check(launch(plan.handle, host_in, v.data_ptr(), m.data_ptr(), ws, nbytes, s), "launch")
    info = N.info(plan.handle, ws, s)
    _check(info, "sweep")
    _mark_synced(X)
    return info


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


def cholesky(X, precision="fp64"):
    """Supernodal multifrontal Cholesky factorisation X = L L^T, in place
    (cbase.c:176-284).  On exit X holds the factor and X.is_factor is True.

    precision (an addition; the reference is FP64 only): "tf32" or "tf32x3"
    run the GEMM tiles (Schur updates, panel solves) on TF32 tensor cores
    with FP32 accumulation, the diagonal tiles in FP64 (see
    chompack_b200.mixed for refined solves and error reports)."""
    if X.is_factor is not False:
        raise ValueError("X must be a cspmatrix")
    prec = _precision(precision)
    if _on_host(X):
        info = _streamed(X, N.OP_CHOLESKY,
                         lambda h, hi, ho, d, ws, nb, s: N.cholesky_prec(h, prec, hi, ho, d, ws, nb, s), prec=prec)
    else:
        v = _values(X)
        plan = X.symb.plan(v.device.index)
        if prec:
            info = _run_and_status(plan, N.OP_CHOLESKY,
                                   lambda ws, nb, s: N.cholesky_prec(plan.handle, prec, None, None, v.data_ptr(),
                                                                     ws, nb, s), flags=N.precision_flags(prec))
        else:
            info = _run_and_status(plan, N.OP_CHOLESKY,
                                   lambda ws, nb, s: N.cholesky(plan.handle, v.data_ptr(), ws, nb, s))
    X.is_factor = True
    if info:
        raise ArithmeticError("factorization failed")


def projected_inverse(L, precision="fp64"):
    """Supernodal multifrontal projected inverse Y = P(L^{-T} L^{-1}), in place
    (cbase.c:393-500).  On exit L holds Y and L.is_factor is False.
    precision: as for cholesky (its GEMM tiles on TF32 tensor cores)."""
    if L.is_factor is not True:
        raise ValueError("X must be a cspmatrix")
    prec = _precision(precision)
    if _on_host(L):
        info = _streamed(L, N.OP_PROJECTED_INVERSE,
                         lambda h, hi, ho, d, ws, nb, s: N.projected_inverse_prec(h, prec, hi, ho, d, ws, nb, s),
                         prec=prec)
    else:
        v = _values(L)
        plan = L.symb.plan(v.device.index)
        if prec:
            info = _run_and_status(plan, N.OP_PROJECTED_INVERSE,
                                   lambda ws, nb, s: N.projected_inverse_prec(plan.handle, prec, None, None,
                                                                              v.data_ptr(), ws, nb, s),
                                   flags=N.precision_flags(prec))
        else:
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
    if _on_host(L):
        _streamed(L, N.OP_LLT, N.llt_io)
    else:
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


def _trsm_reuse(L, B, trans, reuse, slot):
    """trsm on a column-major CUDA tensor B through chb_trsm_reuse, with the
    workspace of `slot`: with reuse the step operands are taken from that
    workspace as the previous call on it (same factor, trans and number of
    right-hand sides) left them.  For repeated solves (mixed.solve)."""
    v = _values(L, "L")
    dev = v.device
    if B.dim() != 2 or B.stride(0) != 1 or B.device != dev or B.dtype != torch.float64:
        raise ValueError("B must be a column-major float64 tensor on the device of L")
    nrhs, ld = B.shape[1], B.stride(1)
    plan = L.symb.plan(dev.index)
    ws, nb = plan.workspace(N.OP_TRSM, nrhs, (1 if trans == 'T' else 0) | (2 if reuse else 0), slot=slot)
    s = _stream(dev)
    _check(N.trsm_reuse(plan.handle, trans.encode(), int(nrhs), 1.0, v.data_ptr(), B.data_ptr(), int(ld), ws, nb,
                        1 if reuse else 0, s), "launch")
    _check(N.info(plan.handle, ws, s), "sweep")


def trmm(L, B, alpha=1.0, trans='N', nrhs=None, offsetB=0, ldB=None):
    """Multiplication with a cspmatrix factor (pybase/trmm.py:4-116):
    B := alpha L B (trans 'N') or alpha L^T B (trans 'T'), in place.

    Arguments and the layout of B are those of trsm: a CUDA float64 tensor
    (element (i, j) at storage offset i + j*ld) or a Fortran-ordered numpy
    array (copied to the GPU and back), rows in the original order."""
    if L.is_factor is not True:
        raise ValueError("L must be a cspmatrix factor")
    if trans not in ('N', 'T'):
        raise ValueError("trans must be 'N' or 'T'")
    v = _values(L, "L")
    dev = v.device
    Bt, host, cols, ld0 = _rhs_on_device(B, dev)
    if nrhs is None:
        nrhs = cols
    if ldB is None:
        ldB = ld0
    plan = L.symb.plan(dev.index)
    ptr = Bt.data_ptr() + 8 * int(offsetB)
    _run_and_status(plan, N.OP_TRMM,
                    lambda ws, nb, s: N.trmm(plan.handle, trans.encode(), int(nrhs), float(alpha), v.data_ptr(), ptr,
                                             int(ldB), ws, nb, s), k=int(nrhs), flags=1 if trans == 'T' else 0)
    if host is not None:
        out = Bt.cpu().numpy()
        if host.ndim == 1:
            host[:] = out
        else:
            host[:, :] = out.reshape(host.shape, order="F")


def _rhs_on_device(B, dev):
    """(tensor on dev, host array or None, columns, leading dimension) of a
    right-hand-side block given as a column-major CUDA float64 tensor or a
    Fortran-ordered float64 numpy array."""
    if isinstance(B, torch.Tensor):
        if B.device != dev or B.dtype != torch.float64:
            raise ValueError("B must be a float64 tensor on the device of L")
        if B.dim() == 1:
            return B, None, 1, B.shape[0]
        if B.stride(0) != 1:
            raise ValueError("B must be column-major (stride(0) == 1)")
        return B, None, B.shape[1], B.stride(1)
    import numpy as np
    host = np.asarray(B)
    if host.dtype != np.float64:
        raise ValueError("B must be float64")
    if host.ndim > 1 and not host.flags["F_CONTIGUOUS"]:
        raise ValueError("B must be column-major (Fortran order)")
    cols = 1 if host.ndim == 1 else host.shape[1]
    return torch.from_numpy(host.reshape(-1, order="F")).to(dev), host, cols, host.shape[0]


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


def completion(X, factored_updates=True):
    """Maximum-determinant positive definite completion (cbase.c:521-620):
    on exit X holds, in place, the Cholesky factor L of the inverse of the
    max-det positive definite completion of X (so L L^T has projected
    inverse X); X.is_factor becomes True.  factored_updates selects the
    update_factor form of the update matrices (the same L up to rounding)."""
    if X.is_factor is not False:
        raise ValueError("X must be a cspmatrix")
    v = _values(X)
    plan = X.symb.plan(v.device.index)
    fu = 1 if factored_updates is True else 0
    info = _run_and_status(plan, N.OP_COMPLETION,
                           lambda ws, nb, s: N.completion(plan.handle, v.data_ptr(), fu, ws, nb, s), k=fu)
    _write_back(X)
    X.is_factor = True
    if info:
        raise ArithmeticError("completion failed")


def hessian(L, Y, U, adj=False, inv=False, factored_updates=True):
    """Hessian factors of the log-det barrier (cbase.c:675-857), applied in
    place to U (a cspmatrix or a list of them, all on L's symbolic
    factorisation):

        adj=False, inv=False:  U := G(U)          adj=True,  inv=False: U := G^adj(U)
        adj=False, inv=True:   U := G^{-1}(U)     adj=True,  inv=True:  U := (G^adj)^{-1}(U)
        adj=None:              U := H(U) = G^adj(G(U))  (inv=True: the inverse)

    L is the Cholesky factor, Y the projected inverse (L.symb's)."""
    symb = L.symb
    Us = U if isinstance(U, list) else [U]
    if Y.symb is not symb or any(u.symb is not symb for u in Us):
        raise ValueError("symbolic factorizations must be the same")
    if L.is_factor is False:
        raise ValueError("L must be a cspmatrix factor")
    if Y.is_factor is True:
        raise ValueError("Y must be a cspmatrix")
    inv_i = 1 if inv is True else 0
    if adj is True:
        adj_i = 1
    elif adj is None:
        adj_i = inv_i
    else:
        adj_i = 0
    fu = 1 if factored_updates is True else 0
    lv = _values(L, "L")
    yv = _values(Y, "Y")
    uv = [_values(u, "U") for u in Us]
    if not Us:
        return
    plan = symb.plan(lv.device.index)
    passes = [adj_i, 1 ^ adj_i] if adj is None else [adj_i]
    info = 0
    for a in passes:
        for c0 in range(0, len(uv), N.HESSIAN_MAX_U):
            chunk = uv[c0:c0 + N.HESSIAN_MAX_U]
            arr = (ctypes.c_void_p * len(chunk))(*[u.data_ptr() for u in chunk])
            flags = a | inv_i << 1 | fu << 2
            info |= _run_and_status(
                plan, N.OP_HESSIAN,
                lambda ws, nb, s: N.hessian(plan.handle, lv.data_ptr(), yv.data_ptr(), arr, len(chunk), a, inv_i,
                                            fu, ws, nb, s), k=len(chunk), flags=flags)
    for u in Us:
        _write_back(u)
    if info:
        raise ArithmeticError("hessian failed")


# ------------------------------------------------------- product-form factor
# cbase.pfchol / pftrsm / pftrmm (cbase.c:859-942) over the GPU kernels of
# csrc/pf.cu.  V, L, B and U are n x k (n x nrhs) column-major float64: CUDA
# tensors with stride(0) == 1 (transformed in place on the device) or
# Fortran-ordered numpy arrays (copied to the current device and back).

def _dense_on_device(M, name, dev=None):
    """(tensor, host array or None, rows, cols, ld) of a column-major block."""
    import numpy as np
    if isinstance(M, torch.Tensor):
        if M.device.type != "cuda" or M.dtype != torch.float64:
            raise ValueError("%s must be a float64 CUDA tensor" % name)
        if dev is not None and M.device != dev:
            raise ValueError("%s must be on %s" % (name, dev))
        if M.dim() == 1:
            return M, None, M.shape[0], 1, max(1, M.shape[0])
        if M.dim() != 2 or (M.shape[0] > 1 and M.stride(0) != 1):
            raise ValueError("%s must be column-major (stride(0) == 1)" % name)
        return M, None, M.shape[0], M.shape[1], max(1, M.stride(1) if M.shape[1] > 1 else M.shape[0])
    host = np.asarray(M)
    if host.dtype != np.float64:
        raise ValueError("%s must be float64" % name)
    if host.ndim > 2 or (host.ndim == 2 and not host.flags["F_CONTIGUOUS"]):
        raise ValueError("%s must be column-major (Fortran order)" % name)
    d = dev if dev is not None else torch.device("cuda", torch.cuda.current_device())
    rows = host.shape[0]
    cols = 1 if host.ndim == 1 else host.shape[1]
    return torch.from_numpy(host.reshape(-1, order="F")).to(d), host, rows, cols, max(1, rows)


def _copy_back(t, host):
    if host is not None:
        out = t.cpu().numpy()
        if host.ndim == 1:
            host[:] = out
        else:
            host[:, :] = out.reshape(host.shape, order="F")


def _pf_workspace(n, ncols, dev):
    sz = ctypes.c_size_t()
    with torch.cuda.device(dev):
        _check(N.pf_workspace_size(int(n), int(ncols), ctypes.byref(sz)), "pf_workspace_size")
    buf = torch.empty(sz.value + 256, dtype=torch.uint8, device=dev)
    return buf, (buf.data_ptr() + 255) // 256 * 256, sz.value


def _pf_status(ws, dev):
    info = N.pf_info(ws, _stream(dev))
    if info < -1:
        raise RuntimeError("product-form sweep failed: %s" % N.last_error().decode())
    return info


def pfchol(alpha, V, L, B):
    """Product-form Cholesky factorisation of I + V diag(alpha) V^T
    (cbase.c:862-880 / dpftrf): V (n x k) is overwritten, L and B receive
    the factors.  ArithmeticError when the matrix is not positive definite."""
    Vt, Vh, n, k, ldv = _dense_on_device(V, "V")
    dev = Vt.device
    Lt, Lh, nl, kl, ldl = _dense_on_device(L, "L", dev)
    Bt, Bh, nb, kb, ldb = _dense_on_device(B, "B", dev)
    if (nl, kl) != (n, k) or (nb, kb) != (n, k):
        raise ValueError("V, L and B must have the same size")
    a = torch.as_tensor(alpha, dtype=torch.float64).reshape(-1).to(dev).contiguous()
    if a.numel() < k:
        raise ValueError("alpha must have at least k entries")
    buf, ws, nbytes = _pf_workspace(n, k, dev)
    with torch.cuda.device(dev):
        _check(N.pftrf(n, k, a.data_ptr(), Vt.data_ptr(), ldv, Lt.data_ptr(), ldl, Bt.data_ptr(), ldb, ws, nbytes,
                       _stream(dev)), "pftrf")
        info = _pf_status(ws, dev)
    for t, h in ((Vt, Vh), (Lt, Lh), (Bt, Bh)):
        _copy_back(t, h)
    if info:
        raise ArithmeticError("factorization failed")


def _pf_apply(fn, what, V, L, B, U, trans):
    if trans not in ('N', 'T'):
        raise ValueError("trans must be 'N' or 'T'")
    Vt, _, n, k, ldv = _dense_on_device(V, "V")
    dev = Vt.device
    Lt, _, _, _, ldl = _dense_on_device(L, "L", dev)
    Bt, _, _, _, ldb = _dense_on_device(B, "B", dev)
    Ut, Uh, nu, nrhs, ldu = _dense_on_device(U, "U", dev)
    if nu != n:
        raise ValueError("U must have n rows")
    buf, ws, nbytes = _pf_workspace(n, nrhs, dev)
    with torch.cuda.device(dev):
        _check(fn(n, k, trans.encode(), Vt.data_ptr(), ldv, Lt.data_ptr(), ldl, Bt.data_ptr(), ldb, Ut.data_ptr(),
                  ldu, nrhs, ws, nbytes, _stream(dev)), what)
        _pf_status(ws, dev)
    _copy_back(Ut, Uh)


def pftrsm(V, L, B, U, trans='N'):
    """U := (L_1...L_k)^{-1} U ('N') or (L_k^T...L_1^T)^{-1} U ('T'), in place
    (cbase.c:885-911 / dpfsv)."""
    _pf_apply(N.pfsv, "pfsv", V, L, B, U, trans)


def pftrmm(V, L, B, U, trans='N'):
    """U := L_1...L_k U ('N') or L_k^T...L_1^T U ('T'), in place
    (cbase.c:916-942 / dpfmv)."""
    _pf_apply(N.pfmv, "pfmv", V, L, B, U, trans)
