"""Mixed precision for the chordal sweeps (no counterpart in the reference,
which is FP64 only).

`cbase.cholesky(X, precision="tf32")` and `projected_inverse(L,
precision=...)` run every GEMM tile of the sweep (Schur-complement updates,
panel solves through the inverse of the diagonal tile, the projected
inverse's products) on TF32 tensor cores with FP32 accumulation; the
diagonal tiles, look-ahead steps, split-K sums, assembly and extraction
stay FP64, and so does the storage.  "tf32x3" splits each operand into high
and low TF32 parts (three products, about 22 bits).

This module adds what makes such a factor usable at FP64 accuracy and
states the error of every result:

* `symv`: y = X x in FP64 on the GPU (the refinement residual);
* `solve`: X^{-1} B by iterative refinement (FP64 residual, corrections
  through the mixed factor with the FP64 triangular solves) to a stated
  normwise relative residual;
* `logdet_and_gradient`: log det X and its gradient P(X^{-1}) (the projected
  inverse) in mixed precision, with their errors against an FP64 run.
"""
import ctypes

import torch

from . import _native as N
from . import cbase

__all__ = ["symv", "solve", "logdet_and_gradient"]


def _device_index(symb):
    return symb.plan().device


def _sym_arrays(symb, dev):
    """sncolptr / snrowidx of the symbolic on the device (cached)."""
    from .cspmatrix import _symbolic_arrays
    return _symbolic_arrays(symb, dev)


def _as_columns(B, dev):
    if B.dim() == 1:
        B = B[:, None]
    if B.device != dev or B.dtype != torch.float64:
        B = B.to(device=dev, dtype=torch.float64)
    return B.t().contiguous().t()   # column-major n x nrhs


def symv(X, x, alpha=1.0, y=None):
    """y = alpha X x (+ y when given) for the symmetric chordal matrix X in
    FP64; x, y are n-vectors or n x nrhs matrices in the original order."""
    if X.is_factor is not False:
        raise ValueError("X must be a cspmatrix")
    v = cbase._values(X)
    dev = v.device
    xs = _as_columns(x, dev)
    n, nrhs = xs.shape
    out = torch.zeros_like(xs) if y is None else _as_columns(y, dev).clone()
    plan = X.symb.plan(dev.index)
    colptr, rowidx = _sym_arrays(X.symb, dev)
    s = torch.cuda.current_stream(dev).cuda_stream
    rc = N.symv(plan.handle, v.data_ptr(), colptr.data_ptr(), rowidx.data_ptr(), xs.data_ptr(), out.data_ptr(),
                nrhs, out.stride(1) if nrhs > 1 else n, float(alpha), s)
    if rc < 0:
        raise RuntimeError("symv failed: %s" % N.last_error().decode())
    return out if x.dim() > 1 else out[:, 0]


def solve(X, L, B, tol=1e-12, maxiter=30):
    """X^{-1} B by iterative refinement: corrections d = (L L^T)^{-1} r with
    the (mixed-precision) factor L of X, residuals r = B - X x in FP64.
    Stops when the normwise relative residual max_j ||r_j|| / ||b_j|| is at
    most tol.  Returns (x, report) with the iterations and residuals."""
    if L.is_factor is not True:
        raise ValueError("L must be a cspmatrix factor")
    dev = cbase._values(L).device
    Bc = _as_columns(B, dev)
    bn = torch.linalg.vector_norm(Bc, dim=0).clamp_min(torch.finfo(torch.float64).tiny)
    x = torch.zeros_like(Bc)
    r = Bc.clone()
    history = []
    it = 0
    # the solves' step operands (diagonal-tile inverses and their coupling
    # products, from L alone) are computed by the first iteration and reused
    slots = ("refine_N", "refine_T")
    for it in range(1, maxiter + 1):
        d = r.clone()
        cbase._trsm_reuse(L, d, 'N', it > 1, slots[0])
        cbase._trsm_reuse(L, d, 'T', it > 1, slots[1])
        x += d
        r = symv(X, x, alpha=-1.0, y=Bc)
        res = float((torch.linalg.vector_norm(r, dim=0) / bn).max())
        history.append(res)
        if res <= tol:
            break
    out = x if B.dim() > 1 else x[:, 0]
    return out, {"iterations": it, "residuals": history, "converged": history[-1] <= tol}


def _logdet(L):
    v = cbase._values(L)
    plan = L.symb.plan(v.device.index)
    ws, nb = plan.workspace(N.OP_DOT)
    out = torch.empty(1, dtype=torch.float64, device=v.device)
    s = torch.cuda.current_stream(v.device).cuda_stream
    if N.logdet(plan.handle, v.data_ptr(), out.data_ptr(), ws, nb, s) < 0:
        raise RuntimeError("logdet failed: %s" % N.last_error().decode())
    return float(out.item())


def logdet_and_gradient(X, precision="tf32", reference=True):
    """log det X (FP64 accumulation of the factor's diagonal) and its
    gradient Y = P(X^{-1}) with cholesky and projected_inverse in the given
    precision.  X is left unchanged.  With reference=True the same values
    are computed in FP64 and the report states the errors: |logdet error| /
    |logdet|, max |Y - Y64| / max |Y64|, and the factor's max |L - L64| /
    max |L64|."""
    from .cspmatrix import cspmatrix
    if X.is_factor is not False:
        raise ValueError("X must be a cspmatrix")
    v = cbase._values(X)
    Lm = cspmatrix(X.symb, blkval=v.clone())
    cbase.cholesky(Lm, precision=precision)
    ld = _logdet(Lm)
    Lfac = Lm.blkval.clone()
    cbase.projected_inverse(Lm, precision=precision)
    report = {"precision": precision, "logdet": ld}
    if reference:
        R = cspmatrix(X.symb, blkval=v.clone())
        cbase.cholesky(R)
        ld64 = _logdet(R)
        L64 = R.blkval.clone()
        cbase.projected_inverse(R)
        report["logdet_rel_error"] = abs(ld - ld64) / max(abs(ld64), 1e-300)
        report["gradient_rel_error"] = float((Lm.blkval - R.blkval).abs().max() / R.blkval.abs().max())
        report["factor_rel_error"] = float((Lfac - L64).abs().max() / L64.abs().max())
    return ld, Lm, report
