"""Differentiable chordal log-determinant.

    f(X) = log det X,     X symmetric positive definite with chordal pattern

on the values of a cspmatrix (its `blkval` tensor, the reference block
layout).  A function of the stored entries x (lower trapezoid of each
supernode block) sees the symmetric matrix X with X_ij = X_ji = x_ij, so

    df/dx = w .* Y,       Y = P(X^{-1}) = projected_inverse(cholesky(X))

with w = 2 below the diagonal, 1 on it, 0 in the strict upper part of a
diagonal block (the weights of `dot`: <A, B> = sum w a b).  The second
derivative is the Hessian of the barrier: d<Y, C>/dX = -H_X(C), with
H_X(C) = P(X^{-1} C X^{-1}) = hessian(L, Y, C, adj=None), so the backward
of the gradient is -w .* H_X(unpack(c)).

Forward: one `cholesky` sweep and a log-det reduction of the factor's
diagonal.  Backward: one `projected_inverse` sweep (the reverse multifrontal
adjoint of the factorisation).  Double backward: one full `hessian`
application.  All three run as the package's CUDA sweeps; torch only holds
the tensors and the autograd graph.

A leading batch dimension of value sets on one pattern (values of shape
(B, blkptr[Nsn])) runs every sweep over all B value sets in ONE launch: a
merged plan over B copies of the clique tree (chompack_b200.batch), cached
on the symbolic object, with per-set log dets from a segmented reduction.

What the backward keeps is the factor L (the size of X per value set), not
the fronts or update matrices of the forward sweep: the projected inverse
needs only L.  Two options trade time for memory where that does not fit:
`recompute_factor=True` keeps only X (which autograd holds anyway) and
recomputes L by one more cholesky sweep in the backward, and
`scratch_limit` (bytes) puts the update matrices of the cholesky and
projected_inverse sweeps, by default several times the factor, in a shared
pool of about that size (the plan option CHB_OPT_SCRATCH_LIMIT: fronts
reuse the memory of update matrices already consumed, as the reference's
postorder stack does, waiting for their readers).  Neither changes a bit
of the results.
"""
import torch

from . import _native as N
from . import cbase
from .cspmatrix import cspmatrix

__all__ = ["logdet", "logdet_values", "logdet_gradient", "logdet_hvp"]


def _stream(dev):
    return torch.cuda.current_stream(dev).cuda_stream


def _check(rc, what):
    if rc < 0:
        raise RuntimeError("%s failed: %s" % (what, N.last_error().decode()))


def _limit_scratch(plan, limit):
    """Sets a plan's scratch limit (bytes, None: no limit) when it changes
    (changing it drops the plan's compiled programs)."""
    if getattr(plan, "_scratch_limit", None) != limit:
        plan.set_option("scratch_limit", limit)
        plan._scratch_limit = limit


def _factor(symb, x):
    """Cholesky factor values of one value set (a new tensor)."""
    L = cspmatrix(symb, blkval=x.detach().clone().contiguous())
    cbase.cholesky(L)
    return L


def _logdet_of_factor(symb, L):
    v = L.blkval
    plan = symb.plan(v.device.index)
    ws, nb = plan.workspace(N.OP_DOT)
    out = torch.empty(1, dtype=torch.float64, device=v.device)
    _check(N.logdet(plan.handle, v.data_ptr(), out.data_ptr(), ws, nb, _stream(v.device)), "logdet")
    return out[0]


def _sym_weight(symb, x, alpha=1.0):
    """alpha * w .* x (a new tensor)."""
    y = torch.empty_like(x)
    plan = symb.plan(x.device.index)
    _check(N.sym_weight(plan.handle, x.data_ptr(), y.data_ptr(), float(alpha), _stream(x.device)), "sym_weight")
    return y


class _LogdetGrad(torch.autograd.Function):
    """x -> w .* P(X^{-1}), given the factor values L of X."""

    @staticmethod
    def forward(ctx, x, L, symb):
        Y = cspmatrix(symb, blkval=L.clone(), factor=True)
        cbase.projected_inverse(Y)
        ctx.save_for_backward(L, Y.blkval)
        ctx.symb = symb
        return _sym_weight(symb, Y.blkval)

    @staticmethod
    def backward(ctx, c):
        L, Yv = ctx.saved_tensors
        symb = ctx.symb
        U = cspmatrix(symb, blkval=c.detach().to(torch.float64).contiguous().clone())
        cbase.hessian(cspmatrix(symb, blkval=L, factor=True), cspmatrix(symb, blkval=Yv), U, adj=None)
        return _sym_weight(symb, U.blkval, -1.0), None, None


class _Logdet(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, symb, recompute):
        L = _factor(symb, x)
        ctx.recompute = recompute
        if recompute:
            ctx.save_for_backward(x)
        else:
            ctx.save_for_backward(x, L.blkval)
        ctx.symb = symb
        return _logdet_of_factor(symb, L)

    @staticmethod
    def backward(ctx, g):
        if ctx.recompute:
            (x,) = ctx.saved_tensors
            Lv = _factor(ctx.symb, x).blkval
        else:
            x, Lv = ctx.saved_tensors
        return g * _LogdetGrad.apply(x, Lv, ctx.symb), None, None


def _value_sets(symb, count, device):
    """Merged plan over `count` copies of symb's clique tree (cached)."""
    from .batch import batch
    cache = symb.__dict__.setdefault("_value_set_batches", {})
    key = (int(count), int(device.index))
    if key not in cache:
        cache[key] = batch([symb] * int(count), device=device.index)
    return cache[key]


class _LogdetGradBatch(torch.autograd.Function):
    """x (B, nv) -> w .* P(X_b^{-1}) for every value set, given the factors."""

    @staticmethod
    def forward(ctx, x, L, symb):
        Bt = _value_sets(symb, x.shape[0], x.device)
        Y = L.reshape(-1).clone()
        Bt.projected_inverse(Y)
        ctx.save_for_backward(L, Y)
        ctx.symb = symb
        return Bt.sym_weight(Y).reshape(x.shape)

    @staticmethod
    def backward(ctx, c):
        L, Y = ctx.saved_tensors
        Bt = _value_sets(ctx.symb, L.shape[0], L.device)
        U = c.detach().to(torch.float64).reshape(-1).contiguous().clone()
        Bt.hessian(L.reshape(-1), Y, U, adj=None)
        return Bt.sym_weight(U, -1.0).reshape(L.shape), None, None


def _factor_sets(Bt, x):
    L = x.detach().reshape(-1).clone()
    Bt.cholesky(L)
    return L.reshape(x.shape)


class _LogdetBatch(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, symb, recompute):
        Bt = _value_sets(symb, x.shape[0], x.device)
        L = _factor_sets(Bt, x)
        ctx.recompute = recompute
        if recompute:
            ctx.save_for_backward(x)
        else:
            ctx.save_for_backward(x, L)
        ctx.symb = symb
        return Bt.logdet(L.reshape(-1))

    @staticmethod
    def backward(ctx, g):
        if ctx.recompute:
            (x,) = ctx.saved_tensors
            L = _factor_sets(_value_sets(ctx.symb, x.shape[0], x.device), x)
        else:
            x, L = ctx.saved_tensors
        return g[:, None] * _LogdetGradBatch.apply(x, L, ctx.symb), None, None


def logdet_values(x, symb, scratch_limit=None, recompute_factor=False):
    """log det of the chordal SPD matrix with block values x (1-D, or
    (B, n_values) for B value sets on `symb`'s pattern, swept together),
    differentiable (first and second order).  scratch_limit: bytes for the
    update matrices of the sweeps (None: each its own memory);
    recompute_factor: keep only x for the backward and factor again there."""
    if not isinstance(x, torch.Tensor) or x.device.type != "cuda" or x.dtype != torch.float64:
        raise ValueError("values must be a float64 CUDA tensor")
    if x.dim() == 1:
        _limit_scratch(symb.plan(x.device.index), scratch_limit)
        return _Logdet.apply(x, symb, bool(recompute_factor))
    if x.dim() != 2 or x.shape[1] != int(symb.blkptr[-1]):
        raise ValueError("batched values must have shape (B, %d)" % int(symb.blkptr[-1]))
    _limit_scratch(_value_sets(symb, x.shape[0], x.device).plan, scratch_limit)
    return _LogdetBatch.apply(x.contiguous(), symb, bool(recompute_factor))


def logdet(X, scratch_limit=None, recompute_factor=False):
    """log det of a cspmatrix X (not a factor), differentiable through
    X.blkval (options as logdet_values)."""
    if X.is_factor is not False:
        raise ValueError("X must be a cspmatrix")
    return logdet_values(X.blkval, X.symb, scratch_limit, recompute_factor)


def logdet_gradient(X):
    """The gradient of log det at X as a cspmatrix: Y = P(X^{-1})
    (cholesky followed by projected_inverse, without autograd)."""
    Y = cspmatrix(X.symb, blkval=X.blkval.detach().clone())
    cbase.cholesky(Y)
    cbase.projected_inverse(Y)
    return Y


def logdet_hvp(L, Y, U):
    """The second directional derivative of log det at X = L L^T along the
    cspmatrix U: -H_X(U) = -P(X^{-1} U X^{-1}), as a new cspmatrix (L the
    factor, Y the projected inverse)."""
    V = cspmatrix(U.symb, blkval=U.blkval.detach().clone())
    cbase.hessian(L, Y, V, adj=None)
    V.blkval.mul_(-1.0)
    return V
