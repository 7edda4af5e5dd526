"""Batches of chordal matrices swept together.

A `batch` holds a list of symbolic factorisations (repeat one of them for
several value sets on a shared pattern) and one merged plan over the
disjoint union of their clique trees (chb_plan_merge).  The block values of
all matrices live in one float64 tensor, matrix m at [offsets[m],
offsets[m+1]), each in the reference block layout, so every sweep runs
over the whole batch in ONE launch of the persistent kernel: the fronts of
different matrices are independent tasks of one task graph, scheduled
together.  Per-matrix reductions (log det, dot) come back as one vector.

    B = batch([symb_1, symb_2, ...])
    x = B.assemble([A_1, A_2, ...])        # values of every matrix
    B.cholesky(x); ld = B.logdet(x)        # factors and log dets, in place
    B.projected_inverse(x)                 # gradients of the log dets
"""
import numpy as np
import torch

from . import _native as N
from .cspmatrix import cspmatrix
from .plan import Plan

__all__ = ["batch"]


def _stream(dev):
    return torch.cuda.current_stream(dev).cuda_stream


class batch(object):
    def __init__(self, symbs, device=None):
        if device is None:
            if not torch.cuda.is_available():
                raise RuntimeError("chompack_b200 sweeps need a CUDA device (no CPU fallback)")
            device = torch.cuda.current_device()
        self.symbs = list(symbs)
        if not self.symbs:
            raise ValueError("empty batch")
        self.device = torch.device("cuda", int(device)) if int(device) >= 0 else None
        host = {}
        for s in self.symbs:
            if id(s) not in host:
                host[id(s)] = Plan(s, device=-1)
        self._host_plans = host
        self.plan = Plan.merged([host[id(s)] for s in self.symbs], int(device))
        sizes = [int(s.blkptr[-1]) for s in self.symbs]
        self.offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        self.size = int(self.offsets[-1])

    def __len__(self):
        return len(self.symbs)

    # ---------------------------------------------------------------- values
    def empty(self):
        return torch.zeros(self.size, dtype=torch.float64, device=self.device)

    def assemble(self, As):
        """Values of cspmatrix(symb_m) + A_m for every matrix, assembled on
        the host and copied to the device once."""
        if len(As) != len(self.symbs):
            raise ValueError("one matrix per symbolic factorisation")
        host = np.empty(self.size)
        for m, (s, A) in enumerate(zip(self.symbs, As)):
            host[self.offsets[m]:self.offsets[m + 1]] = (cspmatrix(s, device="cpu") + A).blkval.numpy()
        return torch.from_numpy(host).to(self.device)

    def matrices(self, values, factor=False):
        """cspmatrix views of the batch values (no copies)."""
        return [cspmatrix(s, blkval=values[self.offsets[m]:self.offsets[m + 1]], factor=factor)
                for m, s in enumerate(self.symbs)]

    # ---------------------------------------------------------------- sweeps
    def _check_values(self, v):
        if not isinstance(v, torch.Tensor) or v.device != self.device or v.dtype != torch.float64 \
                or not v.is_contiguous() or v.numel() != self.size:
            raise ValueError("batch values must be a contiguous float64 tensor of %d entries on %s"
                             % (self.size, self.device))

    def _run(self, op, call, k=0, flags=0):
        ws, nb = self.plan.workspace(op, k, flags)
        s = _stream(self.device)
        rc = call(ws, nb, s)
        if rc < 0:
            raise RuntimeError("batch sweep failed: %s" % N.last_error().decode())
        info = N.info(self.plan.handle, ws, s)
        if info < 0:
            raise RuntimeError("batch sweep failed: %s" % N.last_error().decode())
        return info

    def cholesky(self, values):
        """Factor every matrix in place (one launch)."""
        self._check_values(values)
        h = self.plan.handle
        if self._run(N.OP_CHOLESKY, lambda w, nb, s: N.cholesky(h, values.data_ptr(), w, nb, s)):
            raise ArithmeticError("factorization failed")

    def projected_inverse(self, values):
        """Factors -> projected inverses, in place (one launch)."""
        self._check_values(values)
        h = self.plan.handle
        if self._run(N.OP_PROJECTED_INVERSE, lambda w, nb, s: N.projected_inverse(h, values.data_ptr(), w, nb, s)):
            raise ArithmeticError("partial inverse failed")

    def llt(self, values):
        self._check_values(values)
        h = self.plan.handle
        self._run(N.OP_LLT, lambda w, nb, s: N.llt(h, values.data_ptr(), w, nb, s))

    def completion(self, values, factored_updates=True):
        self._check_values(values)
        h = self.plan.handle
        fu = 1 if factored_updates else 0
        if self._run(N.OP_COMPLETION, lambda w, nb, s: N.completion(h, values.data_ptr(), fu, w, nb, s), k=fu):
            raise ArithmeticError("completion failed")

    def hessian(self, factor_values, pinv_values, u_values, adj=None, inv=False, factored_updates=True):
        """Hessian factors of every matrix's log-det barrier applied in place
        to one direction per matrix (u_values, the batch layout): the modes
        of cbase.hessian, adj=None the full H_X(U) (two passes), one launch
        per pass for the whole batch."""
        for v in (factor_values, pinv_values, u_values):
            self._check_values(v)
        import ctypes
        inv_i = 1 if inv is True else 0
        adj_i = inv_i if adj is None else (1 if adj is True else 0)
        fu = 1 if factored_updates is True else 0
        h = self.plan.handle
        arr = (ctypes.c_void_p * 1)(u_values.data_ptr())
        info = 0
        for a in ([adj_i, 1 ^ adj_i] if adj is None else [adj_i]):
            info |= self._run(N.OP_HESSIAN,
                              lambda w, nb, s: N.hessian(h, factor_values.data_ptr(), pinv_values.data_ptr(), arr, 1,
                                                         a, inv_i, fu, w, nb, s),
                              k=1, flags=a | inv_i << 1 | fu << 2)
        if info:
            raise ArithmeticError("hessian failed")

    def sym_weight(self, values, alpha=1.0):
        """alpha * w .* values with the weights of `dot` (2 below the
        diagonal, 1 on it, 0 in the strict upper part of a diagonal block),
        for every matrix: a new tensor."""
        self._check_values(values)
        out = torch.empty_like(values)
        rc = N.sym_weight(self.plan.handle, values.data_ptr(), out.data_ptr(), float(alpha), _stream(self.device))
        if rc < 0:
            raise RuntimeError("sym_weight failed: %s" % N.last_error().decode())
        return out

    # ------------------------------------------------------------ reductions
    def logdet(self, factor_values):
        """log det of every matrix from its factor: a (count,) tensor."""
        self._check_values(factor_values)
        ws, nb = self.plan.workspace(N.OP_DOT)
        out = torch.empty(len(self), dtype=torch.float64, device=self.device)
        rc = N.logdet_batch(self.plan.handle, factor_values.data_ptr(), out.data_ptr(), ws, nb,
                            _stream(self.device))
        if rc < 0:
            raise RuntimeError("logdet failed: %s" % N.last_error().decode())
        return out

    def dot(self, x, y):
        """<X_m, Y_m> for every matrix: a (count,) tensor."""
        self._check_values(x)
        self._check_values(y)
        ws, nb = self.plan.workspace(N.OP_DOT)
        out = torch.empty(len(self), dtype=torch.float64, device=self.device)
        rc = N.dot_batch(self.plan.handle, x.data_ptr(), y.data_ptr(), out.data_ptr(), ws, nb,
                         _stream(self.device))
        if rc < 0:
            raise RuntimeError("dot failed: %s" % N.last_error().decode())
        return out
