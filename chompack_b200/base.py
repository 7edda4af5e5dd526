"""Projected rank-2 update of a cspmatrix (src/python/base.py:28-67 of the
reference, a Python loop over supernodes there), on the values' device.

    X := alpha P(u v^T + v u^T) + beta X

P projects onto the chordal pattern; only the lower trapezoid of each block
changes.  u and v are n-vectors (numpy arrays or tensors) in the original
numbering, or in the reordered one when reordered=True.
"""
import numpy as np
import torch

from . import _native as N
from . import cbase
from .cspmatrix import _symbolic_arrays

__all__ = ["syr2"]


def _vector(x, n, dev, name):
    t = x if isinstance(x, torch.Tensor) else torch.from_numpy(np.asarray(x, dtype=np.float64))
    t = t.to(device=dev, dtype=torch.float64).reshape(-1).contiguous()
    if t.numel() != n:
        raise ValueError("%s must have %d entries" % (name, n))
    return t


def syr2(X, u, v, alpha=1.0, beta=1.0, reordered=False):
    """X := alpha*P(u v^T + v u^T) + beta*X, in place (chb_syr2)."""
    assert X.is_factor is False, "cspmatrix factor object"
    s = X.symb
    xv = cbase._values(X)
    dev = xv.device
    ut = _vector(u, s.n, dev, "u")
    vt = _vector(v, s.n, dev, "v")
    colptr, rowidx = _symbolic_arrays(s, dev)
    rc = N.syr2(s.plan(dev.index).handle, xv.data_ptr(), colptr.data_ptr(), rowidx.data_ptr(), ut.data_ptr(),
                vt.data_ptr(), float(alpha), float(beta), 1 if reordered else 0,
                torch.cuda.current_stream(dev).cuda_stream)
    if rc < 0:
        raise RuntimeError("syr2 failed: %s" % N.last_error().decode())
    cbase._write_back(X)
