"""chompack_b200 — B200-native (sm_100a) numeric multifrontal sweeps over a
supernodal clique tree, with the API of CHOMPACK.

    import chompack_b200 as cp
    symb = cp.symbolic(A, p=cp.amd.order, merge_function=cp.merge_size_fill(32, 32))
    X = cp.cspmatrix(symb) + A          # values live in a CUDA float64 tensor
    cp.cholesky(X)                      # X now holds the factor
    cp.projected_inverse(X)             # X now holds P(A^{-1})

The symbolic analysis runs on the host (native C++); the numeric sweeps
(`cholesky`, `llt`, `projected_inverse`, `completion`, `hessian`, `trsm`,
`trmm`, `dot`) run as CUDA kernels on the GPU through the C ABI in
include/chompack_b200.h.  There is no CPU fallback for the sweeps.
"""
from .sparse import spmatrix, tril, triu, symmetrize, perm, eye
from .symbolic import symbolic, merge_size_fill, peo
from .cspmatrix import cspmatrix
from . import amd

__all__ = ["spmatrix", "tril", "triu", "symmetrize", "perm", "eye", "symbolic", "merge_size_fill", "peo",
           "cspmatrix", "amd"]

from .cbase import cholesky, llt, projected_inverse, completion, hessian, trsm, trmm, dot  # noqa: E402,F401
from . import autograd  # noqa: E402,F401
from .batch import batch  # noqa: E402,F401
from . import mixed  # noqa: E402,F401
from .pfcholesky import pfcholesky  # noqa: E402,F401
from .base import syr2  # noqa: E402,F401
from .completions import psdcompletion, mrcompletion  # noqa: E402,F401
from .autotune import tune  # noqa: E402,F401

__all__ += ["cholesky", "llt", "projected_inverse", "completion", "hessian", "trsm", "trmm", "dot", "autograd", "batch",
            "pfcholesky", "syr2", "psdcompletion", "mrcompletion", "tune"]
