"""Shared helpers for the parity tests: problem construction (the shared
seeded value recipe of chompack_b200.grids, AMD ordering, merge rule) and
block-wise comparison against the oracle.

Tolerance of the FP64 parity checks (stated once, used everywhere):
    |x - x_ref| <= RTOL * max(|x_ref|, FLOOR * max|block_ref|)
with RTOL = 1e-12 and FLOOR = 1e-3, over the lower trapezoid of each
supernode block (the only part the reference defines, symbolic.py:1087-1094);
the floor covers entries that are the result of near cancellation.
"""
import numpy as np

import chompack_b200 as cp
from chompack_b200 import grids
from oracle import workload

RTOL = 1e-12
FLOOR = workload.FLOOR


def problem(kind, *args, merge=None, seed=0, order="amd"):
    if kind == "grid2d":
        A = grids.grid2d(*args, seed=seed)
    elif kind == "grid3d":
        A = grids.grid3d(*args, seed=seed)
    elif kind == "grid2d_extra":
        A = grids.grid2d_extra(*args, seed=seed)
    elif kind == "random":
        A = grids.random_lower(*args, seed=seed)
    else:
        raise ValueError(kind)
    p = cp.amd.order(A) if order == "amd" else None
    s = cp.symbolic(A, p=p, merge_function=cp.merge_size_fill(*merge) if merge else None)
    return A, s


def block_errors(symb, x, ref):
    """Worst scaled error over all supernode blocks (lower trapezoid); the
    measure the benchmark's parity report uses too."""
    return workload.block_errors(symb, x, ref)


def assert_blocks_close(symb, x, ref, rtol=RTOL):
    e = block_errors(symb, x, ref)
    assert e <= rtol, "scaled block error %.3e exceeds %.1e" % (e, rtol)


def rowsign_errors(symb, x, ref):
    """Like block_errors, but each row of a supernode's off-diagonal block may
    match the reference up to its sign.  Used for single applications of the
    factored-update Hessian factors (adj == inv): those rows are multiplied
    by the update factor L_k of update_factor.c, whose row signs are fixed by
    Householder pivots that can be exactly zero in exact arithmetic, where the
    reference's sign comes from its BLAS's rounding."""
    x = np.asarray(x)
    ref = np.asarray(ref)
    worst = 0.0
    for k in range(symb.Nsn):
        nn = int(symb.snptr[k + 1] - symb.snptr[k])
        nj = int(symb.sncolptr[k + 1] - symb.sncolptr[k])
        b = slice(int(symb.blkptr[k]), int(symb.blkptr[k + 1]))
        xm = x[b].reshape((nj, nn), order="F").copy()
        rm = ref[b].reshape((nj, nn), order="F")
        for i in range(nn, nj):
            if np.abs(xm[i] + rm[i]).max() < np.abs(xm[i] - rm[i]).max():
                xm[i] = -xm[i]
        mask = np.tril(np.ones((nj, nn), dtype=bool))
        rv = rm[mask]
        scale = np.maximum(np.abs(rv), FLOOR * max(np.abs(rv).max(), 1e-300))
        worst = max(worst, float((np.abs(xm[mask] - rv) / scale).max()))
    return worst
