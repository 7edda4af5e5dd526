"""Inputs of the benchmark workloads for the reference's own kernels, built
without the product library.

TEST INFRASTRUCTURE (the checker's side): used by bench.py's reference and
CPU-baseline legs and by tests/.  Nothing in chompack_b200 imports it, and it
imports nothing from chompack_b200, so a process that runs only the reference
kernels (oracle/_ref) maps no library of the product.

* `grid3d_lower(side, seed)` restates the seeded value recipe of the synthetic
  grids: 7-point pattern, strictly lower entries in compressed-column order
  drawn N(0, 1) from numpy.random.default_rng(seed), each diagonal = the sum
  of |off-diagonal| over its full symmetric row + 1.
* `load_symbolic(name)` reads a symbolic factorisation committed under
  tests/golden (written by tests/golden/make_golden.py from the reference's own
  symbolic.py, with the AMD permutation passed explicitly) and checks every
  array against the SHA-256 digests committed beside it.
* `assemble(symb, n, I, J, V)` restates the reference's cspmatrix += spmatrix
  (src/python/symbolic.py:1138-1174): the lower triangle of P·sym(A)·Pᵀ is
  scattered into the supernode blocks, column j of supernode k at
  blkptr[k] + nj·(j - snptr[k]) and row i at its position in the clique's
  row list snrowidx[sncolptr[k]:sncolptr[k+1]].
* `block_errors(symb, x, ref)` is the FP64 parity measure of the tests: the
  worst |x - x_ref| / max(|x_ref|, 1e-3·max|block_ref|) over the lower
  trapezoid of every supernode block.
"""
import hashlib
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(os.path.dirname(HERE), "tests", "golden")

# arrays of a symbolic factorisation that the reference's kernels and the
# assembly read (cbase.c:229-246, symbolic.py:1138-1174)
SYMB_ARRAYS = ("snode", "snptr", "snpar", "snpost", "relptr", "relidx", "chptr", "chidx", "sncolptr",
               "snrowidx", "blkptr", "p", "ip")
FLOOR = 1e-3


def grid3d_lower(side, seed=0):
    """(n, I, J, V): lower triangle (diagonal included) of the seeded SPD
    matrix on the side^3 7-point grid, node = x + side*(y + side*z)."""
    n = side ** 3
    idx = np.arange(n).reshape(side, side, side)
    I = np.concatenate([idx[:, :, 1:].ravel(), idx[:, 1:, :].ravel(), idx[1:, :, :].ravel()])
    J = np.concatenate([idx[:, :, :-1].ravel(), idx[:, :-1, :].ravel(), idx[:-1, :, :].ravel()])
    key = np.unique(J.astype(np.int64) * n + I)          # compressed-column order
    I, J = key % n, key // n
    v = np.random.default_rng(seed).standard_normal(I.size)
    d = np.ones(n)
    np.add.at(d, I, np.abs(v))
    np.add.at(d, J, np.abs(v))
    ar = np.arange(n, dtype=np.int64)
    return n, np.concatenate([I, ar]), np.concatenate([J, ar]), np.concatenate([v, d])


class Symbolic(object):
    """Symbolic factorisation read from a committed fixture: the arrays of
    SYMB_ARRAYS, n, Nsn, clique_number and memory, as the reference's
    symbolic object exposes them."""

    def __init__(self, arrays, scalars, memory):
        for k, v in arrays.items():
            setattr(self, k, v)
        self.n, self.Nsn, self.nnz, self.clique_number = (int(x) for x in scalars)
        self.memory = dict(memory)


def _digests(name):
    want = {}
    for line in open(os.path.join(GOLDEN, name + ".sha256")):
        parts = line.split()
        want[parts[0]] = parts[1:]
    return want


def load_symbolic(name="grid3d_40_m32"):
    """The committed symbolic factorisation `name` (tests/golden/<name>_symbolic.npz),
    each array checked against tests/golden/<name>.sha256 (int64 bytes)."""
    d = np.load(os.path.join(GOLDEN, name + "_symbolic.npz"))
    want = _digests(name)
    arrays = {}
    for a in SYMB_ARRAYS:
        arr = np.ascontiguousarray(d[a], dtype=np.int64)
        got = [str(arr.size), hashlib.sha256(arr.tobytes()).hexdigest()]
        if got != want[a]:
            raise ValueError("fixture %s: array %s does not match its digest" % (name, a))
        arrays[a] = arr
    scalars = [int(x) for x in d["scalars"]]
    if [str(x) for x in scalars] != want["scalars"]:
        raise ValueError("fixture %s: scalars do not match" % name)
    mem = dict(zip(("stack_depth", "stack_mem", "frontal_mem", "stack_solve"), (int(x) for x in d["memory"])))
    return Symbolic(arrays, scalars, mem)


def assemble(symb, n, I, J, V):
    """blkval of the cspmatrix holding the lower triangle (I >= J) of the
    symmetric matrix given by its lower entries (symbolic.py:1138-1174)."""
    ip = np.asarray(symb.ip, dtype=np.int64)
    lo = I >= J
    I, J, V = I[lo], J[lo], V[lo]
    st = I > J
    # symmetrise, permute, keep the lower triangle of the permuted matrix
    Is = np.concatenate([I, J[st]])
    Js = np.concatenate([J, I[st]])
    Vs = np.concatenate([V, V[st]])
    Ip, Jp = ip[Is], ip[Js]
    keep = Ip >= Jp
    Ip, Jp, Vs = Ip[keep], Jp[keep], Vs[keep]
    snptr = np.asarray(symb.snptr, dtype=np.int64)
    sncolptr = np.asarray(symb.sncolptr, dtype=np.int64)
    snrowidx = np.asarray(symb.snrowidx, dtype=np.int64)
    blkptr = np.asarray(symb.blkptr, dtype=np.int64)
    nsn = snptr.size - 1
    col_owner = np.repeat(np.arange(nsn, dtype=np.int64), np.diff(snptr))
    k = col_owner[Jp]
    # each clique's rows are ascending: one search over (owner, row) keys
    row_owner = np.repeat(np.arange(nsn, dtype=np.int64), np.diff(sncolptr))
    keys = row_owner * (n + 1) + snrowidx
    q = np.searchsorted(keys, k * (n + 1) + Ip)
    if np.any(q >= keys.size) or np.any(keys[np.minimum(q, keys.size - 1)] != k * (n + 1) + Ip):
        raise ValueError("entry outside the chordal pattern")
    nj = sncolptr[k + 1] - sncolptr[k]
    pos = blkptr[k] + nj * (Jp - snptr[k]) + (q - sncolptr[k])
    out = np.zeros(int(blkptr[-1]))
    np.add.at(out, pos, Vs)
    return out


def block_errors(symb, x, ref):
    """Worst scaled error over the lower trapezoid of all supernode blocks:
    |x - x_ref| / max(|x_ref|, FLOOR * max|block_ref|)."""
    x = np.asarray(x)
    ref = np.asarray(ref)
    snptr = np.asarray(symb.snptr)
    sncolptr = np.asarray(symb.sncolptr)
    blkptr = np.asarray(symb.blkptr)
    worst = 0.0
    for k in range(snptr.size - 1):
        nn = int(snptr[k + 1] - snptr[k])
        nj = int(sncolptr[k + 1] - sncolptr[k])
        b = slice(int(blkptr[k]), int(blkptr[k + 1]))
        xm = x[b].reshape((nj, nn), order="F")
        rm = ref[b].reshape((nj, nn), order="F")
        mask = np.tril(np.ones((nj, nn), dtype=bool))
        rv = rm[mask]
        scale = np.maximum(np.abs(rv), FLOOR * max(np.abs(rv).max(), 1e-300))
        worst = max(worst, float((np.abs(xm[mask] - rv) / scale).max()))
    return worst
