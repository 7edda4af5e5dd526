"""Generate the golden fixtures under tests/golden/ (run where the reference
tree is available; the fixtures are committed and the GPU box never needs
the reference).

    python tests/golden/make_golden.py

For every case it records the input pattern and values, the permutation
given to `symbolic`, and what the *reference* produces for them:

* the symbolic arrays, scalars and workspace sizes of the reference's own
  `src/python/symbolic.py` (run unmodified under the cvxopt stand-in in
  ./shim; see refload.py);
* the block values of `cspmatrix(symb) + A` from the reference's
  `_iadd_spmatrix` (symbolic.py:1138-1174);
* for the smaller cases, the outputs of the reference's numeric C kernels
  (oracle/_ref): cholesky, llt, projected_inverse, completion (both update
  modes), hessian (all adj/inv modes, both update modes), trsm ('N'/'T') and
  dot, on seeded inputs.

Permutations: `None` for the natural-order cases; otherwise the AMD ordering
of chompack_b200 (cvxopt's AMD is not part of the reference), stored in the
fixture so both sides see the same explicit permutation.
"""
import hashlib
import os
import random
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from refload import load_reference  # noqa: E402

SYMB_ARRAYS = ["snode", "snptr", "snpar", "snpost", "relptr", "relidx", "chptr", "chidx", "sncolptr",
               "snrowidx", "blkptr", "p", "ip"]


def _case_inputs():
    import chompack_b200 as cp
    from chompack_b200 import grids
    cases = {}
    I = list(range(17)) + [2, 2, 3, 3, 4, 14, 4, 14, 8, 14, 15, 8, 15, 7, 8, 14, 8, 14, 14, 15, 10, 12, 13, 16, 12, 13,
                           16, 12, 13, 15, 16, 13, 15, 16, 15, 16, 15, 16, 16]
    J = list(range(17)) + [0, 1, 1, 2, 2, 2, 3, 3, 4, 4, 4, 5, 5, 6, 6, 6, 7, 7, 8, 8, 9, 9, 9, 9, 10, 10, 10, 11, 11,
                           11, 11, 12, 12, 12, 13, 13, 14, 14, 15]
    A17 = cp.spmatrix(np.arange(len(I), dtype=float), I, J, (17, 17))   # tests/test_symbolic.py:9-11
    cases["chordal17"] = (A17, None, None)
    cases["chordal17_m22"] = (A17, None, (2, 2))
    n = 23
    nz = [1, 2, 10, 12, 13, 14, 15, 16, 19, 24, 48, 58, 71, 76, 81, 85, 91, 103, 108, 109, 111, 114, 116, 117, 118,
          134, 143, 145, 161, 174, 178, 180, 183, 192, 194, 202, 203, 205, 212, 214, 219, 224, 226, 227, 228, 229,
          235, 240, 241, 243, 247, 255, 256, 260, 269, 273, 275, 279, 280, 314, 315, 320, 321, 328, 340, 342, 344,
          345, 349, 350, 357, 359, 370, 372, 375, 384, 385, 394, 399, 402, 411, 412, 419, 420, 422, 433, 439, 441,
          447, 452, 454, 458, 460, 474, 476, 479, 481, 483, 485, 497, 506, 517, 519, 523, 526, 527]
    Anc = cp.tril(cp.spmatrix(np.arange(1, len(nz) + 1) / len(nz), [v % n for v in nz], [v // n for v in nz], (n, n))) \
        + cp.spmatrix(10.0, range(n), range(n))                           # tests/test_symbolic.py:13-16
    cases["nc23"] = (Anc, None, None)
    cases["nc23_amd"] = (Anc, "amd", None)
    cases["nc23_amd_m44"] = (Anc, "amd", (4, 4))
    A7 = cp.spmatrix([0.1 * (i + 1) for i in range(15)], [0, 1, 3, 1, 5, 2, 6, 3, 4, 5, 4, 5, 6, 5, 6],
                     [0, 0, 0, 1, 1, 2, 2, 3, 3, 3, 4, 4, 4, 5, 6], (7, 7)) + cp.spmatrix(10.0, range(7), range(7))
    cases["quick7"] = (A7, "amd", None)                                  # doc/source/quick_start.rst:200-205
    n = 31                                                               # tests/test_numeric.py:8-15
    nnz = int(round(0.15 * n ** 2))
    random.seed(1)
    nzs = random.sample(range(n ** 2), nnz)
    A31 = cp.tril(cp.spmatrix(np.arange(1, nnz + 1) / nnz, [v % n for v in nzs], [v // n for v in nzs], (n, n))) \
        + cp.spmatrix(10.0, range(n), range(n))
    cases["numeric31"] = (A31, "amd", None)
    L17 = [[0, 2, 3, 4, 14], [1, 2, 3], [2, 3, 4, 14], [3, 4, 14], [4, 8, 14, 15], [5, 8, 15], [6, 7, 8, 14], [7, 8, 14],
           [8, 14, 15], [9, 10, 12, 13, 16], [10, 12, 13, 16], [11, 12, 13, 15, 16], [12, 13, 15, 16], [13, 15, 16],
           [14, 15, 16], [15, 16], [16]]                                 # doc/source/examples.rst:275-290
    Ie, Je = [], []
    for k, lst in enumerate(L17):
        Ie.extend(lst)
        Je.extend(len(lst) * [k])
    cases["ex17"] = (cp.spmatrix(1.0, Ie, Je, (17, 17)) + cp.spmatrix(16.0, range(17), range(17)), "amd", None)
    cases["grid2d_30_m16"] = (grids.grid2d(30, seed=0), "amd", (16, 16))
    cases["grid3d_8"] = (grids.grid3d(8, seed=1), "amd", None)
    cases["grid3d_12_m32"] = (grids.grid3d(12, seed=1), "amd", (32, 32))
    cases["g2dx_20"] = (grids.grid2d_extra(20, seed=3), "amd", None)
    cases["rand200_m164"] = (grids.random_lower(200, 0.02, seed=5), "amd", (16, 4))
    return cases


NUMERIC = {"nc23_amd", "quick7", "numeric31", "ex17", "rand200_m164"}


def _ref_numeric(symb, blk0, seed):
    """Reference C kernel outputs for one case."""
    from oracle import ref
    out = {}
    L = blk0.copy()
    assert ref.cholesky(symb, L) == 0
    out["cholesky"] = L.copy()
    X = L.copy()
    ref.llt(symb, X)
    out["llt"] = X
    Y = L.copy()
    assert ref.projected_inverse(symb, Y) == 0
    out["projected_inverse"] = Y.copy()
    for fu in (0, 1):
        C = Y.copy()
        assert ref.completion(symb, C, factored_updates=bool(fu)) == 0
        out["completion_fu%d" % fu] = C
    rng = np.random.default_rng(seed)
    U0 = blk0 * rng.standard_normal(blk0.size)   # a symmetric direction on the pattern
    out["hessian_U0"] = U0
    for fu in (0, 1):
        for adj in (0, 1):
            for inv in (0, 1):
                U = U0.copy()
                ref.hessian(symb, L, Y, [U], adj=bool(adj), inv=bool(inv), factored_updates=bool(fu))
                out["hessian_a%d_i%d_fu%d" % (adj, inv, fu)] = U
        U = U0.copy()
        ref.hessian(symb, L, Y, [U], adj=None, inv=False, factored_updates=bool(fu))
        out["hessian_full_fu%d" % fu] = U
    B0 = np.asfortranarray(rng.standard_normal((symb.n, 3)))
    out["trsm_B0"] = B0
    for tr in "NT":
        Bt = B0.copy(order="F")
        ref.trsm(symb, L, Bt, alpha=0.5, trans=tr)
        out["trsm_" + tr] = Bt
    out["dot"] = np.array([ref.dot(symb, blk0.copy(), Y.copy())])
    return out


def main():
    import chompack_b200 as cp
    S, M = load_reference()
    from cvxopt import matrix as cmat, spmatrix as cspm
    cases = _case_inputs()
    for name, (A, p, merge) in cases.items():
        pv = cp.amd.order(A) if p == "amd" else None
        Aref = cspm(list(A.V), list(A.I), list(A.J), A.size)
        mf = S.merge_size_fill(*merge) if merge else None
        sr = S.symbolic(Aref, p=None if pv is None else cmat(list(pv)), merge_function=mf)
        d = {"I": A.I, "J": A.J, "V": A.V, "size": np.array(A.size), "perm": pv if pv is not None else np.array([-1]),
             "merge": np.array(merge if merge else (-1, -1))}
        for a in SYMB_ARRAYS:
            d["symb_" + a] = np.array(list(getattr(sr, a)), dtype=np.int64)
        d["symb_scalars"] = np.array([sr.n, sr.Nsn, sr.nnz, sr.clique_number, sr.fill[0], sr.fill[1],
                                      sr.frontal_len, sr.stack_len, sr.stack_size], dtype=np.float64)
        mem = sr.memory
        d["symb_memory"] = np.array([mem["stack_depth"], mem["stack_mem"], mem["frontal_mem"], mem["stack_solve"]],
                                    dtype=np.int64)
        Xr = S.cspmatrix(sr) + Aref                # the reference's own assembly
        blk0 = np.array(list(Xr.blkval), dtype=np.float64)
        d["blkval"] = blk0
        if name in NUMERIC:
            sm = cp.symbolic(A, p=pv, merge_function=cp.merge_size_fill(*merge) if merge else None)
            for k, v in _ref_numeric(sm, blk0, seed=len(name)).items():
                d["ref_" + k] = v
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **d)
        print("%-16s n=%-5d Nsn=%-4d %s" % (name, sr.n, sr.Nsn, "numeric" if name in NUMERIC else ""))

    # the FP64 drop-in configuration (40^3 grid, AMD, merge 32/32): digests
    # of the reference's symbolic arrays (the arrays themselves are large)
    if "--large" in sys.argv:
        from chompack_b200 import grids
        A = grids.grid3d(40, seed=0)
        pv = cp.amd.order(A)
        sr = S.symbolic(cspm(list(A.V), list(A.I), list(A.J), A.size), p=cmat(list(pv)),
                        merge_function=S.merge_size_fill(32, 32))
        lines = []
        for a in SYMB_ARRAYS:
            arr = np.array(list(getattr(sr, a)), dtype=np.int64)
            lines.append("%s %d %s" % (a, arr.size, hashlib.sha256(arr.tobytes()).hexdigest()))
        lines.append("scalars %d %d %d %d" % (sr.n, sr.Nsn, sr.nnz, sr.clique_number))
        with open(os.path.join(HERE, "grid3d_40_m32.sha256"), "w") as f:
            f.write("\n".join(lines) + "\n")
        # the arrays themselves, compact (int32 fits every entry), for the
        # benchmark's reference leg: it runs the reference kernels on them
        # without loading the product library (oracle/workload.py)
        mem = sr.memory
        np.savez_compressed(
            os.path.join(HERE, "grid3d_40_m32_symbolic.npz"),
            scalars=np.array([sr.n, sr.Nsn, sr.nnz, sr.clique_number], dtype=np.int64),
            memory=np.array([mem["stack_depth"], mem["stack_mem"], mem["frontal_mem"], mem["stack_solve"]],
                            dtype=np.int64),
            **{a: np.array(list(getattr(sr, a)), dtype=np.int32) for a in SYMB_ARRAYS})
        print("grid3d_40_m32 digests and arrays written")


if __name__ == "__main__":
    main()
