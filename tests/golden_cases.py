"""Loading of the committed golden fixtures (tests/golden/*.npz, written by
tests/golden/make_golden.py from the reference's own symbolic.py and C
kernels)."""
import glob
import os

import numpy as np

import chompack_b200 as cp

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SYMB_ARRAYS = ["snode", "snptr", "snpar", "snpost", "relptr", "relidx", "chptr", "chidx", "sncolptr",
               "snrowidx", "blkptr", "p", "ip"]


def names(numeric_only=False):
    out = []
    for f in sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))):
        nm = os.path.basename(f)[:-4]
        if nm.endswith("_symbolic"):   # symbolic arrays only (the benchmark's reference leg)
            continue
        if numeric_only:
            with np.load(f) as d:
                if "ref_cholesky" not in d.files:
                    continue
        out.append(nm)
    return out


def load(name):
    d = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    A = cp.spmatrix(d["V"], d["I"], d["J"], tuple(int(x) for x in d["size"]))
    perm = None if d["perm"][0] < 0 else d["perm"]
    merge = None if d["merge"][0] < 0 else (int(d["merge"][0]), int(d["merge"][1]))
    symb = cp.symbolic(A, p=perm, merge_function=cp.merge_size_fill(*merge) if merge else None)
    return d, A, symb
