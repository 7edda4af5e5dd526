"""The C ABI library (CPU): it loads, exports every function that
include/chompack_b200.h declares, and rejects inconsistent input with an
error code and message rather than touching the device."""
import ctypes
import os
import re

import numpy as np

from chompack_b200 import _native as N

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "chompack_b200.h")


def test_every_declared_function_is_exported():
    src = open(HEADER).read()
    names = sorted(set(re.findall(r"^\s*(?:int|const char\*|void)\s+(chb_\w+)\s*\(", src, re.M)))
    assert len(names) > 20
    missing = [n for n in names if not hasattr(N.lib, n)]
    assert not missing, missing


def test_plan_rejects_inconsistent_blkptr():
    import chompack_b200 as cp
    from chompack_b200 import grids
    A = grids.grid2d(8, seed=0)
    s = cp.symbolic(A, p=cp.amd.order(A))
    arrs = [np.ascontiguousarray(getattr(s, a), dtype=np.int64) for a in
            ("snptr", "snpar", "relptr", "relidx", "chptr", "chidx", "blkptr", "snode", "p")]
    arrs[6] = arrs[6].copy()
    arrs[6][-1] += 1
    h = N.PPLAN()
    rc = N.plan_create(s.n, s.Nsn, *[N.ptr(a) for a in arrs], -1, ctypes.byref(h))
    assert rc < 0
    assert b"blkptr" in N.last_error()


def test_host_only_plan_programs_and_workspace():
    import chompack_b200 as cp
    from chompack_b200 import grids
    from chompack_b200.plan import Plan
    A = grids.grid3d(8, seed=0)
    s = cp.symbolic(A, p=cp.amd.order(A), merge_function=cp.merge_size_fill(16, 16))
    pl = Plan(s, device=-1)
    for op in (N.OP_CHOLESKY, N.OP_PROJECTED_INVERSE, N.OP_LLT):
        info = pl.program_info(op)
        assert info["tasks"] > 0 and info["ws_bytes"] >= 256 + 8 * info["upd_doubles"]
    assert pl.workspace_bytes(N.OP_DOT) >= 8 * s.Nsn


def test_trsm_and_trmm_reject_bad_arguments_before_touching_the_device():
    import chompack_b200 as cp
    from chompack_b200 import grids
    from chompack_b200.plan import Plan
    A = grids.grid2d(8, seed=0)
    s = cp.symbolic(A, p=cp.amd.order(A))
    pl = Plan(s, device=-1)
    for fn in (N.trsm, N.trmm):
        assert fn(pl.handle, b"X", 2, 1.0, None, None, s.n, None, 0, None) < 0
        assert b"trans" in N.last_error()
        assert fn(pl.handle, b"N", 2, 1.0, None, None, s.n - 1, None, 0, None) < 0
        assert b"ldB" in N.last_error()
    # the trmm programs exist for both transposes and need the right-hand
    # sides' workspace: Bp and the update blocks, plus u'_k for 'N'
    n_ws = pl.program_info(N.OP_TRMM, k=3, flags=0)["ws_doubles"]
    t_ws = pl.program_info(N.OP_TRMM, k=3, flags=1)["ws_doubles"]
    na = np.diff(np.asarray(s.relptr)).sum()
    assert t_ws == 3 * (s.n + na) and n_ws == 3 * (s.n + 2 * na)


def test_product_form_entry_points_reject_bad_arguments_before_touching_the_device():
    """chb_pfsv / chb_pfmv / chb_pftrf validate trans and the leading
    dimensions on the host (no CUDA call), like cbase.pftrsm's ValueError."""
    from chompack_b200 import _native as N
    for fn in (N.pfsv, N.pfmv):
        assert fn(10, 2, b"X", None, 10, None, 10, None, 10, None, 10, 1, None, 0, None) < 0
        assert "trans" in N.last_error().decode()
        assert fn(10, 2, b"N", 16, 9, 16, 10, 16, 10, 16, 10, 1, None, 0, None) < 0   # never dereferenced
        assert "leading" in N.last_error().decode()
    assert N.pftrf(10, 2, None, None, 10, None, 10, None, 10, None, 0, None) < 0
    assert N.pftrf(-1, 2, None, None, 10, None, 10, None, 10, None, 0, None) < 0
