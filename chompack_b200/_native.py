"""ctypes binding of the in-tree native library `libchompack_b200.so`
(host symbolic analysis + the sm_100a sweeps behind include/chompack_b200.h).

There is no fallback: importing the package fails loudly when the library
has not been built (`python chompack_b200/build.py` or
`__graft_entry__.build()`).
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libchompack_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError("chompack_b200 native library not built: %s is missing "
                      "(run `python chompack_b200/build.py`)" % LIB_PATH)

lib = ctypes.CDLL(LIB_PATH, mode=ctypes.RTLD_GLOBAL)

i64 = ctypes.c_int64
P64 = ctypes.POINTER(ctypes.c_int64)
vp = ctypes.c_void_p
MERGE_FN = ctypes.CFUNCTYPE(ctypes.c_int, i64, i64, i64, i64)


def _sig(name, res, args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = args
    return f


sym_etree = _sig("chb_sym_etree", ctypes.c_int, [i64, P64, P64, P64])
sym_post_order = _sig("chb_sym_post_order", ctypes.c_int, [i64, P64, P64])
sym_counts = _sig("chb_sym_counts", ctypes.c_int, [i64, P64, P64, P64, P64, P64])
sym_supernodes = _sig("chb_sym_supernodes", ctypes.c_int, [i64, P64, P64, P64, P64, P64, P64, P64])
sym_amalgamate = _sig("chb_sym_amalgamate", ctypes.c_int,
                      [i64, P64, P64, P64, P64, P64, P64, P64, i64, i64, MERGE_FN])
sym_embed = _sig("chb_sym_embed", ctypes.c_int, [i64, P64, P64, P64, P64, P64, P64, P64, i64, P64, P64])
sym_relative_idx = _sig("chb_sym_relative_idx", ctypes.c_int, [i64, P64, P64, P64, P64, P64, P64])
amd_order = _sig("chb_amd_order", ctypes.c_int, [i64, P64, P64, P64])

last_error = _sig("chb_last_error", ctypes.c_char_p, [])
version = _sig("chb_version", ctypes.c_char_p, [])


def ptr(a):
    """int64 pointer to a C-contiguous int64 numpy array (or NULL for None)."""
    if a is None:
        return ctypes.cast(None, P64)
    assert a.dtype == np.int64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(P64)


def check(rc, what):
    if rc != 0:
        msg = last_error()
        raise RuntimeError("%s failed (code %d)%s" % (what, rc, (": " + msg.decode()) if msg else ""))

# ---- plan / sweeps (include/chompack_b200.h)
PPLAN = ctypes.c_void_p
plan_create = _sig("chb_plan_create", ctypes.c_int,
                   [i64, i64, P64, P64, P64, P64, P64, P64, P64, P64, P64, ctypes.c_int, ctypes.POINTER(PPLAN)])
plan_destroy = _sig("chb_plan_destroy", ctypes.c_int, [PPLAN])
workspace_size = _sig("chb_workspace_size", ctypes.c_int,
                      [PPLAN, ctypes.c_int, i64, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)])
program_info = _sig("chb_program_info", ctypes.c_int, [PPLAN, ctypes.c_int, i64, ctypes.c_int, P64])
program_pool = _sig("chb_program_pool", ctypes.c_int, [PPLAN, ctypes.c_int, i64, ctypes.c_int, P64])
cholesky = _sig("chb_cholesky", ctypes.c_int, [PPLAN, vp, vp, ctypes.c_size_t, vp])
projected_inverse = _sig("chb_projected_inverse", ctypes.c_int, [PPLAN, vp, vp, ctypes.c_size_t, vp])
llt = _sig("chb_llt", ctypes.c_int, [PPLAN, vp, vp, ctypes.c_size_t, vp])
completion = _sig("chb_completion", ctypes.c_int, [PPLAN, vp, ctypes.c_int, vp, ctypes.c_size_t, vp])
hessian = _sig("chb_hessian", ctypes.c_int, [PPLAN, vp, vp, ctypes.POINTER(vp), i64, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_int, vp, ctypes.c_size_t, vp])
trsm = _sig("chb_trsm", ctypes.c_int, [PPLAN, ctypes.c_char, i64, ctypes.c_double, vp, vp, i64, vp, ctypes.c_size_t, vp])
trsm_reuse = _sig("chb_trsm_reuse", ctypes.c_int, [PPLAN, ctypes.c_char, i64, ctypes.c_double, vp, vp, i64, vp,
                                                   ctypes.c_size_t, ctypes.c_int, vp])
trmm = _sig("chb_trmm", ctypes.c_int, [PPLAN, ctypes.c_char, i64, ctypes.c_double, vp, vp, i64, vp, ctypes.c_size_t, vp])
dot = _sig("chb_dot", ctypes.c_int, [PPLAN, vp, vp, vp, vp, ctypes.c_size_t, vp])
plan_merge = _sig("chb_plan_merge", ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_int,
                                                    ctypes.POINTER(PPLAN)])
plan_batch_info = _sig("chb_plan_batch_info", ctypes.c_int, [PPLAN, ctypes.POINTER(i64), ctypes.POINTER(i64)])
logdet_batch = _sig("chb_logdet_batch", ctypes.c_int, [PPLAN, vp, vp, vp, ctypes.c_size_t, vp])
dot_batch = _sig("chb_dot_batch", ctypes.c_int, [PPLAN, vp, vp, vp, vp, ctypes.c_size_t, vp])
logdet = _sig("chb_logdet", ctypes.c_int, [PPLAN, vp, vp, vp, ctypes.c_size_t, vp])
sym_weight = _sig("chb_sym_weight", ctypes.c_int, [PPLAN, vp, vp, ctypes.c_double, vp])
info = _sig("chb_info", ctypes.c_int, [PPLAN, vp, vp])
set_trace = _sig("chb_set_trace", ctypes.c_int, [PPLAN, vp, i64])
plan_set_schedule = _sig("chb_plan_set_schedule", ctypes.c_int, [PPLAN, ctypes.c_int])
plan_set_spin_limit = _sig("chb_plan_set_spin_limit", ctypes.c_int, [PPLAN, i64])
io_flags = _sig("chb_io_flags", ctypes.c_int, [ctypes.c_int, ctypes.c_int])
io_overlap_available = _sig("chb_io_overlap_available", ctypes.c_int, [])
precision_flags = _sig("chb_precision_flags", ctypes.c_int, [ctypes.c_int])
cholesky_prec = _sig("chb_cholesky_prec", ctypes.c_int, [PPLAN, ctypes.c_int, vp, vp, vp, vp, ctypes.c_size_t, vp])
projected_inverse_prec = _sig("chb_projected_inverse_prec", ctypes.c_int,
                              [PPLAN, ctypes.c_int, vp, vp, vp, vp, ctypes.c_size_t, vp])
symv = _sig("chb_symv", ctypes.c_int, [PPLAN, vp, vp, vp, vp, vp, i64, i64, ctypes.c_double, vp])
PREC = {"fp64": 0, "tf32": 1, "tf32x3": 2}
cholesky_io = _sig("chb_cholesky_io", ctypes.c_int, [PPLAN, vp, vp, vp, vp, ctypes.c_size_t, vp])
projected_inverse_io = _sig("chb_projected_inverse_io", ctypes.c_int, [PPLAN, vp, vp, vp, vp, ctypes.c_size_t, vp])
llt_io = _sig("chb_llt_io", ctypes.c_int, [PPLAN, vp, vp, vp, vp, ctypes.c_size_t, vp])
program_io = _sig("chb_program_io", ctypes.c_int, [PPLAN, ctypes.c_int, i64, ctypes.c_int, P64, vp, vp, vp, vp])

OP_CHOLESKY, OP_LLT, OP_PROJECTED_INVERSE, OP_COMPLETION, OP_HESSIAN, OP_TRSM, OP_DOT, OP_TRMM, OP_CONVENTIONAL = range(9)
HESSIAN_MAX_U = 59   # U matrices per chb_hessian call (base slots 5..63)

# ---- product-form Cholesky factor (chb_pftrf / chb_pfsv / chb_pfmv)
pf_workspace_size = _sig("chb_pf_workspace_size", ctypes.c_int, [i64, i64, ctypes.POINTER(ctypes.c_size_t)])
pftrf = _sig("chb_pftrf", ctypes.c_int, [i64, i64, vp, vp, i64, vp, i64, vp, i64, vp, ctypes.c_size_t, vp])
pfsv = _sig("chb_pfsv", ctypes.c_int, [i64, i64, ctypes.c_char, vp, i64, vp, i64, vp, i64, vp, i64, i64, vp,
                                       ctypes.c_size_t, vp])
pfmv = _sig("chb_pfmv", ctypes.c_int, [i64, i64, ctypes.c_char, vp, i64, vp, i64, vp, i64, vp, i64, i64, vp,
                                       ctypes.c_size_t, vp])
pf_info = _sig("chb_pf_info", ctypes.c_int, [vp, vp])

# ---- block exports and element-wise updates (csrc/export.cu, build_conventional.cpp)
factor_conventional = _sig("chb_factor_conventional", ctypes.c_int, [PPLAN, vp, vp, ctypes.c_size_t, vp])
lower_ccs = _sig("chb_lower_ccs", ctypes.c_int, [PPLAN, vp, vp, vp, vp, vp, vp, vp])
syr2 = _sig("chb_syr2", ctypes.c_int, [PPLAN, vp, vp, vp, vp, vp, ctypes.c_double, ctypes.c_double, ctypes.c_int, vp])
add_projection = _sig("chb_add_projection", ctypes.c_int, [PPLAN, vp, vp, vp, vp, i64, ctypes.c_double,
                                                           ctypes.c_double, ctypes.c_int, vp])
diag = _sig("chb_diag", ctypes.c_int, [PPLAN, vp, vp, vp])
add_sparse = _sig("chb_add_sparse", ctypes.c_int, [PPLAN, vp, vp, vp, i64, vp, vp, vp, ctypes.c_double, ctypes.c_int,
                                                   vp, vp])

# ---- program-build options (chb_plan_set_option)
plan_set_option = _sig("chb_plan_set_option", ctypes.c_int, [PPLAN, ctypes.c_int, i64])
plan_get_option = _sig("chb_plan_get_option", ctypes.c_int, [PPLAN, ctypes.c_int, ctypes.POINTER(i64)])
OPTIONS = {"small_front_nj": 0, "subtrees": 1, "chol_ksplit": 2, "pinv_ksplit": 3, "fused_la": 4,
           "tf32_tcgen05": 5, "ordered_sums": 6, "scratch_limit": 7}
engine_occupancy = _sig("chb_engine_occupancy", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_int)])
