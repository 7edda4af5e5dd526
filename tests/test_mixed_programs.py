"""Mixed-precision program variants, on the CPU: the TF32 / 3xTF32 variants
of cholesky and projected_inverse mark exactly the GEMM tasks (the FP64
steps, diagonal tiles, look-ahead, sums, assembly, are unmarked), keep the
task graph of the FP64 program, and other sweeps refuse the flag."""
import ctypes

import numpy as np
import pytest

from chompack_b200 import _native as N
from chompack_b200.plan import Plan
from helpers import problem
import taskvm


@pytest.mark.parametrize("op", [N.OP_CHOLESKY, N.OP_PROJECTED_INVERSE])
@pytest.mark.parametrize("prec", ["tf32", "tf32x3"])
def test_gemm_tasks_carry_the_precision(op, prec):
    A, s = problem("grid3d", 10, merge=(32, 32), seed=1)
    pl = Plan(s, device=-1)
    code = N.PREC[prec]
    base = taskvm.Program(pl.handle, op, nsn=s.Nsn)
    mixed = taskvm.Program(pl.handle, op, flags=N.precision_flags(code), nsn=s.Nsn)
    assert mixed.ntasks == base.ntasks and np.array_equal(mixed.waits, base.waits)
    gemm = mixed.tasks["op"] == taskvm.T_GEMM
    assert gemm.sum() > 0
    assert np.all(mixed.tasks["c"]["prec"][gemm] == code)
    assert np.all(mixed.tasks["c"]["prec"][~gemm] == 0)
    assert np.all(base.tasks["c"]["prec"] == 0)
    for f in ("a", "b"):
        assert np.all(mixed.tasks[f]["prec"] == 0)


def test_mixed_precision_only_for_two_sweeps():
    A, s = problem("grid2d", 8, merge=(8, 8), seed=1)
    pl = Plan(s, device=-1)
    info = (ctypes.c_int64 * 8)()
    assert N.program_info(pl.handle, N.OP_COMPLETION, 1, N.precision_flags(1), info) != 0
    assert b"mixed precision" in N.last_error()
