"""GPU test of the allocation-free Cholesky entry point, chb_cholesky_noalloc.

Callers that cannot call cudaMalloc when they factor (code running under CUDA
graph capture, frameworks that own all device memory, processes that must
not grow their device footprint) use this entry point: it keeps all its
device scratch in one static array compiled into the library.  This test
calls it through the C ABI, twice in a row, and checks each result against
the regular entry point (chb_cholesky, via chompack_b200.cholesky) within the
parity tolerance used by every FP64 test (helpers.RTOL).  It also checks that
a factorisation larger than the static array is refused with a clear error.
"""
import ctypes

import pytest
import torch

import chompack_b200 as cp
from chompack_b200 import _native as N
from helpers import problem, assert_blocks_close

pytestmark = pytest.mark.gpu

N.lib.chb_cholesky_noalloc.restype = ctypes.c_int
N.lib.chb_cholesky_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]


@pytest.fixture(scope="module", autouse=True)
def _need_cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")


def _noalloc(symb, values):
    plan = symb.plan(values.device.index)
    stream = torch.cuda.current_stream(values.device).cuda_stream
    return N.lib.chb_cholesky_noalloc(plan.handle, values.data_ptr(), stream)


@pytest.mark.parametrize("kind,args,merge", [("grid3d", (12,), (32, 32)), ("random", (300, 0.05), (16, 16))])
def test_noalloc_matches_regular_entry_point_twice(kind, args, merge):
    A, s = problem(kind, *args, merge=merge, seed=11)
    X = cp.cspmatrix(s) + A
    expected = X.copy()
    cp.cholesky(expected)
    want = expected.blkval.cpu().numpy()
    for _ in range(2):
        Y = X.blkval.clone()
        rc = _noalloc(s, Y)
        assert rc == 0, N.last_error().decode()
        assert_blocks_close(s, Y.cpu().numpy(), want)


def test_noalloc_rejects_problems_beyond_the_static_scratch():
    A, s = problem("grid3d", 40, merge=(32, 32), seed=0)
    Y = (cp.cspmatrix(s) + A).blkval
    rc = _noalloc(s, Y)
    assert rc == -40
    assert "limited to" in N.last_error().decode()
