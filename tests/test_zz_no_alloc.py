"""GPU test of the allocation-free Cholesky entry point, chb_cholesky_noalloc.

Callers that cannot call cudaMalloc when they factor (frameworks whose device
memory all comes from their own pool, processes held to a fixed device
footprint after start-up) use this entry point: it keeps all its device
scratch in one static array compiled into the library.  This test calls it
through the C ABI, twice in a row, and checks each result against the
regular entry point (chb_cholesky, via chompack_b200.cholesky) and against
the reference's own kernels (oracle/_ref), within the parity tolerance used
by every FP64 test (helpers.RTOL).  It also checks that a call allocates no
device memory, that a matrix that is not positive definite gives the same
LAPACK-style info as chb_cholesky, that a host-only plan works, and that a
factorisation larger than the static array is refused with a clear error.

The file is named to be collected last: a run that stops at the first
failure has run every other test by the time it gets here.
"""
import ctypes

import pytest
import torch

import chompack_b200 as cp
from chompack_b200 import _native as N
from chompack_b200.plan import Plan
from helpers import problem, assert_blocks_close
from oracle import ref

pytestmark = pytest.mark.gpu

N.lib.chb_cholesky_noalloc.restype = ctypes.c_int
N.lib.chb_cholesky_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]


@pytest.fixture(scope="module", autouse=True)
def _need_cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")


def _noalloc(plan, values):
    stream = torch.cuda.current_stream(values.device).cuda_stream
    return N.lib.chb_cholesky_noalloc(plan.handle, values.data_ptr(), stream)


def _regular_info(symb, values):
    """Status of the regular entry point (chb_cholesky + chb_info) on `values`."""
    plan = symb.plan(values.device.index)
    ws, nbytes = plan.workspace(N.OP_CHOLESKY)
    stream = torch.cuda.current_stream(values.device).cuda_stream
    assert N.cholesky(plan.handle, values.data_ptr(), ws, nbytes, stream) == 0, N.last_error().decode()
    return N.info(plan.handle, ws, stream)


@pytest.mark.parametrize("kind,args,merge", [("grid3d", (12,), (32, 32)), ("random", (300, 0.05), (16, 16))])
def test_noalloc_matches_regular_entry_point_and_reference_twice(kind, args, merge):
    A, s = problem(kind, *args, merge=merge, seed=11)
    X = cp.cspmatrix(s) + A
    oracle_values = X.blkval.cpu().numpy().copy()
    assert ref.cholesky(s, oracle_values) == 0
    expected = X.copy()
    cp.cholesky(expected)
    want = expected.blkval.cpu().numpy()
    plan = s.plan(X.blkval.device.index)
    for _ in range(2):
        Y = X.blkval.clone()
        rc = _noalloc(plan, Y)
        assert rc == 0, N.last_error().decode()
        got = Y.cpu().numpy()
        assert_blocks_close(s, got, want)
        assert_blocks_close(s, got, oracle_values)


def test_noalloc_allocates_no_device_memory_and_takes_host_only_plans():
    A, s = problem("grid3d", 10, merge=(16, 16), seed=3)
    X = cp.cspmatrix(s) + A
    oracle_values = X.blkval.cpu().numpy().copy()
    assert ref.cholesky(s, oracle_values) == 0
    warm = X.blkval.clone()
    assert _noalloc(s.plan(warm.device.index), warm) == 0, N.last_error().decode()
    host_plan = Plan(s, device=-1)      # uploads nothing
    Y = X.blkval.clone()
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    rc = _noalloc(host_plan, Y)
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert rc == 0, N.last_error().decode()
    assert free_after == free_before, "device memory changed by %d bytes" % (free_before - free_after)
    assert_blocks_close(s, Y.cpu().numpy(), oracle_values)


def test_noalloc_reports_the_same_info_as_chb_cholesky_when_not_positive_definite():
    A, s = problem("grid2d", 10, merge=None, seed=2)
    X = cp.cspmatrix(s) + A
    X.blkval.mul_(-1.0)
    info = _regular_info(s, X.blkval.clone())
    assert info > 0
    rc = _noalloc(s.plan(X.blkval.device.index), X.blkval.clone())
    assert rc == info


def test_noalloc_rejects_problems_beyond_the_static_scratch():
    A, s = problem("grid3d", 40, merge=(32, 32), seed=0)
    Y = (cp.cspmatrix(s) + A).blkval
    rc = _noalloc(s.plan(Y.device.index), Y)
    assert rc == -40
    assert "limited to" in N.last_error().decode()


def test_noalloc_under_a_scratch_limit():
    """Under a scratch limit the program carries its own update-matrix
    offsets (a pool); the allocation-free entry point stages those, and
    the result is bit-identical to the unlimited layout."""
    A, s = problem("grid3d", 12, merge=(32, 32), seed=13)
    X = cp.cspmatrix(s) + A
    plan = Plan(s, device=-1)
    Y0 = X.blkval.clone()
    assert _noalloc(plan, Y0) == 0, N.last_error().decode()
    plan.set_option("scratch_limit", 0)
    assert plan.pool_info(N.OP_CHOLESKY)["pool_bytes"] is not None
    Y1 = X.blkval.clone()
    assert _noalloc(plan, Y1) == 0, N.last_error().decode()
    torch.cuda.synchronize()
    assert torch.equal(Y0, Y1)
