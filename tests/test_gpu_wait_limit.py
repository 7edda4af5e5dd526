"""The bounded-wait failure path on the GPU, without a fault: a sweep whose
waits give up returns status -30 (RuntimeError from cbase), the kernel
returns, and the next sweep on the same plan is correct.

The waits are made to run out by a plan-level limit of zero polls on a
streamed cholesky of host values: its arrival tasks wait for chunks of
about 10 MB that the copy stream starts only when the kernel is launched
(about 0.2 ms each over PCIe), so a wait that may poll only once gives up.
Nothing faults or hangs: every wait in the engine is bounded, and the last
CTA to leave raises every output flag so the copy streams finish."""
import numpy as np
import pytest
import torch

import chompack_b200 as cp
from helpers import problem, assert_blocks_close
from oracle import ref

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")


def test_streamed_arrival_waits_run_out_then_the_plan_recovers():
    A, s = problem("grid3d", 40, merge=(32, 32), seed=0)
    x0 = (cp.cspmatrix(s, device="cpu") + A).blkval
    r = x0.numpy().copy()
    assert ref.cholesky(s, r) == 0
    plan = s.plan()
    plan.set_spin_limit(0)
    X = cp.cspmatrix(s, blkval=x0.clone().pin_memory())
    with pytest.raises(RuntimeError, match="timed out"):
        cp.cholesky(X)
    torch.cuda.synchronize()              # the kernel and the copy streams have finished
    plan.set_spin_limit(None)
    for _ in range(2):
        Y = cp.cspmatrix(s, blkval=x0.clone().pin_memory())
        cp.cholesky(Y)
        assert_blocks_close(s, Y.blkval.numpy(), r)
    Z = cp.cspmatrix(s, blkval=x0.clone().cuda())
    cp.cholesky(Z)
    assert_blocks_close(s, Z.blkval.cpu().numpy(), r)


def test_spin_limit_setter_accepts_default_and_values():
    A, s = problem("grid2d", 12, seed=1)
    plan = s.plan()
    plan.set_spin_limit(123)
    plan.set_spin_limit(None)
    X = cp.cspmatrix(s) + A
    r = X.blkval.cpu().numpy().copy()
    assert ref.cholesky(s, r) == 0
    cp.cholesky(X)
    assert_blocks_close(s, X.blkval.cpu().numpy(), r)
