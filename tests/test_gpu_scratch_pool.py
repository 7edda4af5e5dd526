"""Update matrices under a scratch limit on the GPU: cholesky and
projected_inverse with their update matrices in a shared pool
(CHB_OPT_SCRATCH_LIMIT) give bit-identical results to the default layout
(every task computes the same thing in the same order; only the memory a
front's update matrix lives in, and the waits that protect its reuse,
change), under both schedules, and match the reference's kernels; the
workspace shrinks.  Batched value sets on a merged plan and the
differentiable log det take the limit too."""
import numpy as np
import pytest
import torch

import chompack_b200 as cp
from chompack_b200 import _native as N
from helpers import problem, assert_blocks_close
from oracle import ref

pytestmark = pytest.mark.gpu

CASES = [("grid3d", (16,), (32, 32)), ("grid3d", (14,), None), ("grid2d", (90,), (64, 64))]


@pytest.fixture(scope="module", autouse=True)
def _need_cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")


def _sweeps(s, blk0, limit, mode=None):
    pl = s.plan(0)
    pl.set_schedule(mode)
    pl.set_option("scratch_limit", limit)
    try:
        X = cp.cspmatrix(s, blkval=torch.from_numpy(blk0.copy()).cuda(), factor=False)
        cp.cholesky(X)
        L = X.blkval.clone()
        Y = cp.cspmatrix(s, blkval=L.clone(), factor=True)
        cp.projected_inverse(Y)
        torch.cuda.synchronize()
        info = (pl.pool_info(N.OP_CHOLESKY), pl.pool_info(N.OP_PROJECTED_INVERSE))
        return L.cpu().numpy(), Y.blkval.cpu().numpy(), info
    finally:
        pl.set_schedule(None)
        pl.set_option("scratch_limit", None)


@pytest.mark.parametrize("kind,args,merge", CASES)
@pytest.mark.parametrize("mode", ["static", "dynamic"])
def test_pooled_sweeps_bit_identical(kind, args, merge, mode):
    A, s = problem(kind, *args, merge=merge, seed=7)
    blk0 = (cp.cspmatrix(s, device="cpu") + A).blkval.numpy().copy()
    L0, Y0, info0 = _sweeps(s, blk0, None, mode)
    assert info0[0]["pool_bytes"] is None
    stack = int(s.memory["stack_mem"]) * 8
    for limit in (0, stack, 1 << 40):
        L1, Y1, info = _sweeps(s, blk0, limit, mode)
        assert np.array_equal(L0, L1), limit
        assert np.array_equal(Y0, Y1), limit
        for a, b in zip(info, info0):
            assert a["pool_bytes"] is not None
            assert a["workspace_bytes"] < b["workspace_bytes"]
    # and the reference's kernels
    xr = blk0.copy()
    assert ref.cholesky(s, xr) == 0
    assert_blocks_close(s, L0, xr)
    assert ref.projected_inverse(s, xr) == 0
    assert_blocks_close(s, Y0, xr)


def test_pooled_value_sets_batch():
    """A merged plan over value sets takes the limit on its own plan."""
    A, s = problem("grid3d", 12, merge=None, seed=9)
    blk0 = (cp.cspmatrix(s, device="cpu") + A).blkval.numpy()
    rng = np.random.default_rng(1)
    xs = np.stack([blk0 * (1.0 + 0.01 * rng.standard_normal(blk0.size)) for _ in range(4)])
    xs = np.stack([np.where(blk0 != 0, x, 0.0) for x in xs])
    Bt = cp.batch([s] * 4, device=0)
    out = []
    for limit in (None, 0):
        Bt.plan.set_option("scratch_limit", limit)
        v = torch.from_numpy(xs.reshape(-1).copy()).cuda()
        Bt.cholesky(v)
        L = v.clone()
        Bt.projected_inverse(v)
        torch.cuda.synchronize()
        out.append((L.cpu().numpy(), v.cpu().numpy()))
    Bt.plan.set_option("scratch_limit", None)
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


def test_logdet_scratch_limit_and_recompute():
    """The differentiable log det with a scratch limit and with the factor
    recomputed in the backward instead of kept: the same values and
    gradients as the default."""
    from chompack_b200 import autograd as ag
    A, s = problem("grid3d", 12, merge=(32, 32), seed=11)
    blk0 = (cp.cspmatrix(s, device="cpu") + A).blkval.numpy()
    res = []
    for kw in ({}, {"scratch_limit": 0}, {"recompute_factor": True}, {"scratch_limit": 0, "recompute_factor": True}):
        x = torch.from_numpy(blk0.copy()).cuda().requires_grad_(True)
        f = ag.logdet_values(x, s, **kw)
        (g,) = torch.autograd.grad(f, x)
        xb = torch.from_numpy(np.stack([blk0, blk0 * 1.5])).cuda().requires_grad_(True)
        fb = ag.logdet_values(xb, s, **kw)
        (gb,) = torch.autograd.grad(fb.sum(), xb)
        res.append((f.item(), g.cpu().numpy(), fb.detach().cpu().numpy(), gb.cpu().numpy()))
    for r in res[1:]:
        assert r[0] == res[0][0]
        assert np.array_equal(r[1], res[0][1])
        assert np.array_equal(r[2], res[0][2])
        assert np.array_equal(r[3], res[0][3])


@pytest.mark.parametrize("precision", ["tf32", "tf32x3"])
def test_pooled_mixed_precision_bit_identical(precision):
    """The mixed-precision programs (TF32 GEMM tiles) take the limit too,
    with bit-identical results."""
    A, s = problem("grid3d", 16, merge=(32, 32), seed=5)
    blk0 = (cp.cspmatrix(s, device="cpu") + A).blkval.numpy().copy()
    pl = s.plan(0)
    out = []
    for limit in (None, 0):
        pl.set_option("scratch_limit", limit)
        X = cp.cspmatrix(s, blkval=torch.from_numpy(blk0.copy()).cuda(), factor=False)
        cp.cholesky(X, precision=precision)
        L = X.blkval.clone()
        cp.projected_inverse(X, precision=precision)
        torch.cuda.synchronize()
        out.append((L.cpu().numpy(), X.blkval.cpu().numpy()))
    pl.set_option("scratch_limit", None)
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
