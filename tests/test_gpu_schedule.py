"""The dynamic task schedule on the GPU: every sweep gives bit-identical
results under the dynamic schedule (finished tasks release their waiters)
and the static list order, and both match the reference's kernels.  The
task graph fixes the order of every accumulation, so no result may depend
on which CTA ran which task when; the triangular solve does so with its
ordered-sums option (CHB_OPT_ORDERED_SUMS), while its default adds into
vector blocks with atomics, whose order varies: there the two schedules
agree to rounding (1e-13 relative per column)."""
import numpy as np
import pytest
import torch

import chompack_b200 as cp
from helpers import problem, assert_blocks_close
from oracle import ref

pytestmark = pytest.mark.gpu

CASES = [
    ("grid3d", (14,), (32, 32)),
    ("random", (400, 0.03), (16, 16)),
]


@pytest.fixture(scope="module", autouse=True)
def _need_cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")


def _dev(s, v, factor):
    return cp.cspmatrix(s, blkval=torch.from_numpy(np.array(v, dtype=np.float64)).cuda(), factor=factor)


def _sweeps(s, blk0, mode, ordered_sums=1):
    s.plan(0).set_schedule(mode)
    s.plan(0).set_option("ordered_sums", ordered_sums)
    try:
        out = {}
        X = _dev(s, blk0, False)
        cp.cholesky(X)
        out["cholesky"] = X.blkval.cpu().numpy()
        L = out["cholesky"]
        Y = _dev(s, L, True)
        cp.projected_inverse(Y)
        out["projected_inverse"] = Y.blkval.cpu().numpy()
        Z = _dev(s, L, True)
        cp.llt(Z)
        out["llt"] = Z.blkval.cpu().numpy()
        for fu in (False, True):
            C = _dev(s, out["projected_inverse"], False)
            cp.completion(C, factored_updates=fu)
            out["completion_fu%d" % fu] = C.blkval.cpu().numpy()
            rng = np.random.default_rng(3)
            U = [_dev(s, blk0 * rng.standard_normal(blk0.size), False) for _ in range(2)]
            cp.hessian(_dev(s, L, True), _dev(s, out["projected_inverse"], False), U, adj=None, inv=False,
                       factored_updates=fu)
            out["hessian_fu%d" % fu] = np.concatenate([u.blkval.cpu().numpy() for u in U])
        B = torch.from_numpy(np.asfortranarray(np.random.default_rng(4).standard_normal((s.n, 5)))).cuda()
        for tr in ("N", "T"):
            Bt = B.clone()
            cp.trsm(_dev(s, L, True), Bt, trans=tr)
            out["trsm_" + tr] = Bt.cpu().numpy()
        return out
    finally:
        s.plan(0).set_schedule(None)
        s.plan(0).set_option("ordered_sums", None)


@pytest.mark.parametrize("kind,args,merge", CASES)
def test_dynamic_and_static_are_bit_identical(kind, args, merge):
    A, s = problem(kind, *args, merge=merge, seed=21)
    blk0 = (cp.cspmatrix(s, device="cpu") + A).blkval.numpy().copy()
    dyn = _sweeps(s, blk0, "dynamic")
    sta = _sweeps(s, blk0, "static")
    for key in dyn:
        assert np.array_equal(dyn[key], sta[key]), key
    # the default (atomic) solve: the same to rounding under both schedules
    # and close to the ordered one
    dyn_a = _sweeps(s, blk0, "dynamic", ordered_sums=0)
    sta_a = _sweeps(s, blk0, "static", ordered_sums=0)
    for key in ("trsm_N", "trsm_T"):
        for got in (dyn_a[key], sta_a[key]):
            err = np.max(np.abs(got - sta[key]) / np.maximum(np.abs(sta[key]).max(axis=0), 1e-300))
            assert err <= 1e-13, (key, err)
    L = blk0.copy()
    assert ref.cholesky(s, L) == 0
    assert_blocks_close(s, dyn["cholesky"], L)
    Y = L.copy()
    assert ref.projected_inverse(s, Y) == 0
    assert_blocks_close(s, dyn["projected_inverse"], Y)
    for fu in (False, True):
        r = Y.copy()
        assert ref.completion(s, r, factored_updates=fu) == 0
        assert_blocks_close(s, dyn["completion_fu%d" % fu], r)


@pytest.mark.parametrize("mode", ["dynamic", "static"])
def test_repeated_runs_reuse_the_workspace(mode):
    A, s = problem("grid3d", 10, merge=(16, 16), seed=5)
    blk0 = (cp.cspmatrix(s, device="cpu") + A).blkval.numpy().copy()
    s.plan(0).set_schedule(mode)
    try:
        first = None
        for _ in range(4):
            X = _dev(s, blk0, False)
            cp.cholesky(X)
            cp.projected_inverse(X)
            got = X.blkval.cpu().numpy()
            if first is None:
                first = got
            assert np.array_equal(got, first)
    finally:
        s.plan(0).set_schedule(None)
