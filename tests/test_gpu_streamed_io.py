"""Host-resident values on the GPU (chb_cholesky_io, chb_projected_inverse_io,
chb_llt_io through chompack_b200.cbase): the values stream in while the
sweep runs and each finished chunk streams back out.  The results are
bit-identical to the sweeps on device values (the same tile tasks, plus
waits and signals), the device mirror is reused while the host values are
unchanged and refreshed when they change, and the other sweeps accept host
values through the mirror."""
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
    ("grid2d", (40,), (16, 16)),
]


@pytest.fixture(scope="module", autouse=True)
def _need_cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")


def _host(s, v, factor=False, pinned=True):
    t = torch.from_numpy(np.array(v, dtype=np.float64))
    if pinned:
        t = t.pin_memory()
    return cp.cspmatrix(s, blkval=t, factor=factor)


def _dev(s, v, factor=False):
    return cp.cspmatrix(s, blkval=torch.from_numpy(np.array(v, dtype=np.float64)).cuda(), factor=factor)


@pytest.mark.parametrize("kind,args,merge", CASES)
@pytest.mark.parametrize("pinned", [True, False])
def test_host_sweeps_match_device_sweeps(kind, args, merge, pinned):
    A, s = problem(kind, *args, merge=merge, seed=31)
    blk0 = (cp.cspmatrix(s, device="cpu") + A).blkval.numpy().copy()
    Xd = _dev(s, blk0)
    cp.cholesky(Xd)
    Ld = Xd.blkval.cpu().numpy()
    cp.projected_inverse(Xd)
    Yd = Xd.blkval.cpu().numpy()
    Xh = _host(s, blk0, pinned=pinned)
    assert Xh.blkval.device.type == "cpu"
    cp.cholesky(Xh)
    assert Xh.is_factor is True
    assert np.array_equal(Xh.blkval.numpy(), Ld)
    cp.projected_inverse(Xh)   # the mirror holds L: nothing goes in
    assert np.array_equal(Xh.blkval.numpy(), Yd)
    Lr = blk0.copy()
    assert ref.cholesky(s, Lr) == 0
    assert_blocks_close(s, Ld, Lr)


@pytest.mark.parametrize("kind,args,merge", CASES[:2])
def test_host_llt_and_stale_mirror(kind, args, merge):
    A, s = problem(kind, *args, merge=merge, seed=32)
    blk0 = (cp.cspmatrix(s, device="cpu") + A).blkval.numpy().copy()
    X = _host(s, blk0)
    cp.cholesky(X)
    L = X.blkval.numpy().copy()
    # the host values change: the next sweep must take them, not the mirror
    X.blkval.mul_(2.0)
    cp.llt(X)
    Z = _dev(s, 2.0 * L, factor=True)
    cp.llt(Z)
    assert np.array_equal(X.blkval.numpy(), Z.blkval.cpu().numpy())


def test_host_values_through_the_mirror():
    A, s = problem("grid3d", 10, merge=(16, 16), seed=33)
    blk0 = (cp.cspmatrix(s, device="cpu") + A).blkval.numpy().copy()
    L = blk0.copy()
    assert ref.cholesky(s, L) == 0
    Y = L.copy()
    assert ref.projected_inverse(s, Y) == 0
    for fu in (False, True):
        Ch, Cd = _host(s, Y), _dev(s, Y)
        cp.completion(Ch, factored_updates=fu)
        cp.completion(Cd, factored_updates=fu)
        assert np.array_equal(Ch.blkval.numpy(), Cd.blkval.cpu().numpy())
    rng = np.random.default_rng(5)
    U0 = blk0 * rng.standard_normal(blk0.size)
    Uh, Ud = _host(s, U0), _dev(s, U0)
    cp.hessian(_host(s, L, factor=True), _host(s, Y), [Uh], adj=None)
    cp.hessian(_dev(s, L, factor=True), _dev(s, Y), [Ud], adj=None)
    assert np.array_equal(Uh.blkval.numpy(), Ud.blkval.cpu().numpy())
    assert cp.dot(_host(s, Y), _host(s, U0)) == pytest.approx(cp.dot(_dev(s, Y), _dev(s, U0)), rel=1e-14)


def test_host_cholesky_reports_a_bad_pivot():
    A, s = problem("grid2d", 12, merge=(8, 8), seed=34)
    X = cp.cspmatrix(s, device="cpu") + A
    X.blkval.mul_(-1.0)
    with pytest.raises(ArithmeticError):
        cp.cholesky(X)
    # the sweep ran to its end: the plan still works
    Y = cp.cspmatrix(s, device="cpu") + A
    cp.cholesky(Y)
    assert Y.is_factor is True
