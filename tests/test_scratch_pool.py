"""Update matrices under a scratch limit (CHB_OPT_SCRATCH_LIMIT), on the CPU.

With a limit, cholesky and projected_inverse place the fronts' update
matrices in a shared pool: a front that takes memory another front's update
matrix held waits for that matrix's readers.  The task interpreter runs the
pooled programs in random orders allowed by their waits (a missing reuse
wait shows up as a wrong result: the workspace starts as NaN and a reused
region holds another front's values) and under the dynamic release rules,
against the oracle's C restatement of the reference's sweeps."""
import os

import numpy as np
import pytest

import chompack_b200 as cp
from chompack_b200 import _native as N
from chompack_b200.plan import Plan
from helpers import problem, assert_blocks_close
from oracle import oracle
import taskvm

# (kind, args, merge): fronts of several 64-column blocks (merged 3-D and
# 2-D grids) and a tree of many small fronts in bundles (unmerged 3-D grid)
CASES = [("grid3d", (10,), (32, 32)), ("grid2d", (70,), (64, 64)), ("grid3d", (12,), None)]


@pytest.fixture(autouse=True)
def _pool_every_matrix():
    old = os.environ.get("CHB_SCRATCH_POOL_MIN")
    os.environ["CHB_SCRATCH_POOL_MIN"] = "1"
    yield
    if old is None:
        os.environ.pop("CHB_SCRATCH_POOL_MIN", None)
    else:
        os.environ["CHB_SCRATCH_POOL_MIN"] = old


def _programs(s, op, limit):
    pl = Plan(s, device=-1)
    if limit is not None:
        pl.set_option("scratch_limit", limit)
    prog = taskvm.Program(pl.handle, op, nsn=s.Nsn)
    sch = taskvm.Schedule(pl.handle, op)
    return pl, prog, sch


def _unlimited_workspace(s, op):
    return Plan(s, device=-1).pool_info(op)["workspace_bytes"]


def _upd_bytes(s):
    nn = np.diff(np.asarray(s.snptr))
    na = np.diff(np.asarray(s.blkptr)) // nn - nn
    return int((na.astype(np.int64) ** 2).sum()) * 8


def _stack_bytes(s):
    """The reference's postorder stack of update matrices (its largest
    size), the least memory a sequential sweep needs."""
    return int(s.memory["stack_mem"]) * 8


@pytest.mark.parametrize("kind,args,merge", CASES)
@pytest.mark.parametrize("limit", [0, "stack"])
@pytest.mark.parametrize("order,seed", [("random", 0), ("random", 1), ("dynamic", 2)])
def test_pooled_cholesky(kind, args, merge, limit, order, seed):
    A, s = problem(kind, *args, merge=merge, seed=3)
    lim = _stack_bytes(s) if limit == "stack" else limit
    pl, prog, sch = _programs(s, N.OP_CHOLESKY, lim)
    info = pl.pool_info(N.OP_CHOLESKY)
    assert info["pool_bytes"] is not None
    assert info["workspace_bytes"] < _unlimited_workspace(s, N.OP_CHOLESKY)
    assert info["reuse_waits"] > 0
    x0 = (cp.cspmatrix(s, device="cpu") + A).blkval.numpy().copy()
    ref = x0.copy()
    assert oracle.cholesky(s, ref) == 0
    x = x0.copy()
    bases = {0: x, 1: np.full(prog.ws_doubles, np.nan)}
    assert taskvm.VM(prog, bases, s.relidx, s.chidx).run(order, seed=seed, schedule=sch) == 0
    assert_blocks_close(s, x, ref)


@pytest.mark.parametrize("kind,args,merge", CASES)
@pytest.mark.parametrize("limit", [0, "stack"])
@pytest.mark.parametrize("order,seed", [("random", 3), ("dynamic", 4)])
def test_pooled_projected_inverse(kind, args, merge, limit, order, seed):
    A, s = problem(kind, *args, merge=merge, seed=3)
    lim = _stack_bytes(s) if limit == "stack" else limit
    pl, prog, sch = _programs(s, N.OP_PROJECTED_INVERSE, lim)
    info = pl.pool_info(N.OP_PROJECTED_INVERSE)
    assert info["pool_bytes"] is not None
    assert info["workspace_bytes"] < _unlimited_workspace(s, N.OP_PROJECTED_INVERSE)
    L = (cp.cspmatrix(s, device="cpu") + A).blkval.numpy().copy()
    assert oracle.cholesky(s, L) == 0
    ref = L.copy()
    assert oracle.projected_inverse(s, ref) == 0
    x = L.copy()
    bases = {0: x, 1: np.full(prog.ws_doubles, np.nan)}
    assert taskvm.VM(prog, bases, s.relidx, s.chidx).run(order, seed=seed, schedule=sch) == 0
    assert_blocks_close(s, x, ref)


@pytest.mark.parametrize("op", [N.OP_CHOLESKY, N.OP_PROJECTED_INVERSE])
def test_pool_shrinks_workspace(op):
    """Without a limit there is no pool; with one the update matrices and
    the fronts' scratch take less memory than their sum, and a generous
    limit bounds the pool."""
    A, s = problem("grid3d", 12, merge=None, seed=3)
    total = _upd_bytes(s)
    base = None
    for lim in (None, total, 4 * _stack_bytes(s), _stack_bytes(s), 0):
        pl = Plan(s, device=-1)
        if lim is not None:
            pl.set_option("scratch_limit", lim)
        assert pl.option("scratch_limit") == (-1 if lim is None else lim)
        info = pl.pool_info(op)
        if lim is None:
            assert info["pool_bytes"] is None and info["reuse_waits"] == 0
            base = info["workspace_bytes"]
            continue
        assert info["workspace_bytes"] < base
        if lim >= total:
            assert info["pool_bytes"] <= lim


def test_pooled_program_same_arithmetic():
    """A pooled program computes what the unpooled one does, in the same
    order per task: the results in list order are bit-identical."""
    A, s = problem("grid3d", 10, merge=(32, 32), seed=5)
    x0 = (cp.cspmatrix(s, device="cpu") + A).blkval.numpy().copy()
    out = []
    for lim in (None, 0):
        pl, prog, sch = _programs(s, N.OP_CHOLESKY, lim)
        x = x0.copy()
        bases = {0: x, 1: np.full(prog.ws_doubles, np.nan)}
        assert taskvm.VM(prog, bases, s.relidx, s.chidx).run("list") == 0
        out.append(x)
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("seed", [0, 1])
def test_pooled_merged_plan(seed):
    """A merged plan (three trees: two value sets on one pattern and a
    second pattern) under a scratch limit: buffers of one tree take memory
    of another's, and random orders still give each tree's results."""
    from chompack_b200.batch import batch
    A1, s1 = problem("grid3d", 9, merge=(32, 32), seed=3)
    A2, s2 = problem("grid2d", 40, merge=(16, 16), seed=4)
    symbs, As = [s1, s2, s1], [A1, A2, A1]
    Bt = batch(symbs, device=-1)
    Bt.plan.set_option("scratch_limit", 0)
    info = Bt.plan.pool_info(N.OP_CHOLESKY)
    assert info["pool_bytes"] is not None and info["reuse_waits"] > 0
    relidx = np.concatenate([np.asarray(s.relidx) for s in symbs])
    chidx = np.concatenate([np.asarray(s.chidx) + off for s, off in
                            zip(symbs, np.cumsum([0] + [s.Nsn for s in symbs[:-1]]))])
    xs = [(cp.cspmatrix(s, device="cpu") + A).blkval.numpy().copy() for s, A in zip(symbs, As)]
    xs[2] = np.where(xs[2] != 0, xs[2] * 1.25, 0.0)
    x = np.concatenate(xs)
    nsn = Bt.plan.batch_segments()[-1]
    for op, fn in ((N.OP_CHOLESKY, oracle.cholesky), (N.OP_PROJECTED_INVERSE, oracle.projected_inverse)):
        prog = taskvm.Program(Bt.plan.handle, op, nsn=nsn)
        sch = taskvm.Schedule(Bt.plan.handle, op)
        bases = {0: x, 1: np.full(prog.ws_doubles, np.nan)}
        order = "random" if op == N.OP_CHOLESKY else "dynamic"
        assert taskvm.VM(prog, bases, relidx, chidx).run(order, seed=seed, schedule=sch) == 0
        for m, s in enumerate(symbs):
            assert fn(s, xs[m]) == 0
            assert_blocks_close(s, x[Bt.offsets[m]:Bt.offsets[m + 1]], xs[m])
