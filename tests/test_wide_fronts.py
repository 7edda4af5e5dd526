"""Task programs of problems whose fronts span several 64-column blocks, on
the CPU: the fused diagonal task of cholesky (factor the diagonal tile, then
wait mid task for the next tiles' updates and do the look-ahead) and the
separate look-ahead task it replaces, and projected_inverse with small
fronts (one task each) next to tiled ones, executed by the task interpreter
in random orders allowed by the waits and under the dynamic release rules,
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

CASES = [("grid3d", (10,), (32, 32)), ("grid2d", (70,), (64, 64))]


def _setup(kind, args, merge, fused):
    old = os.environ.pop("CHB_NO_FUSED_LA", None)
    if not fused:
        os.environ["CHB_NO_FUSED_LA"] = "1"
    try:
        A, s = problem(kind, *args, merge=merge, seed=3)
        pl = Plan(s, device=-1)
        prog = taskvm.Program(pl.handle, N.OP_CHOLESKY, nsn=s.Nsn)
        sch = taskvm.Schedule(pl.handle, N.OP_CHOLESKY)
    finally:
        os.environ.pop("CHB_NO_FUSED_LA", None)
        if old is not None:
            os.environ["CHB_NO_FUSED_LA"] = old
    return A, s, pl, prog, sch


@pytest.mark.parametrize("kind,args,merge", CASES)
@pytest.mark.parametrize("fused", [True, False])
@pytest.mark.parametrize("order,seed", [("random", 0), ("random", 1), ("dynamic", 2)])
def test_wide_front_cholesky(kind, args, merge, fused, order, seed):
    A, s, pl, prog, sch = _setup(kind, args, merge, fused)
    ops = prog.tasks["op"]
    n_fused = int(np.sum((ops == taskvm.T_POTRF) & (prog.tasks["k"] > 0)))
    n_la = int(np.sum(ops == taskvm.T_LA))
    assert int(np.max(np.diff(s.snptr))) > 64
    assert (n_fused > 0 and n_la == 0) if fused else (n_fused == 0 and n_la > 0)
    x0 = (cp.cspmatrix(s, device="cpu") + A).blkval.numpy().copy()
    ref = x0.copy()
    assert oracle.cholesky(s, ref) == 0
    x = x0.copy()
    bases = {0: x, 1: np.full(prog.ws_doubles, np.nan)}
    assert taskvm.VM(prog, bases, s.relidx, s.chidx).run(order, seed=seed, schedule=sch) == 0
    assert_blocks_close(s, x, ref)


def test_fused_task_waits():
    """The fused task's first Task::cdiag waits gate its start (and its
    pending count in the dynamic schedule); the rest are mid-task waits on
    the updates of the next panel and diagonal tiles."""
    A, s, pl, prog, sch = _setup("grid3d", (10,), (32, 32), True)
    seen_mid = 0
    for i, t in enumerate(prog.tasks):
        if int(t["op"]) != taskvm.T_POTRF or int(t["k"]) == 0:
            continue
        npre, nw = int(t["cdiag"]), int(t["nwait"])
        assert 0 <= npre <= nw
        assert sch.npend[i] == npre
        w0 = int(t["wait_off"])
        for cid, _ in prog.waits[w0 + npre:w0 + nw]:
            assert cid < prog.ntasks and int(prog.tasks[cid]["op"]) == taskvm.T_GEMM
            seen_mid += 1
        assert int(t["aux"][3]) > 0     # the early signal of the next panel tile
    assert seen_mid > 0


@pytest.mark.parametrize("kind,args,merge", CASES)
@pytest.mark.parametrize("order,seed", [("random", 3), ("dynamic", 4)])
def test_wide_front_projected_inverse(kind, args, merge, order, seed):
    A, s = problem(kind, *args, merge=merge, seed=3)
    pl = Plan(s, device=-1)
    prog = taskvm.Program(pl.handle, N.OP_PROJECTED_INVERSE, nsn=s.Nsn)
    sch = taskvm.Schedule(pl.handle, N.OP_PROJECTED_INVERSE)
    nj = np.diff(np.asarray(s.sncolptr))
    small = int(np.sum(prog.tasks["op"] == taskvm.T_PFRONT))
    assert small == int(np.sum(nj <= 64))
    x0 = (cp.cspmatrix(s, device="cpu") + A).blkval.numpy().copy()
    L = x0.copy()
    assert oracle.cholesky(s, L) == 0
    ref = L.copy()
    assert oracle.projected_inverse(s, ref) == 0
    y = L.copy()
    bases = {0: y, 1: np.full(prog.ws_doubles, np.nan)}
    assert taskvm.VM(prog, bases, s.relidx, s.chidx).run(order, seed=seed, schedule=sch) == 0
    assert_blocks_close(s, y, ref)


@pytest.mark.parametrize("kind,args,merge", [("grid3d", (12,), (128, 128)), ("grid2d", (60,), (256, 256))])
@pytest.mark.parametrize("order,seed", [("random", 5), ("dynamic", 6)])
def test_split_schur_cholesky(kind, args, merge, order, seed):
    """cholesky with the Schur-complement tiles U_k -= S_k S_k^T split along
    K (CHB_CHOL_KSPLIT=128): partial products in scratch, summed in a fixed
    order by T_SUM tasks into U_k."""
    old = os.environ.get("CHB_CHOL_KSPLIT")
    os.environ["CHB_CHOL_KSPLIT"] = "128"
    try:
        A, s = problem(kind, *args, merge=merge, seed=3)
        pl = Plan(s, device=-1)
        prog = taskvm.Program(pl.handle, N.OP_CHOLESKY, nsn=s.Nsn)
        sch = taskvm.Schedule(pl.handle, N.OP_CHOLESKY)
    finally:
        if old is None:
            os.environ.pop("CHB_CHOL_KSPLIT", None)
        else:
            os.environ["CHB_CHOL_KSPLIT"] = old
    assert int(np.sum(prog.tasks["op"] == taskvm.T_SUM)) > 0
    x0 = (cp.cspmatrix(s, device="cpu") + A).blkval.numpy().copy()
    ref = x0.copy()
    assert oracle.cholesky(s, ref) == 0
    x = x0.copy()
    bases = {0: x, 1: np.full(prog.ws_doubles, np.nan)}
    assert taskvm.VM(prog, bases, s.relidx, s.chidx).run(order, seed=seed, schedule=sch) == 0
    assert_blocks_close(s, x, ref)


@pytest.mark.parametrize("ksplit", ["128", "1024"])
@pytest.mark.parametrize("order,seed", [("random", 7), ("dynamic", 8)])
def test_projected_inverse_split_sizes(ksplit, order, seed):
    """projected_inverse with other split-K chunk sizes (CHB_PINV_KSPLIT):
    the number of partial products changes, the result stays the
    reference's within the FP64 tolerance."""
    old = os.environ.get("CHB_PINV_KSPLIT")
    os.environ["CHB_PINV_KSPLIT"] = ksplit
    try:
        A, s = problem("grid3d", 12, merge=(128, 128), seed=3)
        pl = Plan(s, device=-1)
        prog = taskvm.Program(pl.handle, N.OP_PROJECTED_INVERSE, nsn=s.Nsn)
        sch = taskvm.Schedule(pl.handle, N.OP_PROJECTED_INVERSE)
    finally:
        if old is None:
            os.environ.pop("CHB_PINV_KSPLIT", None)
        else:
            os.environ["CHB_PINV_KSPLIT"] = old
    nsum = int(np.sum(prog.tasks["op"] == taskvm.T_SUM))
    assert (nsum > 0) if ksplit == "128" else True
    x0 = (cp.cspmatrix(s, device="cpu") + A).blkval.numpy().copy()
    L = x0.copy()
    assert oracle.cholesky(s, L) == 0
    ref = L.copy()
    assert oracle.projected_inverse(s, ref) == 0
    y = L.copy()
    bases = {0: y, 1: np.full(prog.ws_doubles, np.nan)}
    assert taskvm.VM(prog, bases, s.relidx, s.chidx).run(order, seed=seed, schedule=sch) == 0
    assert_blocks_close(s, y, ref)


@pytest.mark.parametrize("nj", ["0", "32"])
@pytest.mark.parametrize("order,seed", [("random", 9), ("dynamic", 10)])
def test_small_front_threshold(nj, order, seed):
    """CHB_SMALL_FRONT_NJ: with 0 every front is a tile graph, with 32 the
    fronts of order <= 32 are single shared-memory tasks and the others tile
    graphs; both sweeps reproduce the reference in either case."""
    old = os.environ.get("CHB_SMALL_FRONT_NJ")
    os.environ["CHB_SMALL_FRONT_NJ"] = nj
    try:
        A, s = problem("grid2d", 40, merge=(16, 16), seed=5)
        pl = Plan(s, device=-1)
        progs = {op: (taskvm.Program(pl.handle, op, nsn=s.Nsn), taskvm.Schedule(pl.handle, op))
                 for op in (N.OP_CHOLESKY, N.OP_PROJECTED_INVERSE)}
    finally:
        if old is None:
            os.environ.pop("CHB_SMALL_FRONT_NJ", None)
        else:
            os.environ["CHB_SMALL_FRONT_NJ"] = old
    fronts = np.diff(np.asarray(s.sncolptr))
    want = int(np.sum(fronts <= int(nj)))

    def bundled(prog, op):
        """Fronts inside small-subtree bundles (one warp per range)."""
        tot = 0
        for t in prog.tasks[prog.tasks["op"] == op]:
            ends = (int(t["m"]), int(t["n"]), int(t["k"]), int(t["cdiag"]))
            tot += sum(ends[w] - int(t["aux"][w]) + 1 for w in range(4) if int(t["aux"][w]) >= 0)
        return tot
    pc, pp = progs[N.OP_CHOLESKY][0], progs[N.OP_PROJECTED_INVERSE][0]
    assert int(np.sum(pc.tasks["op"] == taskvm.T_FRONT)) + bundled(pc, taskvm.T_SUBTREE) == want
    assert int(np.sum(pp.tasks["op"] == taskvm.T_PFRONT)) + bundled(pp, taskvm.T_PSUBTREE) == want
    assert bundled(pc, taskvm.T_SUBTREE) == bundled(pp, taskvm.T_PSUBTREE)
    if nj == "32":
        assert bundled(pc, taskvm.T_SUBTREE) > 0
    if nj == "32":
        assert 0 < want < len(fronts)
    x0 = (cp.cspmatrix(s, device="cpu") + A).blkval.numpy().copy()
    L = x0.copy()
    assert oracle.cholesky(s, L) == 0
    Y = L.copy()
    assert oracle.projected_inverse(s, Y) == 0
    x = x0.copy()
    prog, sch = progs[N.OP_CHOLESKY]
    assert taskvm.VM(prog, {0: x, 1: np.full(prog.ws_doubles, np.nan)}, s.relidx, s.chidx).run(
        order, seed=seed, schedule=sch) == 0
    assert_blocks_close(s, x, L)
    y = L.copy()
    prog, sch = progs[N.OP_PROJECTED_INVERSE]
    assert taskvm.VM(prog, {0: y, 1: np.full(prog.ws_doubles, np.nan)}, s.relidx, s.chidx).run(
        order, seed=seed + 1, schedule=sch) == 0
    assert_blocks_close(s, y, Y)
