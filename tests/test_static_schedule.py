"""Progress of the static list order, on the CPU: CTAs claim tasks strictly
in list order (one atomic counter), wait for a task's waits, run it and
publish its counter; a fused diagonal task (POTRF with k > 0) publishes its
own counter after its first part, then waits mid task for the updates of
the next tiles, raises its early signal and publishes its end group.  Mid
waits may point forward in the list, so progress depends on the list order
and on the number of CTAs.  These tests run the engine's protocol with the
grid it launches (296 CTAs: 148 SMs x 2), claiming and completing in random
interleavings, and require every program to finish."""
import numpy as np
import pytest

from chompack_b200 import _native as N
from chompack_b200.plan import Plan
from helpers import problem
import golden_cases as G
import taskvm

T_POTRF, T_LA = taskvm.T_POTRF, taskvm.T_LA


def simulate(prog, ctas, seed):
    """Returns the number of tasks finished before no CTA could move."""
    tasks, waits = prog.tasks, prog.waits
    nt = len(tasks)
    cnt = np.zeros(prog.ncounters, dtype=np.int64)
    op = tasks["op"].astype(int)
    fused = (op == T_POTRF) & (tasks["k"] > 0)
    npre = np.where(fused, tasks["cdiag"], tasks["nwait"]).astype(int)
    w0 = tasks["wait_off"].astype(int)
    nw = tasks["nwait"].astype(int)
    early = np.where(((op == T_LA) | fused), tasks["aux"][:, 3].astype(int) - 1, -1)
    group = tasks["group"].astype(int)

    def met(i, a, b):
        for cid, target in waits[w0[i] + a:w0[i] + b]:
            if cnt[cid] < target:
                return False
        return True

    rng = np.random.default_rng(seed)
    nxt = 0
    state = [None] * ctas     # (task, phase): phase 0 waits before, 1 waits mid
    done = 0
    while done < nt:
        moved = False
        for c in rng.permutation(ctas):
            if state[c] is None:
                if nxt >= nt:
                    continue
                state[c] = (nxt, 0)
                nxt += 1
                moved = True
            i, ph = state[c]
            if ph == 0:
                if not met(i, 0, npre[i]):
                    continue
                if fused[i]:
                    cnt[i] += 1            # first part done: L_cc and M_cc published
                    state[c] = (i, 1)
                    ph = 1
                    moved = True
            if ph == 1 and not met(i, npre[i], nw[i]):
                continue
            if early[i] >= 0:
                cnt[early[i]] += 1
            cnt[i] += 1
            if group[i] >= 0:
                cnt[group[i]] += 1
            state[c] = None
            done += 1
            moved = True
        if not moved:
            return done
    return done


def _fused_program(kind, args, merge):
    A, s = problem(kind, *args, merge=merge, seed=3)
    pl = Plan(s, device=-1)
    prog = taskvm.Program(pl.handle, N.OP_CHOLESKY, nsn=s.Nsn)
    return prog


@pytest.mark.parametrize("kind,args,merge", [("grid3d", (10,), (32, 32)), ("grid3d", (16,), (32, 32)),
                                             ("grid2d", (70,), (64, 64))])
@pytest.mark.parametrize("seed", [0, 1])
def test_cholesky_static_order_always_progresses(kind, args, merge, seed):
    prog = _fused_program(kind, args, merge)
    fused = int(np.sum((prog.tasks["op"] == T_POTRF) & (prog.tasks["k"] > 0)))
    assert fused > 0
    mid = int(np.sum(np.where((prog.tasks["op"] == T_POTRF) & (prog.tasks["k"] > 0),
                              prog.tasks["nwait"] - prog.tasks["cdiag"], 0)))
    assert mid > 0 or kind == "grid2d"   # two-block fronts have no mid waits
    assert simulate(prog, 296, seed) == prog.ntasks


def test_bench_workload_static_order_progresses():
    """The 3-D 7-point grid 40^3 (AMD, merge_size_fill(32, 32)) cholesky
    program, 80,265 tasks, under the same protocol."""
    from chompack_b200 import grids
    import chompack_b200 as cp
    A = grids.grid3d(40, seed=0)
    s = cp.symbolic(A, p=cp.amd.order(A), merge_function=cp.merge_size_fill(32, 32))
    pl = Plan(s, device=-1)  # keeps the native plan alive while its program is read
    prog = taskvm.Program(pl.handle, N.OP_CHOLESKY, nsn=s.Nsn)
    assert simulate(prog, 296, 0) == prog.ntasks


@pytest.mark.parametrize("name", ["nc23_amd", "numeric31", "rand200_m164"])
@pytest.mark.parametrize("op", [N.OP_CHOLESKY, N.OP_LLT, N.OP_TRSM, N.OP_TRMM])
def test_static_sweeps_progress_on_one_cta(name, op):
    """Sweeps without mid waits (every wait points backwards in the list)
    finish even on a single CTA."""
    d, A, s = G.load(name)
    k = 3 if op in (N.OP_TRSM, N.OP_TRMM) else 0
    pl = Plan(s, device=-1)
    prog = taskvm.Program(pl.handle, op, k=k, nsn=s.Nsn)
    has_mid = bool(np.any((prog.tasks["op"] == T_POTRF) & (prog.tasks["k"] > 0)
                          & (prog.tasks["nwait"] > prog.tasks["cdiag"])))
    if has_mid:
        pytest.skip("program has mid-task waits")
    assert simulate(prog, 1, 0) == prog.ntasks
