"""The dynamic schedule of the task programs, on the CPU: the pending counts,
successor lists, counter completion values and initial ready bitmaps that
the planner emits are checked against the programs' waits, and every sweep
executed in the order the device's dynamic release rules produce (finished
tasks, completed groups and look-ahead early signals release their
waiters; claims take one of the lowest ready list positions) reproduces
the reference's golden outputs."""
import numpy as np
import pytest

from chompack_b200 import _native as N
from chompack_b200.plan import Plan
import golden_cases as G
import taskvm
from helpers import assert_blocks_close

NAMES = ["nc23_amd", "numeric31", "rand200_m164"]
PROGRAMS = ((N.OP_CHOLESKY, 0, 0), (N.OP_PROJECTED_INVERSE, 0, 0), (N.OP_LLT, 0, 0), (N.OP_COMPLETION, 0, 0),
            (N.OP_COMPLETION, 1, 0), (N.OP_HESSIAN, 2, 5), (N.OP_HESSIAN, 1, 2), (N.OP_TRSM, 3, 1))


def _programs(s):
    pl = Plan(s, device=-1)
    for op, k, flags in PROGRAMS:
        yield (op, k, flags), taskvm.Program(pl.handle, op, k=k, flags=flags, nsn=s.Nsn), \
            taskvm.Schedule(pl.handle, op, k=k, flags=flags)


@pytest.mark.parametrize("name", NAMES)
def test_schedule_matches_waits(name):
    d, A, s = G.load(name)
    for key, prog, sch in _programs(s):
        nt = prog.ntasks
        assert len(sch.npend) == nt and len(sch.ctarget) == prog.ncounters
        assert len(sch.succ_off) == prog.ncounters + 1 and sch.succ_off[-1] == len(sch.succ)
        waiters = [[] for _ in range(prog.ncounters)]
        for i, t in enumerate(prog.tasks):
            w0, nw = int(t["wait_off"]), int(t["nwait"])
            assert sch.npend[i] == nw, key
            for cid, target in prog.waits[w0:w0 + nw]:
                waiters[cid].append(i)
                assert sch.ctarget[cid] == target, key
        for c in range(prog.ncounters):
            got = sorted(sch.succ[sch.succ_off[c]:sch.succ_off[c + 1]].tolist())
            assert got == waiters[c], key
        # group sizes: members that count into each group counter
        members = np.bincount(prog.tasks["group"][prog.tasks["group"] >= 0], minlength=prog.ncounters)
        for c in range(nt, prog.ncounters):
            if members[c]:
                assert sch.ctarget[c] == members[c], key
        ready = np.zeros(len(sch.ready0) * 64, dtype=bool)
        ready[np.nonzero(sch.npend == 0)[0]] = True
        assert np.array_equal(np.packbits(ready, bitorder="little").view(np.uint64), sch.ready0)
        words = np.nonzero(sch.ready0)[0]
        summ = np.zeros(len(sch.summ0) * 64, dtype=bool)
        summ[words] = True
        assert np.array_equal(np.packbits(summ, bitorder="little").view(np.uint64), sch.summ0)


def _run(s, op, bases, k=0, flags=0, seed=0, **kw):
    pl = Plan(s, device=-1)
    prog = taskvm.Program(pl.handle, op, k=k, flags=flags, nsn=s.Nsn)
    sch = taskvm.Schedule(pl.handle, op, k=k, flags=flags)
    bases = dict(bases)
    bases[1] = np.full(prog.ws_doubles, np.nan)
    vm = taskvm.VM(prog, bases, s.relidx, s.chidx, **kw)
    return vm.run("dynamic", seed=seed, schedule=sch)


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("seed", [0, 1])
def test_dynamic_cholesky_and_inverse(name, seed):
    d, A, s = G.load(name)
    x = d["blkval"].copy()
    assert _run(s, N.OP_CHOLESKY, {0: x}, seed=seed) == 0
    assert_blocks_close(s, x, d["ref_cholesky"])
    assert _run(s, N.OP_PROJECTED_INVERSE, {0: x}, seed=seed + 7) == 0
    assert_blocks_close(s, x, d["ref_projected_inverse"])


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("fu", [0, 1])
def test_dynamic_completion(name, fu):
    d, A, s = G.load(name)
    x = d["ref_projected_inverse"].copy()
    assert _run(s, N.OP_COMPLETION, {0: x}, k=fu, seed=3 + fu) == 0
    assert_blocks_close(s, x, d["ref_completion_fu%d" % fu])


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("fu,adj,inv", [(0, 0, 0), (1, 1, 0), (0, 1, 1), (1, 0, 1)])
def test_dynamic_hessian(name, fu, adj, inv):
    d, A, s = G.load(name)
    u = d["ref_hessian_U0"].copy()
    bases = {2: d["ref_cholesky"].copy(), 3: d["ref_projected_inverse"].copy(), 5: u}
    _run(s, N.OP_HESSIAN, bases, k=1, flags=adj | inv << 1 | fu << 2, seed=11)
    assert_blocks_close(s, u, d["ref_hessian_a%d_i%d_fu%d" % (adj, inv, fu)])


@pytest.mark.parametrize("name", NAMES)
def test_dynamic_llt_and_trsm(name):
    d, A, s = G.load(name)
    x = d["ref_cholesky"].copy()
    _run(s, N.OP_LLT, {0: x}, seed=5)
    assert_blocks_close(s, x, d["ref_llt"])
    B0 = d["ref_trsm_B0"]
    for trans in ("N", "T"):
        Bf = B0.reshape(-1, order="F").copy()
        _run(s, N.OP_TRSM, {0: d["ref_cholesky"].copy(), 4: Bf}, k=B0.shape[1], flags=1 if trans == "T" else 0,
             seed=6, perm=s.p, ldb=s.n, alpha=0.5)
        got = Bf.reshape(B0.shape, order="F")
        want = d["ref_trsm_" + trans]
        assert np.max(np.abs(got - want)) <= 1e-12 * max(1.0, np.max(np.abs(want)))
