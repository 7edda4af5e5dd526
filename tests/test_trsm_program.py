"""The triangular-solve task program (csrc/build_trsm.cpp) on fronts large
enough for every one of its forms, run by the interpreter (taskvm) in
random and dynamic orders and compared with the reference's trsm
(src/C/trsm.c, oracle/_ref) on the same factor:

* diagonal blocks of several 64-row tiles, so that the substitution steps
  (T_TRSV tasks, their operand staged before their mid waits) carry the
  updates of the two neighbouring blocks ([-G2_c | -G_c | M_c] for 'N',
  [M_c; -H_c; -H2_c] for 'T');
* long products W x_k (K = nn) and W^T u_k (K = na) beyond 128, in chunks
  whose products add into the target with atomics, like the far updates of
  the substitution;
* extend-add (atomic adds) and extract tasks split by right-hand-side
  columns and row chunks.

Tolerance: 1e-12 relative to the largest entry of the column (the GPU
tests use the same measure)."""
import numpy as np
import pytest

import chompack_b200 as cp
from chompack_b200 import _native as N
from chompack_b200.plan import Plan
import taskvm
from helpers import problem
from oracle import ref


@pytest.fixture(scope="module")
def grid16():
    if not ref.available():
        pytest.skip("reference kernels not built")
    # merge_size_fill(300, 300) on the 16^3 grid: 12 supernodes, fronts with
    # nn up to 525 and na up to 303, ten with nn > 256 below the root
    A, s = problem("grid3d", 16, merge=(300, 300), seed=1)
    x = (cp.cspmatrix(s, device="cpu") + A).blkval.numpy().copy()
    assert ref.cholesky(s, x) == 0
    return s, x


def _tasks(s, nrhs, trans):
    pl = Plan(s, device=-1)
    return taskvm.Program(pl.handle, N.OP_TRSM, k=nrhs, flags=1 if trans == "T" else 0, nsn=s.Nsn)


def test_ordered_form_has_no_atomics(grid16):
    s, _ = grid16
    pl = Plan(s, device=-1)
    pl.set_option("ordered_sums", 1)
    assert pl.option("ordered_sums") == 1
    for trans in ("N", "T"):
        t = taskvm.Program(pl.handle, N.OP_TRSM, k=8, flags=1 if trans == "T" else 0, nsn=s.Nsn).tasks
        assert int(np.sum(t["cmode"][t["op"] == taskvm.T_GEMM] == 2)) == 0, trans
        assert int(np.sum((t["op"] == taskvm.T_VEC) & (t["aux"][:, 0] == 4))) == 0, trans
        assert int(np.sum(t["op"] == taskvm.T_SUM)) > 0, trans


def test_program_has_every_form(grid16):
    s, _ = grid16
    nn = np.diff(np.asarray(s.snptr))
    na = np.diff(np.asarray(s.sncolptr)) - nn
    assert np.any((nn > 256) & (na > 0)) and na.max() > 256
    for trans in ("N", "T"):
        prog = _tasks(s, 8, trans)
        t = prog.tasks
        gemm = t[t["op"] == taskvm.T_GEMM]
        assert int(np.sum(gemm["cmode"] == 2)) > 0, trans       # products that add with atomics
        if trans == "N":
            assert int(np.sum((t["op"] == taskvm.T_VEC) & (t["aux"][:, 0] == 4))) > 0   # atomic extend-add
        steps = t[t["op"] == taskvm.T_TRSV]
        assert int(np.sum(steps["k"] > 128)) > 0, trans        # steps that take two neighbouring updates
        # a step starts on its operand's producers and is split: the x tiles
        # it reads (after the first step of a chain) are mid waits, after the
        # first cdiag waits
        assert np.all(steps["cdiag"] <= steps["nwait"]), trans
        assert int(np.sum(steps["cdiag"] < steps["nwait"])) > 0, trans
        vec = t[(t["op"] == taskvm.T_VEC) & (t["aux"][:, 0] >= 2)]
        assert int(np.sum(vec["aux"][:, 3] - vec["aux"][:, 2] < 8)) > 0, trans   # column-split tasks


@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("nrhs", [1, 8, 70])
@pytest.mark.parametrize("order", ["random", "dynamic"])
@pytest.mark.parametrize("ordered_sums", [0, 1])
def test_program_matches_reference(grid16, trans, nrhs, order, ordered_sums):
    """Both forms of the additions into vector blocks: atomic (default) and
    ordered (CHB_OPT_ORDERED_SUMS: chains and split-K sums)."""
    s, L = grid16
    B0 = np.asfortranarray(np.random.default_rng(nrhs).standard_normal((s.n, nrhs)))
    want = B0.copy(order="F")
    ref.trsm(s, L.copy(), want, alpha=0.5, trans=trans)
    pl = Plan(s, device=-1)
    pl.set_option("ordered_sums", ordered_sums)
    flags = 1 if trans == "T" else 0
    prog = taskvm.Program(pl.handle, N.OP_TRSM, k=nrhs, flags=flags, nsn=s.Nsn)
    Bf = B0.reshape(-1, order="F").copy()
    bases = {0: L.copy(), 1: np.full(prog.ws_doubles, np.nan), 4: Bf}
    vm = taskvm.VM(prog, bases, s.relidx, s.chidx, perm=s.p, ldb=s.n, alpha=0.5)
    if order == "dynamic":
        vm.run("dynamic", seed=nrhs, schedule=taskvm.Schedule(pl.handle, N.OP_TRSM, k=nrhs, flags=flags))
    else:
        vm.run("random", seed=nrhs)
    got = Bf.reshape(B0.shape, order="F")
    err = np.max(np.abs(got - want) / np.maximum(np.abs(want).max(axis=0), 1e-300))
    assert err <= 1e-12, err


@pytest.mark.parametrize("trans", ["N", "T"])
def test_reuse_program_takes_the_step_operands_from_the_workspace(grid16, trans):
    """chb_trsm_reuse: the program with flag 2 has no-ops for the diagonal-tile
    inverse and coupling tasks and, run on the workspace a full solve left,
    solves again (a second right-hand side) to the reference's result."""
    s, L = grid16
    flags = 1 if trans == "T" else 0
    pl = Plan(s, device=-1)
    full = taskvm.Program(pl.handle, N.OP_TRSM, k=8, flags=flags, nsn=s.Nsn)
    again = taskvm.Program(pl.handle, N.OP_TRSM, k=8, flags=flags | 2, nsn=s.Nsn)
    assert again.ws_doubles == full.ws_doubles
    # the same tasks and counters (so the same workspace layout on the
    # device), the operand tasks turned into no-ops
    assert again.ntasks == full.ntasks and again.ncounters == full.ncounters
    assert int(np.sum(again.tasks["op"] == taskvm.T_POTRF)) == 0
    assert int(np.sum(full.tasks["op"] == taskvm.T_POTRF)) > 0
    ws = np.full(full.ws_doubles, np.nan)
    for prog, seed in ((full, 1), (again, 2)):
        B0 = np.asfortranarray(np.random.default_rng(seed).standard_normal((s.n, 8)))
        want = B0.copy(order="F")
        ref.trsm(s, L.copy(), want, alpha=0.5, trans=trans)
        Bf = B0.reshape(-1, order="F").copy()
        vm = taskvm.VM(prog, {0: L.copy(), 1: ws, 4: Bf}, s.relidx, s.chidx, perm=s.p, ldb=s.n, alpha=0.5)
        vm.run("random", seed=seed)
        got = Bf.reshape(B0.shape, order="F")
        err = np.max(np.abs(got - want) / np.maximum(np.abs(want).max(axis=0), 1e-300))
        assert err <= 1e-12, err
