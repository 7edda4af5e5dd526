"""The sweeps' task programs, executed on the CPU by the task interpreter in
random orders allowed by their recorded waits, against the golden outputs
of the reference's own C kernels.  This checks the planner (operands and
dependency lists) without a GPU; the GPU executes the same task bytes."""
import numpy as np
import pytest

from chompack_b200 import _native as N
from chompack_b200.plan import Plan
import golden_cases as G
import taskvm
from helpers import assert_blocks_close

NUM = G.names(numeric_only=True)


def _run(s, op, bases, k=0, flags=0, seed=0, **kw):
    pl = Plan(s, device=-1)
    prog = taskvm.Program(pl.handle, op, k=k, flags=flags, nsn=s.Nsn)
    ws = np.full(prog.ws_doubles, np.nan)
    bases = dict(bases)
    bases[1] = ws
    vm = taskvm.VM(prog, bases, s.relidx, s.chidx, **kw)
    return vm.run("random", seed=seed)


@pytest.mark.parametrize("name", NUM)
@pytest.mark.parametrize("seed", [0, 1])
def test_cholesky_program(name, seed):
    d, A, s = G.load(name)
    x = d["blkval"].copy()
    assert _run(s, N.OP_CHOLESKY, {0: x}, seed=seed) == 0
    assert_blocks_close(s, x, d["ref_cholesky"])


@pytest.mark.parametrize("name", NUM)
def test_projected_inverse_program(name):
    d, A, s = G.load(name)
    x = d["ref_cholesky"].copy()
    assert _run(s, N.OP_PROJECTED_INVERSE, {0: x}, seed=2) == 0
    assert_blocks_close(s, x, d["ref_projected_inverse"])


@pytest.mark.parametrize("name", NUM)
def test_llt_program(name):
    d, A, s = G.load(name)
    x = d["ref_cholesky"].copy()
    _run(s, N.OP_LLT, {0: x}, seed=3)
    assert_blocks_close(s, x, d["ref_llt"])


@pytest.mark.parametrize("name", NUM)
@pytest.mark.parametrize("trans", ["N", "T"])
def test_trsm_program(name, trans):
    d, A, s = G.load(name)
    B0 = d["ref_trsm_B0"]
    Bf = B0.reshape(-1, order="F").copy()
    _run(s, N.OP_TRSM, {0: d["ref_cholesky"].copy(), 4: Bf}, k=B0.shape[1], flags=1 if trans == "T" else 0,
         seed=4, perm=s.p, ldb=s.n, alpha=0.5)
    got = Bf.reshape(B0.shape, order="F")
    want = d["ref_trsm_" + trans]
    assert np.max(np.abs(got - want)) <= 1e-12 * max(1.0, np.max(np.abs(want)))


@pytest.mark.parametrize("name", NUM)
@pytest.mark.parametrize("fu", [0, 1])
def test_completion_program(name, fu):
    d, A, s = G.load(name)
    x = d["ref_projected_inverse"].copy()
    assert _run(s, N.OP_COMPLETION, {0: x}, k=fu, seed=5 + fu) == 0
    assert_blocks_close(s, x, d["ref_completion_fu%d" % fu])


@pytest.mark.parametrize("name", NUM)
@pytest.mark.parametrize("fu", [0, 1])
@pytest.mark.parametrize("adj", [0, 1])
@pytest.mark.parametrize("inv", [0, 1])
def test_hessian_program(name, fu, adj, inv):
    d, A, s = G.load(name)
    u = d["ref_hessian_U0"].copy()
    bases = {2: d["ref_cholesky"].copy(), 3: d["ref_projected_inverse"].copy(), 5: u}
    _run(s, N.OP_HESSIAN, bases, k=1, flags=adj | inv << 1 | fu << 2, seed=7)
    assert_blocks_close(s, u, d["ref_hessian_a%d_i%d_fu%d" % (adj, inv, fu)])


def test_program_waits_point_backwards():
    d, A, s = G.load("rand200_m164")
    pl = Plan(s, device=-1)
    for op, k, flags in ((N.OP_CHOLESKY, 0, 0), (N.OP_PROJECTED_INVERSE, 0, 0), (N.OP_LLT, 0, 0),
                         (N.OP_COMPLETION, 1, 0), (N.OP_HESSIAN, 2, 5), (N.OP_TRSM, 3, 1)):
        prog = taskvm.Program(pl.handle, op, k=k, flags=flags, nsn=s.Nsn)
        for i, t in enumerate(prog.tasks):
            w0, nw = int(t["wait_off"]), int(t["nwait"])
            for cid, target in prog.waits[w0:w0 + nw]:
                if cid < prog.ntasks:
                    assert cid < i and target == 1
