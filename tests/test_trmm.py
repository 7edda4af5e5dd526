"""trmm (B := alpha L B or alpha L^T B with the supernodal factor), on the
CPU: the oracle's restatement of the reference's pybase/trmm.py is pinned
by the reference's own test identity (tests/test_numeric.py:92-104), and
the task programs, executed by the task interpreter in list order, in
random orders allowed by their waits and under the dynamic release rules,
reproduce it."""
import numpy as np
import pytest

import chompack_b200 as cp
from chompack_b200 import _native as N
from chompack_b200.plan import Plan
from helpers import problem
from oracle import oracle
from oracle import trmm as OT
import golden_cases as G
import taskvm

NAMES = ["nc23_amd", "numeric31", "rand200_m164"]


def _dense_lower(d):
    n = int(d["size"][0])
    A = np.zeros((n, n))
    np.add.at(A, (d["I"].astype(int), d["J"].astype(int)), d["V"])
    return np.tril(A) + np.tril(A, -1).T


@pytest.mark.parametrize("name", NAMES)
def test_oracle_pinned_by_the_reference_identity(name):
    d, A, s = G.load(name)
    L = d["ref_cholesky"]
    p = np.asarray(s.p)
    Ld = OT.dense_factor(s, L)
    Ap = _dense_lower(d)[np.ix_(p, p)]
    assert np.allclose(Ld, np.tril(Ld))
    assert np.max(np.abs(Ld @ Ld.T - Ap)) <= 1e-12 * np.max(np.abs(Ap))
    for trans, want in (("N", Ld), ("T", Ld.T)):
        B = np.asfortranarray(np.eye(s.n))
        OT.trmm(s, L, B, trans=trans)
        assert np.max(np.abs(B[np.ix_(p, p)] - want)) <= 1e-13 * np.max(np.abs(want))


def _vm(s, L, B0, trans, alpha, order, seed):
    pl = Plan(s, device=-1)
    nrhs = B0.shape[1]
    flags = 1 if trans == "T" else 0
    prog = taskvm.Program(pl.handle, N.OP_TRMM, k=nrhs, flags=flags, nsn=s.Nsn)
    sch = taskvm.Schedule(pl.handle, N.OP_TRMM, k=nrhs, flags=flags)
    Bf = B0.reshape(-1, order="F").copy()
    bases = {0: L.copy(), 1: np.full(prog.ws_doubles, np.nan), 4: Bf}
    taskvm.VM(prog, bases, s.relidx, s.chidx, perm=s.p, ldb=s.n, alpha=alpha).run(order, seed=seed, schedule=sch)
    return Bf.reshape(B0.shape, order="F"), prog


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("nrhs,order,seed", [(1, "list", 0), (5, "random", 1), (70, "dynamic", 2)])
def test_trmm_program_matches_the_oracle(name, trans, nrhs, order, seed):
    d, A, s = G.load(name)
    L = d["ref_cholesky"]
    B0 = np.asfortranarray(np.random.default_rng(seed).standard_normal((s.n, nrhs)))
    got, _ = _vm(s, L, B0, trans, 0.7, order, seed)
    want = OT.trmm(s, L, B0.copy(order="F"), alpha=0.7, trans=trans)
    assert np.max(np.abs(got - want)) <= 1e-12 * max(1.0, np.max(np.abs(want)))


@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("order,seed", [("random", 3), ("dynamic", 4)])
def test_trmm_wide_fronts(trans, order, seed):
    """Fronts of several 64-column blocks (the in-place block products and
    their write-after-read waits) and three right-hand-side tiles."""
    A, s = problem("grid3d", 12, merge=(128, 128), seed=3)
    assert int(np.max(np.diff(np.asarray(s.snptr)))) > 128
    L = (cp.cspmatrix(s, device="cpu") + A).blkval.numpy().copy()
    assert oracle.cholesky(s, L) == 0
    B0 = np.asfortranarray(np.random.default_rng(seed).standard_normal((s.n, 130)))
    got, prog = _vm(s, L, B0, trans, -1.5, order, seed)
    assert int(np.sum(prog.tasks["op"] == taskvm.T_SUM)) > 0 if trans == "N" else True
    want = OT.trmm(s, L, B0.copy(order="F"), alpha=-1.5, trans=trans)
    assert np.max(np.abs(got - want)) <= 1e-12 * max(1.0, np.max(np.abs(want)))


def test_trmm_then_trsm_is_the_identity():
    """trsm undoes trmm (programs of both, chained in the interpreter)."""
    d, A, s = G.load("numeric31")
    L = d["ref_cholesky"]
    B0 = np.asfortranarray(np.random.default_rng(5).standard_normal((s.n, 3)))
    for trans in ("N", "T"):
        X, _ = _vm(s, L, B0, trans, 2.0, "random", 6)
        pl = Plan(s, device=-1)
        flags = 1 if trans == "T" else 0
        prog = taskvm.Program(pl.handle, N.OP_TRSM, k=3, flags=flags, nsn=s.Nsn)
        Xf = X.reshape(-1, order="F").copy()
        bases = {0: L.copy(), 1: np.full(prog.ws_doubles, np.nan), 4: Xf}
        taskvm.VM(prog, bases, s.relidx, s.chidx, perm=s.p, ldb=s.n, alpha=0.5).run("random", seed=7)
        assert np.max(np.abs(Xf.reshape(B0.shape, order="F") - B0)) <= 1e-11 * np.max(np.abs(B0))
