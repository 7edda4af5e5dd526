"""The oracle itself, pinned (CPU): our C restatement of the reference's
sweeps (oracle/oracle.c) against the golden outputs of the reference's own C
kernels, and the reference kernels (oracle/_ref, when built here) against the
same goldens."""
import numpy as np
import pytest

import golden_cases as G
from helpers import assert_blocks_close, rowsign_errors
from oracle import oracle, ref

NUM = G.names(numeric_only=True)


@pytest.mark.parametrize("name", NUM)
def test_restated_cholesky_matches_reference_golden(name):
    d, A, s = G.load(name)
    x = d["blkval"].copy()
    assert oracle.cholesky(s, x) == 0
    assert_blocks_close(s, x, d["ref_cholesky"])


@pytest.mark.skipif(not ref.available(), reason="reference kernels not built here")
@pytest.mark.parametrize("name", NUM)
def test_reference_build_reproduces_goldens(name):
    d, A, s = G.load(name)
    x = d["blkval"].copy()
    assert ref.cholesky(s, x) == 0
    assert np.array_equal(x, d["ref_cholesky"])
    y = x.copy()
    assert ref.projected_inverse(s, y) == 0
    assert np.array_equal(y, d["ref_projected_inverse"])


def test_restated_cholesky_reports_failure():
    d, A, s = G.load("quick7")
    x = -d["blkval"].copy()          # negative definite: first pivot fails
    assert oracle.cholesky(s, x) > 0


@pytest.mark.parametrize("name", NUM)
def test_restated_llt_and_projected_inverse(name):
    d, A, s = G.load(name)
    x = d["ref_cholesky"].copy()
    oracle.llt(s, x)
    assert_blocks_close(s, x, d["ref_llt"])
    y = d["ref_cholesky"].copy()
    assert oracle.projected_inverse(s, y) == 0
    assert_blocks_close(s, y, d["ref_projected_inverse"])


@pytest.mark.parametrize("name", NUM)
@pytest.mark.parametrize("fu", [0, 1])
def test_restated_completion(name, fu):
    d, A, s = G.load(name)
    x = d["ref_projected_inverse"].copy()
    assert oracle.completion(s, x, factored_updates=bool(fu)) == 0
    assert_blocks_close(s, x, d["ref_completion_fu%d" % fu])


@pytest.mark.parametrize("name", NUM)
@pytest.mark.parametrize("fu", [0, 1])
@pytest.mark.parametrize("adj,inv", [(0, 0), (0, 1), (1, 0), (1, 1), (None, 0)])
def test_restated_hessian(name, fu, adj, inv):
    d, A, s = G.load(name)
    u = d["ref_hessian_U0"].copy()
    oracle.hessian(s, d["ref_cholesky"], d["ref_projected_inverse"], [u], adj=None if adj is None else bool(adj),
                   inv=bool(inv), factored_updates=bool(fu))
    key = "ref_hessian_full_fu%d" % fu if adj is None else "ref_hessian_a%d_i%d_fu%d" % (adj, inv, fu)
    assert_blocks_close(s, u, d[key])


@pytest.mark.parametrize("name", NUM)
@pytest.mark.parametrize("trans", ["N", "T"])
def test_restated_trsm(name, trans):
    d, A, s = G.load(name)
    B = d["ref_trsm_B0"].copy(order="F")
    oracle.trsm(s, d["ref_cholesky"], B, alpha=0.5, trans=trans)
    want = d["ref_trsm_" + trans]
    assert np.max(np.abs(B - want)) <= 1e-12 * max(1.0, np.max(np.abs(want)))


@pytest.mark.parametrize("name", NUM)
def test_restated_dot(name):
    d, A, s = G.load(name)
    v = oracle.dot(s, d["blkval"], d["ref_projected_inverse"])
    assert abs(v - float(d["ref_dot"][0])) <= 1e-12 * max(1.0, abs(float(d["ref_dot"][0])))


def test_restated_completion_reports_failure():
    d, A, s = G.load("quick7")
    x = -d["ref_projected_inverse"].copy()
    assert oracle.completion(s, x, factored_updates=False) != 0


@pytest.mark.skipif(not ref.available(), reason="reference kernels not built here")
@pytest.mark.parametrize("kind,args,merge", [("grid2d", (30,), (16, 16)), ("random", (150, 0.05), (8, 8))])
def test_restated_sweeps_match_reference_build(kind, args, merge):
    """All restated sweeps against the reference's kernels run live, on the
    CPU configuration (2-D 5-point 30x30, merge_size_fill(16,16)) and a
    random pattern."""
    from helpers import problem
    import chompack_b200 as cp
    A, s = problem(kind, *args, merge=merge, seed=3)
    blk0 = (cp.cspmatrix(s, device="cpu") + A).blkval.numpy().copy()
    L_r, L_o = blk0.copy(), blk0.copy()
    assert ref.cholesky(s, L_r) == 0 and oracle.cholesky(s, L_o) == 0
    assert_blocks_close(s, L_o, L_r)
    X_r, X_o = L_r.copy(), L_r.copy()
    ref.llt(s, X_r)
    oracle.llt(s, X_o)
    assert_blocks_close(s, X_o, X_r)
    Y_r, Y_o = L_r.copy(), L_r.copy()
    assert ref.projected_inverse(s, Y_r) == 0 and oracle.projected_inverse(s, Y_o) == 0
    assert_blocks_close(s, Y_o, Y_r)
    for fu in (False, True):
        C_r, C_o = Y_r.copy(), Y_r.copy()
        assert ref.completion(s, C_r, factored_updates=fu) == 0
        assert oracle.completion(s, C_o, factored_updates=fu) == 0
        assert_blocks_close(s, C_o, C_r)
        rng = np.random.default_rng(1)
        U0 = [blk0 * rng.standard_normal(blk0.size) for _ in range(2)]
        for adj, inv in [(False, False), (True, True), (True, False), (False, True), (None, False), (None, True)]:
            U_r = [u.copy() for u in U0]
            U_o = [u.copy() for u in U0]
            ref.hessian(s, L_r, Y_r, U_r, adj=adj, inv=inv, factored_updates=fu)
            oracle.hessian(s, L_r, Y_r, U_o, adj=adj, inv=inv, factored_updates=fu)
            for u0, a, b in zip(U0, U_o, U_r):
                if not fu or adj is None:
                    assert_blocks_close(s, a, b)       # sign-invariant: exact parity
                elif adj == inv:
                    assert rowsign_errors(s, a, b) <= 1e-12
                elif kind == "random":                 # no zero pivots: exact parity
                    assert_blocks_close(s, a, b)
                # adj != inv with zero pivots: G(U) = G_ref(D U) for a row-sign
                # pattern D the reference's rounding picks; covered by the
                # round trips of the GPU tests instead
    B0 = np.asfortranarray(np.random.default_rng(2).standard_normal((s.n, 5)))
    for tr in "NT":
        B_r, B_o = B0.copy(order="F"), B0.copy(order="F")
        ref.trsm(s, L_r, B_r, alpha=1.5, trans=tr)
        oracle.trsm(s, L_r, B_o, alpha=1.5, trans=tr)
        assert np.max(np.abs(B_o - B_r)) <= 1e-12 * max(1.0, np.max(np.abs(B_r)))
    assert abs(oracle.dot(s, blk0, Y_r) - ref.dot(s, blk0.copy(), Y_r.copy())) <= 1e-12 * s.n
