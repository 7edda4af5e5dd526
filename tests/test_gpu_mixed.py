"""Mixed precision on the GPU: TF32 / 3xTF32 GEMM tiles with FP64 diagonal
tiles.  The factor's error against the FP64 factor is bounded by the
products' precision; solves refined with FP64 residuals reach a normwise
relative residual of 1e-12; log det and its gradient (the projected
inverse) state their errors against FP64; the FP64 chordal SYMV matches a
dense product."""
import numpy as np
import pytest
import torch

import chompack_b200 as cp
from chompack_b200 import mixed
from helpers import problem

pytestmark = pytest.mark.gpu

CASES = [("grid3d", (14,), (32, 32)), ("grid2d", (60,), (64, 64))]


@pytest.fixture(scope="module", autouse=True)
def _need_cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")


def _dev(s, A):
    return cp.cspmatrix(s, device="cuda") + A


def test_symv_matches_dense():
    A, s = problem("grid2d", 12, merge=(8, 8), seed=4)
    X = _dev(s, A)
    n = s.n
    D = np.zeros((n, n))
    I, J, V = np.asarray(A.I).ravel(), np.asarray(A.J).ravel(), np.asarray(A.V).ravel()
    D[I, J] = V
    D = np.tril(D) + np.tril(D, -1).T
    x = torch.from_numpy(np.random.default_rng(0).standard_normal((n, 3))).cuda()
    y = mixed.symv(X, x).cpu().numpy()
    assert np.max(np.abs(y - D @ x.cpu().numpy())) <= 1e-12 * np.max(np.abs(D)) * n


@pytest.mark.parametrize("kind,args,merge", CASES)
@pytest.mark.parametrize("prec,bound", [("tf32", 2e-2), ("tf32x3", 2e-5)])
def test_mixed_factor_and_refined_solve(kind, args, merge, prec, bound):
    A, s = problem(kind, *args, merge=merge, seed=5)
    X = _dev(s, A)
    L64 = cp.cspmatrix(s, blkval=X.blkval.clone())
    cp.cholesky(L64)
    L = cp.cspmatrix(s, blkval=X.blkval.clone())
    cp.cholesky(L, precision=prec)
    err = float((L.blkval - L64.blkval).abs().max() / L64.blkval.abs().max())
    assert 0.0 < err <= bound, err
    B = torch.from_numpy(np.asfortranarray(np.random.default_rng(6).standard_normal((s.n, 8)))).cuda()
    x, rep = mixed.solve(X, L, B, tol=1e-12, maxiter=30)
    assert rep["converged"], rep
    assert rep["residuals"][-1] <= 1e-12
    # the refined solution agrees with the FP64 factor's solve
    x64 = B.clone()
    cp.trsm(L64, x64, trans='N')
    cp.trsm(L64, x64, trans='T')
    assert float((x - x64).abs().max() / x64.abs().max()) <= 1e-10


@pytest.mark.parametrize("prec", ["tf32", "tf32x3"])
def test_logdet_and_gradient_report(prec):
    A, s = problem("grid3d", 12, merge=(32, 32), seed=7)
    X = _dev(s, A)
    before = X.blkval.clone()
    ld, Y, rep = mixed.logdet_and_gradient(X, precision=prec)
    assert torch.equal(X.blkval, before)
    assert Y.is_factor is False
    bound = 1e-2 if prec == "tf32" else 2e-5
    assert rep["logdet_rel_error"] <= bound and rep["gradient_rel_error"] <= bound, rep


def test_host_values_in_mixed_precision():
    A, s = problem("grid3d", 12, merge=(32, 32), seed=8)
    base = (cp.cspmatrix(s, device="cpu") + A).blkval
    Xh = cp.cspmatrix(s, blkval=base.clone().pin_memory())
    Xd = cp.cspmatrix(s, blkval=base.clone().cuda())
    cp.cholesky(Xh, precision="tf32x3")
    cp.cholesky(Xd, precision="tf32x3")
    assert torch.equal(Xh.blkval, Xd.blkval.cpu())
    cp.projected_inverse(Xh, precision="tf32x3")
    cp.projected_inverse(Xd, precision="tf32x3")
    assert torch.equal(Xh.blkval, Xd.blkval.cpu())


def test_tcgen05_tiles_agree_with_mma_sync_tiles(tmp_path):
    """The TF32 tiles run as warp-level mma.sync; with CHB_TF32_TCGEN05 set
    they run on tcgen05 (tensor-memory accumulators).  Both round the
    same FP64 operands to TF32 and accumulate in FP32 (in different orders),
    so the factors agree far below the TF32 error itself (which the FP64
    comparison bounds), and both are far from garbage."""
    import os
    import subprocess
    import sys
    A, s = problem("grid3d", 14, merge=(32, 32), seed=5)
    X = _dev(s, A)
    L = cp.cspmatrix(s, blkval=X.blkval.clone())
    cp.cholesky(L, precision="tf32")
    L64 = cp.cspmatrix(s, blkval=X.blkval.clone())
    cp.cholesky(L64)
    out = tmp_path / "tcgen05.npy"
    code = ("import sys, numpy as np; sys.path.insert(0, %r); sys.path.insert(0, %r)\n"
            "import chompack_b200 as cp\nfrom helpers import problem\n"
            "A, s = problem('grid3d', 14, merge=(32, 32), seed=5)\n"
            "X = cp.cspmatrix(s, device='cuda') + A\ncp.cholesky(X, precision='tf32')\n"
            "np.save(%r, X.blkval.cpu().numpy())\n") % (os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                                        os.path.dirname(os.path.abspath(__file__)), str(out))
    env = dict(os.environ, CHB_TF32_TCGEN05="1")
    subprocess.run([sys.executable, "-c", code], env=env, check=True, timeout=600)
    other = np.load(out)
    got = L.blkval.cpu().numpy()
    ref64 = L64.blkval.cpu().numpy()
    scale = np.abs(ref64).max()
    e_tc = np.abs(got - ref64).max() / scale
    e_ms = np.abs(other - ref64).max() / scale
    assert 0.0 < e_tc <= 2e-3 and 0.0 < e_ms <= 2e-3, (e_tc, e_ms)
    assert np.abs(got - other).max() / scale <= 0.5 * max(e_tc, e_ms), (e_tc, e_ms)


@pytest.mark.parametrize("trans", ["N", "T"])
def test_trsm_reuse_matches_trsm(trans):
    """chb_trsm_reuse (the refinement's solves): a first call computes the
    step operands, later calls on the same workspace reuse them; every
    result agrees with cbase.trsm to rounding."""
    from chompack_b200 import cbase
    A, s = problem("grid3d", 14, merge=(32, 32), seed=4)
    L = cp.cspmatrix(s, device="cuda") + A
    cp.cholesky(L)
    for it in range(3):
        B = torch.randn(5, s.n, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(it)).t()
        want = B.clone()
        cbase.trsm(L, want, trans=trans)
        got = B.clone()
        cbase._trsm_reuse(L, got, trans, it > 0, "test_reuse_" + trans)
        err = float(((got - want).abs().max(dim=0).values / want.abs().max(dim=0).values).max())
        assert err <= 1e-13, (it, err)
