"""Product-form Cholesky factor on the GPU (csrc/pf.cu; cbase.pfchol /
pftrsm / pftrmm and the pfcholesky class) against the reference's own
dpftrf / dpfsv / dpfmv (src/C/pfcholesky.c, compiled into oracle/_ref) on
the same inputs, and the reference test suite's identities for the class
(tests/test_numeric.py:120-159 of the reference).

Tolerance.  The GPU evaluates the recurrences as parallel scans (the
running sums as affine scans, dpftrf's alpha through the prefix sum of v^2
in 1/alpha), the reference sequentially, so the last bits differ, and the
recurrences amplify them on entries near zero.  The parity measure is
normwise per column: max |x - x_ref| <= 1e-12 max |x_ref| (helpers.RTOL), at
every size; entry-wise (|x - x_ref| <= 1e-12 max(|x_ref|, 1e-3 max|column|),
the block measure of the other tests) holds up to n = 1000.  Beyond that the
reference itself is about 1.5e-12 entry-wise off an extended-precision
evaluation of its own recurrences (n = 20,000, k = 8), so the entry-wise
check there is against that evaluation (oracle/pf_extended.py): the GPU's
error may not exceed four times the reference's own."""
import numpy as np
import pytest
import torch

import chompack_b200 as cp
from chompack_b200 import cbase
import golden_cases
from helpers import RTOL, FLOOR
from oracle import ref

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")


def _cm(a):
    """Column-major CUDA copy of a Fortran-ordered numpy array."""
    return torch.from_numpy(np.ascontiguousarray(a.T)).cuda().t()


def _entrywise(got, want):
    got = np.asarray(got)
    want = np.asarray(want)
    if want.ndim == 1:
        got, want = got[:, None], want[:, None]
    scale = np.maximum(np.abs(want), FLOOR * np.maximum(np.abs(want).max(axis=0), 1e-300))
    return float(np.max(np.abs(got - want) / scale))


def _close(got, want):
    got = np.asarray(got)
    want = np.asarray(want)
    if want.ndim == 1:
        got, want = got[:, None], want[:, None]
    err = float(np.max(np.abs(got - want).max(axis=0) / np.maximum(np.abs(want).max(axis=0), 1e-300)))
    assert err <= RTOL, "normwise error %.3e" % err
    if want.shape[0] <= 1000:
        e = _entrywise(got, want)
        assert e <= RTOL, "entry-wise scaled error %.3e" % e


def _problem(n, k, seed):
    rng = np.random.default_rng(seed)
    V = np.asfortranarray(rng.random((n, k)) / np.sqrt(n))
    a = np.concatenate([[1.2, -0.01], rng.uniform(-0.2, 2.0, size=max(0, k - 2))])[:k]
    return a, V


SIZES = [(31, 2), (1000, 5), (70000, 16), (1500000, 3)]


@pytest.mark.parametrize("n,k", SIZES)
def test_pfchol_matches_reference(n, k):
    a, V = _problem(n, k, seed=n + k)
    Vr = V.copy(order="F")
    Lr, Br, info = ref.pfchol(a, Vr)
    assert info == 0
    Vg = _cm(V)
    Lg = _cm(np.zeros((n, k), order="F"))
    Bg = _cm(np.zeros((n, k), order="F"))
    cbase.pfchol(a, Vg, Lg, Bg)
    _close(Vg.cpu().numpy(), Vr)
    _close(Lg.cpu().numpy(), Lr)
    _close(Bg.cpu().numpy(), Br)


@pytest.mark.parametrize("n,k", SIZES)
@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("nrhs", [1, 3, 70])
def test_pftrsm_pftrmm_match_reference(n, k, trans, nrhs):
    if n * nrhs > 4_000_000:
        nrhs = 1
    a, V = _problem(n, k, seed=7 * n + k)
    Vr = V.copy(order="F")
    Lr, Br, info = ref.pfchol(a, Vr)
    assert info == 0
    U0 = np.asfortranarray(np.random.default_rng(n + nrhs).standard_normal((n, nrhs)))
    for gpu_fn, ref_fn in ((cbase.pftrsm, ref.pftrsm), (cbase.pftrmm, ref.pftrmm)):
        Ur = U0.copy(order="F")
        ref_fn(Vr, Lr, Br, Ur, trans=trans)
        Ug = _cm(U0)
        gpu_fn(_cm(Vr), _cm(Lr), _cm(Br), Ug, trans=trans)
        _close(Ug.cpu().numpy(), Ur)


def test_pftrsm_on_host_arrays_and_leading_dimension():
    """numpy (Fortran-ordered) right-hand sides are copied to the device and
    back; a device block with a leading dimension larger than n."""
    n, k = 500, 4
    a, V = _problem(n, k, seed=3)
    Vr = V.copy(order="F")
    Lr, Br, _ = ref.pfchol(a, Vr)
    U0 = np.asfortranarray(np.random.default_rng(4).standard_normal((n, 6)))
    Ur = U0.copy(order="F")
    ref.pftrsm(Vr, Lr, Br, Ur, trans="N")
    Uh = U0.copy(order="F")
    cbase.pftrsm(Vr, Lr, Br, Uh, trans="N")
    _close(Uh, Ur)
    big = torch.zeros((6, n + 13), dtype=torch.float64).cuda()
    Ug = big.t()[:n]                       # n x 6, stride (1, n + 13)
    Ug.copy_(torch.from_numpy(U0))
    cbase.pftrsm(_cm(Vr), _cm(Lr), _cm(Br), Ug, trans="N")
    _close(Ug.cpu().numpy(), Ur)


def test_pfchol_not_positive_definite_raises():
    n, k = 2000, 2
    V = np.asfortranarray(np.ones((n, k)) / np.sqrt(n))
    a = np.array([-2.0, 1.0])             # I - 2 v v^T with |v| = 1 is indefinite
    Vr = V.copy(order="F")
    _, _, info = ref.pfchol(a, Vr)
    assert info == -1
    with pytest.raises(ArithmeticError):
        cbase.pfchol(a, _cm(V), _cm(np.zeros((n, k), order="F")), _cm(np.zeros((n, k), order="F")))


def test_bad_trans_is_rejected():
    V = _cm(np.asfortranarray(np.ones((4, 1))))
    with pytest.raises(ValueError):
        cbase.pftrsm(V, V, V, V.clone(), trans="X")


def _identities(Lpf, Xsym, U, D, V):
    """The reference test's identities: L L^T V = (X + U D U^T) V and
    L^{-T} L^{-1} L L^T V = V."""
    Vt = V.copy(order="F")
    Lpf.trmm(Vt, trans="T")
    Lpf.trmm(Vt, trans="N")
    want = Xsym @ V + U @ (D @ (U.T @ V))
    assert np.max(np.abs(Vt - want)) <= 1e-10 * np.max(np.abs(want))
    Lpf.trsm(Vt, trans="N")
    Lpf.trsm(Vt, trans="T")
    assert np.max(np.abs(Vt - V)) <= 1e-10 * np.max(np.abs(V))


def test_pfcholesky_class_identities_reference_suite_case():
    """tests/test_numeric.py:120-159: the n = 31 matrix of the suite, U =
    (1..2n)/n as an n x 2 matrix, alpha = (1.2, -0.01), V random n x 3; the
    product-form factor from an spmatrix (with AMD) and from a cspmatrix."""
    d, A, s = golden_cases.load("numeric31")
    n = s.n
    U = np.asfortranarray(np.arange(1, 2 * n + 1, dtype=np.float64).reshape((n, 2), order="F") / n)
    alpha = np.array([1.2, -0.01])
    D = np.diag(alpha)
    V = np.asfortranarray(np.random.default_rng(1).random((n, 3)))
    Xd = np.zeros((n, n))
    Xd[np.asarray(A.I), np.asarray(A.J)] = np.asarray(A.V)
    Xsym = np.tril(Xd) + np.tril(Xd, -1).T
    Lpf = cp.pfcholesky(A, U, alpha, p=cp.amd.order)
    _identities(Lpf, Xsym, U, D, V)
    X = cp.cspmatrix(s) + A
    Lpf2 = cp.pfcholesky(X, U, alpha)
    _identities(Lpf2, Xsym, U, D, V)
    Lf = X.copy()
    cp.cholesky(Lf)
    Lpf3 = cp.pfcholesky(Lf, U, alpha)
    _identities(Lpf3, Xsym, U, D, V)


def test_pfcholesky_class_on_a_grid():
    """A 3-D grid (n = 4,096) with a rank-8 update, device right-hand sides."""
    from chompack_b200 import grids
    A = grids.grid3d(16, seed=2)
    n = A.size[0]
    rng = np.random.default_rng(8)
    U = np.asfortranarray(rng.standard_normal((n, 8)))
    alpha = rng.uniform(0.1, 1.0, size=8)
    Lpf = cp.pfcholesky(A, U, alpha, p=cp.amd.order)
    Xd = np.zeros((n, n))
    Xd[np.asarray(A.I), np.asarray(A.J)] = np.asarray(A.V)
    Xsym = np.tril(Xd) + np.tril(Xd, -1).T
    V = np.asfortranarray(rng.standard_normal((n, 5)))
    Vt = _cm(V)
    Lpf.trmm(Vt, trans="T")
    Lpf.trmm(Vt, trans="N")
    want = Xsym @ V + U @ (np.diag(alpha) @ (U.T @ V))
    assert np.max(np.abs(Vt.cpu().numpy() - want)) <= 1e-10 * np.max(np.abs(want))
    Lpf.trsm(Vt, trans="N")
    Lpf.trsm(Vt, trans="T")
    assert np.max(np.abs(Vt.cpu().numpy() - V)) <= 1e-10 * np.max(np.abs(V))


def test_pfchol_entrywise_accuracy_against_extended_precision():
    """n = 20,000, k = 8: entry-wise, the GPU is as close to an
    extended-precision evaluation of the reference's recurrences as the
    reference itself (within a factor of four)."""
    from oracle.pf_extended import dpftrf_extended
    n, k = 20000, 8
    a, V = _problem(n, k, seed=5)
    Vr = V.copy(order="F")
    Lr, Br, info = ref.pfchol(a, Vr)
    assert info == 0
    Vt, Lt, Bt = dpftrf_extended(a, V)
    Vg, Lg, Bg = _cm(V), _cm(np.zeros((n, k), order="F")), _cm(np.zeros((n, k), order="F"))
    cbase.pfchol(a, Vg, Lg, Bg)
    for got, mine, truth in ((Vg, Vr, Vt), (Lg, Lr, Lt), (Bg, Br, Bt)):
        e_gpu = _entrywise(got.cpu().numpy(), truth)
        e_ref = _entrywise(mine, truth)
        assert e_gpu <= 4.0 * e_ref + 1e-15, (e_gpu, e_ref)
