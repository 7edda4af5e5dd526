"""Differentiable chordal log det (chompack_b200.autograd) on the GPU:
value, gradient and Hessian-vector product against the reference's own C
kernels (cholesky, projected_inverse, hessian), and against central finite
differences with h = 1e-6."""
import numpy as np
import pytest
import torch

import chompack_b200 as cp
from chompack_b200 import autograd as ag
from helpers import problem
from oracle import ref

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")


def _weights(s):
    """w = 2 below the diagonal, 1 on it, 0 in the strict upper part."""
    w = np.zeros(int(s.blkptr[-1]))
    for k in range(s.Nsn):
        nn = int(s.snptr[k + 1] - s.snptr[k])
        nj = int(s.sncolptr[k + 1] - s.sncolptr[k])
        m = np.tril(np.ones((nj, nn)), -1) * 2 + np.eye(nj, nn)
        w[int(s.blkptr[k]):int(s.blkptr[k + 1])] = m.reshape(-1, order="F")
    return w


def _ref_logdet_grad(s, x):
    L = x.copy()
    assert ref.cholesky(s, L) == 0
    ld = 0.0
    for k in range(s.Nsn):
        nn = int(s.snptr[k + 1] - s.snptr[k])
        nj = int(s.sncolptr[k + 1] - s.sncolptr[k])
        blk = L[int(s.blkptr[k]):int(s.blkptr[k + 1])].reshape((nj, nn), order="F")
        ld += 2.0 * np.sum(np.log(np.diag(blk[:nn])))
    Y = L.copy()
    assert ref.projected_inverse(s, Y) == 0
    return ld, L, Y


CASES = [("grid3d", (10,), (16, 16)), ("grid2d", (30,), (16, 16)), ("random", (200, 0.03), (8, 8))]


@pytest.mark.parametrize("kind,args,merge", CASES)
def test_logdet_value_and_gradient(kind, args, merge):
    A, s = problem(kind, *args, merge=merge, seed=21)
    X = cp.cspmatrix(s) + A
    x0 = X.blkval.cpu().numpy().copy()
    ld_ref, L, Y = _ref_logdet_grad(s, x0)
    x = X.blkval.clone().requires_grad_(True)
    f = ag.logdet_values(x, s)
    assert abs(float(f.detach()) - ld_ref) <= 1e-12 * abs(ld_ref)
    (g,) = torch.autograd.grad(f, x)
    want = _weights(s) * Y
    got = g.cpu().numpy()
    err = np.max(np.abs(got - want)) / np.max(np.abs(want))
    assert err <= 1e-12, err


@pytest.mark.parametrize("kind,args,merge", CASES)
def test_logdet_finite_differences(kind, args, merge):
    A, s = problem(kind, *args, merge=merge, seed=22)
    X = cp.cspmatrix(s) + A
    x = X.blkval.clone().requires_grad_(True)
    rng = np.random.default_rng(5)
    w = _weights(s)
    u = torch.from_numpy(rng.standard_normal(x.numel()) * (w > 0)).cuda()
    f = ag.logdet_values(x, s)
    (g,) = torch.autograd.grad(f, x, create_graph=True)
    h = 1e-6
    with torch.no_grad():
        fp = float(ag.logdet_values(x + h * u, s))
        fm = float(ag.logdet_values(x - h * u, s))
    fd = (fp - fm) / (2 * h)
    an = float((g * u).sum().detach())
    assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (fd, an)
    # second order: d/dt <grad f(x + t u), u> = u^T H u
    (hv,) = torch.autograd.grad((g * u).sum(), x)
    xp = (x + h * u).detach().requires_grad_(True)
    xm = (x - h * u).detach().requires_grad_(True)
    (gp,) = torch.autograd.grad(ag.logdet_values(xp, s), xp)
    (gm,) = torch.autograd.grad(ag.logdet_values(xm, s), xm)
    fd2 = float(((gp - gm) * u).sum()) / (2 * h)
    an2 = float((hv * u).sum().detach())
    assert an2 < 0.0                                   # log det is concave
    assert abs(fd2 - an2) <= 1e-5 * abs(an2), (fd2, an2)


def test_hvp_matches_reference_hessian():
    A, s = problem("grid3d", 8, merge=(16, 16), seed=23)
    X = cp.cspmatrix(s) + A
    x0 = X.blkval.cpu().numpy().copy()
    _, L, Y = _ref_logdet_grad(s, x0)
    rng = np.random.default_rng(6)
    u0 = x0 * rng.standard_normal(x0.size)
    Hu = u0.copy()
    ref.hessian(s, L, Y, [Hu], adj=None, inv=False, factored_updates=True)
    x = X.blkval.clone().requires_grad_(True)
    (g,) = torch.autograd.grad(ag.logdet_values(x, s), x, create_graph=True)
    c = torch.from_numpy(u0).cuda()
    (hv,) = torch.autograd.grad(g, x, grad_outputs=c)
    # <c, d(w .* Y)> = -<H(C), dX>: the vjp is -w .* H(C)
    want = -_weights(s) * Hu
    err = np.max(np.abs(hv.cpu().numpy() - want)) / np.max(np.abs(want))
    assert err <= 1e-11, err
    # the explicit helper: -H(U) as a cspmatrix
    Lg = cp.cspmatrix(s, blkval=torch.from_numpy(L).cuda(), factor=True)
    Yg = cp.cspmatrix(s, blkval=torch.from_numpy(Y).cuda())
    V = ag.logdet_hvp(Lg, Yg, cp.cspmatrix(s, blkval=torch.from_numpy(u0).cuda()))
    got = V.blkval.cpu().numpy()
    mask = _weights(s) > 0
    assert np.max(np.abs(got[mask] + Hu[mask])) <= 1e-11 * np.max(np.abs(Hu))


def test_batched_value_sets():
    A, s = problem("grid2d", 20, merge=(8, 8), seed=24)
    X = cp.cspmatrix(s) + A
    base = X.blkval
    B = 4
    scale = torch.linspace(1.0, 2.0, B, dtype=torch.float64, device=base.device)[:, None]
    xs = (base[None, :] * scale).clone().requires_grad_(True)
    f = ag.logdet_values(xs, s)
    assert f.shape == (B,)
    f.sum().backward()
    for b in range(B):
        ld_ref, L, Y = _ref_logdet_grad(s, xs[b].detach().cpu().numpy().copy())
        assert abs(float(f[b].detach()) - ld_ref) <= 1e-12 * abs(ld_ref)
        want = _weights(s) * Y
        assert np.max(np.abs(xs.grad[b].cpu().numpy() - want)) <= 1e-12 * np.max(np.abs(want))


def test_logdet_of_cspmatrix_and_gradient_helper():
    A, s = problem("grid2d", 12, seed=25)
    X = cp.cspmatrix(s) + A
    ld_ref, L, Y = _ref_logdet_grad(s, X.blkval.cpu().numpy().copy())
    assert abs(float(ag.logdet(X)) - ld_ref) <= 1e-12 * abs(ld_ref)
    Yg = ag.logdet_gradient(X)
    assert np.max(np.abs(Yg.blkval.cpu().numpy() - Y)) <= 1e-12 * np.max(np.abs(Y))
    with pytest.raises(ValueError):
        ag.logdet(cp.cspmatrix(s, blkval=Yg.blkval, factor=True))


def test_batched_hvp_matches_reference_hessian_per_value_set():
    """Double backward of the batched Function (one merged-plan hessian
    launch per pass for all value sets) against the reference hessian of
    each value set."""
    A, s = problem("grid3d", 8, merge=(16, 16), seed=26)
    X = cp.cspmatrix(s) + A
    base = X.blkval
    B = 3
    scale = torch.tensor([1.0, 1.3, 2.1], dtype=torch.float64, device=base.device)[:, None]
    xs = (base[None, :] * scale).clone().requires_grad_(True)
    (g,) = torch.autograd.grad(ag.logdet_values(xs, s).sum(), xs, create_graph=True)
    rng = np.random.default_rng(9)
    c = torch.from_numpy(rng.standard_normal(tuple(xs.shape))).cuda()
    (hv,) = torch.autograd.grad(g, xs, grad_outputs=c)
    assert (B, int(s.blkptr[-1])) == tuple(hv.shape)
    assert (B, base.device.index) in s.__dict__["_value_set_batches"]
    for b in range(B):
        _, L, Y = _ref_logdet_grad(s, xs[b].detach().cpu().numpy().copy())
        Hu = c[b].cpu().numpy().copy()
        ref.hessian(s, L, Y, [Hu], adj=None, inv=False, factored_updates=True)
        want = -_weights(s) * Hu
        err = np.max(np.abs(hv[b].cpu().numpy() - want)) / np.max(np.abs(want))
        assert err <= 1e-11, (b, err)
