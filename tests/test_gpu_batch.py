"""Batched sweeps on the GPU (one launch per sweep for the whole batch):
matrices of different patterns and value sets on one pattern, against the
reference's own C kernels matrix by matrix."""
import numpy as np
import pytest
import torch

import chompack_b200 as cp
from chompack_b200 import grids
from helpers import assert_blocks_close
from oracle import ref

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")


def _logdet_ref(s, L):
    ld = 0.0
    for k in range(s.Nsn):
        nn = int(s.snptr[k + 1] - s.snptr[k])
        nj = int(s.sncolptr[k + 1] - s.sncolptr[k])
        blk = L[int(s.blkptr[k]):int(s.blkptr[k + 1])].reshape((nj, nn), order="F")
        ld += 2.0 * np.sum(np.log(np.diag(blk[:nn])))
    return ld


def _problems():
    rng = np.random.default_rng(7)
    As, symbs = [], []
    for i, side in enumerate(rng.integers(12, 40, size=6)):   # 2-D grids + 2 random neighbours
        A = grids.grid2d_extra(int(side), seed=100 + i)
        As.append(A)
        symbs.append(cp.symbolic(A, p=cp.amd.order(A)))
    # value sets on one shared pattern
    A0 = grids.grid2d(24, seed=5)
    s0 = cp.symbolic(A0, p=cp.amd.order(A0), merge_function=cp.merge_size_fill(16, 16))
    for v in range(5):
        As.append(grids.grid2d(24, seed=200 + v))
        symbs.append(s0)
    return As, symbs


def test_batch_cholesky_logdet_pinv_completion():
    As, symbs = _problems()
    B = cp.batch(symbs)
    x = B.assemble(As)
    x0 = x.cpu().numpy().copy()
    B.cholesky(x)
    L = x.cpu().numpy().copy()
    ld = B.logdet(x).cpu().numpy()
    for m, s in enumerate(symbs):
        r = x0[B.offsets[m]:B.offsets[m + 1]].copy()
        assert ref.cholesky(s, r) == 0
        assert_blocks_close(s, L[B.offsets[m]:B.offsets[m + 1]], r)
        lr = _logdet_ref(s, r)
        assert abs(ld[m] - lr) <= 1e-12 * abs(lr)
    B.projected_inverse(x)
    Y = x.cpu().numpy().copy()
    for m, s in enumerate(symbs):
        r = L[B.offsets[m]:B.offsets[m + 1]].copy()
        assert ref.projected_inverse(s, r) == 0
        assert_blocks_close(s, Y[B.offsets[m]:B.offsets[m + 1]], r)
    # <Y, X> = n for every matrix (trace identity), batched dot
    d = B.dot(x, torch.from_numpy(x0).cuda()).cpu().numpy()
    for m, s in enumerate(symbs):
        assert abs(d[m] - s.n) <= 1e-9 * s.n
    for fu in (False, True):
        c = x.clone()
        B.completion(c, factored_updates=fu)
        C = c.cpu().numpy()
        for m, s in enumerate(symbs):
            r = Y[B.offsets[m]:B.offsets[m + 1]].copy()
            assert ref.completion(s, r, factored_updates=fu) == 0
            assert_blocks_close(s, C[B.offsets[m]:B.offsets[m + 1]], r)


def test_batch_matrices_are_views():
    As, symbs = _problems()
    B = cp.batch(symbs[:3])
    x = B.assemble(As[:3])
    Ms = B.matrices(x)
    cp.cholesky(Ms[1])                  # one matrix through the single-matrix API
    B2 = x.clone()
    assert Ms[1].blkval.data_ptr() == x.data_ptr() + 8 * int(B.offsets[1])
    r = B2[B.offsets[1]:B.offsets[2]].cpu().numpy()
    assert np.array_equal(r, Ms[1].blkval.cpu().numpy())


def test_batch_failure_raises():
    As, symbs = _problems()
    B = cp.batch(symbs[:2])
    x = B.assemble(As[:2])
    x[B.offsets[1]:B.offsets[2]] *= -1.0    # second matrix negative definite
    with pytest.raises(ArithmeticError):
        B.cholesky(x)
