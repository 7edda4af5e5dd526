"""GPU parity of trmm (B := alpha L B or alpha L^T B with the supernodal
factor) against the oracle's restatement of the reference's pybase/trmm.py,
through the public API (device tensors and host numpy arrays)."""
import numpy as np
import pytest
import torch

import chompack_b200 as cp
from helpers import problem
from oracle import oracle
from oracle import trmm as OT
import golden_cases as G

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")


def _factor(s, L):
    return cp.cspmatrix(s, blkval=torch.from_numpy(np.array(L, dtype=np.float64)).cuda(), factor=True)


@pytest.mark.parametrize("name", ["nc23_amd", "numeric31", "rand200_m164"])
@pytest.mark.parametrize("trans", ["N", "T"])
def test_trmm_matches_the_oracle(name, trans):
    d, A, s = G.load(name)
    L = d["ref_cholesky"]
    B0 = np.asfortranarray(np.random.default_rng(1).standard_normal((s.n, 5)))
    Bt = torch.from_numpy(B0.copy(order="F")).cuda().t().contiguous().t()  # column-major on the device
    cp.trmm(_factor(s, L), Bt, alpha=0.7, trans=trans)
    want = OT.trmm(s, L, B0.copy(order="F"), alpha=0.7, trans=trans)
    assert np.max(np.abs(Bt.cpu().numpy() - want)) <= 1e-12 * max(1.0, np.max(np.abs(want)))


@pytest.mark.parametrize("trans", ["N", "T"])
def test_trmm_wide_fronts_host_array(trans):
    A, s = problem("grid3d", 12, merge=(128, 128), seed=3)
    L = (cp.cspmatrix(s, device="cpu") + A).blkval.numpy().copy()
    assert oracle.cholesky(s, L) == 0
    B = np.asfortranarray(np.random.default_rng(2).standard_normal((s.n, 130)))
    want = OT.trmm(s, L, B.copy(order="F"), alpha=-1.5, trans=trans)
    cp.trmm(_factor(s, L), B, alpha=-1.5, trans=trans)
    assert np.max(np.abs(B - want)) <= 1e-12 * max(1.0, np.max(np.abs(want)))
