"""The autotuner on the GPU: it times the sweeps of a batch (a merged plan)
under the candidate task cuttings, applies the fastest, and the tuned plan's
results still match the reference's kernels (the choice changes only how the
sweep is cut into tasks)."""
import numpy as np
import pytest
import torch

import chompack_b200 as cp
from chompack_b200 import autotune, grids
from helpers import assert_blocks_close
from oracle import ref

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")


def test_tuned_batch_matches_reference():
    autotune._cache.clear()
    specs = grids.uneven_batch_specs(count=12, lo=20, hi=60)
    As = [grids.grid2d_extra(sd, seed=seed) for sd, seed in specs]
    symbs = [cp.symbolic(A, p=cp.amd.order(A)) for A in As]
    B = cp.batch(symbs)
    x0 = B.assemble(As)
    rep = cp.tune(B, x0, reps=2)
    assert rep["cached"] is False and rep["ms"] <= rep["default_ms"]
    assert len(rep["trials"]) == 1 + sum(len(v) - 1 for _, v in autotune.CANDIDATES)
    for name, value in rep["choice"].items():
        if name != "schedule":
            want = value if name != "chol_ksplit" or value == 0 else value
            assert B.plan.option(name) == want
    x = x0.clone()
    B.cholesky(x)
    L = x.cpu().numpy().copy()
    B.projected_inverse(x)
    Y = x.cpu().numpy()
    xh = x0.cpu().numpy()
    for m, s in enumerate(symbs):
        seg = slice(B.offsets[m], B.offsets[m + 1])
        r = xh[seg].copy()
        assert ref.cholesky(s, r) == 0
        assert_blocks_close(s, L[seg], r)
        assert ref.projected_inverse(s, r) == 0
        assert_blocks_close(s, Y[seg], r)
    # the same pattern again: remembered, not timed
    B2 = cp.batch(symbs)
    assert cp.tune(B2, x0)["cached"] is True
    autotune._cache.clear()
