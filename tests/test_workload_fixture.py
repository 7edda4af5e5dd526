"""CPU checks of the benchmark's reference-leg inputs (oracle/workload.py):
the committed 40^3 symbolic factorisation equals this package's symbolic
analysis (both equal the reference's symbolic.py, by the SHA-256 digests in
tests/golden/grid3d_40_m32.sha256), and the oracle's own assembly of the
seeded values gives the same block values as cspmatrix + A."""
import numpy as np

import chompack_b200 as cp
from chompack_b200 import grids
from oracle import workload as W


def test_fixture_equals_package_symbolic_and_assembly():
    s = W.load_symbolic("grid3d_40_m32")
    A = grids.grid3d(40, seed=0)
    sc = cp.symbolic(A, p=cp.amd.order(A), merge_function=cp.merge_size_fill(32, 32))
    for a in W.SYMB_ARRAYS:
        assert np.array_equal(np.asarray(getattr(sc, a), dtype=np.int64), getattr(s, a)), a
    assert (s.n, s.Nsn, s.clique_number) == (sc.n, sc.Nsn, sc.clique_number)
    assert s.memory == dict(sc.memory)
    n, I, J, V = W.grid3d_lower(40, seed=0)
    x = W.assemble(s, n, I, J, V)
    want = (cp.cspmatrix(sc, device="cpu") + A).blkval.numpy()
    assert np.array_equal(x, want)


def test_grid_recipe_matches_package_on_small_grids():
    for side, seed in ((3, 0), (5, 7)):
        n, I, J, V = W.grid3d_lower(side, seed=seed)
        A = grids.grid3d(side, seed=seed)
        got = sorted(zip(I.tolist(), J.tolist(), V.tolist()))
        want = sorted(zip(np.asarray(A.I).tolist(), np.asarray(A.J).tolist(), np.asarray(A.V).tolist()))
        assert got == want
