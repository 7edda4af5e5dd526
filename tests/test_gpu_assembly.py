"""cspmatrix += spmatrix on the device (chb_add_sparse; the reference's
_iadd_spmatrix, symbolic.py:1138-1174): the values must equal the
reference's own assembly bit for bit (the `blkval` arrays of the golden
fixtures, written by the reference's symbolic.py), at n = 10^6 they must
equal the host restatement's, and an entry outside the chordal pattern
raises ValueError as the reference's row lookup does."""
import numpy as np
import pytest
import torch

import chompack_b200 as cp
import golden_cases as G
from chompack_b200 import grids
from chompack_b200.sparse import spmatrix

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")


@pytest.mark.parametrize("name", G.names())
def test_device_assembly_is_the_references(name):
    d, A, s = G.load(name)
    X = cp.cspmatrix(s, device="cuda") + A
    assert X.blkval.is_cuda
    assert np.array_equal(X.blkval.cpu().numpy(), d["blkval"])
    X -= A
    assert not np.any(X.blkval.cpu().numpy())
    Y = cp.cspmatrix(s, device="cuda") + A
    Y += A
    assert np.array_equal(Y.blkval.cpu().numpy(), 2.0 * d["blkval"])


def test_device_assembly_matches_host_at_a_million_columns():
    """2-D 5-point grid 1000^2, AMD, merge_size_fill(64,64): 174.7 M block
    values; device and host assembly agree exactly."""
    A = grids.grid2d(1000, seed=0)
    s = cp.symbolic(A, p=cp.amd.order(A), merge_function=cp.merge_size_fill(64, 64))
    Xd = cp.cspmatrix(s, device="cuda") + A
    Xh = cp.cspmatrix(s, device="cpu") + A
    assert torch.equal(Xd.blkval.cpu(), Xh.blkval)


def test_upper_entries_are_ignored_and_repeated_entries_summed():
    """Only A's lower triangle is read (symmetrize, misc.py:32-40): adding
    A + (a strictly upper matrix) changes nothing."""
    d, A, s = G.load("numeric31")
    I, J, V = np.asarray(A.I), np.asarray(A.J), np.asarray(A.V)
    lo = I > J
    upper = spmatrix(V[lo] * 3.0, J[lo], I[lo], A.size)      # mirror images, upper triangle only
    X = cp.cspmatrix(s, device="cuda") + A
    X += upper
    assert np.array_equal(X.blkval.cpu().numpy(), d["blkval"])


def test_entry_outside_the_pattern_raises():
    """Two disconnected 3x3 cliques: (5, 0) joins them and lies outside
    the chordal pattern."""
    I, J = [], []
    for b in (0, 3):
        for j in range(3):
            for i in range(j, 3):
                I.append(b + i)
                J.append(b + j)
    A = spmatrix([4.0 if i == j else 1.0 for i, j in zip(I, J)], I, J, (6, 6))
    s = cp.symbolic(A, p=cp.amd.order)
    X = cp.cspmatrix(s, device="cuda") + A
    with pytest.raises(ValueError):
        X += spmatrix([1.0], [5], [0], (6, 6))
    with pytest.raises(ValueError):
        X += spmatrix([1.0], [2], [0], (7, 7))
