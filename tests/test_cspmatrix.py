"""cspmatrix assembly on the host (CPU tensors): bit-exact against the
reference's own _iadd_spmatrix.  The exports (spmatrix(), diag(),
add_projection) run on the device and are tested in test_gpu_export.py."""
import numpy as np
import pytest

import chompack_b200 as cp
import golden_cases as G


@pytest.mark.parametrize("name", G.names())
def test_assembly_matches_reference(name):
    d, A, s = G.load(name)
    X = cp.cspmatrix(s, device="cpu") + A
    assert np.array_equal(X.blkval.numpy(), d["blkval"])


def test_pattern_mismatch_raises():
    d, A, s = G.load("quick7")
    bad = cp.spmatrix([1.0], [6], [0], (7, 7))
    X = cp.cspmatrix(s, device="cpu")
    # (6, 0) of the original order is outside the chordal pattern
    with pytest.raises(ValueError):
        X += bad
