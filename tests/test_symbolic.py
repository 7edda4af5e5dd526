"""Host symbolic analysis against the reference (CPU).

* every array, scalar and workspace size equals what the reference's own
  symbolic.py produced for the same pattern / permutation / merge rule
  (golden fixtures, bit-exact);
* the known answers of the reference's tests/test_symbolic.py;
* the AMD goldens of the reference's tests and documentation.
"""
import hashlib
import os

import numpy as np
import pytest

import chompack_b200 as cp
from chompack_b200 import grids
import golden_cases as G


@pytest.mark.parametrize("name", G.names())
def test_symbolic_bit_exact_vs_reference(name):
    d, A, s = G.load(name)
    for a in G.SYMB_ARRAYS:
        assert np.array_equal(getattr(s, a), d["symb_" + a]), a
    sc = d["symb_scalars"]
    assert (s.n, s.Nsn, s.nnz, s.clique_number) == tuple(int(x) for x in sc[:4])
    assert s.fill == (int(sc[4]), int(sc[5]))
    assert (s.frontal_len, s.stack_len, s.stack_size) == tuple(int(x) for x in sc[6:9])
    m = d["symb_memory"]
    assert s.memory == {"stack_depth": int(m[0]), "stack_mem": int(m[1]), "frontal_mem": int(m[2]),
                        "stack_solve": int(m[3])}


def _A17():
    d, A, _ = G.load("chordal17")
    return A


def _Anc():
    d, A, _ = G.load("nc23")
    return A


def test_known_answers_chordal17():       # reference tests/test_symbolic.py:24-34
    s = cp.symbolic(_A17(), p=None)
    assert (s.n, s.nnz, s.clique_number, s.Nsn, s.fill) == (17, 56, 5, 9, (0, 0))
    assert cp.peo(_A17(), list(range(17)))


def test_known_answers_merge():            # :43-60
    s = cp.symbolic(_A17(), p=None, merge_function=cp.merge_size_fill(0, 0))
    assert (s.n, s.nnz, s.Nsn, s.fill, s.clique_number) == (17, 56, 9, (0, 0), 5)
    s = cp.symbolic(_A17(), p=None, merge_function=cp.merge_size_fill(2, 2))
    assert s.n == 17 and s.nnz > 56 and s.Nsn < 9 and s.fill[0] >= 0 and s.fill[1] > 0


def test_known_answers_nonchordal():       # :62-80
    s = cp.symbolic(_Anc(), p=None)
    assert (s.n, s.nnz, s.clique_number, s.Nsn, s.fill) == (23, 150, 12, 10, (73, 0))
    s = cp.symbolic(_Anc(), p=cp.amd.order)
    assert (s.n, s.nnz, s.clique_number, s.Nsn, s.fill) == (23, 113, 9, 15, (36, 0))


def test_known_answers_merge_nonchordal():  # :82-98
    s = cp.symbolic(_Anc(), p=None, merge_function=cp.merge_size_fill(0, 0))
    assert (s.n, s.nnz, s.clique_number, s.Nsn, s.fill) == (23, 150, 12, 10, (73, 0))
    s = cp.symbolic(_Anc(), p=cp.amd.order, merge_function=cp.merge_size_fill(4, 4))
    assert s.n == 23 and s.nnz > 150 and s.Nsn < 10 and s.fill[0] >= 36 and s.fill[1] > 0


def test_amd_quick_start_golden():         # doc/source/quick_start.rst:76-128
    A = cp.spmatrix(1.0, [0, 1, 3, 1, 5, 2, 6, 3, 4, 5, 4, 5, 6, 5, 6], [0, 0, 0, 1, 1, 2, 2, 3, 3, 3, 4, 4, 4, 5, 6],
                    (7, 7))
    s = cp.symbolic(A, p=cp.amd.order)
    assert s.p.tolist() == [2, 6, 4, 1, 3, 5, 0]
    assert s.cliques() == [[0, 1], [1, 2], [2, 4, 5], [3, 5, 6], [4, 5, 6]]
    assert s.parent() == [1, 2, 4, 4, 4]
    assert s.supernodes() == [[0], [1], [2], [3], [4, 5, 6]]
    assert s.separators() == [[1], [2], [4, 5], [5, 6], []]


def test_amd_examples_table_golden():      # doc/source/examples.rst:320-340
    d, A, _ = G.load("ex17")
    s = cp.symbolic(A, p=cp.amd.order)
    assert s.parent() == [4, 2, 4, 4, 5, 7, 7, 7]
    assert s.supernodes() == [[0], [1], [2, 3, 4], [5, 6], [7, 8], [9], [10, 11], [12, 13, 14, 15, 16]]


def test_custom_merge_callable_matches_builtin_rule():
    A = grids.grid2d(20, seed=1)
    p = cp.amd.order(A)
    s1 = cp.symbolic(A, p=p, merge_function=cp.merge_size_fill(8, 8))
    rule = cp.merge_size_fill(8, 8)
    s2 = cp.symbolic(A, p=p, merge_function=lambda a, b, c, d: rule(a, b, c, d))
    for a in G.SYMB_ARRAYS:
        assert np.array_equal(getattr(s1, a), getattr(s2, a))


def test_benchmark_workload_digests():
    """40^3 grid (the FP64 drop-in configuration): SHA-256 of every symbolic
    array equals that of the reference's symbolic.py on the same input."""
    path = os.path.join(G.GOLDEN, "grid3d_40_m32.sha256")
    want = {}
    for line in open(path):
        parts = line.split()
        want[parts[0]] = parts[1:]
    A = grids.grid3d(40, seed=0)
    s = cp.symbolic(A, p=cp.amd.order(A), merge_function=cp.merge_size_fill(32, 32))
    for a in G.SYMB_ARRAYS:
        arr = np.ascontiguousarray(getattr(s, a), dtype=np.int64)
        assert [str(arr.size), hashlib.sha256(arr.tobytes()).hexdigest()] == want[a], a
    assert want["scalars"] == [str(s.n), str(s.Nsn), str(s.nnz), str(s.clique_number)]


def test_diagonal_required():
    A = cp.spmatrix([1.0, 1.0], [1, 0], [0, 0], (2, 2))
    with pytest.raises(AssertionError):
        cp.symbolic(A)
