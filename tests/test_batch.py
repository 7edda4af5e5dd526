"""Batches (chb_plan_merge), on the CPU: the task program of a merged plan,
executed by the task interpreter in a random order allowed by its waits,
reproduces every matrix's golden reference output, for distinct patterns
and for value sets repeated on one pattern."""
import numpy as np
import pytest

from chompack_b200 import _native as N
from chompack_b200.batch import batch
import golden_cases as G
import taskvm
from helpers import assert_blocks_close

NAMES = ["nc23_amd", "quick7", "numeric31", "rand200_m164", "numeric31"]


def _merged(names):
    loaded = [G.load(nm) for nm in names]
    # repeated names share one symbolic object: value sets on one pattern
    symb_of = {}
    symbs = []
    for nm, (d, A, s) in zip(names, loaded):
        symb_of.setdefault(nm, s)
        symbs.append(symb_of[nm])
    B = batch(symbs, device=-1)
    relidx = np.concatenate([np.asarray(s.relidx) for s in symbs])
    chidx = np.concatenate([np.asarray(s.chidx) + off for s, off in
                            zip(symbs, np.cumsum([0] + [s.Nsn for s in symbs[:-1]]))])
    return B, [d for d, A, s in loaded], symbs, relidx, chidx


def _run(B, op, bases, relidx, chidx, k=0, flags=0, seed=0):
    nsn = B.plan.batch_segments()[-1]
    prog = taskvm.Program(B.plan.handle, op, k=k, flags=flags, nsn=nsn)
    bases = dict(bases)
    bases[1] = np.full(prog.ws_doubles, np.nan)
    return taskvm.VM(prog, bases, relidx, chidx).run("random", seed=seed)


def test_segments_and_offsets():
    B, ds, symbs, relidx, chidx = _merged(NAMES)
    seg = B.plan.batch_segments()
    assert seg == list(np.cumsum([0] + [s.Nsn for s in symbs]))
    assert list(B.offsets) == list(np.cumsum([0] + [int(s.blkptr[-1]) for s in symbs]))


@pytest.mark.parametrize("seed", [0, 1])
def test_merged_cholesky_and_projected_inverse(seed):
    B, ds, symbs, relidx, chidx = _merged(NAMES)
    x = np.concatenate([d["blkval"] for d in ds])
    assert _run(B, N.OP_CHOLESKY, {0: x}, relidx, chidx, seed=seed) == 0
    for m, (d, s) in enumerate(zip(ds, symbs)):
        assert_blocks_close(s, x[B.offsets[m]:B.offsets[m + 1]], d["ref_cholesky"])
    assert _run(B, N.OP_PROJECTED_INVERSE, {0: x}, relidx, chidx, seed=seed + 2) == 0
    for m, (d, s) in enumerate(zip(ds, symbs)):
        assert_blocks_close(s, x[B.offsets[m]:B.offsets[m + 1]], d["ref_projected_inverse"])


@pytest.mark.parametrize("fu", [0, 1])
def test_merged_completion(fu):
    B, ds, symbs, relidx, chidx = _merged(NAMES)
    x = np.concatenate([d["ref_projected_inverse"] for d in ds])
    assert _run(B, N.OP_COMPLETION, {0: x}, relidx, chidx, k=fu, seed=4) == 0
    for m, (d, s) in enumerate(zip(ds, symbs)):
        assert_blocks_close(s, x[B.offsets[m]:B.offsets[m + 1]], d["ref_completion_fu%d" % fu])


def test_merge_rejects_empty():
    with pytest.raises(ValueError):
        batch([], device=-1)
