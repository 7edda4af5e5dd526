"""Streamed values (chb_cholesky_io and friends), on the CPU: the programs
that copy the values in and out while the sweep runs.  Every task that
touches a chunk of the values waits for that chunk's arrival task; every
chunk's output signal comes after every task that writes the chunk; and
the programs, executed by the task interpreter in random orders allowed by
their waits and under the dynamic release rules, still reproduce the
reference's golden outputs."""
import ctypes

import numpy as np
import pytest

from chompack_b200 import _native as N
from chompack_b200.plan import Plan
import golden_cases as G
import taskvm
from helpers import assert_blocks_close

NAMES = ["nc23_amd", "numeric31", "rand200_m164"]
IN_OUT = N.io_flags(1, 1)
OUT = N.io_flags(0, 1)
IN = N.io_flags(1, 0)


def _io(pl, op, flags):
    counts = (ctypes.c_int64 * 2)()
    N.check(N.program_io(pl.handle, op, 0, flags, counts, None, None, None, None), "program_io")
    in_off = np.zeros(counts[0] + 1, dtype=np.int64)
    in_order = np.zeros(counts[0], dtype=np.int32)
    out_off = np.zeros(counts[1] + 1, dtype=np.int64)
    order = np.zeros(counts[1], dtype=np.int32)
    N.check(N.program_io(pl.handle, op, 0, flags, counts, in_off.ctypes.data, in_order.ctypes.data,
                         out_off.ctypes.data, order.ctypes.data), "program_io")
    if counts[0]:
        assert sorted(in_order.tolist()) == list(range(counts[0]))
    return in_off[:counts[0] + 1] if counts[0] else np.zeros(0, np.int64), \
        out_off[:counts[1] + 1] if counts[1] else np.zeros(0, np.int64), order


def _in_chunks(t, off):
    """Incoming chunks a task touches: those holding the start of each of
    its operands on the values (base 0)."""
    op = int(t["op"])
    if op in (taskvm.T_NOP, taskvm.T_SIGNAL, taskvm.T_ARRIVAL):
        return set()
    starts = [int(t[nm]["off"]) for nm in "abc" if int(t[nm]["base"]) == 0 and int(t[nm]["ld"]) > 0]
    if op == taskvm.T_MROW and int(t["aux"][0]) == 0:
        starts.append((int(t["aux"][2]) & 0xffffffff) | (int(t["aux"][3]) << 32))
    out = {int(np.searchsorted(off, x, side="right")) - 1 for x in starts}
    return {j for j in out if 0 <= j < len(off) - 1}


def _written_ranges(t):
    """Value ranges [lo, hi) a task writes (a tile of at most e = max(m, n)
    rows and columns, a plain copy's m x n strip, a small front's block, or
    an extend-add's front columns)."""
    op = int(t["op"])
    e = max(int(t["m"]), int(t["n"]), 1)

    def tile(nm):
        o = t[nm]
        if int(o["base"]) == 0 and int(o["ld"]) > 0:
            return [(int(o["off"]), int(o["off"]) + (e - 1) * int(o["ld"]) + e)]
        return []
    if op in (taskvm.T_NOP, taskvm.T_SIGNAL, taskvm.T_ARRIVAL, taskvm.T_EXTRACT):
        return []
    if op in (taskvm.T_FRONT, taskvm.T_PFRONT):
        o = t["a"]
        return [(int(o["off"]), int(o["off"]) + int(t["m"]) * int(t["n"]))] if int(o["base"]) == 0 else []
    if op == taskvm.T_COPY and int(t["aux"][0]) & 24 == 0:
        o = t["c"]
        if int(o["base"]) == 0 and int(o["ld"]) > 0:
            return [(int(o["off"]), int(o["off"]) + (max(int(t["n"]), 1) - 1) * int(o["ld"]) + max(int(t["m"]), 1))]
        return []
    if op in (taskvm.T_GEMM, taskvm.T_MROW, taskvm.T_COPY, taskvm.T_SUM):
        return tile("c")
    if op == taskvm.T_LA:
        return tile("a") + tile("c")
    if op == taskvm.T_POTRF:
        return tile("a") + (tile("c") if int(t["aux"][1]) else [])
    if op == taskvm.T_ASM:
        a = t["a"]
        r = []
        if int(a["base"]) == 0 and int(a["ld"]) > 0:
            r.append((int(a["off"]) + int(t["aux"][1]) * int(a["ld"]), int(a["off"]) + int(t["aux"][2]) * int(a["ld"])))
        return r + tile("c")
    return tile("a") + tile("b") + tile("c")


def _predecessors(prog, i, memo):
    """Tasks that must finish before task i starts (transitively)."""
    if i in memo:
        return memo[i]
    tasks, waits = prog.tasks, prog.waits
    members = getattr(prog, "_members", None)
    if members is None:
        members = {}
        for u, t in enumerate(tasks):
            if int(t["group"]) >= 0:
                members.setdefault(int(t["group"]), []).append(u)
        prog._members = members
    out = set()
    stack = [i]
    while stack:
        v = stack.pop()
        w0, nw = int(tasks[v]["wait_off"]), int(tasks[v]["nwait"])
        for cid, _ in waits[w0:w0 + nw]:
            deps = [int(cid)] if cid < prog.ntasks else members.get(int(cid), [])
            for d in deps:
                if d not in out:
                    out.add(d)
                    stack.append(d)
    memo[i] = out
    return out


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("op,flags", [(N.OP_CHOLESKY, IN_OUT), (N.OP_CHOLESKY, IN), (N.OP_PROJECTED_INVERSE, OUT),
                                      (N.OP_PROJECTED_INVERSE, IN_OUT), (N.OP_LLT, IN_OUT)])
def test_streamed_program_structure(name, op, flags):
    d, A, s = G.load(name)
    pl = Plan(s, device=-1)
    prog = taskvm.Program(pl.handle, op, flags=flags, nsn=s.Nsn)
    in_off, out_off, order = _io(pl, op, flags)
    blkptr = set(int(x) for x in s.blkptr)
    total = int(s.blkptr[-1])
    if flags & IN:
        assert in_off[0] == 0 and in_off[-1] == total and np.all(np.diff(in_off) > 0)
        assert set(int(x) for x in in_off) <= blkptr          # whole supernodes
        assert 1 <= len(in_off) - 1 <= 24
    else:
        assert len(in_off) == 0
    arrival = {int(t["aux"][0]): i for i, t in enumerate(prog.tasks) if int(t["op"]) == taskvm.T_ARRIVAL}
    assert sorted(arrival) == list(range(max(len(in_off) - 1, 0)))
    nout = max(len(out_off) - 1, 0)
    if flags & OUT:
        assert out_off[0] == 0 and out_off[-1] == total and np.all(np.diff(out_off) > 0)
        assert 1 <= nout <= 24
        # a cut inside a supernode falls between 64-column tiles
        for x in out_off:
            if int(x) not in blkptr:
                k = int(np.searchsorted(s.blkptr, x, side="right")) - 1
                nj = int(s.sncolptr[k + 1] - s.sncolptr[k])
                col, row = divmod(int(x) - int(s.blkptr[k]), nj)
                assert row == 0 and col % 64 == 0
    writers = [[] for _ in range(nout)]
    for i, t in enumerate(prog.tasks):
        w0, nw = int(t["wait_off"]), int(t["nwait"])
        waited = {int(c) for c, _ in prog.waits[w0:w0 + nw]}
        if flags & IN:
            for j in _in_chunks(t, in_off):
                assert arrival[j] in waited, (i, j)
        for lo, hi in _written_ranges(t):
            for j in range(nout):
                if out_off[j] < hi and lo < out_off[j + 1]:
                    writers[j].append(i)
    if not flags & OUT:
        assert not np.any(prog.tasks["op"] == taskvm.T_SIGNAL)
        return
    sig = {int(t["aux"][0]): i for i, t in enumerate(prog.tasks) if int(t["op"]) == taskvm.T_SIGNAL}
    assert sorted(sig) == list(range(nout))
    assert sorted(order.tolist()) == list(range(nout))
    assert [sig[j] for j in order] == sorted(sig.values())   # listed in signal order
    memo = {}
    for j in range(nout):
        pred = _predecessors(prog, sig[j], memo)
        missing = [u for u in writers[j] if u not in pred]
        assert not missing, (j, missing[:5])


def _run(s, op, bases, flags, seed, order="random"):
    pl = Plan(s, device=-1)
    prog = taskvm.Program(pl.handle, op, flags=flags, nsn=s.Nsn)
    sch = taskvm.Schedule(pl.handle, op, flags=flags)
    bases = dict(bases)
    bases[1] = np.full(prog.ws_doubles, np.nan)
    return taskvm.VM(prog, bases, s.relidx, s.chidx).run(order, seed=seed, schedule=sch)


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("seed,order", [(0, "random"), (1, "random"), (2, "dynamic")])
def test_streamed_programs_match_the_reference(name, seed, order):
    d, A, s = G.load(name)
    x = d["blkval"].copy()
    assert _run(s, N.OP_CHOLESKY, {0: x}, IN_OUT, seed, order) == 0
    assert_blocks_close(s, x, d["ref_cholesky"])
    y = x.copy()
    assert _run(s, N.OP_PROJECTED_INVERSE, {0: y}, OUT, seed + 2, order) == 0
    assert_blocks_close(s, y, d["ref_projected_inverse"])
    z = x.copy()
    _run(s, N.OP_LLT, {0: z}, IN_OUT, seed + 4, order)
    assert_blocks_close(s, z, d["ref_llt"])


def test_streamed_values_only_for_three_sweeps():
    d, A, s = G.load("numeric31")
    pl = Plan(s, device=-1)
    info = (ctypes.c_int64 * 8)()
    assert N.program_info(pl.handle, N.OP_COMPLETION, 1, OUT, info) != 0
    assert b"streamed" in N.last_error()
