"""Per-task traces of a sweep and the critical path through them.

The engine records, when a trace buffer is set on a plan
(`chb_set_trace`), four 64-bit words per task: the global timer (ns) when a
CTA took the task, when its waits were met, when it ended, and the SM id |
task kind << 32.  `record` runs a sweep with tracing on; `critical_path`
walks back from the last task to end through, at each step, the wait that
was met last, and splits the path's time into execution, wait after
release and claim delay (a ready task that no CTA had taken yet: under the
static list order its list position had not been reached, under the
dynamic schedule every CTA was busy).

    python -m chompack_b200.trace --side 40 --merge 32 32 [--trsm 8]

prints the summary for cholesky and projected_inverse on the 3-D 7-point
grid side^3 (--grid2d: the 2-D 5-point grid side^2; AMD order,
merge_size_fill(merge)), and with --trsm R for the
triangular solves 'N' and 'T' with R right-hand sides; it needs a GPU.
"""
import argparse
import ctypes
import json

import numpy as np

from . import _native as N

_OPERAND = np.dtype([("off", "<i8"), ("ld", "<i4"), ("base", "u1"), ("mode", "u1"), ("prec", "<i2"),
                     ("diag", "<i4"), ("pad2", "<i4")])
TASK = np.dtype({
    "names": ["op", "cmode", "nwait", "wait_off", "group", "m", "n", "k", "cdiag", "aux", "alpha", "beta",
              "a", "b", "c", "off2"],
    "formats": ["u1", "u1", "<u2", "<i4", "<i4", "<i4", "<i4", "<i4", "<i4", ("<i4", 4), "<f8", "<f8",
                _OPERAND, _OPERAND, _OPERAND, "<i8"],
    "offsets": [0, 1, 2, 4, 8, 12, 16, 20, 24, 28, 48, 56, 64, 88, 112, 136],
    "itemsize": 144,
})

OP_NAMES = ["GEMM", "POTRF", "ASM", "MROW", "EXTRACT", "COPY", "INV", "RPOTRF", "QL", "VEC", "NOP", "LA",
            "SUM", "SIGNAL", "ARRIVAL", "FRONT", "PFRONT", "SUBTREE", "PSUBTREE", "TRSV"]
T_POTRF, T_LA = 1, 11

N.lib.chb_program_info.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_int64)]
N.lib.chb_program_export.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_int,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]


def program(plan, op, k=0, flags=0):
    """The task list and (counter, target) waits of a compiled sweep."""
    info = (ctypes.c_int64 * 8)()
    N.check(N.lib.chb_program_info(plan.handle, op, k, flags, info), "program_info")
    if info[7] != TASK.itemsize:
        raise RuntimeError("task record is %d bytes, expected %d" % (info[7], TASK.itemsize))
    tasks = np.zeros(info[0], dtype=TASK)
    waits = np.zeros((info[1], 2), dtype=np.int32)
    N.check(N.lib.chb_program_export(plan.handle, op, k, flags, tasks.ctypes.data, waits.ctypes.data, None),
            "program_export")
    return tasks, waits


def record(plan, op, run, k=0, flags=0):
    """Run `run()` (which must launch exactly the sweep `op` on `plan`) with
    tracing on; returns (tasks, waits, trace) with trace an (ntasks, 4)
    int64 array."""
    import torch
    tasks, waits = program(plan, op, k, flags)
    buf = torch.zeros(4 * len(tasks), dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    N.check(N.set_trace(plan.handle, buf.data_ptr(), len(tasks)), "set_trace")
    try:
        run()
        torch.cuda.synchronize()
    finally:
        N.check(N.set_trace(plan.handle, None, 0), "set_trace")
    return tasks, waits, buf.cpu().numpy().reshape(-1, 4)


def critical_path(tasks, waits, trace):
    """The chain of tasks that ended last, each preceded by the wait met
    last.  A fused diagonal task (POTRF with k > 0) is entered through its
    first Task::cdiag waits; group counters are met when their last member
    ends; early signals (aux[3] - 1 of fused diagonal and look-ahead tasks)
    at the end of the raising task at the latest, so their release is taken
    as min(that end, the waiter's start)."""
    nt = len(tasks)
    t0 = int(trace[:, 0].min())
    claim = trace[:, 0].astype(np.int64) - t0
    start = trace[:, 1].astype(np.int64) - t0
    end = trace[:, 2].astype(np.int64) - t0
    op = tasks["op"].astype(int)
    producers = {}
    for i in range(nt):
        g = int(tasks["group"][i])
        if g >= 0:
            producers.setdefault(g, []).append(i)
        if (op[i] == T_POTRF and int(tasks["k"][i]) > 0) or op[i] == T_LA:
            a3 = int(tasks["aux"][i][3])
            if a3 > 0:
                producers.setdefault(a3 - 1, []).append(i)

    def release(cid):
        if cid < nt:
            return int(end[cid]), cid
        m = producers.get(cid)
        if not m:
            return 0, -1
        j = max(m, key=lambda u: end[u])
        return int(end[j]), j

    cur = int(np.argmax(end))
    path = []
    while cur >= 0:
        w0, nw = int(tasks["wait_off"][cur]), int(tasks["nwait"][cur])
        fused = op[cur] == T_POTRF and int(tasks["k"][cur]) > 0
        npre = int(tasks["cdiag"][cur]) if fused else nw
        best_r, best_p = 0, -1
        for cid, _ in waits[w0:w0 + npre]:
            r, p = release(int(cid))
            r = min(r, int(start[cur]))
            if r > best_r or best_p < 0:
                best_r, best_p = r, p
        path.append({"task": cur, "op": OP_NAMES[op[cur]] if op[cur] < len(OP_NAMES) else str(op[cur]),
                     "exec_ns": int(end[cur] - start[cur]),
                     "wait_ns": int(start[cur] - max(claim[cur], best_r)),
                     "claim_delay_ns": int(max(0, claim[cur] - best_r)) if best_p >= 0 else int(claim[cur])})
        cur = best_p
    path.reverse()
    by_op, count = {}, {}
    for p in path:
        by_op[p["op"]] = by_op.get(p["op"], 0) + p["exec_ns"]
        count[p["op"]] = count.get(p["op"], 0) + 1
    dur = end - start
    per_op = {}
    for o in sorted(set(op.tolist())):
        sel = op == o
        per_op[OP_NAMES[o] if o < len(OP_NAMES) else str(o)] = {
            "tasks": int(sel.sum()), "mean_us": round(float(dur[sel].mean()) / 1e3, 2),
            "total_ms": round(float(dur[sel].sum()) / 1e6, 3)}
    return {
        "span_ms": round(float(end.max()) / 1e6, 4),
        "path_tasks": len(path),
        "path_exec_ms": {k: round(v / 1e6, 4) for k, v in sorted(by_op.items(), key=lambda x: -x[1])},
        "path_count": count,
        "path_wait_ms": round(sum(p["wait_ns"] for p in path) / 1e6, 4),
        "path_claim_delay_ms": round(sum(p["claim_delay_ns"] for p in path) / 1e6, 4),
        "cta_time_ms": round(float(dur.sum()) / 1e6, 2),
        "per_op": per_op,
        "path": path,
    }


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--side", type=int, default=40)
    ap.add_argument("--merge", type=int, nargs=2, default=(32, 32))
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--path", action="store_true", help="also list the path's tasks")
    ap.add_argument("--trsm", type=int, default=0, help="also trace trsm with this many right-hand sides")
    ap.add_argument("--batch", type=int, default=0,
                    help="trace the first BATCH matrices of the uneven 2-D batch in one merged plan instead")
    ap.add_argument("--grid2d", action="store_true", help="the 2-D 5-point grid side^2 instead")
    ap.add_argument("--dump", default="", help="also save each sweep's task records and raw trace (.npz)")
    args = ap.parse_args()
    import torch
    import chompack_b200 as cp
    from chompack_b200 import grids
    if args.batch:
        return trace_batch(args)
    A = grids.grid2d(args.side, seed=0) if args.grid2d else grids.grid3d(args.side, seed=0)
    s = cp.symbolic(A, p=cp.amd.order(A), merge_function=cp.merge_size_fill(*args.merge))
    x0 = (cp.cspmatrix(s, device="cpu") + A).blkval.cuda()
    plan = s.plan(0)
    X = cp.cspmatrix(s, blkval=x0.clone(), factor=False)
    cp.cholesky(X)
    l0 = X.blkval.clone()
    sweeps = (("cholesky", N.OP_CHOLESKY, lambda: cp.cholesky(cp.cspmatrix(s, blkval=x0.clone(), factor=False))),
              ("projected_inverse", N.OP_PROJECTED_INVERSE,
               lambda: cp.projected_inverse(cp.cspmatrix(s, blkval=l0.clone(), factor=True))))
    if args.trsm > 0:
        L = cp.cspmatrix(s, blkval=l0, factor=True)
        B0 = torch.randn(args.trsm, s.n, dtype=torch.float64, device="cuda").t()   # column-major
        for trans in ("N", "T"):
            sweeps += (("trsm_" + trans, N.OP_TRSM, lambda tr=trans: cp.trsm(L, B0.clone().t().contiguous().t(),
                                                                              trans=tr)),)
    out = {"workload": "%s grid %d^%d (n=%d), AMD, merge_size_fill(%d,%d)"
                       % ("2-D 5-point" if args.grid2d else "3-D 7-point", args.side, 2 if args.grid2d else 3, s.n,
                          args.merge[0], args.merge[1])}
    for name, op, fn in sweeps:
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        k, flags = (args.trsm, int(name == "trsm_T")) if op == N.OP_TRSM else (0, 0)
        tasks, waits, tr = record(plan, op, fn, k, flags)
        if args.dump:
            np.savez_compressed("%s_%s.npz" % (args.dump, name), tasks=tasks, waits=waits, trace=tr)
        res = critical_path(tasks, waits, tr)
        if not args.path:
            res.pop("path")
        out[name] = res
    print(json.dumps(out, indent=1))


def trace_batch(args):
    """cholesky and projected_inverse over the first args.batch matrices of
    the uneven batch (2-D grids of side 20..120 with two extra neighbours,
    AMD, no merging), one merged plan."""
    import torch
    import chompack_b200 as cp
    from chompack_b200 import grids
    specs = grids.uneven_batch_specs()[:args.batch]
    As = [grids.grid2d_extra(sd, seed=seed) for sd, seed in specs]
    Bt = cp.batch([cp.symbolic(A, p=cp.amd.order(A)) for A in As])
    x0 = Bt.assemble(As)
    l0 = x0.clone()
    Bt.cholesky(l0)
    plan = Bt.plan
    sweeps = (("cholesky", N.OP_CHOLESKY, lambda: Bt.cholesky(x0.clone())),
              ("projected_inverse", N.OP_PROJECTED_INVERSE, lambda: Bt.projected_inverse(l0.clone())))
    out = {"workload": "uneven 2-D batch, first %d matrices, one merged plan" % args.batch}
    for name, op, fn in sweeps:
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        tasks, waits, tr = record(plan, op, fn)
        res = critical_path(tasks, waits, tr)
        if not args.path:
            res.pop("path")
        out[name] = res
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
