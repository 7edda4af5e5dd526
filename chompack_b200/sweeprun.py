"""Run one sweep of a synthetic grid a few times and print its CUDA-event
times (for profiling a single kernel launch, e.g. under ncu):

    python -m chompack_b200.sweeprun --side 40 --merge 32 --sweep cholesky --precision fp64 --reps 3
    python -m chompack_b200.sweeprun --side 40 --merge 32 --sweep trsm --nrhs 8 --trans N --reps 3

The matrix is the seeded 3-D 7-point grid side^3 (or the 2-D 5-point grid
with --grid2d) with AMD ordering and merge_size_fill(merge, merge), or with
--batch N the first N matrices of the uneven batch (2-D grids of side 20..120
with two extra neighbours per node, AMD, no merging) in one merged plan;
each repetition refreshes the values and launches the sweep once
(projected_inverse and trsm run on the factor of a preceding, untimed
cholesky; trsm on --nrhs seeded N(0,1) right-hand sides).  With
--scratch-limit (bytes, or 'stack' / '<m>stack' for m times the
reference's postorder stack size) the update matrices and the fronts'
scratch share a pool of about that size; the line then also reports the
pool (chb_program_pool).
"""
import argparse
import json

import numpy as np
import torch

from . import grids
from . import cbase
from .cspmatrix import cspmatrix
from .symbolic import symbolic, merge_size_fill
from . import amd


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--side", type=int, default=40)
    ap.add_argument("--grid2d", action="store_true")
    ap.add_argument("--merge", type=int, default=32)
    ap.add_argument("--sweep", default="cholesky", choices=["cholesky", "projected_inverse", "trsm"])
    ap.add_argument("--nrhs", type=int, default=8)
    ap.add_argument("--trans", default="N", choices=["N", "T"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "tf32", "tf32x3"])
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--batch", type=int, default=0)
    ap.add_argument("--scratch-limit", default=None,
                    help="bytes for the update matrices and fronts' scratch (plan option scratch_limit), or "
                         "'stack' / '<m>stack' for (m times) the reference's postorder stack size")
    args = ap.parse_args()
    if args.batch:
        return run_batch(args)
    A = grids.grid2d(args.side, seed=0) if args.grid2d else grids.grid3d(args.side, seed=0)
    s = symbolic(A, p=amd.order(A), merge_function=merge_size_fill(args.merge, args.merge))
    limit = _scratch_limit(args, s)
    X0 = cspmatrix(s) + A
    base = X0.blkval
    if args.sweep == "trsm":
        return run_trsm(args, s, base)
    if args.sweep == "projected_inverse":
        L = cspmatrix(s, blkval=base.clone())
        cbase.cholesky(L, precision=args.precision)
        base = L.blkval
    X = cspmatrix(s, blkval=base.clone(), factor=args.sweep == "projected_inverse")
    times = []
    for _ in range(args.reps):
        X.blkval.copy_(base)
        X.is_factor = args.sweep == "projected_inverse"
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        getattr(cbase, args.sweep)(X, precision=args.precision)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    out = {"sweep": args.sweep, "precision": args.precision, "n": s.n, "nsn": s.Nsn,
           "ms": [round(t, 3) for t in times], "median_ms": round(float(np.median(times)), 3)}
    if limit is not None:
        from . import _native as N
        op = N.OP_CHOLESKY if args.sweep == "cholesky" else N.OP_PROJECTED_INVERSE
        out["scratch_limit"] = limit
        out["pool"] = s.plan(base.device.index).pool_info(op)
    print(json.dumps(out))


def _scratch_limit(args, s):
    if args.scratch_limit is None:
        return None
    v = args.scratch_limit
    if v.endswith("stack"):   # "stack", "2stack", ...: multiples of the reference's stack size
        limit = int(float(v[:-5] or 1) * int(s.memory["stack_mem"]) * 8)
    else:
        limit = int(v)
    s.plan(torch.cuda.current_device()).set_option("scratch_limit", limit)
    return limit


def run_trsm(args, s, base):
    L = cspmatrix(s, blkval=base.clone())
    cbase.cholesky(L, precision=args.precision)
    B0 = torch.randn(args.nrhs, s.n, dtype=torch.float64, device=base.device,
                     generator=torch.Generator(base.device).manual_seed(5)).t()   # column-major n x nrhs
    Bt = B0.clone().t().contiguous().t()
    times = []
    for _ in range(args.reps):
        Bt.copy_(B0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        cbase.trsm(L, Bt, trans=args.trans)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    print(json.dumps({"sweep": "trsm", "trans": args.trans, "nrhs": args.nrhs, "n": s.n, "nsn": s.Nsn,
                      "ms": [round(t, 3) for t in times], "median_ms": round(float(np.median(times)), 3)}))


def run_batch(args):
    from .batch import batch
    specs = grids.uneven_batch_specs()[:args.batch]
    As = [grids.grid2d_extra(sd, seed=seed) for sd, seed in specs]
    B = batch([symbolic(A, p=amd.order(A)) for A in As])
    x0 = B.assemble(As)
    base = x0
    if args.sweep == "projected_inverse":
        base = x0.clone()
        B.cholesky(base)
    x = base.clone()
    times = []
    for _ in range(args.reps):
        x.copy_(base)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        getattr(B, args.sweep)(x)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    print(json.dumps({"sweep": args.sweep, "batch": args.batch, "values": B.size,
                      "ms": [round(t, 3) for t in times], "median_ms": round(float(np.median(times)), 3)}))


if __name__ == "__main__":
    main()
