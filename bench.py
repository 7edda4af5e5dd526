#!/usr/bin/env python
"""Benchmark of the FP64 chordal Cholesky + adjoint sweeps on B200.

Workload: the FP64 drop-in configuration — 3-D 7-point grid 40x40x40
(n = 64,000), seeded values (off-diagonals N(0,1), diagonal = row |sum| + 1),
AMD ordering, merge_size_fill(32, 32).  One step = refresh the values, then
`cholesky` (factor) followed by `projected_inverse` (the adjoint sweep:
Y = P(X^{-1}) = gradient of log det X), each a single persistent-kernel
launch.  The inputs (246 MB of block values) exceed the 126 MB L2, so no
explicit flush is done between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Metric: algorithmic GFLOP/s of the two sweeps (flop formulas summed over
supernodes from the symbolic arrays).  `--impl reference` times the
reference's own C kernels (compiled from its sources against OpenBLAS,
oracle/_ref) on the host cores, same workload.  With N > 1 (torchrun) every
rank factors its own replica of the matrix (the path has no cross-GPU
exchange for independent matrices): value = total flops / max rank time.
"""
import argparse
import json
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.environ.get("CHB_OUT_DIR", "gpurun_out")  # the folder whose files are kept after a run
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "chordal Cholesky+adjoint ms & GFLOP/s, mixed vs FP64 on B200 at stated error"
WORKLOAD = "FP64 drop-in: 3-D 7-point grid 40^3 (n=64000), AMD, merge_size_fill(32,32); cholesky + projected_inverse"


def sweep_flops(symb):
    """Algorithmic flops per supernode (the reference's BLAS sequence)."""
    nn = np.diff(symb.snptr).astype(np.float64)
    na = np.diff(symb.relptr).astype(np.float64)
    nj = nn + na
    chol = nn ** 3 / 3 + 2 * nn ** 2 * na + nn * na ** 2
    pinv = nn ** 3 / 3 + nn ** 3 + 2 * na ** 2 * nn + 2 * nn ** 2 * na
    llt = na * nn ** 2 + nn * nj ** 2
    comp = na ** 3 / 3 + 2 * na ** 2 * nn + nn ** 2 * na + 2 * nn ** 3 / 3
    hess = 4 * na ** 2 * nn + 2 * na * nn ** 2 + nj * nn ** 2 + nn ** 3 + na ** 2 * nn   # one G application
    trsm = 2 * (nn ** 2 + 2 * na * nn)                                                   # per right-hand side
    return {"cholesky": float(chol.sum()), "projected_inverse": float(pinv.sum()), "llt": float(llt.sum()),
            "completion": float(comp.sum()), "hessian_G": float(hess.sum()), "trsm_rhs": float(trsm.sum()),
            "potrf_updates": float((na ** 3 / 3).sum())}


def build_problem(side=40, merge=(32, 32), seed=0):
    import chompack_b200 as cp
    from chompack_b200 import grids
    A = grids.grid3d(side, seed=seed)
    s = cp.symbolic(A, p=cp.amd.order(A), merge_function=cp.merge_size_fill(*merge))
    return A, s


class ClockSampler(object):
    """SM clock and clock-event-reason sampling during the timed region, by
    NVML polling from a thread (every 2 ms; read-only queries).  The samples
    are also written as CSV beside the run's other outputs (OUT_DIR)."""

    # NVML clocks-event-reason bits
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, dev):
        self.dev = dev
        self.thread = None
        self.samples = []
        self.path = os.path.join(ROOT, OUT_DIR, "clocks_bench_%d.csv" % os.getpid())

    def _handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        uuid = getattr(torch.cuda.get_device_properties(self.dev), "uuid", None)
        if uuid is not None:
            u = str(uuid)
            try:
                return pynvml.nvmlDeviceGetHandleByUUID(u if u.startswith("GPU-") else "GPU-" + u)
            except Exception:
                pass
        return pynvml.nvmlDeviceGetHandleByIndex(self.dev.index or 0)

    def start(self):
        import threading
        try:
            import pynvml
            self.nv = pynvml
            self.h = self._handle()
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
        except Exception:
            self.h = None
            return
        self.stop_flag = threading.Event()

        def run():
            nv = self.nv
            while not self.stop_flag.is_set():
                try:
                    sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                    rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                    pw = nv.nvmlDeviceGetPowerUsage(self.h) / 1000.0
                    self.samples.append((time.time(), float(sm), int(rs), pw))
                except Exception:
                    pass
                time.sleep(0.002)
        self.thread = threading.Thread(target=run, daemon=True)
        self.thread.start()

    def stop(self):
        if self.thread is None:
            return None
        self.stop_flag.set()
        self.thread.join(timeout=5)
        if not self.samples:
            return None
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            with open(self.path, "w") as f:
                f.write("time,sm_mhz,reasons_mask,power_w\n")
                for t, sm, rs, pw in self.samples:
                    f.write("%.4f,%.0f,0x%x,%.1f\n" % (t, sm, rs, pw))
        except OSError:
            pass
        reasons = set()
        for _, _, rs, _ in self.samples:
            for bit, nm in self.REASONS.items():
                if rs & bit:
                    reasons.add(nm)
        sm = [x[1] for x in self.samples]
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": self.max_mhz, "reasons": sorted(reasons),
                "samples": len(sm), "power_w_max": round(max(x[3] for x in self.samples), 1)}


def profiled_traffic(name="engine_kernel_grid3d40.md"):
    """DRAM bytes (read + write) per launch from the committed ncu summary."""
    try:
        for line in open(os.path.join(ROOT, "profiles", name)):
            if line.startswith("traffic_bytes_per_launch:"):
                return {k: int(v) for k, v in (kv.split("=") for kv in line.split(":", 1)[1].split())}
    except OSError:
        pass
    return {}


def fp64_peak_tflops(dev):
    """Measured FP64 GEMM throughput (cuBLAS DGEMM via torch.matmul)."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize(dev)
    best = 1e9
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    return 2.0 * n ** 3 / best / 1e12


def run_reference(args, rank, world):
    """The reference's own C kernels on the host cores."""
    if rank != 0:
        return 0
    from oracle import ref
    import chompack_b200 as cp
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "reference kernels not built (oracle/_ref)"}))
        return 0
    cores = os.cpu_count() or 1
    ref.set_threads(cores)
    A, s = build_problem()
    fl = sweep_flops(s)
    step_flops = fl["cholesky"] + fl["projected_inverse"]
    X = cp.cspmatrix(s, device="cpu") + A
    x0 = X.blkval.numpy().copy()

    def step():
        x = x0.copy()
        assert ref.cholesky(s, x) == 0
        assert ref.projected_inverse(s, x) == 0
        return x

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = time.perf_counter() - t0
    ms = dt / args.steps * 1e3
    val = step_flops * args.steps / dt / 1e9
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(val, 3), "unit": "GFLOP/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD + " [reference C kernels + OpenBLAS on host]", "n": s.n, "nsn": s.Nsn},
        "cpu_baseline": {"value": round(val, 3), "unit": "GFLOP/s", "cores": cores, "kind": "reference",
                         "sample": "full workload per step (cholesky + projected_inverse), %d steps" % args.steps},
        "e2e": {"value": round(val, 3), "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))
    return 0


def cpu_baseline(s, A, budget_s=15.0):
    from oracle import ref
    import chompack_b200 as cp
    cores = os.cpu_count() or 1
    ref.set_threads(cores)
    fl = sweep_flops(s)
    step_flops = fl["cholesky"] + fl["projected_inverse"]
    X = cp.cspmatrix(s, device="cpu") + A
    x0 = X.blkval.numpy().copy()
    times = []
    t_start = time.perf_counter()
    while len(times) < 5 and (time.perf_counter() - t_start) < budget_s:
        x = x0.copy()
        t0 = time.perf_counter()
        ref.cholesky(s, x)
        ref.projected_inverse(s, x)
        times.append(time.perf_counter() - t0)
    med = float(np.median(times))
    out = {"value": round(step_flops / med / 1e9, 3), "unit": "GFLOP/s", "cores": cores, "kind": "reference",
           "sample": "%d full runs of cholesky+projected_inverse (median %.1f ms)" % (len(times), med * 1e3)}
    # the other drop-in sweeps once each, for the same comparison
    L = x0.copy()
    ref.cholesky(s, L)
    Y = L.copy()
    ref.projected_inverse(s, Y)
    other = {}

    def once(name, fn, flops):
        t0 = time.perf_counter()
        fn()
        dt = time.perf_counter() - t0
        other[name] = {"ms": round(dt * 1e3, 2), "gflops": round(flops / dt / 1e9, 3)}
    once("completion", lambda: ref.completion(s, Y.copy(), factored_updates=True), fl["completion"])
    once("completion_unfactored", lambda: ref.completion(s, Y.copy(), factored_updates=False), fl["completion"])
    once("llt", lambda: ref.llt(s, L.copy()), fl["llt"])
    B = np.asfortranarray(np.random.default_rng(5).standard_normal((s.n, 8)))
    once("trsm_N_nrhs8", lambda: ref.trsm(s, L, B.copy(order="F"), trans="N"), fl["trsm_rhs"] * 8)
    U = Y * np.random.default_rng(6).standard_normal(Y.size)
    for fu in (1, 0):
        once("hessian_full_fu%d" % fu, lambda: ref.hessian(s, L, Y, [U.copy()], adj=None, factored_updates=bool(fu)),
             2 * fl["hessian_G"] + (0 if fu else 2 * fl["potrf_updates"]))
    out["other_sweeps"] = other
    return out


def mixed_precision_section(dev, side=48, merge=(64, 64), nrhs=8, reps=5):
    """Mixed-precision form (GEMM tiles on TF32 tensor cores, FP64 diagonal
    tiles): log det forward + backward (cholesky + projected_inverse) on the
    3-D 7-point grid side^3 with merge_size_fill(merge), timed in FP64,
    TF32 and 3xTF32, with the errors of log det, its gradient and the factor
    against the FP64 path, and an nrhs solve refined with FP64 residuals to
    a normwise relative residual of 1e-12."""
    import torch
    import chompack_b200 as cp
    from chompack_b200 import mixed
    A, s = build_problem(side=side, merge=merge)
    fl = sweep_flops(s)
    flops = fl["cholesky"] + fl["projected_inverse"]
    X0 = cp.cspmatrix(s, device=dev) + A
    out = {"workload": "3-D 7-point grid %d^3 (n=%d), AMD, merge_size_fill(%d,%d); log det forward + backward "
                       "(cholesky + projected_inverse)" % (side, s.n, merge[0], merge[1]),
           "flops": flops}
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for prec in ("fp64", "tf32", "tf32x3"):
        X = cp.cspmatrix(s, blkval=X0.blkval.clone())
        times = []
        for it in range(reps + 2):
            X.blkval.copy_(X0.blkval)
            X.is_factor = False
            torch.cuda.synchronize(dev)
            ev0.record()
            cp.cholesky(X, precision=prec)
            cp.projected_inverse(X, precision=prec)
            ev1.record()
            torch.cuda.synchronize(dev)
            if it >= 2:
                times.append(ev0.elapsed_time(ev1))
        ms = float(np.median(times))
        entry = {"ms": round(ms, 3), "gflops": round(flops / ms / 1e6, 1)}
        if prec != "fp64":
            ld, Y, rep = mixed.logdet_and_gradient(X0, precision=prec)
            entry.update({k: rep[k] for k in ("logdet_rel_error", "gradient_rel_error", "factor_rel_error")})
            L = cp.cspmatrix(s, blkval=X0.blkval.clone())
            cp.cholesky(L, precision=prec)
            B = torch.from_numpy(np.asfortranarray(np.random.default_rng(11).standard_normal((s.n, nrhs)))).to(dev)
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            x, srep = mixed.solve(X0, L, B, tol=1e-12, maxiter=40)
            torch.cuda.synchronize(dev)
            entry["solve"] = {"nrhs": nrhs, "iterations": srep["iterations"],
                              "residual": srep["residuals"][-1], "ms": round((time.perf_counter() - t0) * 1e3, 2)}
        out[prec] = entry
    out["speedup_tf32"] = round(out["fp64"]["ms"] / out["tf32"]["ms"], 3)
    out["speedup_tf32x3"] = round(out["fp64"]["ms"] / out["tf32x3"]["ms"], 3)
    return out


def _event_ms(dev, fn, reps):
    """Median CUDA-event time of fn() over reps runs after two warm-ups."""
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    times = []
    for it in range(reps + 2):
        torch.cuda.synchronize(dev)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize(dev)
        if it >= 2:
            times.append(e0.elapsed_time(e1))
    return float(np.median(times))


def batch_section(dev, count=256, value_sets=64, reps=5):
    """Batched FP64 factorisation: `count` independent 2-D 5-point grids
    (side uniform in 20..120, each node with 2 extra random neighbours
    within grid distance 5, AMD ordering), and `value_sets` value sets on
    one 64x64 grid pattern.  Each batch is one merged plan: cholesky and
    projected_inverse of all its matrices take one launch each."""
    import chompack_b200 as cp
    from chompack_b200 import grids
    out = {}
    rng = np.random.default_rng(2024)
    sides = rng.integers(20, 121, size=count)
    As, symbs = [], []
    for i, sd in enumerate(sides):
        A = grids.grid2d_extra(int(sd), seed=1000 + i)
        As.append(A)
        symbs.append(cp.symbolic(A, p=cp.amd.order(A)))
    for name, Bs, Xs in (("uneven_grids", symbs, As), ("value_sets_64x64", None, None)):
        if Bs is None:
            A0 = grids.grid2d(64, seed=7)
            s0 = cp.symbolic(A0, p=cp.amd.order(A0))
            Bs = [s0] * value_sets
            Xs = [grids.grid2d(64, seed=7 + v) for v in range(value_sets)]
        B = cp.batch(Bs, device=dev.index)
        x0 = B.assemble(Xs)
        x = x0.clone()

        def step():
            x.copy_(x0)
            B.cholesky(x)
            B.projected_inverse(x)
        ms = _event_ms(dev, step, reps)
        flops = sum(sweep_flops(sb)["cholesky"] + sweep_flops(sb)["projected_inverse"] for sb in Bs)
        out[name] = {"matrices": len(Bs), "n_total": int(sum(sb.n for sb in Bs)), "values": int(B.size),
                     "launches_per_step": 2, "ms": round(ms, 3), "gflops": round(flops / ms / 1e6, 1),
                     "matrices_per_s": round(len(Bs) / ms * 1e3, 1), "step": "cholesky + projected_inverse (copy of "
                     "the values included)"}
    return out


def autograd_section(dev, side=32, value_sets=16, reps=5, h=1e-6):
    """Differentiation: log det and its gradient (the projected inverse) for
    `value_sets` value sets on the 3-D 7-point grid side^3 in one batch
    (forward + backward = two launches), a central finite-difference check
    of the gradient and of the second derivative (hessian) along a random
    symmetric direction on the pattern, for the first value set."""
    import torch
    import chompack_b200 as cp
    from chompack_b200 import grids, autograd
    A0 = grids.grid3d(side, seed=0)
    s = cp.symbolic(A0, p=cp.amd.order(A0), merge_function=cp.merge_size_fill(32, 32))
    B = cp.batch([s] * value_sets, device=dev.index)
    x0 = B.assemble([grids.grid3d(side, seed=v) for v in range(value_sets)])
    x = x0.clone()
    res = {}

    def fwd_bwd():
        x.copy_(x0)
        B.cholesky(x)
        res["ld"] = B.logdet(x)
        B.projected_inverse(x)
    ms = _event_ms(dev, fwd_bwd, reps)
    fl = sweep_flops(s)
    flops = value_sets * (fl["cholesky"] + fl["projected_inverse"])
    # checks on value set 0
    X = cp.cspmatrix(s, blkval=x0[:int(s.blkptr[-1])].clone())
    rng = np.random.default_rng(5)
    U = cp.cspmatrix(s, blkval=torch.from_numpy(rng.standard_normal(int(s.blkptr[-1]))).to(dev))

    def ld_at(t):
        return float(autograd.logdet_values(X.blkval + t * U.blkval, s))
    Y = autograd.logdet_gradient(X)
    g = cp.dot(Y, U)
    fd = (ld_at(h) - ld_at(-h)) / (2 * h)
    L = cp.cspmatrix(s, blkval=X.blkval.clone())
    cp.cholesky(L)
    HU = autograd.logdet_hvp(L, Y, U)
    second = cp.dot(U, HU)

    def g_at(t):
        Xt = cp.cspmatrix(s, blkval=X.blkval + t * U.blkval)
        return cp.dot(autograd.logdet_gradient(Xt), U)
    fd2 = (g_at(1e-4) - g_at(-1e-4)) / 2e-4
    return {"workload": "3-D 7-point grid %d^3 (n=%d), AMD, merge_size_fill(32,32), %d value sets in one batch"
                        % (side, s.n, value_sets),
            "fwd_bwd_ms": round(ms, 3), "gflops": round(flops / ms / 1e6, 1), "launches": 2,
            "gradient_fd_rel_error": abs(g - fd) / max(abs(fd), 1e-300),
            "hvp_fd_rel_error": abs(second - fd2) / max(abs(fd2), 1e-300),
            "fd_steps": [h, 1e-4]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-other", action="store_true", help="skip the timings of the other sweeps")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision section (48^3)")
    ap.add_argument("--no-batch", action="store_true", help="skip the batch and autograd sections")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", device_id=dev, timeout=datetime.timedelta(seconds=120))

    import chompack_b200 as cp
    from chompack_b200 import _native as N

    A, s = build_problem()
    fl = sweep_flops(s)
    ops = ["cholesky", "projected_inverse"]
    step_flops = sum(fl[o] for o in ops)
    X0 = cp.cspmatrix(s, device=dev) + A
    Xw = X0.blkval.clone()
    plan = s.plan(local)
    # one workspace sized for the larger of the two sweeps, shared by both
    nbytes = max(plan.workspace_bytes(N.OP_CHOLESKY), plan.workspace_bytes(N.OP_PROJECTED_INVERSE))
    wbuf = torch.empty(nbytes + 256, dtype=torch.uint8, device=dev)
    ws = (wbuf.data_ptr() + 255) // 256 * 256
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    ev_k = {"cholesky": [], "projected_inverse": []}
    launch = {"cholesky": N.cholesky, "projected_inverse": N.projected_inverse}

    def step(timed=False):
        Xw.copy_(X0.blkval)
        for op in ops:
            if timed:
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            rc = launch[op](plan.handle, Xw.data_ptr(), ws, nbytes, sp)
            if rc < 0:
                raise RuntimeError(N.last_error().decode())
            if timed:
                e1.record(stream)
                ev_k[op].append((e0, e1))

    for _ in range(args.warmup):
        step()
    info = N.info(plan.handle, ws, sp)
    if info != 0:
        raise RuntimeError("sweep status %d (%s)" % (info, N.last_error().decode()))

    sampler = ClockSampler(dev)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    sampler.start()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(args.steps):
        step(timed=True)
    t1.record(stream)
    torch.cuda.synchronize(dev)
    clocks = sampler.stop()
    if world > 1:
        dist.barrier()
    elapsed = t0.elapsed_time(t1) / 1e3
    kern = {op: float(np.mean([a.elapsed_time(b) for a, b in ev_k[op]])) / 1e3 for op in ops}
    # the job ends with the slowest rank (chompack_b200.shard, NCCL here)
    from chompack_b200 import shard
    elapsed = shard.max_over_ranks(elapsed, device=dev)
    kern = {o: shard.max_over_ranks(kern[o], device=dev) for o in ops}
    value = step_flops * args.steps * world / elapsed / 1e9

    # the other drop-in sweeps of the workload, timed alone after the step
    # loop (not part of the step): completion of the projected inverse the
    # step produced (both update modes) and llt of the factor
    other = {}
    sweeps_other = not args.no_other
    Yw = Xw.clone()
    Lw = X0.blkval.clone()
    launch["cholesky"](plan.handle, Lw.data_ptr(), ws, nbytes, sp)
    Cw = torch.empty_like(Yw)
    reps = max(3, min(args.steps, 10))
    for name, op, k, src, call in () if not sweeps_other else (
            ("completion", N.OP_COMPLETION, 1, Yw, lambda w, nb: N.completion(plan.handle, Cw.data_ptr(), 1, w, nb, sp)),
            ("completion_unfactored", N.OP_COMPLETION, 0, Yw,
             lambda w, nb: N.completion(plan.handle, Cw.data_ptr(), 0, w, nb, sp)),
            ("llt", N.OP_LLT, 0, Lw, lambda w, nb: N.llt(plan.handle, Cw.data_ptr(), w, nb, sp))):
        w2, nb2 = plan.workspace(op, k)
        ts = []
        for it in range(reps + 1):
            Cw.copy_(src)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            if call(w2, nb2) < 0:
                raise RuntimeError(N.last_error().decode())
            e1.record(stream)
            ts.append((e0, e1))
        torch.cuda.synchronize(dev)
        if N.info(plan.handle, w2, sp) != 0:
            raise RuntimeError("%s status %s" % (name, N.last_error().decode()))
        ms = float(np.median([a.elapsed_time(b) for a, b in ts[1:]]))
        fkey = "completion" if name.startswith("completion") else name
        other[name] = {"ms": round(ms, 4), "gflops": round(fl[fkey] / ms / 1e6, 3)}

    # triangular solves with 8 right-hand sides, and the full Hessian H(U)
    # (adj=None: two passes) on one direction U, both update forms
    def timed(fn, reps):
        ts = []
        for it in range(reps + 1):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            ts.append((e0, e1))
        torch.cuda.synchronize(dev)
        return float(np.median([a.elapsed_time(b) for a, b in ts[1:]]))
    nrhs = 8 if sweeps_other else 0
    Bd = torch.randn(s.n, nrhs, dtype=torch.float64, device=dev, generator=torch.Generator(dev).manual_seed(5))
    for tr in ("NT" if sweeps_other else ""):
        wt, nbt = plan.workspace(N.OP_TRSM, nrhs, 1 if tr == "T" else 0)
        Bt = Bd.t().contiguous()   # column-major n x nrhs
        ms = timed(lambda: N.trsm(plan.handle, tr.encode(), nrhs, 1.0, Lw.data_ptr(), Bt.data_ptr(), s.n, wt, nbt, sp),
                   reps)
        other["trsm_%s_nrhs%d" % (tr, nrhs)] = {"ms": round(ms, 4), "gflops": round(fl["trsm_rhs"] * nrhs / ms / 1e6, 3)}
    import ctypes
    Ud = Yw * torch.randn(Yw.shape, dtype=torch.float64, device=dev, generator=torch.Generator(dev).manual_seed(6))
    Uw = torch.empty_like(Ud)
    uarr = (ctypes.c_void_p * 1)(Uw.data_ptr())
    for fu in ((1, 0) if sweeps_other else ()):
        for a in (0, 1):
            plan.workspace(N.OP_HESSIAN, 1, a | fu << 2)
        def full_hessian():
            Uw.copy_(Ud)
            for a in (0, 1):   # adj = inv = False first, then adj toggled (the reference's adj=None)
                wh, nbh = plan.workspace(N.OP_HESSIAN, 1, a | fu << 2)
                if N.hessian(plan.handle, Lw.data_ptr(), Yw.data_ptr(), uarr, 1, a, 0, fu, wh, nbh, sp) < 0:
                    raise RuntimeError(N.last_error().decode())
        ms = timed(full_hessian, max(2, reps // 2))
        hf = 2 * fl["hessian_G"] + (0 if fu else 2 * fl["potrf_updates"])
        other["hessian_full_fu%d" % fu] = {"ms": round(ms, 4), "gflops": round(hf / ms / 1e6, 3)}

    # end-to-end through the public API with host values, the reference's
    # calling pattern: each step factors a fresh cspmatrix whose values are
    # in pinned host memory; cholesky streams them in and L back out while it
    # runs, projected_inverse streams Y back out (its input, L, is already
    # on the device).  Host bytes per step: the values in, L and Y out.
    e2e = None
    if not args.no_e2e:
        host_in = X0.blkval.cpu()
        bufs = [host_in.clone().pin_memory() for _ in range(2 + args.steps)]
        for it in range(2 + args.steps):
            if it == 2:
                torch.cuda.synchronize(dev)
                w0 = time.perf_counter()
            X = cp.cspmatrix(s, blkval=bufs[it])
            cp.cholesky(X)
            cp.projected_inverse(X)
            del X   # its device copy goes back to torch's cache for the next step
        torch.cuda.synchronize(dev)
        w = (time.perf_counter() - w0) / args.steps
        nbytes = host_in.numel() * 8
        e2e = {"value": round(step_flops / w / 1e9, 3), "unit": "GFLOP/s", "h2d_bytes_per_step": nbytes,
               "d2h_bytes_per_step": 2 * nbytes, "ms_per_step": round(w * 1e3, 3),
               "path": "cbase.cholesky + cbase.projected_inverse on host-resident values (streamed chunks)"}

    if rank == 0:
        peak = fp64_peak_tflops(dev)
        na = np.diff(np.asarray(s.relptr)).astype(np.float64)
        alg_bytes = int(16 * int(s.blkptr[-1]) + np.sum(16 * na * (na + 1) / 2))
        achieved = fl["cholesky"] / kern["cholesky"] / 1e12
        out = {
            "metric": METRIC, "value": round(value, 3), "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(elapsed / args.steps * 1e3, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "n": s.n, "nsn": s.Nsn, "sweeps": ops,
                       "flops_per_step": step_flops, "l2": "inputs 246 MB > 126 MB L2; no flush",
                       "parallelism": "replicas x%d" % world},
            "gpu_launches": args.steps * len(ops),
            "roofline": {"bound": "tensor", "achieved": round(achieved, 3), "peak": round(peak, 3),
                         "unit": "TFLOP/s", "frac": round(achieved / peak, 4),
                         "traffic": profiled_traffic().get("cholesky"),
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, one capture "
                                           "(profiles/engine_kernel_grid3d40.md)",
                         "algorithmic_bytes": alg_bytes,
                         "kernel": "chb::engine_kernel (cholesky)",
                         "peak_source": "measured cuBLAS DGEMM 8192^3 on this GPU (FP64; MEASURED_PEAKS.json "
                                        "lists bf16 and HBM only)"},
            "kernel_ms": {o: round(kern[o] * 1e3, 4) for o in ops},
            "other_sweeps": other,
        }
        if clocks:
            out["clocks"] = clocks
        if e2e:
            out["e2e"] = e2e
        if not args.no_mixed and not args.no_other:
            try:
                out["mixed_precision"] = mixed_precision_section(dev)
            except Exception as exc:  # reported beside the headline, never required
                out["mixed_precision"] = {"unavailable": str(exc)}
        if not args.no_batch and not args.no_other:
            for key, fn in (("batch", batch_section), ("autograd", autograd_section)):
                try:
                    out[key] = fn(dev)
                except Exception as exc:  # reported beside the headline, never required
                    out[key] = {"unavailable": str(exc)}
        if not args.no_cpu:
            try:
                out["cpu_baseline"] = cpu_baseline(s, A)
            except Exception as exc:  # the baseline is reported, never required
                out["cpu_baseline"] = {"unavailable": str(exc)}
        print(json.dumps(out))
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
