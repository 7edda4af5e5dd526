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
oracle/_ref) on the host cores, same workload; that process loads no library
of this package (its inputs come from oracle/workload.py and the committed
symbolic fixture).  With N > 1 every rank factors its own replica of the
matrix (the path has no cross-GPU exchange for independent matrices):
value = total flops / max rank time; `--gpus N` without a launcher starts
the N ranks itself.  The batch section shards its 256 matrices over the
ranks.  Every result is compared with the reference's output on the same
inputs (`parity`, outside the timed region).
"""
import argparse
import json
import os
import socket
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.environ.get("CHB_OUT_DIR")  # where the clock samples are written as CSV (unset: not written)
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "chordal Cholesky+adjoint ms & GFLOP/s, mixed vs FP64 on B200 at stated error"
WORKLOAD = "FP64 drop-in: 3-D 7-point grid 40^3 (n=64000), AMD, merge_size_fill(32,32); cholesky + projected_inverse"
RTOL = 1e-12
HBM_FALLBACK_GBS = 6650.0


def sweep_flops(symb):
    """Algorithmic flops per supernode (the reference's BLAS sequence)."""
    nn = np.diff(np.asarray(symb.snptr)).astype(np.float64)
    na = np.diff(np.asarray(symb.relptr)).astype(np.float64)
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


def sweep_bytes(symb):
    """Algorithmic HBM bytes of one sweep: the block values read and written
    once, and each update triangle written and read once."""
    na = np.diff(np.asarray(symb.relptr)).astype(np.float64)
    return int(16 * int(symb.blkptr[-1]) + np.sum(16 * na * (na + 1) / 2))


def bench_config(symb):
    """The workload description both arms print (identical dicts)."""
    fl = sweep_flops(symb)
    return {"workload": WORKLOAD, "n": int(symb.n), "nsn": int(symb.Nsn), "sweeps": ["cholesky", "projected_inverse"],
            "flops_per_step": fl["cholesky"] + fl["projected_inverse"],
            "l2": "inputs 246 MB > 126 MB L2; no flush",
            "parallelism": "replicas: one matrix per rank, no data-path collective"}


def build_problem(side=40, merge=(32, 32), seed=0):
    import chompack_b200 as cp
    from chompack_b200 import grids
    A = grids.grid3d(side, seed=seed)
    s = cp.symbolic(A, p=cp.amd.order(A), merge_function=cp.merge_size_fill(*merge))
    return A, s


def hbm_peak_gbs():
    """Measured copy bandwidth of this pool's B200s when the driver wrote it,
    else the fallback figure."""
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        for k in ("hbm_gbs", "hbm_GBs", "hbm"):
            if k in d:
                v = d[k]
                return float(v["value"] if isinstance(v, dict) else v), "measured (MEASURED_PEAKS.json)"
    except (OSError, ValueError, KeyError, TypeError):
        pass
    return HBM_FALLBACK_GBS, "fallback 6.65 TB/s (no MEASURED_PEAKS.json)"


class ClockSampler(object):
    """SM clock and clock-event-reason sampling during the timed region, by
    NVML polling from a thread (every 2 ms; read-only queries).  With
    CHB_OUT_DIR set the samples are also written there as CSV."""

    # NVML clocks-event-reason bits
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, dev):
        self.dev = dev
        self.thread = None
        self.samples = []
        self.path = os.path.join(OUT_DIR, "clocks_bench_%d.csv" % os.getpid()) if OUT_DIR else None

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
        if self.path:
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


# ------------------------------------------------------------ reference arm

def run_reference(args, rank, world):
    """The reference's own C kernels on the host cores (rank 0 only).  The
    inputs come from oracle/workload.py: no library of this package is
    loaded by this process."""
    if rank != 0:
        return 0
    from oracle import ref, workload
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "reference kernels not built (oracle/_ref)"}))
        return 0
    cores = os.cpu_count() or 1
    ref.set_threads(cores)
    s = workload.load_symbolic("grid3d_40_m32")
    n, I, J, V = workload.grid3d_lower(40, seed=0)
    x0 = workload.assemble(s, n, I, J, V)
    cfg = bench_config(s)
    step_flops = cfg["flops_per_step"]

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
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
        "cpu_baseline": {"value": round(val, 3), "unit": "GFLOP/s", "cores": cores, "kind": "reference",
                         "sample": "full workload per step (cholesky + projected_inverse), %d steps; reference C "
                                   "kernels + OpenBLAS threads on the host" % args.steps},
        "e2e": {"value": round(val, 3), "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))
    return 0


# --------------------------------------------------- reference outputs, CPU

def reference_outputs(s, x0):
    """Reference factor and projected inverse of the workload (all cores)."""
    from oracle import ref
    ref.set_threads(os.cpu_count() or 1)
    L = x0.copy()
    assert ref.cholesky(s, L) == 0
    Y = L.copy()
    assert ref.projected_inverse(s, Y) == 0
    return L, Y


def cpu_baseline(s, x0, budget_s=15.0):
    """The reference's kernels on the host: cholesky + projected_inverse with
    all cores (median of up to 5 runs within the budget) and with 1 thread
    (one run), and the other drop-in sweeps once each with all cores."""
    from oracle import ref
    cores = os.cpu_count() or 1
    ref.set_threads(cores)
    fl = sweep_flops(s)
    step_flops = fl["cholesky"] + fl["projected_inverse"]
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
           "sample": "%d full runs of cholesky+projected_inverse (median %.1f ms), OpenBLAS on %d threads"
                     % (len(times), med * 1e3, cores)}
    ref.set_threads(1)
    x = x0.copy()
    t0 = time.perf_counter()
    ref.cholesky(s, x)
    ref.projected_inverse(s, x)
    t1 = time.perf_counter() - t0
    out["one_thread"] = {"value": round(step_flops / t1 / 1e9, 3), "unit": "GFLOP/s", "cores": 1,
                         "ms": round(t1 * 1e3, 1), "sample": "1 full run of cholesky+projected_inverse"}
    ref.set_threads(cores)
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


def _logdet_of_factor(s, L):
    ld = 0.0
    for k in range(int(s.Nsn)):
        nn = int(s.snptr[k + 1] - s.snptr[k])
        nj = int(s.sncolptr[k + 1] - s.sncolptr[k])
        blk = L[int(s.blkptr[k]):int(s.blkptr[k + 1])].reshape((nj, nn), order="F")
        ld += 2.0 * float(np.sum(np.log(np.diag(blk[:nn]))))
    return ld


# ----------------------------------------------------------- side sections

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


def mixed_precision_section(dev, side=48, merge=(64, 64), nrhs=8, reps=5, grid2d=None):
    """Mixed-precision form (GEMM tiles on TF32 tensor cores, FP64 diagonal
    tiles): log det forward + backward (cholesky + projected_inverse) on the
    3-D 7-point grid side^3 with merge_size_fill(merge), timed in FP64,
    TF32 and 3xTF32.  Errors of log det, its gradient (the projected inverse)
    and the factor are stated against the reference's FP64 kernels run on
    the same inputs; the FP64 GPU path's parity there is reported too.  An
    nrhs solve is refined with FP64 residuals to a normwise relative
    residual of 1e-12 (timed after a warm-up solve)."""
    import torch
    import chompack_b200 as cp
    from chompack_b200 import mixed
    from oracle import workload
    if grid2d:
        from chompack_b200 import grids
        A = grids.grid2d(grid2d, seed=0)
        s = cp.symbolic(A, p=cp.amd.order(A), merge_function=cp.merge_size_fill(*merge))
        what = "2-D 5-point grid %d^2 (n=%d)" % (grid2d, s.n)
    else:
        A, s = build_problem(side=side, merge=merge)
        what = "3-D 7-point grid %d^3 (n=%d)" % (side, s.n)
    fl = sweep_flops(s)
    flops = fl["cholesky"] + fl["projected_inverse"]
    X0 = cp.cspmatrix(s, device=dev) + A
    x0 = X0.blkval.cpu().numpy()
    Lr, Yr = reference_outputs(s, x0)
    ld_ref = _logdet_of_factor(s, Lr)
    out = {"workload": "%s, AMD, merge_size_fill(%d,%d); log det forward + backward (cholesky + "
                       "projected_inverse)" % (what, merge[0], merge[1]),
           "flops": flops, "nsn": int(s.Nsn), "values": int(s.blkptr[-1]),
           "errors_against": "reference C kernels (oracle/_ref), FP64, same inputs"}
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for key in ("fp64", "tf32", "tf32x3", "tf32_tcgen05"):
        prec = "tf32" if key == "tf32_tcgen05" else key
        s.plan().set_option("tf32_tcgen05", 1 if key == "tf32_tcgen05" else None)
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
        ld, Ym, _ = mixed.logdet_and_gradient(X0, precision=prec, reference=False)
        Lm = cp.cspmatrix(s, blkval=X0.blkval.clone())
        cp.cholesky(Lm, precision=prec)
        Lh = Lm.blkval.cpu().numpy()
        Yh = Ym.blkval.cpu().numpy()
        entry["logdet_rel_error"] = abs(ld - ld_ref) / abs(ld_ref)
        entry["gradient_rel_error"] = float(np.abs(Yh - Yr).max() / np.abs(Yr).max())
        entry["factor_rel_error"] = float(np.abs(Lh - Lr).max() / np.abs(Lr).max())
        if prec == "fp64":
            entry["parity_scaled_error"] = max(workload.block_errors(s, Lh, Lr), workload.block_errors(s, Yh, Yr))
        elif key == "tf32_tcgen05":
            entry["tiles"] = "tcgen05.mma kind::tf32, accumulators in tensor memory"
        else:
            B = torch.from_numpy(np.asfortranarray(np.random.default_rng(11).standard_normal((s.n, nrhs)))).to(dev)
            mixed.solve(X0, Lm, B, tol=1e-12, maxiter=40)     # warm-up: builds the solve programs
            torch.cuda.synchronize(dev)
            ev0.record()
            x, srep = mixed.solve(X0, Lm, B, tol=1e-12, maxiter=40)
            ev1.record()
            torch.cuda.synchronize(dev)
            sms = ev0.elapsed_time(ev1)
            entry["solve"] = {"nrhs": nrhs, "iterations": srep["iterations"], "residual": srep["residuals"][-1],
                              "ms": round(sms, 3), "ms_per_iteration": round(sms / srep["iterations"], 3)}
        out[key] = entry
    s.plan().set_option("tf32_tcgen05", None)
    out["speedup_tf32"] = round(out["fp64"]["ms"] / out["tf32"]["ms"], 3)
    out["speedup_tf32_tcgen05"] = round(out["fp64"]["ms"] / out["tf32_tcgen05"]["ms"], 3)
    out["speedup_tf32x3"] = round(out["fp64"]["ms"] / out["tf32x3"]["ms"], 3)
    return out


def batch_section(dev, rank, world, count=256, value_sets=64, reps=5):
    """Batched FP64 factorisation: `count` independent 2-D 5-point grids
    (side uniform in 20..120, each node with 2 extra random neighbours
    within grid distance 5, AMD ordering), and `value_sets` value sets on
    one 64x64 grid pattern.  Each batch is one merged plan: cholesky and
    projected_inverse of all its matrices take one launch each.  With
    world > 1 the uneven grids are sharded over the ranks by estimated
    flops (chompack_b200.shard): every rank sweeps its share with its own
    merged plan, the time is the max over ranks and the per-matrix log dets
    are gathered.  Rank 0 also times the reference's kernels on the same
    matrices and checks parity on a sample."""
    import torch
    import chompack_b200 as cp
    from chompack_b200 import grids, shard
    out = {}
    specs = grids.uneven_batch_specs(count)
    As, symbs = [], []
    for sd, seed in specs:
        A = grids.grid2d_extra(sd, seed=seed)
        As.append(A)
        symbs.append(cp.symbolic(A, p=cp.amd.order(A)))
    costs = [sweep_flops(sb)["cholesky"] for sb in symbs]
    mine = shard.my_share(costs, rank, world) if world > 1 else list(range(count))
    peak, peak_src = hbm_peak_gbs()
    for name in ("uneven_grids", "value_sets_64x64"):
        if name == "uneven_grids":
            Bs = [symbs[i] for i in mine]
            Xs = [As[i] for i in mine]
        else:
            if world > 1 and rank != 0:
                continue
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
        alg = sum(2 * sweep_bytes(sb) for sb in Bs)
        entry = {"matrices": len(Bs), "n_total": int(sum(sb.n for sb in Bs)), "values": int(B.size),
                 "launches_per_step": 2, "ms": round(ms, 3), "gflops": round(flops / ms / 1e6, 1),
                 "matrices_per_s": round(len(Bs) / ms * 1e3, 1),
                 "algorithmic_bytes": alg, "achieved_gbs": round(alg / ms / 1e6, 1),
                 "hbm_frac": round(alg / ms / 1e6 / peak, 4), "hbm_peak_gbs": peak, "hbm_peak_source": peak_src,
                 "step": "cholesky + projected_inverse (copy of the values included)"}
        if name == "uneven_grids" and world > 1:
            x.copy_(x0)
            B.cholesky(x)
            lds = B.logdet(x).cpu().numpy()
            all_ld = shard.gather_results(mine, lds, count)
            t_max = shard.max_over_ranks(ms, device=dev)
            import torch.distributed as dist
            per_rank = [None] * world
            dist.all_gather_object(per_rank, {"rank": rank, "matrices": len(Bs), "ms": round(ms, 3),
                                              "gflops": round(flops / ms / 1e6, 1)})
            entry = {"matrices": count, "ranks": per_rank, "ms": round(t_max, 3),
                     "matrices_per_s": round(count / t_max * 1e3, 1), "logdets_gathered": sum(
                         v is not None for v in all_ld), "sharding": "chompack_b200.shard.partition by cholesky flops"}
        if rank == 0 and name == "uneven_grids":
            entry.update(_batch_reference(Bs, x0, x, B, dev))
        if world == 1:
            # the task cutting picked by the autotuner for this batch, timed again
            tr = cp.tune(B, x0, reps=2)
            tms = _event_ms(dev, step, reps)
            entry["tuned"] = {"choice": tr["choice"], "ms": round(tms, 3),
                              "achieved_gbs": round(alg / tms / 1e6, 1), "hbm_frac": round(alg / tms / 1e6 / peak, 4),
                              "trials": len(tr["trials"])}
        out[name] = entry
    return out


def _batch_reference(Bs, x0, x, B, dev, sample_every=16):
    """Reference kernels on the host for the same batch (all matrices, all
    cores), and parity of cholesky + projected_inverse on every 16th."""
    from oracle import ref, workload
    ref.set_threads(os.cpu_count() or 1)
    xh = x0.cpu().numpy()
    x.copy_(x0)
    B.cholesky(x)
    Lg = x.cpu().numpy().copy()
    B.projected_inverse(x)
    Yg = x.cpu().numpy()
    t0 = time.perf_counter()
    outs = []
    for m, s in enumerate(Bs):
        r = xh[B.offsets[m]:B.offsets[m + 1]].copy()
        ref.cholesky(s, r)
        L = r.copy() if m % sample_every == 0 else None
        ref.projected_inverse(s, r)
        outs.append((L, r))
    dt = time.perf_counter() - t0
    worst = 0.0
    for m in range(0, len(Bs), sample_every):
        seg = slice(B.offsets[m], B.offsets[m + 1])
        worst = max(worst, workload.block_errors(Bs[m], Lg[seg], outs[m][0]),
                    workload.block_errors(Bs[m], Yg[seg], outs[m][1]))
    return {"reference_ms": round(dt * 1e3, 1), "reference_cores": os.cpu_count() or 1,
            "parity": {"max_scaled_error": worst, "rtol": RTOL, "matrices_checked": len(range(0, len(Bs),
                                                                                            sample_every))}}


def autograd_section(dev, side=32, value_sets=16, reps=5, h=1e-6):
    """Differentiation: log det of `value_sets` value sets on the 3-D 7-point
    grid side^3 through the autograd Function (chompack_b200.autograd) with a
    leading batch dimension, forward + backward by torch.autograd.grad: one
    cholesky launch, one projected_inverse launch and three small reduction
    and weight kernels for all value sets.  Checks on value set 0: the
    gradient against the reference's projected inverse (<g,U> = <Y_ref,U>),
    the central finite difference with h = 1e-6, and the Hessian-vector
    product -<U, H(U)> (double backward, one merged hessian launch per pass)
    against the reference hessian."""
    import torch
    import chompack_b200 as cp
    from chompack_b200 import grids, autograd
    from oracle import ref
    A0 = grids.grid3d(side, seed=0)
    s = cp.symbolic(A0, p=cp.amd.order(A0), merge_function=cp.merge_size_fill(32, 32))
    xs = []
    for v in range(value_sets):
        xs.append((cp.cspmatrix(s, device=dev) + grids.grid3d(side, seed=v)).blkval)
    x0 = torch.stack(xs)

    def fwd_bwd():
        x = x0.detach().requires_grad_(True)
        ld = autograd.logdet_values(x, s)
        (g,) = torch.autograd.grad(ld.sum(), x)
        return ld, g
    ms = _event_ms(dev, fwd_bwd, reps)
    fl = sweep_flops(s)
    flops = value_sets * (fl["cholesky"] + fl["projected_inverse"])
    # checks on value set 0 against the reference
    xh = x0[0].cpu().numpy().copy()
    Lr, Yr = reference_outputs(s, xh)
    U = np.random.default_rng(6).standard_normal(xh.size)
    ld, g = fwd_bwd()
    gU = float((g[0] * torch.from_numpy(U).to(dev)).sum())
    want = ref.dot(s, Yr.copy(), U.copy())
    u = torch.from_numpy(U).to(dev)
    fd = (float(autograd.logdet_values(x0[0] + h * u, s)) - float(autograd.logdet_values(x0[0] - h * u, s))) / (2 * h)
    x = x0[:1].detach().requires_grad_(True)
    (g1,) = torch.autograd.grad(autograd.logdet_values(x, s).sum(), x, create_graph=True)
    (hv,) = torch.autograd.grad((g1 * u[None, :]).sum(), x)
    second = float((hv[0] * u).sum())
    Hu = U.copy()
    ref.hessian(s, Lr, Yr, [Hu], adj=None, factored_updates=True)
    second_ref = -ref.dot(s, U.copy(), Hu)
    memory = autograd_memory(dev, s, x0, reps, g)
    return {"workload": "3-D 7-point grid %d^3 (n=%d), AMD, merge_size_fill(32,32), %d value sets through "
                        "chompack_b200.autograd.logdet_values (torch.autograd.grad)" % (side, s.n, value_sets),
            "fwd_bwd_ms": round(ms, 3), "gflops": round(flops / ms / 1e6, 1),
            "launches": {"sweeps": 2, "kernels": 5,
                         "note": "cholesky and projected_inverse engine launches for all value sets, log-det "
                                 "reduction (2 kernels) and the gradient weights (1 kernel)"},
            "gradient_rel_error_vs_reference": abs(gU - want) / abs(want),
            "gradient_fd_rel_error": abs(gU - fd) / abs(fd), "fd_step": h,
            "hvp_rel_error_vs_reference": abs(second - second_ref) / abs(second_ref),
            "memory": memory}


def autograd_memory(dev, s, x0, reps, g_default):
    """Memory against time for the autograd workload: the sweeps' workspace
    (update matrices, per-front scratch, counters) with every update matrix
    in memory of its own (the default), and with them in a pool (plan option
    scratch_limit) limited to the reference's postorder stack size per value
    set, or unlimited (2^40 bytes: the pool reuses only memory the simulated
    schedule has freed, no added delay); the forward + backward time with
    each, and with the factor recomputed in the backward instead of kept
    (recompute_factor).
    Each variant's gradient must be bit-identical to the default's."""
    import torch
    from chompack_b200 import _native as N, autograd
    sets = int(x0.shape[0])
    Bt = autograd._value_sets(s, sets, x0.device)
    ops = (("cholesky", N.OP_CHOLESKY), ("projected_inverse", N.OP_PROJECTED_INVERSE))

    def workspace():
        return {name: Bt.plan.pool_info(op)["workspace_bytes"] for name, op in ops}

    def run(**kw):
        x = x0.detach().requires_grad_(True)
        ld = autograd.logdet_values(x, s, **kw)
        (g,) = torch.autograd.grad(ld.sum(), x)
        return g

    nv = int(s.blkptr[-1])
    limit = int(s.memory["stack_mem"]) * 8 * sets
    out = {"update_matrices_bytes": int(sum(int(f) ** 2 for f in _update_orders(s))) * 8 * sets,
           "reference_stack_bytes": limit, "factor_kept_bytes": nv * 8 * sets,
           "default": {"workspace_bytes": workspace()}}
    variants = (("scratch_limit", {"scratch_limit": limit}),
                ("scratch_limit_no_delay", {"scratch_limit": 1 << 40}),
                ("recompute_factor", {"recompute_factor": True}))
    for label, kw in variants:
        ms = _event_ms(dev, lambda: run(**kw), reps)
        g = run(**kw)
        entry = {"fwd_bwd_ms": round(ms, 3), "gradient_bit_identical": bool(torch.equal(g, g_default))}
        if "scratch_limit" in kw:
            entry["scratch_limit_bytes"] = kw["scratch_limit"]
            entry["workspace_bytes"] = workspace()
            entry["pool_bytes"] = {name: Bt.plan.pool_info(op)["pool_bytes"] for name, op in ops}
        else:
            entry["factor_kept_bytes"] = 0
        out[label] = entry
        autograd._limit_scratch(Bt.plan, None)
    return out


def _update_orders(s):
    """|A_k| of every supernode (the order of its update matrix)."""
    nn = np.diff(np.asarray(s.snptr))
    return np.diff(np.asarray(s.blkptr)) // nn - nn


def _engine_occupancy():
    """Resident CTAs per SM of the persistent kernel's two builds (FP64 and
    the one with tcgen05 TF32 tiles)."""
    import ctypes
    from chompack_b200 import _native as N
    out = {}
    for name, tc in (("fp64", 0), ("tcgen05", 1)):
        v = ctypes.c_int()
        out[name] = v.value if N.engine_occupancy(tc, ctypes.byref(v)) == 0 else None
    return out


# ------------------------------------------------------------------- main

def _spawn(args):
    """Start args.gpus ranks of this script under torch.distributed.run."""
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(args.gpus),
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


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

    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        return _spawn(args)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus:
        raise SystemExit("bench.py: --gpus %d but WORLD_SIZE=%d" % (args.gpus, world))
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
    cfg = bench_config(s)
    step_flops = cfg["flops_per_step"]
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
    info = N.info(plan.handle, ws, sp)
    if info != 0:
        raise RuntimeError("sweep status %d (%s)" % (info, N.last_error().decode()))
    elapsed = t0.elapsed_time(t1) / 1e3
    kern = {op: float(np.mean([a.elapsed_time(b) for a, b in ev_k[op]])) / 1e3 for op in ops}
    # the job ends with the slowest rank (chompack_b200.shard, NCCL here)
    from chompack_b200 import shard
    elapsed = shard.max_over_ranks(elapsed, device=dev)
    kern = {o: shard.max_over_ranks(kern[o], device=dev) for o in ops}
    value = step_flops * args.steps * world / elapsed / 1e9
    Y_step = Xw.cpu().numpy()          # output of the last timed step (steps are bit-identical)

    # the other drop-in sweeps of the workload, timed alone after the step
    # loop (not part of the step): completion of the projected inverse the
    # step produced (both update modes) and llt of the factor
    other = {}
    sweeps_other = not args.no_other
    Yw = Xw.clone()
    Lw = X0.blkval.clone()
    launch["cholesky"](plan.handle, Lw.data_ptr(), ws, nbytes, sp)
    L_gpu = Lw.cpu().numpy()
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
        fb = 8.0 * int(s.blkptr[-1]) + 16.0 * s.n * nrhs     # factor read once, B read and written
        other["trsm_%s_nrhs%d" % (tr, nrhs)] = {"ms": round(ms, 4), "gflops": round(fl["trsm_rhs"] * nrhs / ms / 1e6, 3),
                                                "achieved_gbs": round(fb / ms / 1e6, 1)}
        # the bit-reproducible form (additions into vector blocks in a fixed order)
        plan.set_option("ordered_sums", 1)
        try:
            wt, nbt = plan.workspace(N.OP_TRSM, nrhs, 1 if tr == "T" else 0)
            ms = timed(lambda: N.trsm(plan.handle, tr.encode(), nrhs, 1.0, Lw.data_ptr(), Bt.data_ptr(), s.n, wt,
                                      nbt, sp), reps)
        finally:
            plan.set_option("ordered_sums", None)
        other["trsm_%s_nrhs%d" % (tr, nrhs)]["ordered_sums_ms"] = round(ms, 4)
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
    Y_e2e = None
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
        w = shard.max_over_ranks(w, device=dev)
        nb_in = host_in.numel() * 8
        e2e = {"value": round(step_flops * world / w / 1e9, 3), "unit": "GFLOP/s", "h2d_bytes_per_step": nb_in,
               "d2h_bytes_per_step": 2 * nb_in, "ms_per_step": round(w * 1e3, 3),
               "path": "cbase.cholesky + cbase.projected_inverse on host-resident values (streamed chunks)"}
        Y_e2e = bufs[-1].numpy()

    # sharded batch section: every rank takes part (collectives inside)
    batch_out = None
    if not args.no_batch and not args.no_other:
        try:
            batch_out = batch_section(dev, rank, world)
        except Exception as exc:  # reported beside the headline, never required
            batch_out = {"unavailable": str(exc)}

    if rank == 0:
        x0h = X0.blkval.cpu().numpy()
        parity = None
        try:
            from oracle import workload
            Lr, Yr = reference_outputs(s, x0h)
            parity = {"rtol": RTOL, "against": "reference C kernels (oracle/_ref) on the same inputs",
                      "cholesky": workload.block_errors(s, L_gpu, Lr),
                      "projected_inverse": workload.block_errors(s, Y_step, Yr)}
            if Y_e2e is not None:
                parity["e2e_projected_inverse"] = workload.block_errors(s, Y_e2e, Yr)
            parity["max_scaled_error"] = max(v for k, v in parity.items() if isinstance(v, float) and k != "rtol")
            parity["pass"] = parity["max_scaled_error"] <= RTOL
        except Exception as exc:  # the checker is reported, never required
            parity = {"unavailable": str(exc)}
        peak = fp64_peak_tflops(dev)
        alg_bytes = sweep_bytes(s)
        achieved = fl["cholesky"] / kern["cholesky"] / 1e12
        out = {
            "metric": METRIC, "value": round(value, 3), "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(elapsed / args.steps * 1e3, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
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
            "parity": parity,
            "engine_ctas_per_sm": _engine_occupancy(),
            "kernel_ms": {o: round(kern[o] * 1e3, 4) for o in ops},
            "other_sweeps": other,
        }
        if clocks:
            out["clocks"] = clocks
        if e2e:
            out["e2e"] = e2e
        if batch_out is not None:
            out["batch"] = batch_out
        if not args.no_mixed and not args.no_other:
            try:
                out["mixed_precision"] = mixed_precision_section(dev)
                out["mixed_precision"]["grid2d_1000"] = mixed_precision_section(dev, grid2d=1000, reps=3)
            except Exception as exc:  # reported beside the headline, never required
                out["mixed_precision"] = {"unavailable": str(exc)}
        if not args.no_batch and not args.no_other:
            try:
                out["autograd"] = autograd_section(dev)
            except Exception as exc:  # reported beside the headline, never required
                out["autograd"] = {"unavailable": str(exc)}
        if not args.no_cpu:
            try:
                out["cpu_baseline"] = cpu_baseline(s, x0h)
            except Exception as exc:  # the baseline is reported, never required
                out["cpu_baseline"] = {"unavailable": str(exc)}
        print(json.dumps(out))
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
