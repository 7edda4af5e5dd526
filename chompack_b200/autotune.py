"""Autotuner of how a plan's sweeps are cut into tasks (no counterpart in the
reference, whose sweeps are one BLAS call sequence per front).

The choices are the plan's program-build options (chb_plan_set_option) and
its schedule:

* small_front_nj — largest front run as one shared-memory task (0..64);
* subtrees       — small complete subtrees bundled four per task (1/0);
* pinv_ksplit    — K chunk of projected_inverse's long-K tiles;
* chol_ksplit    — K chunk of cholesky's Schur-complement tiles (0: whole);
* schedule       — static list order, dynamic release, or the per-sweep default.

`tune(target, values)` times the sweeps (cholesky, then projected_inverse on
its factor, CUDA events, after a warm-up launch that builds the programs)
under one choice at a time, in a single pass of coordinate descent from the
defaults, keeps the fastest setting of each, applies the result to the plan
and remembers it per sparsity pattern: a later call for a plan of the same
pattern applies the remembered choice without timing.  Results do not
depend on the choice beyond the FP64 rounding of a different, still fixed,
summation order.
"""
import hashlib

import numpy as np
import torch

from . import _native as N

__all__ = ["tune", "fingerprint", "CANDIDATES"]

CANDIDATES = [
    ("subtrees", [1, 0]),
    ("small_front_nj", [64, 48, 32, 0]),
    ("schedule", [None, "static", "dynamic"]),
    ("pinv_ksplit", [512, 384, 768, 1024]),
    ("chol_ksplit", [0, 256, 512]),
]

_cache = {}


def fingerprint(plan):
    """Identity of a plan's sparsity pattern: the front sizes and the
    relative indices of its supernodes (from the symbolic arrays of every
    matrix of a merged plan)."""
    h = hashlib.sha1()
    symbs = [plan.symb] if getattr(plan, "symb", None) is not None else None
    if symbs is None:
        symbs = [getattr(p, "symb", None) for p in getattr(plan, "_keep", [])]
    for s in symbs:
        if s is None:
            continue
        for a in (s.snptr, s.relptr, s.relidx, s.chptr, s.chidx):
            h.update(np.ascontiguousarray(np.asarray(a), dtype=np.int64).tobytes())
    return h.hexdigest()


def _apply(plan, choice):
    for name, value in choice.items():
        if name == "schedule":
            plan.set_schedule(value)
        else:
            plan.set_option(name, value)


def _sweep_timer(plan, values, reps):
    """Median CUDA-event time (ms) of cholesky + projected_inverse on a copy
    of `values`, after one warm-up run."""
    dev = torch.device("cuda", plan.device)
    x = values.clone()
    s = torch.cuda.current_stream(dev).cuda_stream
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def once():
        x.copy_(values)
        for op, fn in ((N.OP_CHOLESKY, N.cholesky), (N.OP_PROJECTED_INVERSE, N.projected_inverse)):
            ws, nb = plan.workspace(op)
            if fn(plan.handle, x.data_ptr(), ws, nb, s) < 0:
                raise RuntimeError(N.last_error().decode())
            info = N.info(plan.handle, ws, s)
            if info != 0:
                raise RuntimeError("sweep status %d during tuning" % info)

    once()
    times = []
    for _ in range(reps):
        torch.cuda.synchronize(dev)
        e0.record()
        once()
        e1.record()
        torch.cuda.synchronize(dev)
        times.append(e0.elapsed_time(e1))
    return float(np.median(times))


def tune(target, values, reps=3, timer=None, use_cache=True):
    """Pick the fastest task cutting for `target` (a symbolic factorisation,
    a Plan or a batch) on the block values `values` (a CUDA float64 tensor in
    the plan's layout, left unchanged) and apply it to the plan.  Returns
    {"choice": ..., "ms": best time, "default_ms": time with the defaults,
    "trials": [(choice, ms), ...], "cached": bool}.  `timer(plan)` replaces
    the CUDA-event timing (tests)."""
    if hasattr(target, "handle"):          # a Plan
        plan = target
    elif callable(getattr(target, "plan", None)):
        plan = target.plan()               # a symbolic factorisation
    else:
        plan = target.plan                 # a batch
    key = fingerprint(plan)
    if use_cache and key in _cache:
        choice, ms, dms = _cache[key]
        _apply(plan, choice)
        return {"choice": dict(choice), "ms": ms, "default_ms": dms, "trials": [], "cached": True}
    measure = timer if timer is not None else (lambda p: _sweep_timer(p, values, reps))
    choice = {name: vals[0] for name, vals in CANDIDATES}
    choice["schedule"] = None
    _apply(plan, choice)
    best = measure(plan)
    default_ms = best
    trials = [(dict(choice), best)]
    for name, vals in CANDIDATES:
        for v in vals:
            if v == choice[name]:
                continue
            trial = dict(choice)
            trial[name] = v
            _apply(plan, trial)
            ms = measure(plan)
            trials.append((dict(trial), ms))
            if ms < best:
                best = ms
                choice = trial
    _apply(plan, choice)
    _cache[key] = (dict(choice), best, default_ms)
    return {"choice": dict(choice), "ms": best, "default_ms": default_ms, "trials": trials, "cached": False}
