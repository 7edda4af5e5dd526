"""Device plan of a symbolic factorisation: the symbolic arrays uploaded once
(chb_plan_create), the compiled task programs of each sweep, and the device
workspaces they run in (allocated through torch's caching allocator and
reused across calls)."""
import ctypes

import numpy as np
import torch

from . import _native as N

__all__ = ["Plan"]


def _i64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int64))


class Plan(object):
    """Uploaded symbolic factorisation.  device=None picks the current CUDA
    device; device=-1 builds a host-only plan (introspection only)."""

    @classmethod
    def merged(cls, plans, device=None):
        """One plan over the disjoint union of `plans` (chb_plan_merge): a
        batch swept by one launch per sweep."""
        if device is None:
            if not torch.cuda.is_available():
                raise RuntimeError("chompack_b200 sweeps need a CUDA device (no CPU fallback)")
            device = torch.cuda.current_device()
        self = cls.__new__(cls)
        self.device = int(device)
        self.symb = None
        self._keep = list(plans)
        arr = (ctypes.c_void_p * len(plans))(*[p.handle.value if hasattr(p.handle, "value") else p.handle
                                               for p in plans])
        h = N.PPLAN()
        if self.device >= 0:
            with torch.cuda.device(self.device):
                rc = N.plan_merge(arr, len(plans), self.device, ctypes.byref(h))
        else:
            rc = N.plan_merge(arr, len(plans), self.device, ctypes.byref(h))
        N.check(rc, "plan_merge")
        self.handle = h
        self._ws = {}
        return self

    def batch_segments(self):
        """Supernode ranges of the matrices of this plan (count + 1 offsets)."""
        cnt = ctypes.c_int64()
        N.check(N.plan_batch_info(self.handle, ctypes.byref(cnt), None), "plan_batch_info")
        seg = (ctypes.c_int64 * (cnt.value + 1))()
        N.check(N.plan_batch_info(self.handle, None, seg), "plan_batch_info")
        return list(seg)

    def __init__(self, symb, device=None):
        if device is None:
            if not torch.cuda.is_available():
                raise RuntimeError("chompack_b200 sweeps need a CUDA device (no CPU fallback)")
            device = torch.cuda.current_device()
        self.device = int(device)
        self.symb = symb
        arrs = [_i64(getattr(symb, a)) for a in ("snptr", "snpar", "relptr", "relidx", "chptr", "chidx",
                                                 "blkptr", "snode", "p")]
        self._keep = arrs
        h = N.PPLAN()
        if self.device >= 0:
            with torch.cuda.device(self.device):
                rc = N.plan_create(symb.n, symb.Nsn, *[N.ptr(a) for a in arrs], self.device, ctypes.byref(h))
        else:
            rc = N.plan_create(symb.n, symb.Nsn, *[N.ptr(a) for a in arrs], self.device, ctypes.byref(h))
        N.check(rc, "plan_create")
        self.handle = h
        self._ws = {}

    def __del__(self):
        h = getattr(self, "handle", None)
        if h and N is not None and getattr(N, "plan_destroy", None) is not None:  # not during interpreter teardown
            N.plan_destroy(h)
            self.handle = None

    def workspace_bytes(self, op, k=0, flags=0):
        sz = ctypes.c_size_t()
        N.check(N.workspace_size(self.handle, op, int(k), int(flags), ctypes.byref(sz)), "workspace_size")
        return int(sz.value)

    def workspace(self, op, k=0, flags=0, slot=0):
        """Device workspace for an operation (cached; 256-byte aligned)."""
        nbytes = self.workspace_bytes(op, k, flags)
        key = (slot,)
        buf = self._ws.get(key)
        if buf is None or buf.numel() < nbytes + 256:
            buf = torch.empty(nbytes + 256, dtype=torch.uint8, device=torch.device("cuda", self.device))
            self._ws[key] = buf
        base = buf.data_ptr()
        aligned = (base + 255) // 256 * 256
        return aligned, nbytes

    def set_schedule(self, mode):
        """Task scheduling of this plan's sweeps: "dynamic" (finished tasks
        release their waiters), "static" (list order with waits) or None
        (the default).  Results are bit-identical."""
        code = {None: -1, "dynamic": 0, "static": 1}[mode]
        N.check(N.plan_set_schedule(self.handle, code), "plan_set_schedule")

    def set_option(self, name, value=None):
        """Program-build option of this plan's sweeps (chb_plan_set_option):
        "small_front_nj", "subtrees", "chol_ksplit", "pinv_ksplit",
        "fused_la", "tf32_tcgen05", "ordered_sums" (trsm's additions in a
        fixed order, bit-reproducible) or "scratch_limit" (bytes for the
        update matrices of cholesky and projected_inverse, shared where the
        schedule allows; see `pool_info`); None restores the default.
        Drops the compiled programs (the device is synchronised first, so
        no sweep of the plan is in flight)."""
        if self.device >= 0:
            torch.cuda.synchronize(self.device)
        v = -1 if value is None else int(value)
        N.check(N.plan_set_option(self.handle, N.OPTIONS[name], v), "plan_set_option")

    def pool_info(self, op, k=0, flags=0):
        """The update-matrix pool of a sweep's program under a scratch
        limit: {"pool_bytes" (None without a pool), "reuse_waits",
        "workspace_bytes", "model_span_us" (the span of the planner's
        simulated schedule, a model, not a measurement)}."""
        info = (ctypes.c_int64 * 4)()
        N.check(N.program_pool(self.handle, op, int(k), int(flags), info), "program_pool")
        return {"pool_bytes": None if info[0] < 0 else int(info[0]), "reuse_waits": int(info[1]),
                "workspace_bytes": int(info[2]), "model_span_us": info[3] / 1000.0}

    def option(self, name):
        """The value the next program build uses for an option."""
        v = ctypes.c_int64()
        N.check(N.plan_get_option(self.handle, N.OPTIONS[name], ctypes.byref(v)), "plan_get_option")
        return int(v.value)

    def options(self):
        return {k: self.option(k) for k in N.OPTIONS}

    def set_spin_limit(self, polls=None):
        """Bound of every wait inside this plan's sweeps, in polls (None:
        the default, about 10 s); a wait that runs out ends the sweep with
        status -30 (RuntimeError from the sweeps)."""
        N.check(N.plan_set_spin_limit(self.handle, -1 if polls is None else int(polls)), "plan_set_spin_limit")

    def program_info(self, op, k=0, flags=0):
        info = (ctypes.c_int64 * 8)()
        N.check(N.program_info(self.handle, op, int(k), int(flags), info), "program_info")
        keys = ("tasks", "waits", "counters", "ws_doubles", "ws_bytes", "dbl_off", "upd_doubles", "task_bytes")
        return dict(zip(keys, list(info)))
