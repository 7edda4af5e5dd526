"""CPU interpreter of the device task programs (test infrastructure).

The native planner compiles every sweep into a task list (the same bytes the
persistent GPU kernel executes).  This module decodes that list through the
library's introspection API and executes it with numpy, either in list order
or in a random order that only respects the recorded waits.  Running random
topological orders against the reference results checks, without a GPU, that
the planner's operands are right and that its dependency lists are complete.
It is a checker of the planner, never a way to compute a result in the
product.
"""
import ctypes

import numpy as np

from chompack_b200 import _native as N
from chompack_b200 import trace

TASK = trace.TASK  # the engine's 144-byte task record
FRONT = np.dtype([("nn", "<i4"), ("na", "<i4"), ("nj", "<i4"), ("relptr", "<i4"), ("chbeg", "<i4"),
                  ("chend", "<i4"), ("parent", "<i4"), ("level", "<i4"), ("blk", "<i8"), ("upd", "<i8"),
                  ("col0", "<i8"), ("vpos", "<i8")])

OM_N, OM_T, OM_TRI_N, OM_TRI_T, OM_SYM = range(5)
T_GEMM, T_POTRF, T_ASM, T_MROW, T_EXTRACT, T_COPY = 0, 1, 2, 3, 4, 5
T_QL, T_VEC, T_NOP, T_LA, T_SUM, T_SIGNAL, T_ARRIVAL, T_FRONT, T_PFRONT = 8, 9, 10, 11, 12, 13, 14, 15, 16
T_SUBTREE, T_PSUBTREE, T_TRSV = 17, 18, 19
QL_GATHER, QL_PANEL = 0, 1
B_X, B_WS, B_RHS = 0, 1, 4

N.lib.chb_program_info.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_int64)]
N.lib.chb_program_export.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_int,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]


N.lib.chb_program_schedule.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_int64)] + [ctypes.c_void_p] * 6


class Schedule(object):
    """The dynamic-schedule data of a program: pending counts, successors
    per counter (CSR), completion values and the initial ready bitmaps."""

    def __init__(self, plan_handle, op, k=0, flags=0):
        sz = (ctypes.c_int64 * 6)()
        args = (plan_handle, op, k, flags, sz)
        N.check(N.lib.chb_program_schedule(*args, None, None, None, None, None, None), "program_schedule")
        self.npend = np.zeros(sz[0], dtype=np.int32)
        self.succ_off = np.zeros(sz[1], dtype=np.int32)
        self.succ = np.zeros(sz[2], dtype=np.int32)
        self.ctarget = np.zeros(sz[3], dtype=np.int32)
        self.ready0 = np.zeros(sz[4], dtype=np.uint64)
        self.summ0 = np.zeros(sz[5], dtype=np.uint64)
        N.check(N.lib.chb_program_schedule(*args, self.npend.ctypes.data, self.succ_off.ctypes.data,
                                           self.succ.ctypes.data, self.ctarget.ctypes.data,
                                           self.ready0.ctypes.data, self.summ0.ctypes.data),
                "program_schedule")


class Program(object):
    def __init__(self, plan_handle, op, k=0, flags=0, nsn=0):
        info = (ctypes.c_int64 * 8)()
        N.check(N.lib.chb_program_info(plan_handle, op, k, flags, info), "program_info")
        self.ntasks, self.nwaits, self.ncounters, self.ws_doubles = info[0], info[1], info[2], info[3]
        assert info[7] == TASK.itemsize, "Task layout mismatch (%d bytes)" % info[7]
        self.upd_total = info[6]
        self.tasks = np.zeros(self.ntasks, dtype=TASK)
        self.waits = np.zeros((self.nwaits, 2), dtype=np.int32)
        self.fronts = np.zeros(nsn, dtype=FRONT)
        N.check(N.lib.chb_program_export(plan_handle, op, k, flags, self.tasks.ctypes.data,
                                         self.waits.ctypes.data, self.fronts.ctypes.data), "program_export")


def _early_counter(t):
    """The early-signal counter of a look-ahead task or a fused diagonal
    task (aux[3] = counter + 1), or -1."""
    op = int(t["op"])
    if op == T_LA or (op == T_POTRF and int(t["k"]) > 0):
        return int(t["aux"][3]) - 1
    return -1


def _operand(buf, o, rows, K):
    r = np.arange(rows)[:, None]
    k = np.arange(K)[None, :]
    mode = int(o["mode"])
    off, ld, d = int(o["off"]), int(o["ld"]), int(o["diag"])
    if mode == OM_N:
        return buf[off + k * ld + r]
    if mode == OM_T:
        return buf[off + r * ld + k]
    if mode == OM_TRI_N:
        v = buf[off + np.minimum(k * ld + r, buf.size - 1 - off)]
        return np.where(r + d >= k, v, 0.0)
    if mode == OM_TRI_T:
        v = buf[off + np.minimum(r * ld + k, buf.size - 1 - off)]
        return np.where(k + d >= r, v, 0.0)
    gr, gc = r + d, k + int(o["pad2"])
    idx = np.where(gr >= gc, gc * ld + gr, gr * ld + gc)
    return buf[off + idx]


def _store(buf, o, m, n, val, lower, cdiag, beta):
    r = np.arange(m)[:, None]
    c = np.arange(n)[None, :]
    idx = int(o["off"]) + c * int(o["ld"]) + r
    mask = np.ones((m, n), dtype=bool) if not lower else (r + cdiag >= c)
    old = buf[idx]
    new = val + (beta * old if beta != 0.0 else 0.0)
    buf[idx[mask]] = new[mask]


class VM(object):
    """Executes a Program on numpy buffers.  bases: dict slot -> 1-D array."""

    def __init__(self, prog, bases, relidx, chidx, perm=None, ldb=0, alpha=1.0):
        self.p = prog
        self.bases = bases
        self.relidx = np.asarray(relidx)
        self.chidx = np.asarray(chidx)
        self.perm = None if perm is None else np.asarray(perm)
        self.ldb = ldb
        self.alpha = alpha
        self.info = 0

    def run_task(self, t):
        op = int(t["op"])
        if op == T_GEMM or op == T_TRSV:  # a substitution step is a GEMM (its cdiag counts its first waits)
            m, n, K = int(t["m"]), int(t["n"]), int(t["k"])
            A = _operand(self.bases[int(t["a"]["base"])], t["a"], m, K)
            Bm = _operand(self.bases[int(t["b"]["base"])], t["b"], n, K)
            _store(self.bases[int(t["c"]["base"])], t["c"], m, n, float(t["alpha"]) * (A @ Bm.T),
                   int(t["cmode"]) == 1, int(t["cdiag"]), float(t["beta"]))
        elif op == T_MROW:
            m, n, K = int(t["m"]), int(t["n"]), int(t["k"])
            A = _operand(self.bases[int(t["a"]["base"])], t["a"], m, K)
            Bm = _operand(self.bases[int(t["b"]["base"])], t["b"], n, K)
            aux = t["aux"]
            moff = (int(aux[2]) & 0xffffffff) | (int(aux[3]) << 32)
            buf = self.bases[int(aux[0])]
            r = np.arange(m)[:, None]
            k = np.arange(m)[None, :]
            M2 = np.where(r >= k, buf[moff + k * int(aux[1]) + r], 0.0)
            _store(self.bases[int(t["c"]["base"])], t["c"], m, n, float(t["alpha"]) * (M2 @ (A @ Bm.T)),
                   False, 0, 0.0)
        elif op == T_POTRF:
            b = int(t["m"])
            X = self.bases[int(t["a"]["base"])]
            off, ld = int(t["a"]["off"]), int(t["a"]["ld"])
            r = np.arange(b)[:, None]
            c = np.arange(b)[None, :]
            tile = X[off + c * ld + r]
            if int(t["aux"][2]):
                L = np.tril(tile)
                if np.any(np.diag(L) == 0.0) and self.info == 0:
                    self.info = int(t["aux"][0]) + 1
            else:
                S = np.tril(tile) + np.tril(tile, -1).T
                try:
                    L = np.linalg.cholesky(S)
                except np.linalg.LinAlgError:
                    if self.info == 0:
                        self.info = int(t["aux"][0]) + 1
                    L = np.nan_to_num(np.tril(tile))
                idx = off + c * ld + r
                low = r >= c
                X[idx[low]] = L[low]
            if int(t["aux"][1]):
                M = np.linalg.inv(L)
                _store(self.bases[int(t["c"]["base"])], t["c"], b, b, np.tril(M), False, 0, 0.0)
            m2 = int(t["k"])
            if m2 > 0:   # fused look-ahead: next panel tile and next diagonal tile
                r2 = np.arange(m2)[:, None]
                pidx = off + b + c * ld + r2                   # tile (c+1, c): m2 x b
                L2 = X[pidx] @ np.tril(np.linalg.inv(L)).T
                X[pidx] = L2
                c2 = np.arange(m2)[None, :]
                didx = off + b * ld + b + c2 * ld + r2         # tile (c+1, c+1): m2 x m2
                low = r2 >= c2
                X[didx[low]] = (X[didx] - L2 @ L2.T)[low]
        elif op == T_ASM:
            self._asm(t)
        elif op == T_FRONT:
            self._front(t)
        elif op == T_PFRONT:
            self._pfront(t)
        elif op == T_SUBTREE:
            self._subtrees(t, False)
        elif op == T_PSUBTREE:
            self._subtrees(t, True)
        elif op == T_EXTRACT:
            self._extract(t)
        elif op == T_VEC:
            self._vec(t)
        elif op == T_QL:
            self._ql(t)
        elif op in (T_NOP, T_SIGNAL, T_ARRIVAL):
            pass
        elif op == T_SUM:  # C = alpha * sum_q P_q + beta * C (in order)
            m, n, p, stride = int(t["m"]), int(t["n"]), int(t["aux"][0]), int(t["aux"][1])
            Pb, Po, ldp = self.bases[int(t["a"]["base"])], int(t["a"]["off"]), int(t["a"]["ld"])
            r = np.arange(m)[:, None]
            c = np.arange(n)[None, :]
            acc = np.zeros((m, n))
            for q in range(p):
                acc = acc + Pb[Po + q * stride + c * ldp + r]
            _store(self.bases[int(t["c"]["base"])], t["c"], m, n, float(t["alpha"]) * acc,
                   int(t["cmode"]) == 1, int(t["cdiag"]), float(t["beta"]))
        elif op == T_LA:  # L = A M^T -> A; D -= tril(L L^T)
            m, n, K = int(t["m"]), int(t["n"]), int(t["k"])
            A = _operand(self.bases[int(t["a"]["base"])], t["a"], m, K)
            Mt = _operand(self.bases[int(t["b"]["base"])], t["b"], n, K)
            L = A @ Mt.T
            _store(self.bases[int(t["a"]["base"])], t["a"], m, n, L, False, 0, 0.0)
            _store(self.bases[int(t["c"]["base"])], t["c"], m, m, -(L @ L.T), True, 0, 1.0)
        elif op == T_COPY:
            m, n = int(t["m"]), int(t["n"])
            fl = int(t["aux"][0])
            r = np.arange(m)[:, None]
            c = np.arange(n)[None, :]
            C = self.bases[int(t["c"]["base"])]
            cidx = int(t["c"]["off"]) + c * int(t["c"]["ld"]) + r
            if fl & 16:  # transpose (optionally the strict upper part only)
                A = self.bases[int(t["a"]["base"])]
                src = int(t["a"]["off"]) + r * int(t["a"]["ld"]) + c
                sel = (r < c) if (fl & 32) else np.ones((m, n), dtype=bool)
                C[cidx[sel]] = float(t["alpha"]) * A[src[sel]]
                return
            if fl & 8:   # anti-transpose inside an nn x nn matrix
                nn, i0, j0 = int(t["aux"][1]), int(t["aux"][2]), int(t["aux"][3])
                A = self.bases[int(t["a"]["base"])]
                gi, gj = i0 + r + 0 * c, j0 + c + 0 * r
                low = gi >= gj
                src = int(t["a"]["off"]) + (nn - 1 - gi) * int(t["a"]["ld"]) + (nn - 1 - gj)
                dst = int(t["c"]["off"]) + gj * int(t["c"]["ld"]) + gi
                C[dst[low]] = A[src[low]]
                return
            if fl & 4:
                C[cidx] = 0.0
            else:
                A = self.bases[int(t["a"]["base"])]
                v = float(t["alpha"]) * A[int(t["a"]["off"]) + c * int(t["a"]["ld"]) + r]
                low = (r >= c) | (not (fl & 1))
                C[cidx[low]] = v[low]
                if fl & 2:
                    C[cidx[~low]] = 0.0
        else:
            raise NotImplementedError("task op %d" % op)

    def _asm(self, t):
        f = self.p.fronts[int(t["aux"][0])]
        j0, j1 = int(t["aux"][1]), int(t["aux"][2])
        nn, na, nj = int(f["nn"]), int(f["na"]), int(f["nj"])
        WS = self.bases[B_WS]
        Pb, Pof, ldp = self.bases[int(t["a"]["base"])], int(t["a"]["off"]), int(t["a"]["ld"])
        Ub, Uof, ldu = self.bases[int(t["c"]["base"])], int(t["c"]["off"]), int(t["c"]["ld"])
        if int(t["aux"][3]) & 1:
            for j in range(max(j0, nn), j1):
                jj = j - nn
                Ub[Uof + jj * ldu + jj: Uof + jj * ldu + na] = 0.0
        for l in range(int(f["chend"]) - 1, int(f["chbeg"]) - 1, -1):
            ch = self.p.fronts[self.chidx[l]]
            Nc = int(ch["na"])
            r = self.relidx[int(ch["relptr"]): int(ch["relptr"]) + Nc]
            o2 = int(t["off2"])
            Uc = WS[o2 + int(ch["upd"]): o2 + int(ch["upd"]) + Nc * Nc].reshape((Nc, Nc), order="F")
            for q in range(Nc):
                col = int(r[q])
                if not (j0 <= col < j1):
                    continue
                rows = r[q:]
                v = Uc[q:, q]
                if col < nn:
                    Pb[Pof + col * ldp + rows] += v
                else:
                    Ub[Uof + (col - nn) * ldu + (rows - nn)] += v

    def _front(self, t):
        """A whole small cholesky front (T_FRONT)."""
        self._front_k(int(t["aux"][0]), self.bases[int(t["a"]["base"])], int(t["a"]["off"]),
                      self.bases[int(t["c"]["base"])], int(t["c"]["off"]), int(t["c"]["ld"]))

    def _bundle_ranges(self, t):
        ends = (int(t["m"]), int(t["n"]), int(t["k"]), int(t["cdiag"]))
        return [(int(t["aux"][w]), ends[w]) for w in range(4) if int(t["aux"][w]) >= 0]

    def _subtrees(self, t, pinv):
        """A small-subtree bundle: each range's fronts in postorder
        (cholesky) or parents first (projected_inverse), values at their
        blocks and updates at their usual workspace offsets."""
        WS = self.bases[B_WS]
        for lo, hi in self._bundle_ranges(t):
            for k in (range(hi, lo - 1, -1) if pinv else range(lo, hi + 1)):
                f = self.p.fronts[k]
                args = (k, self.bases[B_X], int(f["blk"]), WS, int(f["upd"]), max(int(f["na"]), 1))
                self._pfront_k(*args) if pinv else self._front_k(*args)

    def _front_k(self, k, X, off, Ub, Uof, ldu):
        """A whole small cholesky front: extend-add of the children (last
        to first), partial Cholesky of the nj x nj front, the Schur
        complement into the update matrix, and the off-diagonal block
        stored as L21 L11^{-1} (the reference's layout)."""
        f = self.p.fronts[k]
        nn, na, nj = int(f["nn"]), int(f["na"]), int(f["nj"])
        WS = self.bases[B_WS]
        r = np.arange(nj)[:, None]
        c = np.arange(nn)[None, :]
        F = np.zeros((nj, nj))
        F[:, :nn] = np.where(r >= c, X[off + c * nj + r], 0.0)
        for l in range(int(f["chend"]) - 1, int(f["chbeg"]) - 1, -1):
            ch = self.p.fronts[self.chidx[l]]
            Nc = int(ch["na"])
            rr = np.asarray(self.relidx[int(ch["relptr"]): int(ch["relptr"]) + Nc], dtype=np.int64)
            Uc = WS[int(ch["upd"]): int(ch["upd"]) + Nc * Nc].reshape((Nc, Nc), order="F")
            for q in range(Nc):
                F[rr[q:], rr[q]] += Uc[q:, q]
        S = np.tril(F) + np.tril(F, -1).T
        try:
            L11 = np.linalg.cholesky(S[:nn, :nn])
        except np.linalg.LinAlgError:
            if self.info == 0:
                self.info = 1
            return
        Li = np.linalg.inv(L11)
        L21 = S[nn:, :nn] @ Li.T
        blk = np.vstack([L11, L21 @ Li])              # nj x nn
        low = np.broadcast_to(r >= c, blk.shape)
        X[(off + c * nj + r)[low]] = blk[low]
        if na > 0:
            U = S[nn:, nn:] - L21 @ L21.T
            ri = np.arange(na)[:, None]
            ci = np.arange(na)[None, :]
            lw = ri >= ci
            Ub[(Uof + ci * ldu + ri)[lw]] = U[lw]

    def _pfront(self, t):
        """A whole small projected-inverse front (T_PFRONT)."""
        self._pfront_k(int(t["aux"][0]), self.bases[int(t["a"]["base"])], int(t["a"]["off"]),
                       self.bases[int(t["c"]["base"])], int(t["c"]["off"]), int(t["c"]["ld"]))

    def _pfront_k(self, k, X, off, Ub, Uof, ldu):
        """A whole small projected-inverse front: M = L11^{-1}, Y11 = M^T M,
        S21 = -V W, Y11 -= S21^T W, the children's updates extracted from
        the front [Y11, S21^T; S21, V], the block written back as [Y11
        (strict upper part zeroed); S21]."""
        f = self.p.fronts[k]
        nn, na, nj = int(f["nn"]), int(f["na"]), int(f["nj"])
        WS = self.bases[B_WS]
        r = np.arange(nj)[:, None]
        c = np.arange(nn)[None, :]
        blk = X[off + c * nj + r]
        L11 = np.tril(blk[:nn])
        if np.any(np.diag(L11) == 0.0) and self.info == 0:
            self.info = 1
        M = np.linalg.inv(L11)
        Y11 = M.T @ M
        F = np.zeros((nj, nj))
        if na > 0:
            ri = np.arange(na)[:, None]
            ci = np.arange(na)[None, :]
            Vl = np.where(ri >= ci, Ub[Uof + ci * ldu + ri], 0.0)
            V = Vl + np.tril(Vl, -1).T
            W = blk[nn:]
            S = -V @ W
            Y11 = Y11 - S.T @ W
            F[nn:, :nn] = S
            F[nn:, nn:] = V
        F[:nn, :nn] = Y11
        for l in range(int(f["chbeg"]), int(f["chend"])):
            ch = self.p.fronts[self.chidx[l]]
            Nc = int(ch["na"])
            rr = np.asarray(self.relidx[int(ch["relptr"]): int(ch["relptr"]) + Nc], dtype=np.int64)
            q = np.arange(Nc)[None, :]
            i = np.arange(Nc)[:, None]
            low = i >= q
            vals = F[rr[:, None], rr[None, :]]
            WS[(int(ch["upd"]) + q * Nc + i)[low]] = vals[low]
        out = np.vstack([np.where(r[:nn] >= c, Y11, 0.0), F[nn:, :nn]])
        X[off + c * nj + r] = out

    def _vec(self, t):
        mode, nrhs = int(t["aux"][0]), int(t["n"])
        WS = self.bases[B_WS]
        if mode in (0, 1):
            r0, r1 = int(t["aux"][1]), int(t["aux"][2])
            Bp, off, ld = self.bases[int(t["c"]["base"])], int(t["c"]["off"]), int(t["c"]["ld"])
            Bu = self.bases[B_RHS]
            for j in range(nrhs):
                src = self.perm[r0:r1] + j * self.ldb
                if mode == 0:
                    Bp[off + np.arange(r0, r1) + j * ld] = self.alpha * Bu[src]
                else:
                    Bu[src] = Bp[off + np.arange(r0, r1) + j * ld]
            return
        vbase = int(t["b"]["off"])
        xb, xo, ldx = self.bases[int(t["a"]["base"])], int(t["a"]["off"]), int(t["a"]["ld"])
        ub, uo = self.bases[int(t["c"]["base"])], int(t["c"]["off"])
        # right-hand-side columns [aux[2], aux[3]) (aux[3] == 0: all)
        j0 = int(t["aux"][2])
        j1 = int(t["aux"][3]) if int(t["aux"][3]) > 0 else nrhs
        if mode == 2:
            f = self.p.fronts[int(t["aux"][1])]
            nn, na = int(f["nn"]), int(f["na"])
            for j in range(j0, j1):
                ub[uo + j * na: uo + (j + 1) * na] = 0.0
            for l in range(int(f["chend"]) - 1, int(f["chbeg"]) - 1, -1):
                ch = self.p.fronts[self.chidx[l]]
                Nc = int(ch["na"])
                r = self.relidx[int(ch["relptr"]): int(ch["relptr"]) + Nc]
                uc = WS[vbase + int(ch["vpos"]) * nrhs: vbase + int(ch["vpos"]) * nrhs + Nc * nrhs].reshape((Nc, nrhs), order="F")
                for j in range(j0, j1):
                    top = r < nn
                    xb[xo + r[top] + j * ldx] += uc[top, j]
                    ub[uo + (r[~top] - nn) + j * na] += uc[~top, j]
            return
        if mode == 5:  # VEC_ZERO: m * n doubles of operand c
            ub[uo: uo + int(t["m"]) * nrhs] = 0.0
            return
        ch = self.p.fronts[int(t["aux"][1])]
        f = self.p.fronts[int(ch["parent"])]
        nn, na, Nc = int(f["nn"]), int(f["na"]), int(ch["na"])
        i0 = int(t["m"])
        i1 = int(t["k"]) if int(t["k"]) > 0 else Nc
        r = self.relidx[int(ch["relptr"]) + i0: int(ch["relptr"]) + i1]
        base = vbase + int(ch["vpos"]) * nrhs
        top = r < nn
        for j in range(j0, j1):
            seg = slice(base + j * Nc + i0, base + j * Nc + i1)
            if mode == 4:  # VEC_ADD: [x_p; u_p](r_c) += u_c (rows i0..i1)
                v = WS[seg].copy()
                np.add.at(xb, xo + r[top] + j * ldx, v[top])
                np.add.at(ub, uo + (r[~top] - nn) + j * na, v[~top])
                continue
            vals = np.empty(i1 - i0)
            vals[top] = xb[xo + r[top] + j * ldx]
            vals[~top] = ub[uo + (r[~top] - nn) + j * na]
            WS[seg] = vals

    def _ql(self, t):
        """Blocked Householder QL of update_factor (engine.cu run_ql) with
        numpy: QL_GATHER copies the parent-update columns, QL_PANEL reduces a
        panel and writes the explicit reflectors W' and the T factor."""
        ch = self.p.fronts[int(t["aux"][0])]
        f = self.p.fronts[int(ch["parent"])]
        Nc, nn, na = int(ch["na"]), int(f["nn"]), int(f["na"])
        r = self.relidx[int(ch["relptr"]): int(ch["relptr"]) + Nc]
        N1 = int(np.sum(r < nn))
        N2 = Nc - N1
        c0, c1, sub = int(t["aux"][1]), int(t["aux"][2]), int(t["aux"][3])
        if sub == QL_GATHER:
            Lb, Lo, ldl = self.bases[int(t["a"]["base"])], int(t["a"]["off"]), int(t["a"]["ld"])
            Cb, Co, ldc = self.bases[int(t["c"]["base"])], int(t["c"]["off"]), int(t["c"]["ld"])
            for j in range(c0, c1):
                jj = int(r[N1 + j]) - nn
                col = np.zeros(na)
                col[jj:] = Lb[Lo + jj * ldl + jj: Lo + jj * ldl + na]
                Cb[Co + j * ldc: Co + j * ldc + na] = col
            return
        Cb, Co, ldc = self.bases[int(t["a"]["base"])], int(t["a"]["off"]), int(t["a"]["ld"])
        Wb, Wo, ldw = self.bases[int(t["b"]["base"])], int(t["b"]["off"]), int(t["b"]["ld"])
        Tb, To, ldt = self.bases[int(t["c"]["base"])], int(t["c"]["off"]), int(t["c"]["ld"])
        nb = c1 - c0
        row0 = int(r[N1 + c0]) - nn
        row1 = na - N2 + c1 - 1
        h = row1 - row0 + 1
        ci = Co + (c0 + np.arange(nb))[None, :] * ldc + row0 + np.arange(h)[:, None]
        Pn = Cb[ci].copy()
        taus = np.zeros(nb)
        sup = []
        for i in range(nb):
            col = c1 - 1 - i
            pc = col - c0
            lr0 = int(r[N1 + col]) - nn - row0
            lp = na - N2 + col - row0
            sup.append((lr0, lp))
            if lp <= lr0:
                continue
            x = Pn[lr0:lp, pc]
            xn2 = float(np.dot(x, x))
            if xn2 == 0.0:
                continue
            alpha = Pn[lp, pc]
            beta = -np.copysign(np.hypot(alpha, np.sqrt(xn2)), alpha)
            tau = (beta - alpha) / beta
            Pn[lr0:lp, pc] = x / (alpha - beta)
            v = np.concatenate([Pn[lr0:lp, pc], [1.0]])
            blk = Pn[lr0:lp + 1, :pc]
            Pn[lr0:lp + 1, :pc] = blk - tau * np.outer(v, v @ blk)
            Pn[lp, pc] = beta
            taus[i] = tau
        Cb[ci] = Pn
        Wp = np.zeros((h, nb))
        for i in range(nb):
            lr0, lp = sup[i]
            pc = nb - 1 - i
            Wp[lr0:lp, i] = Pn[lr0:lp, pc]
            Wp[lp, i] = 1.0
        wi = Wo + (c0 + np.arange(nb))[None, :] * ldw + row0 + np.arange(h)[:, None]
        Wb[wi] = Wp
        G = Wp.T @ Wp
        T = np.zeros((nb, nb))
        for i in range(nb - 1, -1, -1):
            T[i, i] = taus[i]
            if i + 1 < nb:
                T[i + 1:, i] = -taus[i] * (T[i + 1:, i + 1:] @ G[i + 1:, i])
        ti = To + np.arange(nb)[None, :] * ldt + np.arange(nb)[:, None]
        Tb[ti] = T

    def _extract(self, t):
        ch = self.p.fronts[int(t["aux"][0])]
        f = self.p.fronts[int(ch["parent"])]
        q0, q1 = int(t["aux"][1]), int(t["aux"][2])
        Nc, nn = int(ch["na"]), int(f["nn"])
        r = self.relidx[int(ch["relptr"]): int(ch["relptr"]) + Nc]
        A = (self.bases[int(t["a"]["base"])], int(t["a"]["off"]), int(t["a"]["ld"]))
        Bb = (self.bases[int(t["b"]["base"])], int(t["b"]["off"]), int(t["b"]["ld"]))
        C = (self.bases[int(t["c"]["base"])], int(t["c"]["off"]), int(t["c"]["ld"]))
        WS = self.bases[B_WS]
        up = int(t["off2"]) + int(ch["upd"])
        for q in range(q0, q1):
            col = int(r[q])
            for i in range(q, Nc):
                row = int(r[i])
                if col >= nn:
                    buf, off, ld = C
                    v = buf[off + (col - nn) * ld + row - nn]
                elif row >= nn:
                    buf, off, ld = Bb
                    v = buf[off + col * ld + row - nn]
                else:
                    buf, off, ld = A
                    v = buf[off + col * ld + row]
                WS[up + q * Nc + i] = v

    def run(self, order="list", seed=0, schedule=None):
        """order: "list", "random" (any order the waits allow) or "dynamic"
        (the device's dynamic release rules applied to `schedule`)."""
        tasks = self.p.tasks
        nt = len(tasks)
        if order == "list":
            seq = range(nt)
        elif order == "dynamic":
            seq = dynamic_order(self.p, schedule, seed)
        else:
            seq = self._random_order(seed)
        for i in seq:
            self.run_task(tasks[i])
        return self.info

    def _random_order(self, seed):
        """A random execution order allowed by the waits alone."""
        rng = np.random.default_rng(seed)
        tasks, waits = self.p.tasks, self.p.waits
        nt = len(tasks)
        counters = np.zeros(self.p.ncounters, dtype=np.int64)
        # waiters per counter
        need = np.zeros(nt, dtype=np.int64)
        watchers = {}
        for i in range(nt):
            w0, nw = int(tasks[i]["wait_off"]), int(tasks[i]["nwait"])
            need[i] = nw
            for (cid, target) in waits[w0:w0 + nw]:
                watchers.setdefault(int(cid), []).append((i, int(target)))
        ready = [i for i in range(nt) if need[i] == 0]
        order = []
        while ready:
            j = int(rng.integers(len(ready)))
            i = ready[j]
            ready[j] = ready[-1]
            ready.pop()
            order.append(i)
            early = _early_counter(tasks[i])
            for cid in (i, int(tasks[i]["group"]), early):
                if cid < 0:
                    continue
                counters[cid] += 1
                for (w, target) in watchers.get(cid, ()):
                    if counters[cid] == target:
                        need[w] -= 1
                        if need[w] == 0:
                            ready.append(w)
        assert len(order) == nt, "task graph has unsatisfiable waits"
        return order


def dynamic_order(prog, sch, seed=0, window=4):
    """The task order of the dynamic device schedule: a finished task (and
    the early signal of a look-ahead task) releases the waiters of its
    counters; a group counter releases its waiters when it reaches its
    completion value; the next task is one of the `window` ready tasks of
    lowest list position (several CTAs claim at once), chosen at random."""
    rng = np.random.default_rng(seed)
    tasks = prog.tasks
    nt = len(tasks)
    pend = sch.npend.astype(np.int64).copy()
    count = np.zeros(len(sch.ctarget), dtype=np.int64)
    ready = sorted(int(i) for i in np.nonzero(pend == 0)[0])
    bits = np.zeros(len(sch.ready0) * 64, dtype=bool)
    bits[ready] = True
    assert np.array_equal(np.packbits(bits, bitorder="little").view(np.uint64), sch.ready0)

    def release(c, out):
        for s in sch.succ[sch.succ_off[c]:sch.succ_off[c + 1]]:
            pend[s] -= 1
            assert pend[s] >= 0
            if pend[s] == 0:
                out.append(int(s))

    # split tasks (a fused diagonal task) wait for their mid waits too: the
    # device runs them in two parts, this interpreter in one
    done = np.zeros(nt, dtype=bool)

    def mid_deps(i):
        t = tasks[i]
        if int(t["op"]) != T_POTRF or int(t["k"]) == 0:
            return []
        w0, nw, npre = int(t["wait_off"]), int(t["nwait"]), int(t["cdiag"])
        return [int(c) for c, _ in prog.waits[w0 + npre:w0 + nw]]

    order = []
    stalled = []
    while ready or stalled:
        still = [i for i in stalled if not all(done[d] for d in mid_deps(i))]
        ready = sorted(ready + [i for i in stalled if i not in still])
        stalled = still
        if not ready:
            raise AssertionError("dynamic schedule: split tasks wait on tasks that never run")
        j = int(rng.integers(min(window, len(ready))))
        i = ready.pop(j)
        if not all(done[d] for d in mid_deps(i)):
            stalled.append(i)
            continue
        done[i] = True
        order.append(i)
        new = []
        early = _early_counter(tasks[i])
        if early >= 0:
            release(early, new)
        release(i, new)
        g = int(tasks[i]["group"])
        if g >= 0:
            count[g] += 1
            assert count[g] <= sch.ctarget[g]
            if count[g] == sch.ctarget[g]:
                release(g, new)
        ready = sorted(ready + new)
    assert len(order) == nt, "dynamic schedule left tasks unreleased"
    return order
