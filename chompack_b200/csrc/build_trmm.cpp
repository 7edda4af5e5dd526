// Task program of the multiplication with the supernodal factor
// (reference: pybase/trmm.py:4-116, Python only):
//
//   B := alpha L B    (trans 'N', postorder)
//   B := alpha L^T B  (trans 'T', reverse postorder)
//
// L is the factor as cholesky leaves it: per supernode the diagonal block
// L_kk and W = blk21 = L21 L_kk^{-1}.  B is n x nrhs column-major in the
// original row order; it is gathered through p (alpha applied) into a
// reordered copy Bp, so that x_k = Bp[snptr[k]:snptr[k+1], :], and
// scattered back at the end, as the triangular solve does.
//
// 'N', per front k (trmm.py:55-83):
//   x_k := L_kk x_k                       (:63)
//   u_k  = W x_k                          (:65-68)
//   [x_k; u_k] += children's updates      (:70-74)
// 'T', per front k (trmm.py:87-114):
//   u_c = [x_k; u_k](r_c) per child       (:99-102), before x_k changes
//   x_k += W^T u_k                        (:104-106)
//   x_k := L_kk^T x_k                     (:109)
//
// Built from the triangular solve's tasks: 64x64 tile products (in place on
// an x tile, as the solve's diagonal steps), the vector extend-add (which
// zeroes u_k and adds the children's updates into x_k and u_k) and extract,
// and a one-part T_SUM.  The extend-add zeroes u_k, so 'N' computes W x_k
// into a second buffer u'_k first and adds it after the extend-add.
#include "dag.h"

namespace chb {

int build_trmm(const chb_plan& P, Program& prog, int64_t nrhs, bool trans) {
  const int T = TILE;
  const int64_t N = P.nsn;
  const int64_t n = P.n;
  DagBuilder B;
  if (nrhs <= 0 || n == 0) {
    prog.ws_doubles = 0;
    return B.finish(prog, 1);
  }

  // workspace: Bp (n x nrhs, ld n), u_k (na x nrhs, ld na) per front in the
  // order the vector extend-add and extract address them, then ('N') u'_k
  int64_t ws = 0;
  const int64_t Bp = ws;
  ws += n * nrhs;
  std::vector<int64_t> uoff(N), voff(N, -1);
  for (int64_t k = 0; k < N; k++) {
    uoff[k] = ws;
    ws += (int64_t)P.fronts[k].na * nrhs;
  }
  if (!trans)
    for (int64_t k = 0; k < N; k++) {
      voff[k] = ws;
      ws += (int64_t)P.fronts[k].na * nrhs;
    }
  prog.ws_doubles = ws;
  const int nrt = ceil_div(nrhs, T);  // right-hand-side column tiles
  auto rw = [&](int s) { return (int)std::min<int64_t>(T, nrhs - (int64_t)s * T); };

  // gather Bp = alpha B[p]
  const int RCH = 4096;
  const int gath = B.new_group();
  for (int64_t r0 = 0; r0 < n; r0 += RCH) {
    Task t = make_task(T_VEC);
    t.aux[0] = VEC_GATHER;
    t.aux[1] = (int32_t)r0;
    t.aux[2] = (int32_t)std::min(n, r0 + RCH);
    t.n = (int)nrhs;
    t.c = opnd(B_WS, Bp, (int)n);
    B.add(t, {-2, 0, 0, 0, (int)(r0 / RCH), 0}, gath, 2.0 + (double)RCH * nrhs / 4000.0);
  }
  // group of each front's outgoing updates: u_k ('N': the sums of u'_k
  // into u_k, read by the parent) or the children's u_c ('T': written by k's
  // extract tasks, one group per child)
  std::vector<int> ugrp(N);
  for (int64_t k = 0; k < N; k++) ugrp[k] = B.new_group();
  const int xfinal = B.new_group();  // the last writer of every x tile

  for (int64_t kk = 0; kk < N; kk++) {
    const int64_t k = trans ? N - 1 - kk : kk;
    const FrontDesc& f = P.fronts[k];
    const int nn = f.nn, na = f.na, nj = f.nj;
    const int lv = trans ? P.nlevels - f.level : f.level;
    const int NBc = ceil_div(nn, T), NBb = ceil_div(na, T);
    const int64_t blk = f.blk, xk = Bp + P.snptr[k], uk = uoff[k];
    auto bw = [&](int c) { return std::min(T, nn - c * T); };
    auto bh = [&](int i) { return std::min(T, na - i * T); };
    // x tile (c, s): rows cT.. of x_k, right-hand sides sT..
    auto xop = [&](int c, int s, uint8_t mode) {
      return opnd(B_WS, xk + c * T + (int64_t)s * T * n, (int)n, mode);
    };
    // L_kk tile (r, c), r >= c
    auto ltile = [&](int r, int c, uint8_t mode) {
      return opnd(B_X, blk + (int64_t)(c * T) * nj + r * T, nj, mode, 0);
    };
    std::vector<int> last(NBc * nrt, -1);            // last writer of x tile (c, s)
    std::vector<std::vector<int>> readers(NBc * nrt);  // products that read x tile (c, s) before it changes
    auto chain = [&](int id, int c, int s) {
      B.wait_task(id, last[c * nrt + s]);
      for (int r : readers[c * nrt + s]) B.wait_task(id, r);
      readers[c * nrt + s].clear();
      last[c * nrt + s] = id;
    };
    if (!trans) {
      // x_k := L_kk x_k in place, block rows last to first: x(r) = L(r,r) x(r)
      // + sum_{c<r} L(r,c) x(c) reads rows c < r before they change
      for (int r = NBc - 1; r >= 0; r--)
        for (int s = 0; s < nrt; s++) {
          Task d = gemm(bw(r), rw(s), bw(r), 1.0, ltile(r, r, OM_TRI_N), xop(r, s, OM_T), 0.0, xop(r, s, OM_N));
          int id = B.add(d, {lv, 2 * (NBc - r), 0, (int)k, s, r});
          B.wait_group(id, gath);
          chain(id, r, s);
          for (int c = 0; c < r; c++) {
            Task u = gemm(bw(r), rw(s), bw(c), 1.0, ltile(r, c, OM_N), xop(c, s, OM_T), 1.0, xop(r, s, OM_N));
            int uid = B.add(u, {lv, 2 * (NBc - r) + 1, 0, (int)k, s, c});
            B.wait_group(uid, gath);
            chain(uid, r, s);
            readers[c * nrt + s].push_back(uid);
          }
        }
      // u'_k = W x_k (x_k final up to the children's updates)
      std::vector<int> wg;
      for (int i = 0; i < NBb; i++)
        for (int s = 0; s < nrt; s++) {
          Operand a = opnd(B_X, blk + nn + i * T, nj);
          Operand c = opnd(B_WS, voff[k] + i * T + (int64_t)s * T * na, na);
          Task t = gemm(bh(i), rw(s), nn, 1.0, a, xop(0, s, OM_T), 0.0, c);
          int id = B.add(t, {lv, 2 * NBc + 2, 0, (int)k, s, i});
          for (int c2 = 0; c2 < NBc; c2++) B.wait_task(id, last[c2 * nrt + s]);
          wg.push_back(id);
        }
      // children's updates into x_k and u_k (u_k zeroed first); the last
      // writer of x_k
      int asm_id;
      {
        Task t = make_task(T_VEC);
        t.aux[0] = VEC_ASM;
        t.aux[1] = (int32_t)k;
        t.n = (int)nrhs;
        t.a = opnd(B_WS, xk, (int)n);
        t.b = opnd(B_WS, uoff[0], 0);
        t.c = opnd(B_WS, uk, std::max(na, 1));
        asm_id = B.add(t, {lv, 2 * NBc + 3, 0, (int)k, 0, 0}, xfinal, 2.0 + (double)nj * nrhs / 2000.0);
        B.wait_group(asm_id, gath);
        for (int id : last) B.wait_task(asm_id, id);
        for (int id : wg) B.wait_task(asm_id, id);
        for (int l = f.chbeg; l < f.chend; l++) B.wait_group(asm_id, ugrp[P.chidx[l]]);
      }
      // u_k += u'_k, tile by tile
      for (int i = 0; i < NBb; i++)
        for (int s = 0; s < nrt; s++) {
          Task t = make_task(T_SUM);
          t.m = bh(i);
          t.n = rw(s);
          t.alpha = 1.0;
          t.beta = 1.0;
          t.a = opnd(B_WS, voff[k] + i * T + (int64_t)s * T * na, na);
          t.c = opnd(B_WS, uk + i * T + (int64_t)s * T * na, na);
          t.aux[0] = 1;
          t.aux[1] = 0;
          int id = B.add(t, {lv, 2 * NBc + 4, 0, (int)k, s, i}, ugrp[k], 3.5);
          B.wait_task(id, asm_id);
        }
    } else {
      const int from_parent = (f.parent != (int)k) ? ugrp[k] : -1;  // u_k, written by the parent
      // children's updates u_c = [x_k; u_k](r_c), from the values before
      // x_k changes
      std::vector<int> ex;
      for (int l = f.chbeg; l < f.chend; l++) {
        const int c = P.chidx[l];
        Task t = make_task(T_VEC);
        t.aux[0] = VEC_EXTRACT;
        t.aux[1] = c;
        t.n = (int)nrhs;
        t.a = opnd(B_WS, xk, (int)n);
        t.b = opnd(B_WS, uoff[0], 0);
        t.c = opnd(B_WS, uk, std::max(na, 1));
        int id = B.add(t, {lv, 0, 0, (int)k, c, 0}, ugrp[c], 2.0 + (double)P.fronts[c].na * nrhs / 2000.0);
        B.wait_group(id, gath);
        B.wait_group(id, from_parent);
        ex.push_back(id);
      }
      // x_k += W^T u_k
      for (int c = 0; c < NBc; c++)
        for (int s = 0; s < nrt; s++) {
          if (na == 0) continue;
          Operand a = opnd(B_X, blk + (int64_t)(c * T) * nj + nn, nj, OM_T);
          Operand b = opnd(B_WS, uk + (int64_t)s * T * na, na, OM_T);
          Task t = gemm(bw(c), rw(s), na, 1.0, a, b, 1.0, xop(c, s, OM_N));
          int id = B.add(t, {lv, 1, 0, (int)k, s, c});
          B.wait_group(id, gath);
          B.wait_group(id, from_parent);
          for (int e : ex) B.wait_task(id, e);
          chain(id, c, s);
        }
      // x_k := L_kk^T x_k in place, block rows first to last: x(r) =
      // L(r,r)^T x(r) + sum_{c>r} L(c,r)^T x(c) reads rows c > r before they
      // change
      for (int r = 0; r < NBc; r++)
        for (int s = 0; s < nrt; s++) {
          Task d = gemm(bw(r), rw(s), bw(r), 1.0, ltile(r, r, OM_TRI_T), xop(r, s, OM_T), 0.0, xop(r, s, OM_N));
          const bool last_of_row = r == NBc - 1;
          int id = B.add(d, {lv, 2 + 2 * r, 0, (int)k, s, r}, last_of_row ? xfinal : -1);
          B.wait_group(id, gath);
          for (int e : ex) B.wait_task(id, e);
          chain(id, r, s);
          for (int c = r + 1; c < NBc; c++) {
            Task u = gemm(bw(r), rw(s), bw(c), 1.0, ltile(c, r, OM_T), xop(c, s, OM_T), 1.0, xop(r, s, OM_N));
            int uid = B.add(u, {lv, 3 + 2 * r, 0, (int)k, s, c}, c == NBc - 1 ? xfinal : -1);
            for (int e : ex) B.wait_task(uid, e);
            B.wait_task(uid, last[c * nrt + s]);  // x(c) has its W^T u_k part
            chain(uid, r, s);
            readers[c * nrt + s].push_back(uid);
          }
        }
    }
  }
  // scatter back B[p] = Bp (every x tile has its last writer in xfinal)
  for (int64_t r0 = 0; r0 < n; r0 += RCH) {
    Task t = make_task(T_VEC);
    t.aux[0] = VEC_SCATTER;
    t.aux[1] = (int32_t)r0;
    t.aux[2] = (int32_t)std::min(n, r0 + RCH);
    t.n = (int)nrhs;
    t.c = opnd(B_WS, Bp, (int)n);
    int id = B.add(t, {1 << 20, 0, 0, 0, (int)(r0 / RCH), 0}, -1, 2.0 + (double)RCH * nrhs / 4000.0);
    B.wait_group(id, xfinal);
  }
  return B.finish(prog, P.grid > 0 ? P.grid : 296);
}

}  // namespace chb
