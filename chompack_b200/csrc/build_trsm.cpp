// Task program of the supernodal triangular solve (reference: trsm.c:3-139).
//
//   B := alpha L^{-1} B  (trans 'N', postorder)
//   B := alpha L^{-T} B  (trans 'T', reverse postorder)
//
// B is n x nrhs column-major in the original row order (leading dimension
// given at run time).  It is gathered through p into a reordered copy Bp, so
// that the rows of supernode k are contiguous (x_k = Bp[snptr[k]:snptr[k+1],
// :]), solved there and scattered back.  alpha is applied by the gather, as
// trsm.c:35-37 does.
//
// 'N', per front k:  x_k, u_k += children's updates   (trsm.c:44-53)
//                    u_k -= W x_k                     (:57)
//                    x_k := L_kk^{-1} x_k              (:63)
// 'T', per front k:  x_k := L_kk^{-T} x_k              (:97)
//                    x_k -= W^T u_k                   (:104)
//                    u_c = [x_k; u_k](r_c) per child  (:108-116)
// L_kk^{-1} is applied block by block with the inverses of its 64x64
// diagonal tiles (computed up front, in parallel) and rank-64 updates.
#include "dag.h"

namespace chb {

int build_trsm(const chb_plan& P, Program& prog, int64_t nrhs, bool trans) {
  const int T = TILE;
  const int64_t N = P.nsn;
  const int64_t n = P.n;
  DagBuilder B;
  if (nrhs <= 0 || n == 0) {
    prog.ws_doubles = 0;
    return B.finish(prog, 1);
  }

  // workspace: Bp (n x nrhs, ld n), u_k (na x nrhs, ld na) per front, the
  // diagonal-tile inverses (nn x 64 per front, tile c at rows cT)
  int64_t ws = 0;
  const int64_t Bp = ws;
  ws += n * nrhs;
  std::vector<int64_t> uoff(N), moff(N);
  for (int64_t k = 0; k < N; k++) {
    uoff[k] = ws;
    ws += (int64_t)P.fronts[k].na * nrhs;
  }
  for (int64_t k = 0; k < N; k++) {
    moff[k] = ws;
    ws += (int64_t)P.fronts[k].nn * T;
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
  // inverses of the diagonal tiles of every L_kk (independent of the sweep)
  std::vector<std::vector<int>> inv(N);
  for (int64_t k = 0; k < N; k++) {
    const FrontDesc& f = P.fronts[k];
    const int NBc = ceil_div(f.nn, T);
    inv[k].resize(NBc);
    for (int c = 0; c < NBc; c++) {
      const int cT = c * T;
      Task t = make_task(T_POTRF);
      t.m = t.n = std::min(T, f.nn - cT);
      t.a = opnd(B_X, f.blk + (int64_t)cT * f.nj + cT, f.nj);
      t.c = opnd(B_WS, moff[k] + cT, f.nn);
      t.aux[0] = cT;
      t.aux[1] = 1;
      t.aux[2] = 1;
      inv[k][c] = B.add(t, {-1, 0, 0, (int)k, c, 0});
    }
  }
  // group of each front's outgoing updates: u_k ('N', read by the parent) or
  // the children's u_c ('T', written by k's extract tasks, group per child)
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
    std::vector<int> last(NBc * nrt, -1);
    if (!trans) {
      // children's updates into x_k and u_k (u_k zeroed first)
      int asm_id;
      {
        Task t = make_task(T_VEC);
        t.aux[0] = VEC_ASM;
        t.aux[1] = (int32_t)k;
        t.n = (int)nrhs;
        t.a = opnd(B_WS, xk, (int)n);
        t.b = opnd(B_WS, uoff[0], 0);
        t.c = opnd(B_WS, uk, std::max(na, 1));
        asm_id = B.add(t, {lv, 0, 0, (int)k, 0, 0}, -1, 2.0 + (double)nj * nrhs / 2000.0);
        B.wait_group(asm_id, gath);
        for (int l = f.chbeg; l < f.chend; l++) B.wait_group(asm_id, ugrp[P.chidx[l]]);
      }
      // u_k -= W x_k (reads x_k before it is solved)
      std::vector<int> ug;
      for (int i = 0; i < NBb; i++)
        for (int s = 0; s < nrt; s++) {
          Operand a = opnd(B_X, blk + nn + i * T, nj);
          Operand c = opnd(B_WS, uk + i * T + (int64_t)s * T * na, na);
          Task t = gemm(bh(i), rw(s), nn, -1.0, a, xop(0, s, OM_T), 1.0, c);
          int id = B.add(t, {lv, 1, 0, (int)k, s, i}, ugrp[k]);
          B.wait_task(id, asm_id);
          ug.push_back(id);
        }
      // x_k := L^{-1} x_k, block forward substitution
      for (int c = 0; c < NBc; c++) {
        for (int s = 0; s < nrt; s++) {
          Operand m = opnd(B_WS, moff[k] + c * T, nn, OM_TRI_N, 0);
          Task t = gemm(bw(c), rw(s), bw(c), 1.0, m, xop(c, s, OM_T), 0.0, xop(c, s, OM_N));
          int sol = B.add(t, {lv, 2 + 2 * c, 0, (int)k, s, c}, xfinal);
          B.wait_task(sol, inv[k][c]);
          B.wait_task(sol, asm_id);
          for (int id : ug) B.wait_task(sol, id);
          B.wait_task(sol, last[c * nrt + s]);
          for (int r = c + 1; r < NBc; r++) {
            Operand a = opnd(B_X, blk + (int64_t)(c * T) * nj + r * T, nj);
            Task u = gemm(bw(r), rw(s), bw(c), -1.0, a, xop(c, s, OM_T), 1.0, xop(r, s, OM_N));
            int uid = B.add(u, {lv, 3 + 2 * c, 0, (int)k, s, r});
            B.wait_task(uid, sol);
            B.wait_task(uid, last[r * nrt + s]);
            last[r * nrt + s] = uid;
          }
        }
      }
    } else {
      const int from_parent = (f.parent != (int)k) ? ugrp[k] : -1;  // u_k, written by the parent
      // x_k := L^{-T} x_k, block backward substitution
      std::vector<int> head(nrt, -1);  // last task of the chain per rhs tile
      for (int c = NBc - 1; c >= 0; c--) {
        for (int s = 0; s < nrt; s++) {
          Operand m = opnd(B_WS, moff[k] + c * T, nn, OM_TRI_T, 0);
          Task t = gemm(bw(c), rw(s), bw(c), 1.0, m, xop(c, s, OM_T), 0.0, xop(c, s, OM_N));
          int sol = B.add(t, {lv, 2 * (NBc - c), 0, (int)k, s, c}, (c == 0 && na == 0) ? xfinal : -1);
          B.wait_task(sol, inv[k][c]);
          B.wait_group(sol, gath);
          B.wait_task(sol, last[c * nrt + s]);
          head[s] = sol;
          for (int r = 0; r < c; r++) {
            Operand a = opnd(B_X, blk + (int64_t)(r * T) * nj + c * T, nj, OM_T);
            Task u = gemm(bw(r), rw(s), bw(c), -1.0, a, xop(c, s, OM_T), 1.0, xop(r, s, OM_N));
            int uid = B.add(u, {lv, 2 * (NBc - c) + 1, 0, (int)k, s, r});
            B.wait_task(uid, sol);
            B.wait_task(uid, last[r * nrt + s]);
            last[r * nrt + s] = uid;
          }
        }
      }
      // the chain of rhs tile s ends with the solve of block 0; it waits
      // (transitively) on every update of that tile
      std::vector<int> wg;
      if (na > 0) {
        // x_k -= W^T u_k
        for (int c = 0; c < NBc; c++)
          for (int s = 0; s < nrt; s++) {
            Operand a = opnd(B_X, blk + (int64_t)(c * T) * nj + nn, nj, OM_T);
            Operand b = opnd(B_WS, uk + (int64_t)s * T * na, na, OM_T);
            Task t = gemm(bw(c), rw(s), na, -1.0, a, b, 1.0, xop(c, s, OM_N));
            int id = B.add(t, {lv, 2 * NBc + 2, 0, (int)k, s, c}, xfinal);
            B.wait_task(id, head[s]);
            B.wait_group(id, from_parent);
            wg.push_back(id);
          }
      }
      // children's updates u_c = [x_k; u_k](r_c)
      for (int l = f.chbeg; l < f.chend; l++) {
        const int c = P.chidx[l];
        Task t = make_task(T_VEC);
        t.aux[0] = VEC_EXTRACT;
        t.aux[1] = c;
        t.n = (int)nrhs;
        t.a = opnd(B_WS, xk, (int)n);
        t.b = opnd(B_WS, uoff[0], 0);
        t.c = opnd(B_WS, uk, std::max(na, 1));
        int id = B.add(t, {lv, 2 * NBc + 3, 0, (int)k, c, 0}, ugrp[c],
                       2.0 + (double)P.fronts[c].na * nrhs / 2000.0);
        for (int s = 0; s < nrt; s++) B.wait_task(id, head[s]);
        for (int w : wg) B.wait_task(id, w);
        B.wait_group(id, from_parent);
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
