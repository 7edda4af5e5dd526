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
//
// L_kk^{-1} is applied block by block (64 rows) with the inverses M_c of its
// diagonal tiles, computed up front and in parallel.  Each step of the
// block substitution also takes the update from the block before it, so
// the dependent chain is one task per block:
//   'N':  x_c := M_c x'_c - G_c x_{c-1},        G_c = M_c L_{c,c-1}
//   'T':  x_c := M_c^T x'_c - H_c^T x_{c+1},    H_c = L_{c+1,c} M_c
// (x'_c: x_c after the updates of the blocks further away, which run as
// independent tile products).  [-G_c | M_c] and [M_c; -H_c] are stored side
// by side per block, so that a step is one GEMM with K = 64 + the block
// width over two adjacent x tiles.  The long products (W x_k with K = nn,
// W^T u_k with K = na) are split along K into chunks of 128, partial tiles
// summed by one T_SUM task.  The extend-add and extract tasks are split by right-hand-side
// columns.
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
  const int nrt = ceil_div(nrhs, T);  // right-hand-side column tiles
  auto rw = [&](int s) { return (int)std::min<int64_t>(T, nrhs - (int64_t)s * T); };
  const int KC = 128;                 // K chunk of the split long products

  // workspace: Bp (n x nrhs, ld n); u_k (na x nrhs, ld na) per front; per
  // diagonal block c of every front the step operand ('N': [-G_c | M_c],
  // bw(c) x (64 + bw(c)) with ld bw(c), M_c alone for c = 0; 'T':
  // [M_c; -H_c], (bw(c) + bw(c+1)) x bw(c) with ld the row count, M_c alone
  // for the last block); split-K partial tiles (64 x rw(s), ld 64)
  int64_t ws = 0;
  const int64_t Bp = ws;
  ws += n * nrhs;
  std::vector<int64_t> uoff(N);
  for (int64_t k = 0; k < N; k++) {
    uoff[k] = ws;
    ws += (int64_t)P.fronts[k].na * nrhs;
  }
  std::vector<std::vector<int64_t>> soff(N);
  std::vector<std::vector<int>> sld(N);
  for (int64_t k = 0; k < N; k++) {
    const int nn = P.fronts[k].nn, NBc = ceil_div(nn, T);
    auto bw = [&](int c) { return std::min(T, nn - c * T); };
    soff[k].resize(NBc);
    sld[k].resize(NBc);
    for (int c = 0; c < NBc; c++) {
      int rows, cols;
      if (!trans) {
        rows = bw(c);
        cols = (c > 0 ? T : 0) + bw(c);
      } else {
        rows = bw(c) + (c + 1 < NBc ? bw(c + 1) : 0);
        cols = bw(c);
      }
      soff[k][c] = ws;
      sld[k][c] = rows;
      ws += (int64_t)rows * cols;
    }
  }
  auto partials = [&](int K, int width) -> int64_t {
    const int p = split_count(K, KC);
    if (p == 1) return 0;
    const int64_t o = ws;
    ws += (int64_t)p * T * width;
    return o;
  };
  // A GEMM split along K into partial tiles (ld 64, 64 x n apart) and one
  // T_SUM into C; returns the parts and the sum (parts = {sum} when K <= KC).
  auto split_gemm = [&](const Task& t, const SchedKey& key, int group, std::vector<int>& parts) -> int {
    const int p = split_count(t.k, KC);
    if (p == 1) {
      const int id = B.add(t, key, group);
      parts.push_back(id);
      return id;
    }
    const int64_t scr = partials(t.k, t.n);
    const int chunk = (t.k + p - 1) / p;
    std::vector<int> mine;
    for (int q = 0; q < p; q++) {
      const int k0 = q * chunk, kq = std::min(chunk, t.k - k0);
      Task u = t;
      u.k = kq;
      u.a = shift_k(t.a, k0);
      u.b = shift_k(t.b, k0);
      u.alpha = 1.0;
      u.beta = 0.0;
      u.cmode = CM_FULL;
      u.c = opnd(B_WS, scr + (int64_t)q * T * t.n, T);
      SchedKey kk = key;
      kk.rank = key.rank * 64 + q;
      mine.push_back(B.add(u, kk));
    }
    Task s = make_task(T_SUM);
    s.m = t.m;
    s.n = t.n;
    s.alpha = t.alpha;
    s.beta = t.beta;
    s.cmode = CM_FULL;
    s.a = opnd(B_WS, scr, T);
    s.c = t.c;
    s.aux[0] = p;
    s.aux[1] = T * t.n;
    const int out = B.add(s, key, group, 2.0 + 0.4 * p);
    for (int id : mine) {
      B.wait_task(out, id);
      parts.push_back(id);
    }
    return out;
  };

  // gather Bp = alpha B[p], 256 rows per task
  const int RCH = 256;
  const int gath = B.new_group();
  for (int64_t r0 = 0; r0 < n; r0 += RCH) {
    Task t = make_task(T_VEC);
    t.aux[0] = VEC_GATHER;
    t.aux[1] = (int32_t)r0;
    t.aux[2] = (int32_t)std::min(n, r0 + RCH);
    t.n = (int)nrhs;
    t.c = opnd(B_WS, Bp, (int)n);
    B.add(t, {-3, 0, 0, 0, (int)(r0 / RCH), 0}, gath, 1.5 + (double)RCH * nrhs / 4000.0);
  }
  // step operands of every diagonal block (independent of the sweep): the
  // inverse M_c, then G_c / H_c from it
  std::vector<std::vector<int>> inv(N), coup(N);
  for (int64_t k = 0; k < N; k++) {
    const FrontDesc& f = P.fronts[k];
    const int nn = f.nn, nj = f.nj, NBc = ceil_div(nn, T);
    auto bw = [&](int c) { return std::min(T, nn - c * T); };
    inv[k].resize(NBc);
    coup[k].assign(NBc, -1);
    for (int c = 0; c < NBc; c++) {
      const int cT = c * T;
      Task t = make_task(T_POTRF);
      t.m = t.n = bw(c);
      t.a = opnd(B_X, f.blk + (int64_t)cT * nj + cT, nj);
      // M_c: columns 64.. of [-G_c | M_c] ('N', c > 0), else the first rows
      const int64_t mo = soff[k][c] + ((!trans && c > 0) ? (int64_t)T * sld[k][c] : 0);
      t.c = opnd(B_WS, mo, sld[k][c]);
      t.aux[0] = cT;
      t.aux[1] = 1;
      t.aux[2] = 1;
      inv[k][c] = B.add(t, {-2, 0, 0, (int)k, c, 0});
    }
    for (int c = 0; c < NBc; c++) {
      const int cT = c * T;
      if (!trans && c > 0) {
        // -G_c = -M_c L_{c,c-1}  (bw(c) x 64), columns 0..63
        const int ld = sld[k][c];
        Operand a = opnd(B_WS, soff[k][c] + (int64_t)T * ld, ld);
        Operand b = opnd(B_X, f.blk + (int64_t)(cT - T) * nj + cT, nj, OM_T);
        Task g = gemm(bw(c), T, bw(c), -1.0, a, b, 0.0, opnd(B_WS, soff[k][c], ld));
        coup[k][c] = B.add(g, {-1, 0, 0, (int)k, c, 0});
        B.wait_task(coup[k][c], inv[k][c]);
      } else if (trans && c + 1 < NBc) {
        // -H_c = -L_{c+1,c} M_c  (bw(c+1) x 64), rows 64.. of [M_c; -H_c]
        const int ld = sld[k][c];
        Operand a = opnd(B_X, f.blk + (int64_t)cT * nj + cT + T, nj);
        Operand b = opnd(B_WS, soff[k][c], ld, OM_T);
        Task h = gemm(bw(c + 1), T, T, -1.0, a, b, 0.0, opnd(B_WS, soff[k][c] + T, ld));
        coup[k][c] = B.add(h, {-1, 0, 0, (int)k, c, 0});
        B.wait_task(coup[k][c], inv[k][c]);
      }
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
    // the step of block c (K spans x_{c-1}, x_c for 'N'; x_c, x_{c+1} for
    // 'T'), a T_TRSV task: its operand is staged before its mid waits
    auto step = [&](int c, int s) {
      const int ld = sld[k][c];
      Task t;
      if (!trans) {
        if (c == 0) t = gemm(bw(0), rw(s), bw(0), 1.0, opnd(B_WS, soff[k][0], ld), xop(0, s, OM_T), 0.0,
                             xop(0, s, OM_N));
        else t = gemm(bw(c), rw(s), T + bw(c), 1.0, opnd(B_WS, soff[k][c], ld), xop(c - 1, s, OM_T), 0.0,
                      xop(c, s, OM_N));
      } else {
        const int K = bw(c) + (c + 1 < NBc ? bw(c + 1) : 0);
        t = gemm(bw(c), rw(s), K, 1.0, opnd(B_WS, soff[k][c], ld, OM_T), xop(c, s, OM_T), 0.0, xop(c, s, OM_N));
      }
      t.op = T_TRSV;
      return t;
    };
    // Waits of a step: the operand's producers (and the inputs every step
    // shares) before it starts, with the step two back, so that at most two
    // steps of a chain hold a CTA; the step before and the last update of
    // its own x tile in the middle, after its operand copies are issued.
    const double STEP_US = 3.0;
    std::vector<int> last(NBc * nrt, -1);
    if (!trans) {
      // children's updates into x_k and u_k (u_k zeroed first), by columns
      int64_t elems = nj;
      for (int l = f.chbeg; l < f.chend; l++) elems += P.fronts[P.chidx[l]].na;
      const int cpt = vec_cols_per_task(elems, nrhs, nj);
      const int agrp = B.new_group();
      for (int64_t j0 = 0; j0 < nrhs; j0 += cpt) {
        Task t = make_task(T_VEC);
        t.aux[0] = VEC_ASM;
        t.aux[1] = (int32_t)k;
        t.aux[2] = (int32_t)j0;
        t.aux[3] = (int32_t)std::min<int64_t>(nrhs, j0 + cpt);
        t.n = (int)nrhs;
        t.a = opnd(B_WS, xk, (int)n);
        t.b = opnd(B_WS, uoff[0], 0);
        t.c = opnd(B_WS, uk, std::max(na, 1));
        const int id = B.add(t, {lv, 0, 0, (int)k, (int)j0, 0}, agrp,
                             1.5 + (double)elems * (t.aux[3] - t.aux[2]) / 1500.0);
        B.wait_group(id, gath);
        for (int l = f.chbeg; l < f.chend; l++) B.wait_group(id, ugrp[P.chidx[l]]);
      }
      // u_k -= W x_k (reads x_k before it is solved), split along K = nn
      std::vector<int> readers;
      for (int i = 0; i < NBb; i++)
        for (int s = 0; s < nrt; s++) {
          Operand a = opnd(B_X, blk + nn + i * T, nj);
          Operand c = opnd(B_WS, uk + i * T + (int64_t)s * T * na, na);
          std::vector<int> parts;
          const int out = split_gemm(gemm(bh(i), rw(s), nn, -1.0, a, xop(0, s, OM_T), 1.0, c),
                                     {lv, 1, 0, (int)k, s, i}, ugrp[k], parts);
          for (int id : parts) B.wait_group(id, agrp);
          B.wait_group(out, agrp);
          readers.insert(readers.end(), parts.begin(), parts.end());
        }
      // x_k := L^{-1} x_k, block forward substitution: the step of block c
      // takes the update from block c-1; the other updates are tile products
      std::vector<int> prev(nrt, -1), prev2(nrt, -1);
      for (int c = 0; c < NBc; c++) {
        for (int s = 0; s < nrt; s++) {
          const int sol = B.add(step(c, s), {lv, 2 + 2 * c, 0, (int)k, s, c}, xfinal);
          B.wait_task(sol, inv[k][c]);
          B.wait_task(sol, coup[k][c]);
          B.wait_group(sol, agrp);
          if (c == 0)
            for (int id : readers) B.wait_task(sol, id);  // the later steps follow this one
          B.wait_task(sol, prev2[s]);
          B.wait_mid(sol, last[c * nrt + s]);
          B.wait_mid(sol, prev[s]);
          B.split_task(sol, STEP_US, true);
          prev2[s] = prev[s];
          prev[s] = sol;
          for (int r = c + 2; r < NBc; r++) {
            Operand a = opnd(B_X, blk + (int64_t)(c * T) * nj + r * T, nj);
            Task u = gemm(bw(r), rw(s), bw(c), -1.0, a, xop(c, s, OM_T), 1.0, xop(r, s, OM_N));
            const int uid = B.add(u, {lv, 3 + 2 * c, 0, (int)k, s, r});
            B.wait_task(uid, sol);
            B.wait_task(uid, last[r * nrt + s]);
            last[r * nrt + s] = uid;
          }
        }
      }
    } else {
      const int from_parent = (f.parent != (int)k) ? ugrp[k] : -1;  // u_k, written by the parent
      // x_k := L^{-T} x_k, block backward substitution
      std::vector<int> prev(nrt, -1), prev2(nrt, -1);
      for (int c = NBc - 1; c >= 0; c--) {
        for (int s = 0; s < nrt; s++) {
          const int sol = B.add(step(c, s), {lv, 2 * (NBc - c), 0, (int)k, s, c}, (c == 0 && na == 0) ? xfinal : -1);
          B.wait_task(sol, inv[k][c]);
          B.wait_task(sol, coup[k][c]);
          B.wait_group(sol, gath);
          B.wait_task(sol, prev2[s]);
          B.wait_mid(sol, last[c * nrt + s]);
          B.wait_mid(sol, prev[s]);
          B.split_task(sol, STEP_US, true);
          prev2[s] = prev[s];
          prev[s] = sol;
          for (int r = 0; r + 1 < c; r++) {
            Operand a = opnd(B_X, blk + (int64_t)(r * T) * nj + c * T, nj, OM_T);
            Task u = gemm(bw(r), rw(s), bw(c), -1.0, a, xop(c, s, OM_T), 1.0, xop(r, s, OM_N));
            const int uid = B.add(u, {lv, 2 * (NBc - c) + 1, 0, (int)k, s, r});
            B.wait_task(uid, sol);
            B.wait_task(uid, last[r * nrt + s]);
            last[r * nrt + s] = uid;
          }
        }
      }
      // prev[s]: the step of block 0, which waits (transitively) on every
      // write of the rhs tile s's x blocks
      std::vector<int> wg;
      if (na > 0) {
        // x_k -= W^T u_k, split along K = na; the parts need only u_k
        for (int c = 0; c < NBc; c++)
          for (int s = 0; s < nrt; s++) {
            Operand a = opnd(B_X, blk + (int64_t)(c * T) * nj + nn, nj, OM_T);
            Operand b = opnd(B_WS, uk + (int64_t)s * T * na, na, OM_T);
            std::vector<int> parts;
            const int out = split_gemm(gemm(bw(c), rw(s), na, -1.0, a, b, 1.0, xop(c, s, OM_N)),
                                       {lv, 2 * NBc + 2, 0, (int)k, s, c}, xfinal, parts);
            for (int id : parts) B.wait_group(id, from_parent);
            B.wait_task(out, prev[s]);
            B.wait_group(out, from_parent);
            wg.push_back(out);
          }
      }
      // children's updates u_c = [x_k; u_k](r_c), by columns
      for (int l = f.chbeg; l < f.chend; l++) {
        const int c = P.chidx[l];
        const int Nc = P.fronts[c].na;
        const int cpt = vec_cols_per_task(Nc, nrhs, 0);
        for (int64_t j0 = 0; j0 < nrhs; j0 += cpt) {
          Task t = make_task(T_VEC);
          t.aux[0] = VEC_EXTRACT;
          t.aux[1] = c;
          t.aux[2] = (int32_t)j0;
          t.aux[3] = (int32_t)std::min<int64_t>(nrhs, j0 + cpt);
          t.n = (int)nrhs;
          t.a = opnd(B_WS, xk, (int)n);
          t.b = opnd(B_WS, uoff[0], 0);
          t.c = opnd(B_WS, uk, std::max(na, 1));
          const int id = B.add(t, {lv, 2 * NBc + 3, 0, (int)k, c, (int)j0}, ugrp[c],
                               1.5 + (double)Nc * (t.aux[3] - t.aux[2]) / 1500.0);
          for (int s = 0; s < nrt; s++) B.wait_task(id, prev[s]);
          for (int w : wg) B.wait_task(id, w);
          B.wait_group(id, from_parent);
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
    const int id = B.add(t, {1 << 20, 0, 0, 0, (int)(r0 / RCH), 0}, -1, 1.5 + (double)RCH * nrhs / 4000.0);
    B.wait_group(id, xfinal);
  }
  prog.ws_doubles = ws;
  return B.finish(prog, P.grid > 0 ? P.grid : 296);
}

}  // namespace chb
