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
// block substitution also takes the updates from the two blocks before it,
// so the dependent chain is one task per block:
//   'N':  x_c := M_c x'_c - G_c x_{c-1} - G2_c x_{c-2},
//         G_c = M_c L_{c,c-1},  G2_c = M_c L_{c,c-2}
//   'T':  x_c := M_c^T x'_c - H_c^T x_{c+1} - H2_c^T x_{c+2},
//         H_c = L_{c+1,c} M_c,  H2_c = L_{c+2,c} M_c
// (x'_c: x_c after the updates from the blocks further away).
// [-G2_c | -G_c | M_c] and [M_c; -H_c; -H2_c] are stored per block, so that
// a step is one product with K up to 192 over adjacent x tiles, a T_TRSV
// task whose operand is staged before it waits for its predecessor.
//
// Everything that only adds into a vector block runs as independent tasks
// with atomic adds (CM_ATOMIC products, VEC_ADD), so that no chain of
// read-modify-write tasks forms on one block: the far updates of the block
// substitution, the long products W x_k (K = nn) and W^T u_k (K = na) in
// chunks of 128, and the children's updates into [x_k; u_k] (split by
// right-hand-side columns and row chunks).  The order of those additions
// varies from run to run, so the last bits of the solution may too.
#include "dag.h"

namespace chb {

int build_trsm(const chb_plan& P, Program& prog, int64_t nrhs, bool trans, bool reuse) {
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
  // diagonal block c of every front the step operand ('N': [-G2_c | -G_c |
  // M_c], bw(c) x (64 min(c, 2) + bw(c)) with ld bw(c); 'T': [M_c; -H_c;
  // -H2_c], (bw(c) + bw(c+1) + bw(c+2)) x bw(c) with ld the row count, the
  // blocks that exist); split-K partial tiles (64 x rw(s), ld 64)
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
        cols = T * std::min(c, 2) + bw(c);
      } else {
        rows = bw(c) + (c + 1 < NBc ? bw(c + 1) : 0) + (c + 2 < NBc ? bw(c + 2) : 0);
        cols = bw(c);
      }
      soff[k][c] = ws;
      sld[k][c] = rows;
      ws += (int64_t)rows * cols;
    }
  }
  const bool ordered = ordered_sums(P);
  // Ordered mode: a long product split along K into partial tiles (ld 64,
  // 64 x n apart) and one T_SUM into C; returns the sum task and appends
  // the parts (parts = {sum} when K <= KC).
  auto split_gemm = [&](const Task& t, const SchedKey& key, int group, std::vector<int>& parts) -> int {
    const int p = split_count(t.k, KC);
    if (p == 1) {
      const int id = B.add(t, key, group);
      parts.push_back(id);
      return id;
    }
    const int64_t scr = ws;
    ws += (int64_t)p * T * t.n;
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
    Task sm = make_task(T_SUM);
    sm.m = t.m;
    sm.n = t.n;
    sm.alpha = t.alpha;
    sm.beta = t.beta;
    sm.cmode = CM_FULL;
    sm.a = opnd(B_WS, scr, T);
    sm.c = t.c;
    sm.aux[0] = p;
    sm.aux[1] = T * t.n;
    const int out = B.add(sm, key, group, 2.0 + 0.4 * p);
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
  // inverse M_c, then G_c, G2_c / H_c, H2_c from it.  With `reuse` they are
  // left in the workspace by an earlier solve with the same factor, trans
  // and nrhs, and each of their tasks is a no-op: the program keeps the
  // same tasks and counters, so its workspace has the same layout
  auto add_step_operand = [&](const Task& t, const SchedKey& key) {
    if (!reuse) return B.add(t, key);
    return B.add(make_task(T_NOP), key, -1, 0.3);
  };
  std::vector<std::vector<int>> inv(N);
  std::vector<std::vector<std::array<int, 2>>> coup(N);
  for (int64_t k = 0; k < N; k++) {
    const FrontDesc& f = P.fronts[k];
    const int nn = f.nn, nj = f.nj, NBc = ceil_div(nn, T);
    auto bw = [&](int c) { return std::min(T, nn - c * T); };
    inv[k].assign(NBc, -1);
    coup[k].assign(NBc, {-1, -1});
    for (int c = 0; c < NBc; c++) {
      const int cT = c * T;
      Task t = make_task(T_POTRF);
      t.m = t.n = bw(c);
      t.a = opnd(B_X, f.blk + (int64_t)cT * nj + cT, nj);
      // M_c: the last columns of the 'N' operand, the first rows of the 'T' one
      const int64_t mo = soff[k][c] + (!trans ? (int64_t)T * std::min(c, 2) * sld[k][c] : 0);
      t.c = opnd(B_WS, mo, sld[k][c]);
      t.aux[0] = cT;
      t.aux[1] = 1;
      t.aux[2] = 1;
      inv[k][c] = add_step_operand(t, {-2, 0, 0, (int)k, c, 0});
    }
    for (int c = 0; c < NBc; c++) {
      const int cT = c * T, ld = sld[k][c];
      for (int d = 1; d <= 2; d++) {
        if (!trans && c >= d) {
          // -G_c (d = 1) / -G2_c (d = 2) = -M_c L_{c,c-d}  (bw(c) x 64), in
          // the columns just before M_c's (d = 1) or before those (d = 2)
          const int64_t mcol = (int64_t)T * std::min(c, 2);
          Operand a = opnd(B_WS, soff[k][c] + mcol * ld, ld);
          Operand b = opnd(B_X, f.blk + (int64_t)(cT - d * T) * nj + cT, nj, OM_T);
          Task g = gemm(bw(c), T, bw(c), -1.0, a, b, 0.0, opnd(B_WS, soff[k][c] + (mcol - (int64_t)d * T) * ld, ld));
          coup[k][c][d - 1] = add_step_operand(g, {-1, 0, 0, (int)k, c, d});
          B.wait_task(coup[k][c][d - 1], inv[k][c]);
        } else if (trans && c + d < NBc) {
          // -H_c (d = 1) / -H2_c (d = 2) = -L_{c+d,c} M_c  (bw(c+d) x 64),
          // rows 64 d.. of [M_c; -H_c; -H2_c] (blocks below the last are full)
          Operand a = opnd(B_X, f.blk + (int64_t)cT * nj + cT + d * T, nj);
          Operand b = opnd(B_WS, soff[k][c], ld, OM_T);
          Task h = gemm(bw(c + d), T, T, -1.0, a, b, 0.0, opnd(B_WS, soff[k][c] + d * T, ld));
          coup[k][c][d - 1] = add_step_operand(h, {-1, 0, 0, (int)k, c, d});
          B.wait_task(coup[k][c][d - 1], inv[k][c]);
        }
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
    // the step of block c (K spans x_{c-2}, x_{c-1}, x_c for 'N'; x_c,
    // x_{c+1}, x_{c+2} for 'T', those that exist), a T_TRSV task: its
    // operand is staged before its mid waits
    auto step = [&](int c, int s) {
      const int ld = sld[k][c];
      Task t;
      if (!trans) {
        const int back = std::min(c, 2);
        t = gemm(bw(c), rw(s), T * back + bw(c), 1.0, opnd(B_WS, soff[k][c], ld), xop(c - back, s, OM_T), 0.0,
                 xop(c, s, OM_N));
      } else {
        t = gemm(bw(c), rw(s), ld, 1.0, opnd(B_WS, soff[k][c], ld, OM_T), xop(c, s, OM_T), 0.0, xop(c, s, OM_N));
      }
      t.op = T_TRSV;
      return t;
    };
    // Waits of a step: the operand's producers, the inputs every step
    // shares, the step two back (so that at most two steps of a chain hold a
    // CTA) and the far updates of its own x tile (from the blocks three or
    // more away, done by then) before it starts; the step before in the
    // middle, after its operand copies are issued.  The far updates of an x
    // tile are independent tile products that add into it with atomics
    // (CM_ATOMIC), each as soon as its block is solved, so that no chain of
    // updates forms behind the steps; a group per tile collects them.
    // (Ordered mode: the far updates of a tile form a chain, each waiting
    // for the one before, and the step waits for the last one in the middle.)
    const double STEP_US = 3.0;
    std::vector<int> far(NBc * nrt, -1);
    std::vector<int> nfar(NBc * nrt, 0), lastu(NBc * nrt, -1);
    if (!ordered)
      for (int i = 0; i < NBc * nrt; i++) far[i] = B.new_group();
    auto far_update = [&](const Operand& a, int r, int c, int s, const SchedKey& key, int sol) {
      Task u = gemm(bw(r), rw(s), bw(c), -1.0, a, xop(c, s, OM_T), 1.0, xop(r, s, OM_N));
      if (!ordered) u.cmode = CM_ATOMIC;
      const int uid = B.add(u, key, far[r * nrt + s]);
      nfar[r * nrt + s]++;
      B.wait_task(uid, sol);
      if (ordered) {
        B.wait_task(uid, lastu[r * nrt + s]);
        lastu[r * nrt + s] = uid;
      }
    };
    auto wait_far = [&](int sol, int c, int s) {
      if (ordered) B.wait_mid(sol, lastu[c * nrt + s]);
      else if (nfar[c * nrt + s] > 0) B.wait_group(sol, far[c * nrt + s]);
    };
    // Column groups and row chunks of the extract / add tasks of child c
    auto child_tasks = [&](int c, int mode, const SchedKey& key0, int group, const std::vector<int>& deps,
                           const std::vector<int>& gdeps, int skip_group) {
      const int Nc = P.fronts[c].na;
      const int cpt = vec_cols_per_task(Nc, nrhs, 0);
      const int rows = std::max(256, (int)(2048 / std::max<int64_t>(1, std::min<int64_t>(cpt, nrhs))));
      for (int64_t j0 = 0; j0 < nrhs; j0 += cpt)
        for (int i0 = 0; i0 < Nc; i0 += rows) {
          Task t = make_task(T_VEC);
          t.aux[0] = mode;
          t.aux[1] = c;
          t.aux[2] = (int32_t)j0;
          t.aux[3] = (int32_t)std::min<int64_t>(nrhs, j0 + cpt);
          t.m = i0;
          t.k = std::min(Nc, i0 + rows);
          t.n = (int)nrhs;
          t.a = opnd(B_WS, xk, (int)n);
          t.b = opnd(B_WS, uoff[0], 0);
          t.c = opnd(B_WS, uk, std::max(na, 1));
          SchedKey key = key0;
          key.j = (int)j0;
          key.i = i0;
          const int id = B.add(t, key, group, 1.5 + (double)(t.k - t.m) * (t.aux[3] - t.aux[2]) / 1500.0);
          for (int d : deps) B.wait_task(id, d);
          for (int g : gdeps)
            if (g != skip_group) B.wait_group(id, g);
        }
    };
    if (!trans) {
      // u_k zeroed; the children's updates added into x_k and u_k with
      // atomics (one task per child, column group and row chunk, all at
      // once); u_k -= W x_k as partial products that add into u_k with
      // atomics (no sum task), after x_k is complete.  Ordered mode: one
      // extend-add task per column group adds the children in order, and
      // the products go through partial tiles and a sum.
      int zero = -1;
      const int agrp = B.new_group();
      int nadd = 0;
      std::vector<int> readers;  // ordered mode: the products that read x_k
      if (ordered) {
        // the children's updates added in order (last child first, as the
        // reference pops its stack), staged in shared memory per column
        // group; the task zeroes u_k's columns first
        int64_t elems = nj;
        for (int l = f.chbeg; l < f.chend; l++) elems += P.fronts[P.chidx[l]].na;
        const int cpt = vec_cols_per_task(elems, nrhs, nj);
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
          nadd++;
        }
      } else if (na > 0) {
        Task t = make_task(T_VEC);
        t.aux[0] = VEC_ZERO;
        t.m = na;
        t.n = (int)nrhs;
        t.c = opnd(B_WS, uk, na);
        zero = B.add(t, {-3, 1, 0, (int)k, 0, 0}, -1, 1.0 + (double)na * nrhs / 20000.0);
      }
      for (int l = f.chbeg; l < f.chend && !ordered; l++) {
        const int c = P.chidx[l];
        std::vector<int> deps;
        if (zero >= 0) deps.push_back(zero);
        child_tasks(c, VEC_ADD, {lv, 0, 0, (int)k, 0, 0}, agrp, deps, {gath, ugrp[c]}, -1);
        nadd++;
      }
      // x_k is complete after the gather and the adds
      auto wait_x = [&](int id) {
        B.wait_group(id, gath);
        if (nadd > 0) B.wait_group(id, agrp);
      };
      // u_k -= W x_k (reads x_k before it is solved), K = nn in chunks of
      // KC, each chunk's product added into u_k
      int nread = 0;
      for (int i = 0; i < NBb && ordered; i++)
        for (int s = 0; s < nrt; s++) {
          Operand a = opnd(B_X, blk + nn + i * T, nj);
          Operand c = opnd(B_WS, uk + i * T + (int64_t)s * T * na, na);
          std::vector<int> parts;
          const int out = split_gemm(gemm(bh(i), rw(s), nn, -1.0, a, xop(0, s, OM_T), 1.0, c),
                                     {lv, 1, 0, (int)k, s, i}, ugrp[k], parts);
          for (int id : parts) wait_x(id);
          wait_x(out);
          readers.insert(readers.end(), parts.begin(), parts.end());
        }
      for (int i = 0; i < NBb && !ordered; i++)
        for (int s = 0; s < nrt; s++)
          for (int k0 = 0; k0 < nn; k0 += KC) {
            const int kq = std::min(KC, nn - k0);
            Operand a = opnd(B_X, blk + nn + i * T + (int64_t)k0 * nj, nj);
            Operand c = opnd(B_WS, uk + i * T + (int64_t)s * T * na, na);
            Task u = gemm(bh(i), rw(s), kq, -1.0, a, shift_k(xop(0, s, OM_T), k0), 1.0, c);
            u.cmode = CM_ATOMIC;
            const int id = B.add(u, {lv, 1, 0, (int)k, s, i}, ugrp[k]);
            wait_x(id);
            B.wait_task(id, zero);
            nread++;
          }
      // x_k := L^{-1} x_k, block forward substitution: the step of block c
      // takes the updates from blocks c-1 and c-2; the others are tile
      // products that add into their x tile
      std::vector<int> prev(nrt, -1), prev2(nrt, -1);
      for (int c = 0; c < NBc; c++) {
        for (int s = 0; s < nrt; s++) {
          const int sol = B.add(step(c, s), {lv, 2 + 2 * c, 0, (int)k, s, c}, xfinal);
          B.wait_task(sol, inv[k][c]);
          B.wait_task(sol, coup[k][c][0]);
          B.wait_task(sol, coup[k][c][1]);
          wait_x(sol);
          if (c == 0 && nread > 0) B.wait_group(sol, ugrp[k]);  // the products that read x_k first
          if (c == 0)
            for (int id : readers) B.wait_task(sol, id);
          B.wait_task(sol, prev2[s]);
          wait_far(sol, c, s);
          B.wait_mid(sol, prev[s]);
          B.split_task(sol, STEP_US, true);
          prev2[s] = prev[s];
          prev[s] = sol;
          for (int r = c + 3; r < NBc; r++)
            far_update(opnd(B_X, blk + (int64_t)(c * T) * nj + r * T, nj), r, c, s, {lv, 3 + 2 * c, 0, (int)k, s, r},
                       sol);
        }
      }
    } else {
      const int from_parent = (f.parent != (int)k) ? ugrp[k] : -1;  // u_k, written by the parent
      // x_k := L^{-T} x_k, block backward substitution
      std::vector<int> prev(nrt, -1), prev2(nrt, -1);
      for (int c = NBc - 1; c >= 0; c--) {
        for (int s = 0; s < nrt; s++) {
          const int sol = B.add(step(c, s), {lv, 2 * (NBc - c), 0, (int)k, s, c}, na == 0 && c == 0 ? xfinal : -1);
          B.wait_task(sol, inv[k][c]);
          B.wait_task(sol, coup[k][c][0]);
          B.wait_task(sol, coup[k][c][1]);
          B.wait_group(sol, gath);
          B.wait_task(sol, prev2[s]);
          wait_far(sol, c, s);
          B.wait_mid(sol, prev[s]);
          B.split_task(sol, STEP_US, true);
          prev2[s] = prev[s];
          prev[s] = sol;
          for (int r = 0; r + 2 < c; r++)
            far_update(opnd(B_X, blk + (int64_t)(r * T) * nj + c * T, nj, OM_T), r, c, s,
                       {lv, 2 * (NBc - c) + 1, 0, (int)k, s, r}, sol);
        }
      }
      // prev[s]: the step of block 0, the end of the chain of rhs tile s
      // (every read and write of its x tiles by the chain precedes it)
      int xdone = -1;
      std::vector<int> chain_end;
      if (na > 0 && ordered) {
        // x_k -= W^T u_k split along K = na into partial tiles and a sum
        // per x tile, the last writer of the tile
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
            chain_end.push_back(out);
          }
      } else if (na > 0) {
        // x_k -= W^T u_k, K = na in chunks of KC, each chunk's product added
        // into the x tile after the chain; then one no-op marks x_k final
        xdone = B.new_group();
        for (int c = 0; c < NBc; c++)
          for (int s = 0; s < nrt; s++)
            for (int k0 = 0; k0 < na; k0 += KC) {
              const int kq = std::min(KC, na - k0);
              Operand a = opnd(B_X, blk + (int64_t)(c * T) * nj + nn + k0, nj, OM_T);
              Operand b = opnd(B_WS, uk + (int64_t)s * T * na + k0, na, OM_T);
              Task t = gemm(bw(c), rw(s), kq, -1.0, a, b, 1.0, xop(c, s, OM_N));
              t.cmode = CM_ATOMIC;
              const int id = B.add(t, {lv, 2 * NBc + 2, 0, (int)k, s, c}, xdone);
              B.wait_task(id, prev[s]);
              B.wait_group(id, from_parent);
            }
        Task nop = make_task(T_NOP);
        const int id = B.add(nop, {lv, 2 * NBc + 3, 0, (int)k, 0, 0}, xfinal, 0.5);
        B.wait_group(id, xdone);
      } else {
        chain_end = prev;
      }
      // children's updates u_c = [x_k; u_k](r_c), by column groups and row chunks
      for (int l = f.chbeg; l < f.chend; l++) {
        const int c = P.chidx[l];
        std::vector<int> gd = {xdone, from_parent};
        child_tasks(c, VEC_EXTRACT, {lv, 2 * NBc + 4, 0, (int)k, c, 0}, ugrp[c], chain_end, gd, -1);
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
