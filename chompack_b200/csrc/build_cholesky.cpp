// Task program of the multifrontal Cholesky sweep (reference: cholesky.c:3-84).
//
// Per supernode k (front F = [blkval panel P, nj x nn, ld nj | update U_k,
// na x na, ld na]) the reference does
//   F := [blk, 0] + extend-add(children's U)          (cholesky.c:33-52)
//   L11 = potrf(F11)                                  (:55)
//   L21 = F21 * L11^{-T}                              (:61)
//   U_k = F22 - L21 * L21^T                           (:64-69)
//   blk21 = L21 * L11^{-1}                            (:72)
// Here the nn columns are processed in 64-wide column blocks, right-looking:
// POTRF of the diagonal tile (which also writes M_cc = L_cc^{-1}), TRSM of the
// tiles below it as a GEMM with M_cc^T, and rank-64 updates of the tiles to
// the right.  L21 goes to scratch S_k (na x nn), the Schur update U_k -= S S^T
// is one K = nn GEMM per tile, and the second triangular solve becomes
// blk21 = S_k * M with M = L11^{-1} assembled block-row by block-row
// (M(c, j) = -M_cc * sum_{l=j}^{c-1} L(c, l) M(l, j)), so no tile of it has a
// sequential dependency on its neighbours.
#include <cstdlib>

#include "dag.h"

namespace chb {

int build_cholesky(const chb_plan& P, Program& prog) {
  const int T = TILE;
  const int small_nj = small_front_nj(P);
  const int CH = 64;  // at most this many front columns per extend-add task
  const int64_t N = P.nsn;
  DagBuilder B;

  // workspace: update matrices first (shared layout), then per-front scratch
  int64_t ws = P.upd_total;
  const int kc = chol_ksplit(P);
  std::vector<int64_t> scrS(N, -1), scrM(N, -1), scrK(N, -1);
  for (int64_t k = 0; k < N; k++) {
    const FrontDesc& f = P.fronts[k];
    const int NBc = ceil_div(f.nn, T);
    if (f.nj <= small_nj) continue;  // a small front needs no scratch (one shared-memory task)
    if (f.na > 0) {
      scrS[k] = ws;
      ws += (int64_t)f.na * f.nn;
    }
    if (NBc > 1 || f.na > 0) {
      scrM[k] = ws;
      ws += (int64_t)f.nn * f.nn;
    }
    if (f.na > 0 && kc > 0 && split_count(f.nn, kc) > 1) {
      // partial products of the split Schur-complement tiles
      const int64_t NBb = ceil_div(f.na, T);
      scrK[k] = ws;
      ws += NBb * (NBb + 1) / 2 * split_count(f.nn, kc) * (int64_t)T * T;
    }
  }
  prog.ws_doubles = ws;
  // pooled update matrices (under a scratch limit): U_k is first written by
  // front k's extend-add tasks (or its one-task front, or its bundle) and
  // dead once the parent's extend-add has read it.  Front k's scratch
  // (S_k, M_k and the split partials, contiguous) is pooled too: first
  // touched after its extend-add tasks (or its first diagonal task), dead
  // once its Schur complement (group uc_group[k]) and its blk21 products
  // are done, or, for a front without update, its last diagonal task,
  // which follows every other task of the front.
  const std::vector<int> ubuf = pool_update_matrices(P, prog, B);
  std::vector<int> sbuf(N, -1);
  if (B.pool_limit >= 0) {
    for (int64_t k = 0; k < N; k++) {
      int64_t lo = -1, hi = -1;
      for (int64_t o : {scrS[k], scrM[k], scrK[k]})
        if (o >= 0) lo = lo < 0 ? o : std::min(lo, o);
      if (lo < 0) continue;
      const FrontDesc& f = P.fronts[k];
      hi = lo;
      if (scrS[k] >= 0) hi = std::max(hi, scrS[k] + (int64_t)f.na * f.nn);
      if (scrM[k] >= 0) hi = std::max(hi, scrM[k] + (int64_t)f.nn * f.nn);
      if (scrK[k] >= 0) {
        const int64_t NBb = ceil_div(f.na, T);
        hi = std::max(hi, scrK[k] + NBb * (NBb + 1) / 2 * split_count(f.nn, kc) * (int64_t)T * T);
      }
      sbuf[k] = B.pool_buffer(lo, hi - lo);
    }
    B.pool_region = ws;
  }

  // small subtrees: one warp per range, four ranges per task; the parent of
  // a range's root waits on the whole task (utask)
  const Bundles bd = make_bundles(P);
  std::vector<int> uc_group(N, -1), utask(N, -1);
  for (int64_t k = 0; k < N; k++)
    if (P.fronts[k].na > 0 && bd.of[k] < 0) uc_group[k] = B.new_group();
  for (size_t b = 0; b < bd.tasks.size(); b++) {
    const int r0 = bd.roots[b].front();
    int id = B.add(bundle_task(P, bd, (int)b, T_SUBTREE), {P.fronts[r0].level, -1, 0, r0, 0, 0}, -1, bd.cost[b]);
    for (int r : bd.roots[b]) utask[r] = id;
  }
  for (int64_t k = 0; k < N; k++)
    if (bd.of[k] >= 0 && ubuf[k] >= 0) {
      const int id = utask[bd.roots[bd.of[k]].front()];
      const int p = P.fronts[k].parent;
      B.pool_entry(ubuf[k], id);
      if (p >= 0 && p < N && p != k && bd.of[p] == bd.of[k]) B.pool_exit_task(ubuf[k], id);
    }
  auto wait_child = [&](int id, int c) {
    if (utask[c] >= 0) B.wait_task(id, utask[c]);
    else B.wait_group(id, uc_group[c]);
  };

  // a dependency on a task's end, or on an early-signal group
  struct Dep {
    int id = -1;
    bool group = false;
  };
  auto wait_dep = [&](int task, const Dep& d) {
    if (d.group) B.wait_group(task, d.id);
    else B.wait_task(task, d.id);
  };
  std::vector<int> last_top, last_bot, trsmb, last_mrow;
  std::vector<Dep> trsm_top, trsm_prev;
  // Fused diagonal tasks wait mid task; under the dynamic schedule at most
  // one per front can wait at a time, so fuse only while such fronts
  // cannot hold half of the CTAs.
  int64_t multi_block_fronts = 0;
  for (int64_t k = 0; k < N; k++)
    if (P.fronts[k].nn > T) multi_block_fronts++;
  const int grid = P.grid > 0 ? P.grid : 296;
  const bool fuse_la = 2 * multi_block_fronts < grid && fused_la_allowed(P);
  for (int64_t k = 0; k < N; k++) {
    const FrontDesc& f = P.fronts[k];
    const int nn = f.nn, na = f.na, nj = f.nj;
    const int lv = f.level;
    const int NBc = ceil_div(nn, T), NBb = ceil_div(na, T);
    const int64_t blk = f.blk, upd = f.upd, S = scrS[k], M = scrM[k];
    auto bw = [&](int c) { return std::min(T, nn - c * T); };  // column block width
    auto bh = [&](int i) { return std::min(T, na - i * T); };  // bottom tile height

    if (bd.of[k] >= 0) continue;  // inside a small-subtree bundle
    // A front that fits one tile is one task: extend-add, partial Cholesky
    // and Schur complement in shared memory (cholesky.c:33-72 for one node).
    if (nj <= small_nj) {
      Task t = make_task(T_FRONT);
      t.m = nj;
      t.n = nn;
      t.aux[0] = (int32_t)k;
      t.a = opnd(B_X, blk, nj);
      t.c = opnd(B_WS, upd, std::max(na, 1));
      const double est = 3.0 + 0.02 * nn * (double)nj + 0.002 * (double)nj * nj;
      int id = B.add(t, {lv, -1, 0, (int)k, 0, 0}, uc_group[k], est);
      for (int l = f.chbeg; l < f.chend; l++) {
        wait_child(id, P.chidx[l]);
        B.pool_exit_task(ubuf[P.chidx[l]], id);
      }
      B.pool_entry(ubuf[k], id);
      continue;
    }

    // --- extend-add (cholesky.c:33-52), split into column chunks of about
    // equal work (children's update entries landing in the chunk)
    int asm_group = -1;
    if (f.chend > f.chbeg || na > 0) {
      asm_group = B.new_group();
      std::vector<double> colwork(nj, 0.0);
      for (int l = f.chbeg; l < f.chend; l++) {
        const FrontDesc& ch = P.fronts[P.chidx[l]];
        for (int q = 0; q < ch.na; q++) colwork[P.relidx[ch.relptr + q]] += ch.na - q;
      }
      for (int j = nn; j < nj; j++) colwork[j] += nj - j;  // zeroing of U_k
      double total = 0.0;
      for (double w : colwork) total += w;
      // (a merged plan, a batch of independent trees, is bound by its total
      // work rather than by one tree's chain: fewer, larger chunks there)
      const double target = std::max(P.seg.size() > 2 ? 16384.0 : 4096.0, total / 256.0);
      int j0 = 0;
      while (j0 < nj) {
        int j1 = j0;
        double w = 0.0;
        while (j1 < nj && (j1 - j0 < 8 || w < target) && j1 - j0 < CH) w += colwork[j1++];
        Task t = make_task(T_ASM);
        t.aux[0] = (int32_t)k;
        t.aux[1] = j0;
        t.aux[2] = j1;
        t.aux[3] = na > 0 ? 1 : 0;
        t.a = opnd(B_X, blk, nj);
        t.c = opnd(B_WS, upd, std::max(na, 1));
        // modelled cost (list order): w / 1000 gave cholesky 6.51 ms at 40^3
        // against 6.55 ms for w / 2000
        int id = B.add(t, {lv, -1, 0, (int)k, j0, 0}, asm_group, 3.0 + w / 1000.0);
        for (int l = f.chbeg; l < f.chend; l++) wait_child(id, P.chidx[l]);
        B.pool_entry(ubuf[k], id);
        B.pool_entry(sbuf[k], id);
        j0 = j1;
      }
      for (int l = f.chbeg; l < f.chend; l++) B.pool_exit_group(ubuf[P.chidx[l]], asm_group);
    }

    last_top.assign((size_t)NBc * NBc, -1);
    last_bot.assign((size_t)std::max(NBb, 1) * NBc, -1);
    trsm_top.assign(NBc, Dep());
    trsm_prev.assign(NBc, Dep());
    trsmb.assign(std::max(NBb, 1), -1);
    last_mrow.assign(NBc, -1);
    int pot = -1;
    int diag_end = -1;  // end group of the previous fused diagonal task
    for (int c = 0; c < NBc; c++) {
      const int bc = bw(c);
      const int cT = c * T;
      // POTRF of the diagonal tile (+ M_cc when anything lies below it).
      // With fusion, the same task then publishes its counter (M_cc is
      // stored: the solves below may start), waits (mid task) for the
      // updates of tiles (c+1, c) and (c+1, c+1) from column c-1, computes
      // L(c+1, c) = A(c+1, c) M_cc^T from M_cc in shared memory, raises an
      // early signal, and applies A(c+1, c+1) -= L L^T; its end group
      // releases POTRF(c+1), so consecutive diagonal tiles are consecutive
      // tasks.
      const bool fuse = fuse_la && c + 1 < NBc;
      {
        Task t = make_task(T_POTRF);
        t.m = t.n = bc;
        t.a = opnd(B_X, blk + (int64_t)cT * nj + cT, nj);
        const bool inv = (cT + bc < nj);
        t.aux[0] = cT;
        t.aux[1] = inv ? 1 : 0;
        if (inv) t.c = opnd(B_WS, M + (int64_t)cT * nn + cT, nn);
        if (fuse) t.k = bw(c + 1);
        const int gend = fuse ? B.new_group() : -1;
        pot = B.add(t, {lv, c, 0, (int)k, 0, 0}, gend);
        if (c == 0 && asm_group < 0) B.pool_entry(sbuf[k], pot);
        if (c == 0) B.wait_group(pot, asm_group);
        else if (diag_end >= 0) B.wait_group(pot, diag_end);
        else B.wait_task(pot, last_top[(size_t)c * NBc + c]);
        diag_end = gend;
      }
      const Operand Mcc = opnd(B_WS, M + (int64_t)cT * nn + cT, nn, OM_TRI_N, 0);
      for (int r = 0; r < NBc; r++) trsm_prev[r] = trsm_top[r];
      if (fuse) {
        const int r = c + 1;
        // modelled second part and early-signal offset of the fused task:
        // list-order parameters, not durations (the look-ahead takes
        // ~13 us; at 40^3, (9, +5) / (6, +3) / (3, +1.5) / (1, +0.5) gave
        // cholesky 6.61 / 6.56 / 6.52 / 6.54 ms)
        B.split_task(pot, 3.0);
        if (c > 0) {
          B.wait_mid(pot, last_top[(size_t)r * NBc + c]);
          B.wait_mid(pot, last_top[(size_t)r * NBc + r]);
        }
        trsm_top[r].id = B.early_signal(pot, B.cost[pot] + 1.5);
        trsm_top[r].group = true;
        last_top[(size_t)r * NBc + r] = pot;
      }
      // TRSM of the top tiles below the diagonal: P(r,c) := P(r,c) * M_cc^T.
      // Without fusion, the next diagonal block's tile goes through the
      // look-ahead task, which also applies that tile's rank-64 update of
      // the next diagonal tile, so the chain POTRF(c) -> POTRF(c+1) has one
      // task between.
      if (!fuse && c + 1 < NBc) {
        const int r = c + 1, rT = r * T;
        Task t = make_task(T_LA);
        t.m = bw(r);
        t.n = bc;
        t.k = bc;
        t.a = opnd(B_X, blk + (int64_t)cT * nj + rT, nj);
        t.b = Mcc;
        t.c = opnd(B_X, blk + (int64_t)rT * nj + rT, nj);
        int id = B.add(t, {lv, c, 1, (int)k, c, r}, -1, 11.0);
        B.wait_task(id, pot);
        if (c > 0) {
          B.wait_task(id, last_top[(size_t)r * NBc + c]);
          B.wait_task(id, last_top[(size_t)r * NBc + r]);
        }
        trsm_top[r].id = B.early_signal(id, 7.0);
        trsm_top[r].group = true;
        last_top[(size_t)r * NBc + r] = id;
      }
      for (int r = c + 2; r < NBc; r++) {
        const int rT = r * T;
        Operand pr = opnd(B_X, blk + (int64_t)cT * nj + rT, nj);
        Task t = gemm(bw(r), bc, bc, 1.0, pr, Mcc, 0.0, pr);
        int id = B.add(t, {lv, c, 1, (int)k, c, r});
        B.wait_task(id, pot);
        if (c > 0) B.wait_task(id, last_top[(size_t)r * NBc + c]);
        trsm_top[r].id = id;
        trsm_top[r].group = false;
      }
      // TRSM of the bottom tiles into S_k
      for (int i = 0; i < NBb; i++) {
        const int iT = i * T;
        Operand pa = opnd(B_X, blk + (int64_t)cT * nj + nn + iT, nj);
        Operand sc = opnd(B_WS, S + (int64_t)cT * na + iT, na);
        Task t = gemm(bh(i), bc, bc, 1.0, pa, Mcc, 0.0, sc);
        int id = B.add(t, {lv, c, 1, (int)k, c, NBc + i});
        B.wait_task(id, pot);
        if (c > 0) B.wait_task(id, last_bot[(size_t)i * NBc + c]);
        trsmb[i] = id;
      }
      // block row c of M = L11^{-1} (needed for the second solve)
      if (na > 0) {
        for (int j = 0; j < c; j++) {
          const int jT = j * T;
          Task t = make_task(T_MROW);
          t.m = bc;
          t.n = T;
          t.k = cT - jT;
          t.alpha = -1.0;
          t.a = opnd(B_X, blk + (int64_t)jT * nj + cT, nj);
          t.b = opnd(B_WS, M + (int64_t)jT * nn + jT, nn, OM_TRI_T, 0);
          t.c = opnd(B_WS, M + (int64_t)jT * nn + cT, nn);
          const int64_t moff = M + (int64_t)cT * nn + cT;
          t.aux[0] = B_WS;
          t.aux[1] = nn;
          t.aux[2] = (int32_t)(uint32_t)(moff & 0xffffffffLL);
          t.aux[3] = (int32_t)(moff >> 32);
          int id = B.add(t, {lv, c, 3, (int)k, j, 0});
          B.wait_task(id, pot);
          wait_dep(id, trsm_prev[c]);
          if (c - 1 > j) B.wait_task(id, last_mrow[j]);
          last_mrow[j] = id;
        }
      }
      // right-looking updates of the tiles right of column block c
      for (int j = c + 1; j < NBc; j++) {
        const int jT = j * T;
        Operand pj = opnd(B_X, blk + (int64_t)cT * nj + jT, nj);
        for (int r = j; r < NBc; r++) {
          if (r == c + 1 && j == c + 1) continue;  // done by the look-ahead task
          const int rT = r * T;
          Operand pr = opnd(B_X, blk + (int64_t)cT * nj + rT, nj);
          Operand cc = opnd(B_X, blk + (int64_t)jT * nj + rT, nj);
          Task t = gemm(bw(r), bw(j), bc, -1.0, pr, pj, 1.0, cc, r == j, 0);
          int id = B.add(t, {lv, c, 2, (int)k, j, r});
          wait_dep(id, trsm_top[r]);
          wait_dep(id, trsm_top[j]);
          if (c > 0) B.wait_task(id, last_top[(size_t)r * NBc + j]);
          last_top[(size_t)r * NBc + j] = id;
        }
        for (int i = 0; i < NBb; i++) {
          const int iT = i * T;
          Operand sa = opnd(B_WS, S + (int64_t)cT * na + iT, na);
          Operand cc = opnd(B_X, blk + (int64_t)jT * nj + nn + iT, nj);
          Task t = gemm(bh(i), bw(j), bc, -1.0, sa, pj, 1.0, cc);
          int id = B.add(t, {lv, c, 2, (int)k, j, NBc + i});
          B.wait_task(id, trsmb[i]);
          wait_dep(id, trsm_top[j]);
          if (c > 0) B.wait_task(id, last_bot[(size_t)i * NBc + j]);
          last_bot[(size_t)i * NBc + j] = id;
        }
      }
    }
    if (na == 0) {
      B.pool_exit_task(sbuf[k], pot);
      continue;
    }
    B.pool_exit_group(sbuf[k], uc_group[k]);
    const int b21 = sbuf[k] >= 0 ? B.new_group() : -1;
    B.pool_exit_group(sbuf[k], b21);
    // Schur complement U_k -= S_k S_k^T (cholesky.c:64-69); with a split
    // K the partial products are summed in a fixed order into U_k
    int64_t part = 0;
    for (int j = 0; j < NBb; j++) {
      for (int i = j; i < NBb; i++) {
        Operand sa = opnd(B_WS, S + i * T, na);
        Operand sb = opnd(B_WS, S + j * T, na);
        Operand cc = opnd(B_WS, upd + (int64_t)(j * T) * na + i * T, na);
        Task t = gemm(bh(i), bh(j), nn, -1.0, sa, sb, 1.0, cc, i == j, 0);
        if (scrK[k] >= 0) {
          const int p = split_count(nn, kc);
          SplitTask st = add_split_gemm(B, t, kc, scrK[k] + part * p * T * T, {lv, NBc, 0, (int)k, j, i},
                                        uc_group[k]);
          part++;
          for (int id : st.parts) {
            B.wait_task(id, trsmb[i]);
            B.wait_task(id, trsmb[j]);
          }
        } else {
          int id = B.add(t, {lv, NBc, 0, (int)k, j, i}, uc_group[k]);
          B.wait_task(id, trsmb[i]);
          B.wait_task(id, trsmb[j]);
        }
      }
    }
    // blk21 = S_k * M  (= L21 L11^{-1}, cholesky.c:72)
    for (int i = 0; i < NBb; i++) {
      for (int j = 0; j < NBc; j++) {
        const int jT = j * T, iT = i * T;
        Operand sa = opnd(B_WS, S + (int64_t)jT * na + iT, na);
        Operand mb = opnd(B_WS, M + (int64_t)jT * nn + jT, nn, OM_TRI_T, 0);
        Operand cc = opnd(B_X, blk + (int64_t)jT * nj + nn + iT, nj);
        Task t = gemm(bh(i), bw(j), nn - jT, 1.0, sa, mb, 0.0, cc);
        int id = B.add(t, {lv, NBc, 1, (int)k, j, i}, b21);
        B.wait_task(id, trsmb[i]);
        B.wait_task(id, pot);
        if (j < NBc - 1) B.wait_task(id, last_mrow[j]);
      }
    }
  }
  const int rc = B.finish(prog, P.grid > 0 ? P.grid : 296);
  if (rc == 0) pooled_fronts(P, B, prog);
  return rc;
}

}  // namespace chb
