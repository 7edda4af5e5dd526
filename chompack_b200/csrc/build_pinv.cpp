// Task program of the projected-inverse sweep Y = P(X^{-1}) from the factor
// (reference: projected_inverse.c:3-75), run in reverse postorder (parents
// before children).
//
// Per supernode k, with L = L_kk (diagonal block of the factor), W = the
// stored off-diagonal block (L_{Ak,Nk} L_kk^{-1}) and V_k = the update the
// parent extracted for k (na x na, in the update buffer of k):
//   M   = L^{-1}                             (dtrtri, :33)
//   Y11 = M^T M                              (dsyrk, :42)
//   S21 = -V_k W                             (dsymm, :53)
//   Y11 = Y11 - S21^T W                      (dgemm, :57)
//   U_c = F[r_c, r_c] for every child c      (:62-71)
//   blk = [Y11 (lower, upper zeroed); S21]   (:36-38, :73)
// M is built tile-wise: inverses of the 64x64 diagonal tiles (independent)
// and, right-looking, the tiles below them (M(c, j) = -M_cc sum_l L(c, l)
// M(l, j), the sum accumulated as the M(l, j) become final).
// Y11 and S21 live in scratch until every reader of the factor block is done,
// then are copied back into blkval.
#include "dag.h"

namespace chb {

int build_projected_inverse(const chb_plan& P, Program& prog) {
  const int T = TILE;
  const int small_nj = small_front_nj(P);
  const int CH = 16;  // child columns per extract task
  const int64_t N = P.nsn;
  DagBuilder B;

  int64_t ws = P.upd_total;
  std::vector<int64_t> scrM(N), scrY(N), scrS(N, -1);
  for (int64_t k = 0; k < N; k++) {
    const FrontDesc& f = P.fronts[k];
    if (f.nj <= small_nj) continue;  // a small front needs no scratch (one shared-memory task)
    scrM[k] = ws;
    ws += (int64_t)f.nn * f.nn;
    scrY[k] = ws;
    ws += (int64_t)f.nn * f.nn;
    if (f.na > 0) {
      scrS[k] = ws;
      ws += (int64_t)f.na * f.nn;
    }
  }
  // split-K scratch, handed out as the long-K tiles are built
  const int KSPLIT = pinv_ksplit(P);
  auto scratch = [&ws](int K, int kc) {
    const int p = split_count(K, kc);
    if (p == 1) return (int64_t)0;
    const int64_t o = ws;
    ws += (int64_t)p * TILE * TILE;
    return o;
  };

  // pooled update matrices (under a scratch limit): V_k is first written by
  // the parent's extract tasks (or the parent's one-task front, or k's
  // bundle) and dead once k's S21 products and its own extract tasks, which
  // read it, are done
  const std::vector<int> ubuf = pool_update_matrices(P, prog, B);

  // group: the parent's extract tasks that produce V_k (k non-root); the
  // parent's own task when the parent is a small front
  std::vector<int> vready(N, -1);
  for (int64_t k = 0; k < N; k++)
    if (P.fronts[k].na > 0) vready[k] = B.new_group();
  std::vector<int> vtask(N, -1);
  auto wait_v = [&](int id, int64_t k) {
    if (vtask[k] >= 0) B.wait_task(id, vtask[k]);
    else B.wait_group(id, vready[k]);
  };

  // small subtrees: one warp per range, four ranges per task, each task
  // added once the parents of all its roots are (their V_k), parents first
  const Bundles bd = make_bundles(P);
  std::vector<std::vector<int>> in_bundle(bd.tasks.size());
  for (int64_t k = 0; k < N; k++)
    if (bd.of[k] >= 0) in_bundle[bd.of[k]].push_back((int)k);
  std::vector<std::pair<int64_t, int>> pending;  // (smallest parent of a root, bundle)
  for (size_t b = 0; b < bd.tasks.size(); b++) {
    int64_t m = N;
    for (int r : bd.roots[b]) {
      const int p = P.fronts[r].parent;
      if (p != r && p >= 0 && p < N) m = std::min<int64_t>(m, p);
    }
    pending.push_back({m, (int)b});
  }
  std::sort(pending.begin(), pending.end(), [](const std::pair<int64_t, int>& x, const std::pair<int64_t, int>& y) {
    return x.first > y.first || (x.first == y.first && x.second < y.second);
  });
  size_t next_bundle = 0;
  auto emit_bundles = [&](int64_t k) {  // every bundle whose roots' parents are all above k
    for (; next_bundle < pending.size() && pending[next_bundle].first > k; next_bundle++) {
      const int b = pending[next_bundle].second;
      const int r0 = bd.roots[b].back();
      Task t = bundle_task(P, bd, b, T_PSUBTREE);
      int id = B.add(t, {P.nlevels - P.fronts[r0].level, 0, 0, r0, 0, 0}, -1, 1.5 * bd.cost[b]);
      for (int r : bd.roots[b])
        if (P.fronts[r].na > 0) wait_v(id, r);
      for (int q : in_bundle[b]) {
        const int p = P.fronts[q].parent;
        if (!(p >= 0 && p < N && p != q && bd.of[p] == b)) B.pool_exit_task(ubuf[q], id);  // a root: V from outside
        else {
          B.pool_entry(ubuf[q], id);
          B.pool_exit_task(ubuf[q], id);
        }
      }
    }
  };

  const int maxlv = P.nlevels;
  std::vector<int> inv, last_mrow;
  for (int64_t k = N - 1; k >= 0; k--) {
    emit_bundles(k);
    if (bd.of[k] >= 0) continue;  // inside a small-subtree bundle
    const FrontDesc& f = P.fronts[k];
    const int nn = f.nn, na = f.na, nj = f.nj;
    const int lv = maxlv - f.level;  // roots first
    const int NBc = ceil_div(nn, T), NBb = ceil_div(na, T);
    const int64_t blk = f.blk, upd = f.upd, M = scrM[k], Y = scrY[k], S = scrS[k];
    // front k's scratch under a scratch limit: [M | Y11 | S21] and the split
    // partials it is handed below, first touched by the inverses of the
    // diagonal tiles and the S21 products (every other task of the front
    // waits on one of them), dead once the copies back and the extractions
    // for the children, which read Y11 and S21 last, are done
    const bool pool_scr = B.pool_limit >= 0;
    const int64_t part0 = ws;
    std::vector<int> scr_entry;
    const int copies = pool_scr ? B.new_group() : -1;
    auto bw = [&](int c) { return std::min(T, nn - c * T); };
    auto bh = [&](int i) { return std::min(T, na - i * T); };

    // A front that fits one tile is one task: the whole node of
    // projected_inverse.c:33-73 in shared memory, including the children's
    // updates, which its children then wait for.
    if (nj <= small_nj) {
      Task t = make_task(T_PFRONT);
      t.m = nj;
      t.n = nn;
      t.aux[0] = (int32_t)k;
      t.a = opnd(B_X, blk, nj);
      t.c = opnd(B_WS, upd, std::max(na, 1));
      double est = 4.0 + 0.03 * (double)nj * nj;
      for (int l = f.chbeg; l < f.chend; l++) est += 0.001 * P.fronts[P.chidx[l]].na * (double)P.fronts[P.chidx[l]].na;
      int id = B.add(t, {lv, 0, 0, (int)k, 0, 0}, -1, est);
      if (na > 0) wait_v(id, k);
      for (int l = f.chbeg; l < f.chend; l++) {
        vtask[P.chidx[l]] = id;
        B.pool_entry(ubuf[P.chidx[l]], id);
      }
      B.pool_exit_task(ubuf[k], id);
      continue;
    }

    // M = L^{-1}: diagonal tiles
    inv.assign(NBc, -1);
    for (int c = 0; c < NBc; c++) {
      const int cT = c * T;
      Task t = make_task(T_POTRF);
      t.m = t.n = bw(c);
      t.a = opnd(B_X, blk + (int64_t)cT * nj + cT, nj);
      t.c = opnd(B_WS, M + (int64_t)cT * nn + cT, nn);
      t.aux[0] = cT;
      t.aux[1] = 1;
      t.aux[2] = 1;  // invert only
      inv[c] = B.add(t, {lv, 0, 0, (int)k, c, 0});
      scr_entry.push_back(inv[c]);
    }
    // M below the diagonal tiles, right-looking by block column j: as soon
    // as M(l, j) is final, T(c, j) += L(c, l) M(l, j) for every c > l
    // (accumulated in place at M(c, j)); then M(l+1, j) = -M_{l+1} T(l+1, j).
    // The chain per column is two 64x64 tiles per block row.
    std::vector<int> fin((size_t)NBc * NBc, -1);  // last writer of M(c, j)
    for (int j = 0; j < NBc; j++) {
      const int jT = j * T;
      fin[(size_t)j * NBc + j] = inv[j];
      for (int l = j; l + 1 < NBc; l++) {
        const int lT = l * T;
        for (int c = l + 1; c < NBc; c++) {
          const int cT = c * T;
          Operand a = opnd(B_X, blk + (int64_t)lT * nj + cT, nj);          // L(c, l)
          Operand b = opnd(B_WS, M + (int64_t)jT * nn + lT, nn, OM_T, 0);  // M(l, j)^T
          Operand cc = opnd(B_WS, M + (int64_t)jT * nn + cT, nn);          // T(c, j)
          Task t = gemm(bw(c), bw(j), bw(l), 1.0, a, b, l == j ? 0.0 : 1.0, cc);
          int id = B.add(t, {lv, 1, l, (int)k, j, c});
          B.wait_task(id, fin[(size_t)l * NBc + j]);
          if (l > j) B.wait_task(id, fin[(size_t)c * NBc + j]);
          fin[(size_t)c * NBc + j] = id;
        }
        const int c = l + 1, cT = c * T;
        Operand a = opnd(B_WS, M + (int64_t)cT * nn + cT, nn);            // M_cc (lower)
        Operand b = opnd(B_WS, M + (int64_t)jT * nn + cT, nn, OM_T, 0);   // T(c, j)^T
        Operand cc = opnd(B_WS, M + (int64_t)jT * nn + cT, nn);
        Task t = gemm(bw(c), bw(j), bw(c), -1.0, a, b, 0.0, cc);
        int id = B.add(t, {lv, 1, c, (int)k, j, c});
        B.wait_task(id, inv[c]);
        B.wait_task(id, fin[(size_t)c * NBc + j]);
        fin[(size_t)c * NBc + j] = id;
      }
    }
    last_mrow.assign(NBc, -1);
    for (int j = 0; j < NBc; j++) last_mrow[j] = fin[(size_t)(NBc - 1) * NBc + j];
    // Y11 = M^T M (lower tiles), long K split
    std::vector<int> y11(NBc * NBc, -1);
    for (int i = 0; i < NBc; i++) {
      for (int j = 0; j <= i; j++) {
        const int iT = i * T, jT = j * T;
        Operand a = opnd(B_WS, M + (int64_t)iT * nn + iT, nn, OM_TRI_T, 0);
        Operand b = opnd(B_WS, M + (int64_t)jT * nn + iT, nn, i == j ? OM_TRI_T : OM_T, 0);
        Operand c = opnd(B_WS, Y + (int64_t)jT * nn + iT, nn);
        Task t = gemm(bw(i), bw(j), nn - iT, 1.0, a, b, 0.0, c, i == j, 0);
        SplitTask st = add_split_gemm(B, t, KSPLIT, scratch(t.k, KSPLIT), {lv, 2, 0, (int)k, j, i});
        for (int id : st.parts) {
          B.wait_task(id, inv[i]);
          B.wait_task(id, inv[j]);
          B.wait_task(id, last_mrow[i]);
          B.wait_task(id, last_mrow[j]);
        }
        y11[i * NBc + j] = st.out;
      }
    }
    const int yfinal = B.new_group();
    const int sgroup = na > 0 ? B.new_group() : -1;
    if (na > 0) {
      // S21 = -V_k W (long K split)
      for (int i = 0; i < NBb; i++) {
        for (int j = 0; j < NBc; j++) {
          const int iT = i * T, jT = j * T;
          Operand a = opnd(B_WS, upd, na, OM_SYM, iT);
          Operand b = opnd(B_X, blk + (int64_t)jT * nj + nn, nj, OM_T, 0);
          Operand c = opnd(B_WS, S + (int64_t)jT * na + iT, na);
          Task t = gemm(bh(i), bw(j), na, -1.0, a, b, 0.0, c);
          SplitTask st = add_split_gemm(B, t, KSPLIT, scratch(t.k, KSPLIT), {lv, 3, 0, (int)k, j, i}, sgroup);
          for (int id : st.parts) {
            wait_v(id, k);
            scr_entry.push_back(id);
          }
        }
      }
      B.pool_exit_group(ubuf[k], sgroup);
      // Y11 -= S21^T W (long K split)
      for (int i = 0; i < NBc; i++) {
        for (int j = 0; j <= i; j++) {
          const int iT = i * T, jT = j * T;
          Operand a = opnd(B_WS, S + (int64_t)iT * na, na, OM_T, 0);
          Operand b = opnd(B_X, blk + (int64_t)jT * nj + nn, nj, OM_T, 0);
          Operand c = opnd(B_WS, Y + (int64_t)jT * nn + iT, nn);
          Task t = gemm(bw(i), bw(j), na, -1.0, a, b, 1.0, c, i == j, 0);
          SplitTask st = add_split_gemm(B, t, KSPLIT, scratch(t.k, KSPLIT), {lv, 4, 0, (int)k, j, i}, yfinal);
          for (int id : st.parts) B.wait_group(id, sgroup);
          B.wait_task(st.out, y11[i * NBc + j]);
        }
      }
    } else {
      // root: Y11 = M^T M is final; mark it with a copy-free group via the
      // tile tasks themselves
      for (int i = 0; i < NBc; i++)
        for (int j = 0; j <= i; j++) {
          B.group_of[y11[i * NBc + j]] = yfinal;
          B.group_size[yfinal]++;
        }
    }
    // children's updates, CH columns per task (on a merged plan, a batch
    // bound by its total work, columns up to about 16k entries per task)
    const bool merged = P.seg.size() > 2;
    for (int l = f.chbeg; l < f.chend; l++) {
      const int c = P.chidx[l];
      const int Nc = P.fronts[c].na;
      for (int q0 = 0, q1 = 0; q0 < Nc; q0 = q1) {
        q1 = std::min(Nc, q0 + CH);
        if (merged) {
          int64_t w = 0;
          for (q1 = q0; q1 < Nc && (q1 - q0 < CH || w < 16384) && q1 - q0 < 4 * CH; q1++) w += Nc - q1;
        }
        Task t = make_task(T_EXTRACT);
        t.aux[0] = c;
        t.aux[1] = q0;
        t.aux[2] = q1;
        t.a = opnd(B_WS, Y, nn);
        t.b = opnd(B_WS, na > 0 ? S : 0, std::max(na, 1));
        t.c = opnd(B_WS, upd, std::max(na, 1));
        int id = B.add(t, {lv, 5, 0, (int)k, c, q0}, vready[c], 3.0 + (double)(Nc - q0) * (q1 - q0) / 2000.0);
        B.wait_group(id, yfinal);
        B.wait_group(id, sgroup);
        B.pool_entry(ubuf[c], id);
      }
      B.pool_exit_group(ubuf[k], vready[c]);
    }
    // copy back into blkval (all readers of the factor block are done once
    // the final Y11 tiles are: they wait on every M tile and S21 tile), one
    // task per column strip and part: the diagonal tile (lower part, zeros
    // above), the rows below it in Y11, the strict upper part (zeros, as
    // projected_inverse.c:36-38 leaves it) and the rows of S21
    for (int j = 0; j < NBc; j++) {
      const int jT = j * T;
      {
        Task t = make_task(T_COPY);
        t.m = bw(j);
        t.n = bw(j);
        t.a = opnd(B_WS, Y + (int64_t)jT * nn + jT, nn);
        t.c = opnd(B_X, blk + (int64_t)jT * nj + jT, nj);
        t.aux[0] = 3;
        int id = B.add(t, {lv, 6, 0, (int)k, j, j}, copies);
        B.wait_group(id, yfinal);
      }
      if (jT + T < nn) {
        Task t = make_task(T_COPY);
        t.m = nn - (jT + T);
        t.n = bw(j);
        t.a = opnd(B_WS, Y + (int64_t)jT * nn + jT + T, nn);
        t.c = opnd(B_X, blk + (int64_t)jT * nj + jT + T, nj);
        int id = B.add(t, {lv, 6, 0, (int)k, j, j + 1}, copies, 3.0 + (double)t.m * t.n / 4096.0);
        B.wait_group(id, yfinal);
      }
      if (jT > 0) {
        Task t = make_task(T_COPY);
        t.m = jT;
        t.n = bw(j);
        t.aux[0] = 4;  // zeros
        t.c = opnd(B_X, blk + (int64_t)jT * nj, nj);
        int id = B.add(t, {lv, 6, 1, (int)k, j, 0}, copies, 3.0 + (double)t.m * t.n / 8192.0);
        B.wait_group(id, yfinal);
      }
      if (na > 0) {
        Task t = make_task(T_COPY);
        t.m = na;
        t.n = bw(j);
        t.a = opnd(B_WS, S + (int64_t)jT * na, na);
        t.c = opnd(B_X, blk + (int64_t)jT * nj + nn, nj);
        int id = B.add(t, {lv, 6, 2, (int)k, j, 0}, copies, 3.0 + (double)t.m * t.n / 4096.0);
        B.wait_group(id, yfinal);
      }
    }
    if (pool_scr) {
      const int main_buf = B.pool_buffer(M, (S >= 0 ? S + (int64_t)na * nn : Y + (int64_t)nn * nn) - M);
      const int part_buf = ws > part0 ? B.pool_buffer(part0, ws - part0) : -1;
      for (int b : {main_buf, part_buf}) {
        if (b < 0) continue;
        for (int id : scr_entry) B.pool_entry(b, id);
        B.pool_exit_group(b, copies);
        for (int l = f.chbeg; l < f.chend; l++) B.pool_exit_group(b, vready[P.chidx[l]]);
      }
    }
  }
  prog.ws_doubles = ws;
  if (B.pool_limit >= 0) B.pool_region = ws;
  emit_bundles(-1);
  const int rc = B.finish(prog, P.grid > 0 ? P.grid : 296);
  if (rc == 0) pooled_fronts(P, B, prog);
  return rc;
}

}  // namespace chb
