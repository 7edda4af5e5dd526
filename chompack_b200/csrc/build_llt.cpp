// Task program of the Cholesky product X = L L^T (reference: llt.c:3-60),
// postorder.  Per supernode k, with P = the nj x nn factor panel
// [L_kk; W] (W = L_{Ak,Nk} L_kk^{-1} as stored by cholesky):
//   Q21 = W L_kk                                  (dtrmm, :32)
//   F   = [L_kk; Q21] [L_kk; Q21]^T  (lower)     (dsyrk over nj x nn, :33)
//   F  += extend-add(children's updates)          (:36-47)
//   U_k = F22;  blk = F(:, 0:nn) (lower)          (:50-57)
// As in the reference's dsyrk, the whole nn x nn diagonal block of the panel
// takes part in the product (not only its lower triangle).  F's leading nn
// columns live in scratch until every reader of the factor block is done.
#include "dag.h"

namespace chb {

int build_llt(const chb_plan& P, Program& prog) {
  const int T = TILE;
  const int CH = 64;
  const int64_t N = P.nsn;
  DagBuilder B;

  int64_t ws = P.upd_total;
  std::vector<int64_t> scrQ(N, -1), scrF(N);
  for (int64_t k = 0; k < N; k++) {
    const FrontDesc& f = P.fronts[k];
    if (f.na > 0) {
      scrQ[k] = ws;
      ws += (int64_t)f.na * f.nn;
    }
    scrF[k] = ws;
    ws += (int64_t)f.nj * f.nn;
  }
  prog.ws_doubles = ws;

  // group "front complete": the update U_k and the panel F are final
  std::vector<int> done(N);
  for (int64_t k = 0; k < N; k++) done[k] = B.new_group();

  for (int64_t k = 0; k < N; k++) {
    const FrontDesc& f = P.fronts[k];
    const int nn = f.nn, na = f.na, nj = f.nj;
    const int lv = f.level;
    const int NBc = ceil_div(nn, T), NBb = ceil_div(na, T);
    const int64_t blk = f.blk, upd = f.upd, Q = scrQ[k], F = scrF[k];
    auto bw = [&](int c) { return std::min(T, nn - c * T); };
    auto bh = [&](int i) { return std::min(T, na - i * T); };
    const bool has_children = f.chend > f.chbeg;
    const int fgroup = has_children ? B.new_group() : done[k];

    // Q21 = W L_kk
    const int qgroup = na > 0 ? B.new_group() : -1;
    for (int i = 0; i < NBb; i++) {
      for (int j = 0; j < NBc; j++) {
        const int iT = i * T, jT = j * T;
        Operand a = opnd(B_X, blk + (int64_t)jT * nj + nn + iT, nj);
        Operand b = opnd(B_X, blk + (int64_t)jT * nj + jT, nj, OM_TRI_T, 0);
        Operand c = opnd(B_WS, Q + (int64_t)jT * na + iT, na);
        Task t = gemm(bh(i), bw(j), nn - jT, 1.0, a, b, 0.0, c);
        B.add(t, {lv, 0, 0, (int)k, j, i}, qgroup);
      }
    }
    // F(:, 0:nn) lower: top tiles from L_kk, bottom tiles from Q21
    for (int j = 0; j < NBc; j++) {
      const int jT = j * T;
      Operand pj = opnd(B_X, blk + jT, nj);  // rows jT.. of the panel, all nn columns
      for (int i = j; i < NBc; i++) {
        const int iT = i * T;
        Operand pi = opnd(B_X, blk + iT, nj);
        Operand c = opnd(B_WS, F + (int64_t)jT * nj + iT, nj);
        Task t = gemm(bw(i), bw(j), nn, 1.0, pi, pj, 0.0, c, i == j, 0);
        B.add(t, {lv, 1, 0, (int)k, j, i}, fgroup);
      }
      for (int i = 0; i < NBb; i++) {
        const int iT = i * T;
        Operand qi = opnd(B_WS, Q + iT, na);
        Operand c = opnd(B_WS, F + (int64_t)jT * nj + nn + iT, nj);
        Task t = gemm(bh(i), bw(j), nn, 1.0, qi, pj, 0.0, c);
        int id = B.add(t, {lv, 1, 1, (int)k, j, i}, fgroup);
        B.wait_group(id, qgroup);
      }
    }
    // U_k = Q21 Q21^T (lower)
    for (int j = 0; j < NBb; j++) {
      for (int i = j; i < NBb; i++) {
        Operand qa = opnd(B_WS, Q + i * T, na);
        Operand qb = opnd(B_WS, Q + j * T, na);
        Operand c = opnd(B_WS, upd + (int64_t)(j * T) * na + i * T, na);
        Task t = gemm(bh(i), bh(j), nn, 1.0, qa, qb, 0.0, c, i == j, 0);
        int id = B.add(t, {lv, 1, 2, (int)k, j, i}, fgroup);
        B.wait_group(id, qgroup);
      }
    }
    // extend-add of the children into [F, U_k] (after F is initialised)
    if (has_children) {
      std::vector<double> colwork(nj, 0.0);
      for (int l = f.chbeg; l < f.chend; l++) {
        const FrontDesc& ch = P.fronts[P.chidx[l]];
        for (int q = 0; q < ch.na; q++) colwork[P.relidx[ch.relptr + q]] += ch.na - q;
      }
      double total = 0.0;
      for (double w : colwork) total += w;
      const double target = std::max(8192.0, total / 64.0);
      int j0 = 0;
      while (j0 < nj) {
        int j1 = j0;
        double w = 0.0;
        while (j1 < nj && (j1 - j0 < 8 || w < target) && j1 - j0 < CH) w += colwork[j1++];
        Task t = make_task(T_ASM);
        t.aux[0] = (int32_t)k;
        t.aux[1] = j0;
        t.aux[2] = j1;
        t.aux[3] = 0;
        t.a = opnd(B_WS, F, nj);
        t.c = opnd(B_WS, upd, std::max(na, 1));
        int id = B.add(t, {lv, 2, 0, (int)k, j0, 0}, done[k], 3.0 + w / 2000.0);
        B.wait_group(id, fgroup);
        for (int l = f.chbeg; l < f.chend; l++) B.wait_group(id, done[P.chidx[l]]);
        j0 = j1;
      }
    }
    // blk = F(:, 0:nn) lower part (the strict upper part of the diagonal
    // block keeps its old values, as the reference's dlacpy('L') does)
    for (int j = 0; j < NBc; j++) {
      const int jT = j * T;
      for (int i = j; i < NBc + NBb; i++) {
        const bool top = i < NBc;
        const int rT = top ? i * T : nn + (i - NBc) * T;
        const int rows = top ? bw(i) : bh(i - NBc);
        Task t = make_task(T_COPY);
        t.m = rows;
        t.n = bw(j);
        t.a = opnd(B_WS, F + (int64_t)jT * nj + rT, nj);
        t.c = opnd(B_X, blk + (int64_t)jT * nj + rT, nj);
        t.aux[0] = (top && i == j) ? 1 : 0;
        int id = B.add(t, {lv, 3, 0, (int)k, j, i});
        B.wait_group(id, done[k]);
      }
    }
  }
  return B.finish(prog, P.grid > 0 ? P.grid : 296);
}

}  // namespace chb
