// Task program of the maximum-determinant positive definite completion
// (reference: completion.c:3-120, update_factor.c:3-108), reverse postorder.
// The factored updates are built by stf_update_factor (stf.h).
//
// Input: Y = P(S^{-1}) in blkval; output: the factor L of S (in place).
// Per supernode k, with P11 = blk(0:nn, 0:nn), P21 = blk(nn:nj, 0:nn) and
// V_k the update the parent produced for k (na x na in the update buffer):
//   children's updates from F = [P11, P21; P21^T, V_k]     (:47-71)
//     factored_updates: U_c = update_factor(r_c, F), a factor of F[r_c, r_c]
//     otherwise:        U_c = F[r_c, r_c]
//   if na > 0:                                             (:74-99)
//     unfactored: V_k = L L^T (potrf); P21 := L^{-1} P21; P11 -= P21^T P21;
//                 P21 := L^{-T} P21
//     factored (V_k = L^T L): P21 := L^{-T} P21; P11 -= P21^T P21;
//                 P21 := L^{-1} P21
//     P21 := -P21
//   P11 := inv(R) where P11 = R^T R, R lower (the reverse Cholesky of
//   :101-113 and dtrtri of :116): with J the order-reversing permutation,
//   J P11 J = L' L'^T (lower Cholesky), R = J L'^T J and
//   inv(R) = J L'^{-T} J, i.e. P11(i, j) = L'^{-1}(nn-1-j, nn-1-i).
#include "stf.h"

namespace chb {

int build_completion(const chb_plan& P, Program& prog, bool factored) {
  const int T = TILE;
  const int64_t N = P.nsn;
  DagBuilder B;
  Stf S(B);

  // workspace: update matrices, then per front: Minv of V (na x 64), R and
  // L'^{-1} (nn x nn each), Minv of R (nn x 64); then the scratch of the
  // factored updates (handed out as they are built)
  int64_t ws = P.upd_total;
  std::vector<int64_t> oMV(N), oR(N), oM(N), oMR(N);
  for (int64_t k = 0; k < N; k++) {
    const FrontDesc& f = P.fronts[k];
    oMV[k] = ws;
    ws += (int64_t)f.na * T;
    oR[k] = ws;
    ws += (int64_t)f.nn * f.nn;
    oM[k] = ws;
    ws += (int64_t)f.nn * f.nn;
    oMR[k] = ws;
    ws += (int64_t)f.nn * T;
  }
  auto alloc = [&ws](int64_t n) {
    const int64_t o = ws;
    ws += n;
    return o;
  };
  S.alloc = alloc;  // long-K products are split

  // update matrices are tracked as matrices of their own
  std::vector<Mat> V(N);
  for (int64_t k = 0; k < N; k++) {
    const FrontDesc& f = P.fronts[k];
    V[k] = S.mat(B_WS, f.upd, std::max(f.na, 1), f.na, f.na);
  }

  for (int64_t k = N - 1; k >= 0; k--) {
    const FrontDesc& f = P.fronts[k];
    const int nn = f.nn, na = f.na, nj = f.nj;
    KeyGen kg{P.nlevels - f.level, (int)k};
    const Mat P11 = S.mat(B_X, f.blk, nj, nn, nn);
    const Mat P21 = S.mat(B_X, f.blk + nn, nj, na, nn);
    const Mat MV = S.mat(B_WS, oMV[k], std::max(na, 1), na, T);
    const Mat R = S.mat(B_WS, oR[k], nn, nn, nn);
    const Mat M = S.mat(B_WS, oM[k], nn, nn, nn);
    const Mat MR = S.mat(B_WS, oMR[k], nn, nn, T);

    // children's updates (read the original F)
    std::vector<Stf::Acc> fread;
    Stf::all(fread, P11, false, true);
    Stf::all(fread, P21, false);
    if (na > 0) Stf::all(fread, V[k], false, true);
    kg.step++;
    for (int l = f.chbeg; l < f.chend; l++) {
      const int c = P.chidx[l];
      const int Nc = P.fronts[c].na;
      if (factored) {
        const int rc = stf_update_factor(S, kg, P, c, P11, P21, V[k], V[c], 0, alloc);
        if (rc) return rc;
        continue;
      }
      // 64-column chunks of the child's update: each writes its own column
      // tile, so the chunks run in parallel
      const int CH = TILE;
      for (int q0 = 0; q0 < Nc; q0 += CH) {
        std::vector<Stf::Acc> acc = fread;
        for (int i = q0 / TILE; i < V[c].ntr(); i++) acc.push_back(Stf::W(V[c], i, q0 / TILE));
        Task t = make_task(T_EXTRACT);
        t.aux[0] = c;
        t.aux[1] = q0;
        t.aux[2] = std::min(Nc, q0 + CH);
        t.a = opnd(B_X, f.blk, nj);
        t.b = opnd(B_X, f.blk + nn, nj);
        t.c = opnd(B_WS, f.upd, std::max(na, 1));
        S.submit(t, kg(0, c, q0), acc, -1, 3.0 + (double)(Nc - q0) * CH / 2000.0);
      }
    }
    if (na > 0) {
      if (!factored) {
        stf_potrf(S, kg, V[k], MV);                        // V_k = L L^T
        stf_trsm_left(S, kg, V[k], MV, P21, false);        // P21 := L^{-1} P21
        stf_syrk_t(S, kg, P21, P11, -1.0, 1.0);            // P11 -= P21^T P21
        stf_trsm_left(S, kg, V[k], MV, P21, true);         // P21 := L^{-T} P21
      } else {
        stf_diag_inverses(S, kg, V[k], MV);                // V_k = L^T L, L given
        stf_trsm_left(S, kg, V[k], MV, P21, true);         // P21 := L^{-T} P21
        stf_syrk_t(S, kg, P21, P11, -1.0, 1.0);
        stf_trsm_left(S, kg, V[k], MV, P21, false);        // P21 := L^{-1} P21
      }
      kg.step++;
      for (int j = 0; j < P21.ntc(); j++)
        for (int i = 0; i < P21.ntr(); i++) {
          Task t = make_task(T_COPY);
          t.m = P21.th(i);
          t.n = P21.tw(j);
          t.alpha = -1.0;
          t.a = P21.op(i, j);
          t.c = P21.op(i, j);
          S.submit(t, kg(i, j, 0), {Stf::W(P21, i, j)});
        }
    }
    // P11 := inv(R), P11 = R^T R: R = anti-transpose(P11) -> Cholesky -> inverse -> anti-transpose
    stf_antitranspose(S, kg, P11, R, nn);
    stf_potrf(S, kg, R, MR);
    stf_tri_inverse(S, kg, R, MR, M);
    stf_antitranspose(S, kg, M, P11, nn);
  }
  prog.ws_doubles = ws;
  return B.finish(prog, P.grid > 0 ? P.grid : 296);
}

}  // namespace chb
