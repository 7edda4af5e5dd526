// Task program of the Hessian factors of the log-det barrier (reference:
// hessian.c:3-374) applied to a batch of U matrices (base slots B_U0 + u):
//
//   hessian(adj, inv):  if adj != inv: _scale;  adj ? _M2T : _Y2K;
//                       if adj == inv: _scale            (hessian.c:368-371)
//
// alpha = -1 (inv: +1).  L = factor (slot B_L), Y = projected inverse (B_Y).
//
// _Y2K (postorder, per U; hessian.c:3-111): F = [U(:, 0:nn); 0]
//   [!inv: F += children's updates]; F22 += a L21 F21^T; F21 += a L21 F11;
//   F22 += a F21 L21^T; [inv: F += children's updates]; update = F22.
// _M2T (reverse postorder, per U; :114-213): F = [U(:, 0:nn); V]
//   [inv: children's updates = F[r_c, r_c]]; F11 += a F21^T L21;
//   F21 += a F22 L21; F11 += a L21^T F21; [!inv: children's updates].
// _scale (reverse postorder, all U; :216-347): children's updates from
//   Y's front (factored: update_factor); unfactored: potrf of the update;
//   for each U: symmetrise its diagonal block, then
//   !inv: U(:, 0:nn) := U op1(L_kk)^{-1}; U11 := op2(L_kk)^{-1} U11;
//         zero U11's strict upper part; U21 := op3(F22) U21
//   inv:  the same with products and solves exchanged,
//   op1 = adj ? N : T, op2 = adj ? T : N, op3 = factored ? (adj ? T : N)
//   : (adj ? N : T).
// The fronts' U blocks are transformed in place (they are tracked tiles, so
// the order between sweeps and between fronts follows from the accesses).
#include <functional>

#include "stf.h"

namespace chb {

namespace {

struct HessCtx {
  Stf& S;
  const chb_plan& P;
  int nu;
};

// C := X * op(T) in place (X m x n tiles, T n x n lower).  transT: op = T^T.
void right_mult(Stf& S, KeyGen& kg, const Mat& X, const Mat& Tm, bool transT) {
  const int nb = X.ntc();
  for (int jj = 0; jj < nb; jj++) {
    const int j = transT ? nb - 1 - jj : jj;
    kg.step++;
    for (int i = 0; i < X.ntr(); i++) {
      Task t;
      std::vector<Stf::Acc> acc{Stf::W(X, i, j)};
      if (!transT) {  // X(i,j) = sum_{l >= j} X(i,l) T(l,j)
        t = gemm(X.th(i), X.tw(j), X.cols - j * TILE, 1.0, X.op(i, j), Tm.op(j, j, OM_TRI_T, 0), 0.0, X.op(i, j));
        for (int l = j; l < nb; l++) {
          acc.push_back(Stf::R(X, i, l));
          acc.push_back(Stf::R(Tm, l, j));
        }
      } else {        // X(i,j) = sum_{l <= j} X(i,l) T(j,l)
        t = gemm(X.th(i), X.tw(j), j * TILE + X.tw(j), 1.0, X.op(i, 0), Tm.op(j, 0, OM_TRI_N, j * TILE), 0.0,
                 X.op(i, j));
        for (int l = 0; l <= j; l++) {
          acc.push_back(Stf::R(X, i, l));
          acc.push_back(Stf::R(Tm, j, l));
        }
      }
      S.gemm(t, kg(i, j, 0), acc);
    }
  }
}

// X := op(T) X in place (X m x n, T m x m lower).  transT: op = T^T.
void left_mult(Stf& S, KeyGen& kg, const Mat& X, const Mat& Tm, bool transT) {
  const int mb = X.ntr();
  for (int ii = 0; ii < mb; ii++) {
    const int i = transT ? ii : mb - 1 - ii;
    kg.step++;
    for (int j = 0; j < X.ntc(); j++) {
      Task t;
      std::vector<Stf::Acc> acc{Stf::W(X, i, j)};
      if (!transT) {  // X(i,j) = sum_{l <= i} T(i,l) X(l,j)
        t = gemm(X.th(i), X.tw(j), i * TILE + X.th(i), 1.0, Tm.op(i, 0, OM_TRI_N, i * TILE), X.op(0, j, OM_T), 0.0,
                 X.op(i, j));
        for (int l = 0; l <= i; l++) {
          acc.push_back(Stf::R(X, l, j));
          acc.push_back(Stf::R(Tm, i, l));
        }
      } else {        // X(i,j) = sum_{l >= i} T(l,i) X(l,j)
        t = gemm(X.th(i), X.tw(j), X.rows - i * TILE, 1.0, Tm.op(i, i, OM_TRI_T, 0), X.op(i, j, OM_T), 0.0,
                 X.op(i, j));
        for (int l = i; l < mb; l++) {
          acc.push_back(Stf::R(X, l, j));
          acc.push_back(Stf::R(Tm, l, i));
        }
      }
      S.gemm(t, kg(i, j, 0), acc);
    }
  }
}

// C (+)= alpha op(A) op(B)^T over tiles; `lower`: only tiles/entries i >= j.
void tile_gemm(Stf& S, KeyGen& kg, const Mat& C, double alpha, double beta, bool lower,
               const std::function<Operand(int)>& aop, const std::function<Operand(int)>& bop, int K,
               const std::vector<Stf::Acc>& reads) {
  kg.step++;
  for (int j = 0; j < C.ntc(); j++)
    for (int i = lower ? j : 0; i < C.ntr(); i++) {
      std::vector<Stf::Acc> acc = reads;
      acc.push_back(Stf::W(C, i, j));
      Task t = gemm(C.th(i), C.tw(j), K, alpha, aop(i), bop(j), beta, C.op(i, j), lower && i == j, 0);
      S.gemm(t, kg(i, j, 0), acc);
    }
}

void zero_tiles(Stf& S, KeyGen& kg, const Mat& M, bool lower) {
  kg.step++;
  for (int j = 0; j < M.ntc(); j++)
    for (int i = lower ? j : 0; i < M.ntr(); i++) {
      Task t = make_task(T_COPY);
      t.m = M.th(i);
      t.n = M.tw(j);
      t.aux[0] = 4;
      t.c = M.op(i, j);
      S.submit(t, kg(i, j, 0), {Stf::W(M, i, j)});
    }
}

}  // namespace

int build_hessian(const chb_plan& P, Program& prog, int nu, int flags) {
  const bool adj = flags & 1, inv = (flags >> 1) & 1, factored = (flags >> 2) & 1;
  const int T = TILE;
  const int64_t N = P.nsn;
  DagBuilder B;
  Stf S(B);
  if (nu <= 0 || nu > MAX_BASES - B_U0) return set_error(-1, "hessian: 1..%d U matrices per call", MAX_BASES - B_U0);
  const double alpha = inv ? 1.0 : -1.0;

  // workspace: V (update matrices of _scale) | per-U update matrices |
  // per front: diag inverses of L_kk (nn x 64), L_kk^{-1} (nn x nn), diag
  // inverses of the front update (na x 64) | scratch of the factored updates
  // (handed out as they are built)
  int64_t ws = 0;
  const int64_t oV = ws;
  ws += P.upd_total;
  std::vector<int64_t> oW(nu);
  for (int u = 0; u < nu; u++) {
    oW[u] = ws;
    ws += P.upd_total;
  }
  std::vector<int64_t> oML(N), oMF(N), oMV(N);
  for (int64_t k = 0; k < N; k++) {
    const FrontDesc& f = P.fronts[k];
    oML[k] = ws;
    ws += (int64_t)f.nn * T;
    oMF[k] = ws;
    ws += (int64_t)f.nn * f.nn;
    oMV[k] = ws;
    ws += (int64_t)f.na * T;
  }
  auto alloc = [&ws](int64_t n) {
    const int64_t o = ws;
    ws += n;
    return o;
  };
  S.alloc = alloc;  // long-K products are split

  // tracked matrices
  std::vector<Mat> L11(N), L21(N), Y11(N), Y21(N), V(N), ML(N), MF(N), MV(N);
  std::vector<std::vector<Mat>> U11(nu, std::vector<Mat>(N)), U21(nu, std::vector<Mat>(N)),
      W(nu, std::vector<Mat>(N));
  for (int64_t k = 0; k < N; k++) {
    const FrontDesc& f = P.fronts[k];
    L11[k] = S.mat(B_L, f.blk, f.nj, f.nn, f.nn);
    L21[k] = S.mat(B_L, f.blk + f.nn, f.nj, f.na, f.nn);
    Y11[k] = S.mat(B_Y, f.blk, f.nj, f.nn, f.nn);
    Y21[k] = S.mat(B_Y, f.blk + f.nn, f.nj, f.na, f.nn);
    V[k] = S.mat(B_WS, oV + f.upd, std::max(f.na, 1), f.na, f.na);
    ML[k] = S.mat(B_WS, oML[k], f.nn, f.nn, T);
    MF[k] = S.mat(B_WS, oMF[k], f.nn, f.nn, f.nn);
    MV[k] = S.mat(B_WS, oMV[k], std::max(f.na, 1), f.na, T);
    for (int u = 0; u < nu; u++) {
      U11[u][k] = S.mat((uint8_t)(B_U0 + u), f.blk, f.nj, f.nn, f.nn);
      U21[u][k] = S.mat((uint8_t)(B_U0 + u), f.blk + f.nn, f.nj, f.na, f.nn);
      W[u][k] = S.mat(B_WS, oW[u] + f.upd, std::max(f.na, 1), f.na, f.na);
    }
  }
  int phase = 0;

  // ----------------------------------------------------------- _Y2K
  auto y2k = [&]() {
    phase++;
    for (int u = 0; u < nu; u++)
      for (int64_t k = 0; k < N; k++) {
        const FrontDesc& f = P.fronts[k];
        const int nn = f.nn, na = f.na, nj = f.nj;
        KeyGen kg{phase * 100000 + f.level, (int)k};
        const Mat& F11 = U11[u][k];
        const Mat& F21 = U21[u][k];
        const Mat& F22 = W[u][k];
        // extend-add in 64-column chunks of the front (each writes its own
        // column tiles of F11/F21 or F22, so the chunks run in parallel)
        auto extend_add = [&](bool zero) {
          kg.step++;
          std::vector<Stf::Acc> rd;
          for (int l = f.chbeg; l < f.chend; l++) Stf::all(rd, W[u][P.chidx[l]], false, true);
          // chunk boundaries on the tile grids of F11/F21 (from 0) and of
          // F22 (from nn), so no two chunks write the same tile
          std::vector<int> cuts;
          for (int j = 0; j < nn; j += T) cuts.push_back(j);
          for (int j = nn; j < nj; j += T) cuts.push_back(j);
          cuts.push_back(nj);
          for (size_t ci = 0; ci + 1 < cuts.size(); ci++) {
            const int j0 = cuts[ci], j1 = std::min(cuts[ci + 1], j0 + T);
            std::vector<Stf::Acc> acc = rd;
            if (j0 < nn) {
              const int jt = j0 / T;  // nn-column tiles: front tile jt spans [jt*T, jt*T+T)
              for (int i = jt; i < F11.ntr(); i++) acc.push_back(Stf::W(F11, i, jt));
              for (int i = 0; i < F21.ntr(); i++) acc.push_back(Stf::W(F21, i, jt));
            }
            if (j1 > nn) {
              const int c0t = (std::max(j0, nn) - nn) / T, c1t = (j1 - 1 - nn) / T;
              for (int ct = c0t; ct <= c1t; ct++)
                for (int i = ct; i < F22.ntr(); i++) acc.push_back(Stf::W(F22, i, ct));
            }
            Task t = make_task(T_ASM);
            t.aux[0] = (int32_t)k;
            t.aux[1] = j0;
            t.aux[2] = j1;
            t.aux[3] = zero ? 1 : 0;
            t.a = opnd((uint8_t)(B_U0 + u), f.blk, nj);
            t.c = opnd(B_WS, oW[u] + f.upd, std::max(na, 1));
            t.off2 = oW[u];
            S.submit(t, kg(0, j0 / T, 0), acc, -1, 3.0 + (double)nj * (j1 - j0) / 4000.0);
          }
        };
        if (!inv) {
          extend_add(true);
        } else if (na > 0) {
          zero_tiles(S, kg, F22, true);
        }
        if (na > 0) {
          std::vector<Stf::Acc> rl, rf21, rf11;
          Stf::all(rl, L21[k], false);
          Stf::all(rf21, F21, false);
          Stf::all(rf11, F11, false, true);
          // F22 += a L21 F21^T (lower tiles)
          {
            std::vector<Stf::Acc> r = rl;
            r.insert(r.end(), rf21.begin(), rf21.end());
            tile_gemm(S, kg, F22, alpha, 1.0, true, [&](int i) { return L21[k].op(i, 0); },
                      [&](int j) { return F21.op(j, 0); }, nn, r);
          }
          // F21 += a L21 F11 (F11 symmetric, lower stored)
          {
            std::vector<Stf::Acc> r = rl;
            r.insert(r.end(), rf11.begin(), rf11.end());
            tile_gemm(S, kg, F21, alpha, 1.0, false, [&](int i) { return L21[k].op(i, 0); },
                      [&](int j) { return opnd(F11.base, F11.off, F11.ld, OM_SYM, j * T); }, nn, r);
          }
          // F22 += a F21 L21^T (lower tiles)
          {
            std::vector<Stf::Acc> r = rl;
            Stf::all(r, F21, false);
            tile_gemm(S, kg, F22, alpha, 1.0, true, [&](int i) { return F21.op(i, 0); },
                      [&](int j) { return L21[k].op(j, 0); }, nn, r);
          }
        }
        if (inv) extend_add(false);
      }
  };

  // children's updates out of the front [F11, F21; ., F22] into dst[c]
  auto extract = [&](KeyGen& kg, int64_t k, const Mat& F11, const Mat& F21, const Mat& F22,
                     const std::vector<Mat>& dst, int64_t dst_base) {
    const FrontDesc& f = P.fronts[k];
    kg.step++;
    std::vector<Stf::Acc> rd;
    Stf::all(rd, F11, false, true);
    Stf::all(rd, F21, false);
    if (f.na > 0) Stf::all(rd, F22, false, true);
    for (int l = f.chbeg; l < f.chend; l++) {
      const int c = P.chidx[l];
      const int Nc = P.fronts[c].na;
      // 64-column chunks of the child's update (disjoint column tiles)
      for (int q0 = 0; q0 < Nc; q0 += TILE) {
        const int qt = q0 / TILE;
        std::vector<Stf::Acc> acc = rd;
        for (int i = qt; i < dst[c].ntr(); i++) acc.push_back(Stf::W(dst[c], i, qt));
        Task t = make_task(T_EXTRACT);
        t.aux[0] = c;
        t.aux[1] = q0;
        t.aux[2] = std::min(Nc, q0 + TILE);
        t.a = opnd(F11.base, F11.off, F11.ld);
        t.b = opnd(F21.base, F21.off, F21.ld);
        t.c = opnd(F22.base, F22.off, F22.ld);
        t.off2 = dst_base;
        S.submit(t, kg(0, c, q0), acc, -1, 3.0 + (double)(Nc - q0) * TILE / 4000.0);
      }
    }
  };

  // ----------------------------------------------------------- _M2T
  auto m2t = [&]() {
    phase++;
    for (int u = 0; u < nu; u++)
      for (int64_t k = N - 1; k >= 0; k--) {
        const FrontDesc& f = P.fronts[k];
        const int na = f.na;
        KeyGen kg{phase * 100000 + P.nlevels - f.level, (int)k};
        const Mat& F11 = U11[u][k];
        const Mat& F21 = U21[u][k];
        const Mat& F22 = W[u][k];
        if (inv) extract(kg, k, F11, F21, F22, W[u], oW[u]);
        if (na > 0) {
          std::vector<Stf::Acc> rl;
          Stf::all(rl, L21[k], false);
          // F11 += a F21^T L21 (lower tiles)
          {
            std::vector<Stf::Acc> r = rl;
            Stf::all(r, F21, false);
            tile_gemm(S, kg, F11, alpha, 1.0, true,
                      [&](int i) { return opnd(F21.base, F21.at(0, i * T), F21.ld, OM_T); },
                      [&](int j) { return opnd(L21[k].base, L21[k].at(0, j * T), L21[k].ld, OM_T); }, na, r);
          }
          // F21 += a F22 L21 (F22 symmetric, lower stored)
          {
            std::vector<Stf::Acc> r = rl;
            Stf::all(r, F22, false, true);
            tile_gemm(S, kg, F21, alpha, 1.0, false,
                      [&](int i) { return opnd(F22.base, F22.off, F22.ld, OM_SYM, i * T); },
                      [&](int j) { return opnd(L21[k].base, L21[k].at(0, j * T), L21[k].ld, OM_T); }, na, r);
          }
          // F11 += a L21^T F21 (lower tiles)
          {
            std::vector<Stf::Acc> r = rl;
            Stf::all(r, F21, false);
            tile_gemm(S, kg, F11, alpha, 1.0, true,
                      [&](int i) { return opnd(L21[k].base, L21[k].at(0, i * T), L21[k].ld, OM_T); },
                      [&](int j) { return opnd(F21.base, F21.at(0, j * T), F21.ld, OM_T); }, na, r);
          }
        }
        if (!inv) extract(kg, k, F11, F21, F22, W[u], oW[u]);
      }
  };

  // ----------------------------------------------------------- _scale
  int err = 0;
  auto scale = [&]() {
    phase++;
    const bool tr1 = !adj;                     // op1 = T when !adj
    const bool tr2 = adj;                      // op2 = T when adj
    const bool tr3 = factored ? adj : !adj;    // op3 = T
    for (int64_t k = N - 1; k >= 0; k--) {
      const FrontDesc& f = P.fronts[k];
      const int nn = f.nn, na = f.na, nj = f.nj;
      KeyGen kg{phase * 100000 + P.nlevels - f.level, (int)k};
      // children's updates out of Y's front
      if (factored) {
        kg.step++;
        for (int l = f.chbeg; l < f.chend; l++) {
          const int rc = stf_update_factor(S, kg, P, P.chidx[l], Y11[k], Y21[k], V[k], V[P.chidx[l]], oV, alloc);
          if (rc) {
            err = rc;
            return;
          }
        }
      } else {
        extract(kg, k, Y11[k], Y21[k], V[k], V, oV);
      }
      if (na > 0) {
        if (!factored) stf_potrf(S, kg, V[k], MV[k]);       // V_k = L L^T
        else if (inv) stf_diag_inverses(S, kg, V[k], MV[k]); // V_k = L^T L, L given
      }
      if (!inv) {
        stf_diag_inverses(S, kg, L11[k], ML[k]);
        stf_tri_inverse(S, kg, L11[k], ML[k], MF[k]);
      }
      for (int u = 0; u < nu; u++) {
        const Mat& X11 = U11[u][k];
        const Mat& X21 = U21[u][k];
        // symmetrise the diagonal block: upper := lower^T
        kg.step++;
        for (int j = 0; j < X11.ntc(); j++)
          for (int i = 0; i <= j; i++) {
            Task t = make_task(T_COPY);
            t.m = X11.th(i);
            t.n = X11.tw(j);
            t.aux[0] = 16 | (i == j ? 32 : 0);
            t.a = X11.op(j, i);
            t.c = X11.op(i, j);
            S.submit(t, kg(i, j, 0), {Stf::W(X11, i, j), Stf::R(X11, j, i)});
          }
        // the full nj x nn panel as one tracked unit is X11 over X21
        const Mat& Tm = inv ? L11[k] : MF[k];
        // U(:, 0:nn) := U op1(L)^{-1} (= U op1(M)) or U op1(L): row blocks of
        // X11 and X21 separately (same column operation)
        right_mult(S, kg, X11, Tm, tr1);
        if (na > 0) right_mult(S, kg, X21, Tm, tr1);
        // U11 := op2(L)^{-1} U11 (= op2(M) U11) or op2(L) U11
        left_mult(S, kg, X11, Tm, tr2);
        // zero the strict upper part of U11
        kg.step++;
        for (int j = 0; j < X11.ntc(); j++)
          for (int i = 0; i <= j; i++) {
            Task t = make_task(T_COPY);
            t.m = X11.th(i);
            t.n = X11.tw(j);
            t.aux[0] = (i == j) ? 3 : 4;
            t.a = X11.op(i, j);
            t.c = X11.op(i, j);
            S.submit(t, kg(i, j, 0), {Stf::W(X11, i, j)});
          }
        if (na > 0) {
          if (!inv) left_mult(S, kg, X21, V[k], tr3);               // U21 := op3(F22) U21
          else stf_trsm_left(S, kg, V[k], MV[k], X21, tr3);         // U21 := op3(F22)^{-1} U21
        }
      }
    }
  };

  if (adj != inv) scale();
  if (adj) m2t();
  else y2k();
  if (adj == inv) scale();
  if (err) return err;
  prog.ws_doubles = ws;
  return B.finish(prog, P.grid > 0 ? P.grid : 296);
}

}  // namespace chb
