// Task program of the factor export's block products (reference:
// cspmatrix.spmatrix() of a factor, src/python/symbolic.py:1052-1068): after
// cholesky the off-diagonal block of supernode k holds W = L_{Ak,Nk} L_kk^{-1}
// (cholesky.c:72); the conventional factor's block is W L_kk, which the
// reference forms with dtrmm('R', 'L', 'N', 'N') (dscal when nn == 1).
// Per supernode with na > 0: Q = W L_kk into scratch as GEMM tiles with a
// lower-triangular operand, then Q copied over W.  Supernodes are
// independent, so every front's tiles can run at once.
#include "dag.h"

namespace chb {

int build_conventional(const chb_plan& P, Program& prog) {
  const int T = TILE;
  const int64_t N = P.nsn;
  DagBuilder B;
  int64_t ws = 0;
  std::vector<int64_t> scrQ(N, -1);
  for (int64_t k = 0; k < N; k++)
    if (P.fronts[k].na > 0) {
      scrQ[k] = ws;
      ws += (int64_t)P.fronts[k].na * P.fronts[k].nn;
    }
  prog.ws_doubles = ws;
  for (int64_t k = 0; k < N; k++) {
    const FrontDesc& f = P.fronts[k];
    const int nn = f.nn, na = f.na, nj = f.nj;
    if (na == 0) continue;
    const int NBc = ceil_div(nn, T), NBb = ceil_div(na, T);
    const int64_t blk = f.blk, Q = scrQ[k];
    auto bw = [&](int c) { return std::min(T, nn - c * T); };
    auto bh = [&](int i) { return std::min(T, na - i * T); };
    const int qgroup = B.new_group();
    for (int i = 0; i < NBb; i++) {
      for (int j = 0; j < NBc; j++) {
        const int iT = i * T, jT = j * T;
        Operand a = opnd(B_X, blk + (int64_t)jT * nj + nn + iT, nj);
        Operand b = opnd(B_X, blk + (int64_t)jT * nj + jT, nj, OM_TRI_T, 0);
        Operand c = opnd(B_WS, Q + (int64_t)jT * na + iT, na);
        Task t = gemm(bh(i), bw(j), nn - jT, 1.0, a, b, 0.0, c);
        B.add(t, {f.level, 0, 0, (int)k, j, i}, qgroup);
      }
    }
    for (int j = 0; j < NBc; j++) {
      for (int i = 0; i < NBb; i++) {
        Task t = make_task(T_COPY);
        t.m = bh(i);
        t.n = bw(j);
        t.a = opnd(B_WS, Q + (int64_t)(j * T) * na + i * T, na);
        t.c = opnd(B_X, blk + (int64_t)(j * T) * nj + nn + i * T, nj);
        int id = B.add(t, {f.level, 1, 0, (int)k, j, i});
        B.wait_group(id, qgroup);
      }
    }
  }
  return B.finish(prog, P.grid > 0 ? P.grid : 296);
}

}  // namespace chb
