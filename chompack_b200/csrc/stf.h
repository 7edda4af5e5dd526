// Sequential task flow on top of DagBuilder: tasks are submitted in program
// order together with the 64x64 tiles they read and write, and the waits
// are inferred (read-after-write, write-after-write and write-after-read),
// so a sweep can be written as the reference's sequential BLAS script.
// Blocked dense routines (Cholesky, triangular solves, SYRK, inverse) are
// expressed as tile tasks through it.
#pragma once
#include <functional>
#include <unordered_map>
#include <vector>

#include "dag.h"

namespace chb {

// A column-major matrix region addressed by tiles of TILE x TILE.
struct Mat {
  int id;          // identity for dependency tracking
  uint8_t base;    // Base slot
  int64_t off;     // element offset of (0, 0)
  int ld;
  int rows, cols;
  int ntr() const { return ceil_div(rows, TILE); }
  int ntc() const { return ceil_div(cols, TILE); }
  int th(int i) const { return std::min(TILE, rows - i * TILE); }
  int tw(int j) const { return std::min(TILE, cols - j * TILE); }
  int64_t at(int r, int c) const { return off + (int64_t)c * ld + r; }
  Operand op(int i, int j, uint8_t mode = OM_N, int diag = 0) const {
    return opnd(base, at(i * TILE, j * TILE), ld, mode, diag);
  }
};

struct Stf {
  struct Acc {
    uint64_t key;
    bool write;
  };
  struct TileState {
    int last = -1;
    std::vector<int> readers;
  };
  DagBuilder& B;
  std::unordered_map<uint64_t, TileState> st;
  int next_mat = 0;
  // Workspace allocator (doubles) for split-K scratch; products with K above
  // ksplit are split along K when it is set.
  std::function<int64_t(int64_t)> alloc;
  int ksplit = 384;

  explicit Stf(DagBuilder& b) : B(b) {}

  Mat mat(uint8_t base, int64_t off, int ld, int rows, int cols) {
    return Mat{next_mat++, base, off, ld, rows, cols};
  }
  // A view of a sub-matrix that shares the tile grid of `m` (the origin must
  // lie on a tile boundary of m).
  static Mat sub(const Mat& m, int r0, int c0, int rows, int cols) {
    Mat s = m;
    s.off = m.at(r0, c0);
    s.rows = rows;
    s.cols = cols;
    s.id = m.id;
    return s;
  }
  static uint64_t key(const Mat& m, int i, int j) {
    return ((uint64_t)(uint32_t)m.id << 32) | ((uint64_t)(i & 0xffff) << 16) | (uint64_t)(j & 0xffff);
  }
  static Acc R(const Mat& m, int i, int j) { return {key(m, i, j), false}; }
  static Acc W(const Mat& m, int i, int j) { return {key(m, i, j), true}; }

  // All tiles of m (or of its lower triangle).
  static void all(std::vector<Acc>& v, const Mat& m, bool write, bool lower_only = false) {
    for (int j = 0; j < m.ntc(); j++)
      for (int i = lower_only ? j : 0; i < m.ntr(); i++) v.push_back({key(m, i, j), write});
  }

  int submit(const Task& t, const SchedKey& k, const std::vector<Acc>& acc, int group = -1, double est = -1.0,
             const std::vector<int>& extra_waits = {}) {
    const int id = B.add(t, k, group, est);
    for (const Acc& a : acc) {
      auto it = st.find(a.key);
      if (it == st.end()) continue;
      if (it->second.last >= 0) B.wait_task(id, it->second.last);
      if (a.write)
        for (int r : it->second.readers) B.wait_task(id, r);
    }
    for (int w : extra_waits) B.wait_task(id, w);
    for (const Acc& a : acc) {
      TileState& s = st[a.key];
      if (a.write) {
        s.last = id;
        s.readers.clear();
      } else if (s.last != id) {
        s.readers.push_back(id);
      }
    }
    return id;
  }
  // Accesses of a task already added to the builder (e.g. by
  // add_split_gemm): the same inference as submit.
  void submit_existing(int id, const std::vector<Acc>& acc) {
    for (const Acc& a : acc) {
      auto it = st.find(a.key);
      if (it == st.end()) continue;
      if (it->second.last >= 0 && it->second.last != id) B.wait_task(id, it->second.last);
      if (a.write)
        for (int r : it->second.readers)
          if (r != id) B.wait_task(id, r);
    }
    for (const Acc& a : acc) {
      TileState& s = st[a.key];
      if (a.write) {
        s.last = id;
        s.readers.clear();
      } else if (s.last != id) {
        s.readers.push_back(id);
      }
    }
  }
  // A GEMM-type task (T_GEMM or T_MROW): split along K into parallel parts
  // and a fixed-order sum when long and a scratch allocator is set; the
  // parts carry the reads of `acc`, the sum its writes.
  int gemm(const Task& t, const SchedKey& key, const std::vector<Acc>& acc) {
    if (!alloc || split_count(t.k, ksplit) == 1) return submit(t, key, acc);
    const int64_t scr = alloc((int64_t)split_count(t.k, ksplit) * TILE * TILE);
    SplitTask sp = add_split_gemm(B, t, ksplit, scr, key);
    const std::vector<Acc> rd = reads_only(acc);
    std::vector<Acc> wr;
    for (const Acc& a : acc)
      if (a.write) wr.push_back(a);
    for (int id : sp.parts) submit_existing(id, rd);
    submit_existing(sp.out, wr);
    return sp.out;
  }
  static std::vector<Acc> reads_only(const std::vector<Acc>& acc) {
    std::vector<Acc> r;
    for (const Acc& a : acc)
      if (!a.write) r.push_back(a);
    return r;
  }
  // A group wait on top of the inferred ones (e.g. a child's update coming
  // from a tracked matrix of another front is handled by tiles; this is for
  // explicit groups).
  void wait_group(int id, int g) { B.wait_group(id, g); }
};

// ---------------------------------------------------------------------------
// Blocked dense routines on tiles.  `key` supplies the scheduling key (level,
// step base, front); `Minv` receives the inverses of the diagonal tiles of L
// (an n x TILE matrix: tile c at rows cT) when a routine needs them.

struct KeyGen {
  int level, front;
  int step = 0;
  SchedKey operator()(int i = 0, int j = 0, int rank = 0) { return SchedKey{level, step, rank, front, j, i}; }
};

// Lower Cholesky of the n x n matrix A in place (lower tiles), writing the
// inverses of its diagonal tiles to Minv (n x 64).  info_base: offset added
// to the failing column.
inline void stf_potrf(Stf& S, KeyGen& kg, const Mat& A, const Mat& Minv, int info_base = 0) {
  const int nb = A.ntr();
  for (int c = 0; c < nb; c++) {
    kg.step++;
    Task t = make_task(T_POTRF);
    t.m = t.n = A.tw(c);
    t.a = A.op(c, c);
    t.c = Minv.op(c, 0);
    t.aux[0] = info_base + c * TILE;
    t.aux[1] = 1;
    S.submit(t, kg(c, c, 0), {Stf::W(A, c, c), Stf::W(Minv, c, 0)});
    for (int r = c + 1; r < nb; r++) {
      Task g = gemm(A.th(r), A.tw(c), A.tw(c), 1.0, A.op(r, c), Minv.op(c, 0, OM_TRI_N, 0), 0.0, A.op(r, c));
      S.submit(g, kg(r, c, 1), {Stf::W(A, r, c), Stf::R(Minv, c, 0)});
    }
    for (int j = c + 1; j < nb; j++)
      for (int r = j; r < nb; r++) {
        Task g = gemm(A.th(r), A.tw(j), A.tw(c), -1.0, A.op(r, c), A.op(j, c), 1.0, A.op(r, j), r == j, 0);
        S.submit(g, kg(r, j, 2), {Stf::W(A, r, j), Stf::R(A, r, c), Stf::R(A, j, c)});
      }
  }
}

// Inverses of the diagonal tiles of a lower-triangular L (already a factor).
inline void stf_diag_inverses(Stf& S, KeyGen& kg, const Mat& L, const Mat& Minv, int info_base = 0) {
  kg.step++;
  for (int c = 0; c < L.ntr(); c++) {
    Task t = make_task(T_POTRF);
    t.m = t.n = L.tw(c);
    t.a = L.op(c, c);
    t.c = Minv.op(c, 0);
    t.aux[0] = info_base + c * TILE;
    t.aux[1] = 1;
    t.aux[2] = 1;
    S.submit(t, kg(c, c, 0), {Stf::R(L, c, c), Stf::W(Minv, c, 0)});
  }
}

// X := op(L)^{-1} X, L lower n x n with diagonal-tile inverses Minv, X n x m
// (in place).  trans = false: forward substitution; true: with L^T,
// backward substitution.
inline void stf_trsm_left(Stf& S, KeyGen& kg, const Mat& L, const Mat& Minv, const Mat& X, bool trans) {
  const int nb = L.ntr(), mb = X.ntc();
  for (int cc = 0; cc < nb; cc++) {
    const int c = trans ? nb - 1 - cc : cc;
    kg.step++;
    for (int s = 0; s < mb; s++) {
      Operand m = trans ? Minv.op(c, 0, OM_TRI_T, 0) : Minv.op(c, 0, OM_TRI_N, 0);
      Task t = gemm(X.th(c), X.tw(s), L.tw(c), 1.0, m, X.op(c, s, OM_T), 0.0, X.op(c, s));
      S.submit(t, kg(c, s, 0), {Stf::W(X, c, s), Stf::R(Minv, c, 0)});
      if (!trans) {
        for (int r = c + 1; r < nb; r++) {
          Task u = gemm(X.th(r), X.tw(s), L.tw(c), -1.0, L.op(r, c), X.op(c, s, OM_T), 1.0, X.op(r, s));
          S.submit(u, kg(r, s, 1), {Stf::W(X, r, s), Stf::R(X, c, s), Stf::R(L, r, c)});
        }
      } else {
        for (int r = 0; r < c; r++) {
          Task u = gemm(X.th(r), X.tw(s), L.tw(c), -1.0, L.op(c, r, OM_T), X.op(c, s, OM_T), 1.0, X.op(r, s));
          S.submit(u, kg(r, s, 1), {Stf::W(X, r, s), Stf::R(X, c, s), Stf::R(L, c, r)});
        }
      }
    }
  }
}

// C (n x n, lower tiles) := alpha X^T X + beta C, X is k x n.
inline void stf_syrk_t(Stf& S, KeyGen& kg, const Mat& X, const Mat& C, double alpha, double beta) {
  kg.step++;
  const int nb = C.ntr();
  for (int j = 0; j < nb; j++)
    for (int i = j; i < nb; i++) {
      std::vector<Stf::Acc> acc{Stf::W(C, i, j)};
      for (int l = 0; l < X.ntr(); l++) {
        acc.push_back(Stf::R(X, l, i));
        acc.push_back(Stf::R(X, l, j));
      }
      Operand a = opnd(X.base, X.at(0, i * TILE), X.ld, OM_T);
      Operand b = opnd(X.base, X.at(0, j * TILE), X.ld, OM_T);
      Task t = gemm(C.th(i), C.tw(j), X.rows, alpha, a, b, beta, C.op(i, j), i == j, 0);
      S.gemm(t, kg(i, j, 0), acc);
    }
}

// M := L^{-1} (both n x n, lower tiles), from the diagonal-tile inverses,
// right-looking by block column j: as soon as M(l, j) is final,
// T(c, j) += L(c, l) M(l, j) for every c > l (accumulated in place at
// M(c, j)), then M(l+1, j) = -Minv_{l+1} T(l+1, j).  The dependent chain per
// column is two 64x64 tiles per block row.
inline void stf_tri_inverse(Stf& S, KeyGen& kg, const Mat& L, const Mat& Minv, const Mat& M) {
  const int nb = L.ntr();
  kg.step++;
  for (int c = 0; c < nb; c++) {  // diagonal tiles of M
    Task t = make_task(T_COPY);
    t.m = L.tw(c);
    t.n = L.tw(c);
    t.a = Minv.op(c, 0);
    t.c = M.op(c, c);
    S.submit(t, kg(c, c, 0), {Stf::R(Minv, c, 0), Stf::W(M, c, c)});
  }
  for (int l = 0; l + 1 < nb; l++) {
    kg.step++;
    for (int j = 0; j <= l; j++) {
      for (int c = l + 1; c < nb; c++) {
        Operand b = opnd(M.base, M.at(l * TILE, j * TILE), M.ld, OM_T, 0);  // M(l, j)^T
        Task t = gemm(L.tw(c), L.tw(j), L.tw(l), 1.0, L.op(c, l), b, l == j ? 0.0 : 1.0, M.op(c, j));
        S.submit(t, kg(c, j, 1), {Stf::W(M, c, j), Stf::R(L, c, l), Stf::R(M, l, j)});
      }
      const int c = l + 1;
      Operand b = opnd(M.base, M.at(c * TILE, j * TILE), M.ld, OM_T, 0);   // T(c, j)^T
      Task t = gemm(L.tw(c), L.tw(j), L.tw(c), -1.0, Minv.op(c, 0), b, 0.0, M.op(c, j));
      S.submit(t, kg(c, j, 2), {Stf::W(M, c, j), Stf::R(Minv, c, 0)});
    }
  }
}

// dst := the anti-transpose of src's lower triangle (both n x n, lower
// tiles): dst(i, j) = src(n-1-j, n-1-i).  With J the order-reversing
// permutation, dst holds J src J (lower part).
inline void stf_antitranspose(Stf& S, KeyGen& kg, const Mat& src, const Mat& dst, int n) {
  kg.step++;
  for (int j = 0; j < dst.ntc(); j++)
    for (int i = j; i < dst.ntr(); i++) {
      Task t = make_task(T_COPY);
      t.m = dst.th(i);
      t.n = dst.tw(j);
      t.a = opnd(src.base, src.off, src.ld);
      t.c = opnd(dst.base, dst.off, dst.ld);
      t.aux[0] = 8 | 1;  // anti-transpose, lower part
      t.aux[1] = n;
      t.aux[2] = i * TILE;
      t.aux[3] = j * TILE;
      // dst rows iT.. come from src columns n-1-r, dst columns jT.. from src rows
      const int c_hi = n - 1 - i * TILE, c_lo = n - i * TILE - dst.th(i);
      const int r_hi = n - 1 - j * TILE, r_lo = n - j * TILE - dst.tw(j);
      std::vector<Stf::Acc> acc{Stf::W(dst, i, j)};
      for (int sj = c_lo / TILE; sj <= c_hi / TILE; sj++)
        for (int si = r_lo / TILE; si <= r_hi / TILE; si++)
          if (si >= sj) acc.push_back(Stf::R(src, si, sj));
      S.submit(t, kg(i, j, 0), acc);
    }
}

// Tile accesses of rows [r0, r1) of column tile j.
inline void rows_acc(std::vector<Stf::Acc>& v, const Mat& m, int r0, int r1, int j, bool write) {
  if (r1 <= r0) return;
  for (int i = r0 / TILE; i <= (r1 - 1) / TILE; i++) v.push_back({Stf::key(m, i, j), write});
}

// The factored update of child c (update_factor.c:3-108), as tile tasks.
// The parent front is F = [F11, F21^T; F21, F22] with F22 = L_k, the lower
// factor of the parent's update V_k = L_k^T L_k; Vc (N x N) receives the
// lower-triangular U_c with U_c^T U_c = F[r_c, r_c], written at
// WS + upd_base + fronts[c].upd.  Steps, with r_c[:N1] < nn <= r_c[N1:]:
//   U_c(:, :N1) = F[r_c, r_c[:N1]]                        (:17-22)
//   [0; L22] = Q^T L_k(:, r_c[N1:] - nn), Householder QL (:24-47), blocked:
//     panels of nb columns factored in shared memory (T_QL), the columns to
//     their left updated by C -= W' T (W'^T C) (MROW + GEMM tiles);
//   U22 = L22; U21 = L22^{-T} U21 (dtrtrs, :51-52); U11 -= U21^T U21 (:54);
//   U11 = L11 with U11 = L11^T L11 (the reversed Cholesky of :57-87).
// `alloc` hands out workspace (doubles).  Returns 0, or a negative code
// (error text set) when a Householder column does not fit shared memory.
inline int stf_update_factor(Stf& S, KeyGen& kg, const chb_plan& P, int c, const Mat& F11, const Mat& F21,
                             const Mat& F22, const Mat& Vc, int64_t upd_base,
                             const std::function<int64_t(int64_t)>& alloc) {
  const FrontDesc& ch = P.fronts[c];
  const FrontDesc& f = P.fronts[ch.parent];
  const int N = ch.na, nn = f.nn, na = f.na;
  const int32_t* r = P.relidx.data() + ch.relptr;
  int N1 = 0;
  while (N1 < N && r[N1] < nn) N1++;
  const int N2 = N - N1;
  const int64_t vbase = upd_base + ch.upd;
  const Mat U11 = S.mat(B_WS, vbase, std::max(N, 1), N1, N1);
  const Mat U21 = S.mat(B_WS, vbase + N1, std::max(N, 1), N2, N1);
  const Mat U22 = S.mat(B_WS, vbase + (int64_t)N1 * N + N1, std::max(N, 1), N2, N2);
  // U_c(:, :N1) = F[r, r[:N1]]
  if (N1 > 0) {
    kg.step++;
    std::vector<Stf::Acc> rd;
    Stf::all(rd, F11, false, true);
    Stf::all(rd, F21, false);
    const int CH = TILE;  // one column tile of U11/U21 per chunk: parallel chunks
    for (int q0 = 0; q0 < N1; q0 += CH) {
      std::vector<Stf::Acc> acc = rd;
      const int qt = q0 / TILE;
      for (int i = qt; i < U11.ntr(); i++) acc.push_back(Stf::W(U11, i, qt));
      for (int i = 0; i < U21.ntr(); i++) acc.push_back(Stf::W(U21, i, qt));
      Task t = make_task(T_EXTRACT);
      t.aux[0] = c;
      t.aux[1] = q0;
      t.aux[2] = std::min(N1, q0 + CH);
      t.a = opnd(F11.base, F11.off, F11.ld);
      t.b = opnd(F21.base, F21.off, F21.ld);
      t.c = opnd(F22.base, F22.off, F22.ld);
      t.off2 = upd_base;
      S.submit(t, kg(0, c, q0), acc, -1, 3.0 + (double)(N - q0) * CH / 2000.0);
    }
  }
  if (N2 > 0) {
    const Mat C = S.mat(B_WS, alloc((int64_t)na * N2), na, na, N2);
    const int64_t woff = alloc((int64_t)na * N2), toff = alloc((int64_t)TILE * N2);
    const Mat Z = S.mat(B_WS, alloc((int64_t)TILE * N2), TILE, TILE, N2);
    // C = L_k(:, jj)
    kg.step++;
    std::vector<Stf::Acc> rd22;
    Stf::all(rd22, F22, false, true);
    for (int j = 0; j < C.ntc(); j++) {
      std::vector<Stf::Acc> acc = rd22;
      rows_acc(acc, C, 0, na, j, true);
      Task t = make_task(T_QL);
      t.aux[0] = c;
      t.aux[1] = j * TILE;
      t.aux[2] = j * TILE + C.tw(j);
      t.aux[3] = QL_GATHER;
      t.a = opnd(F22.base, F22.off, F22.ld);
      t.c = opnd(B_WS, C.off, na);
      S.submit(t, kg(0, c, j), acc, -1, 2.0 + (double)na * C.tw(j) / 4000.0);
    }
    // panels, right to left; a panel never crosses a 64-column tile
    int c1 = N2;
    while (c1 > 0) {
      const int tile = (c1 - 1) / TILE, tstart = tile * TILE;
      const int row1 = na - N2 + c1 - 1;
      auto h_of = [&](int nb) { return row1 - (r[N1 + c1 - nb] - nn) + 1; };
      int nb = 0;
      while (nb < c1 - tstart && ql_panel_doubles(h_of(nb + 1), nb + 1) <= ENGINE_SMEM_DOUBLES) nb++;
      if (nb == 0) return set_error(-1, "update_factor: a Householder column of %d rows exceeds shared memory", h_of(1));
      const int c0 = c1 - nb;
      const int row0 = r[N1 + c0] - nn, h = row1 - row0 + 1;
      const Mat Wp = S.mat(B_WS, woff + (int64_t)c0 * na, na, na, nb);
      const Mat Tp = S.mat(B_WS, toff + (int64_t)c0 * TILE, TILE, nb, nb);
      kg.step++;
      {
        std::vector<Stf::Acc> acc;
        rows_acc(acc, C, row0, row1 + 1, tile, true);
        Stf::all(acc, Wp, true);
        Stf::all(acc, Tp, true);
        Task t = make_task(T_QL);
        t.aux[0] = c;
        t.aux[1] = c0;
        t.aux[2] = c1;
        t.aux[3] = QL_PANEL;
        t.a = opnd(B_WS, C.off, na);
        t.b = opnd(B_WS, woff, na);
        t.c = opnd(B_WS, Tp.off, TILE);
        S.submit(t, kg(0, c, c1), acc, -1, 4.0 + (double)nb * h * nb / 3000.0);
      }
      // columns [0, c0): C(row0:row1, :) -= W' T (W'^T C(row0:row1, :))
      kg.step++;
      for (int t2 = 0; t2 * TILE < c0; t2++) {
        const int x0 = t2 * TILE, w = std::min(TILE, c0 - x0);
        {
          // Z = T (W'^T C): long K (the panel's row span) is split, each
          // part carrying the T factor (it distributes over the sum)
          std::vector<Stf::Acc> acc{Stf::W(Z, 0, t2), Stf::R(Tp, 0, 0)};
          rows_acc(acc, Wp, row0, row1 + 1, 0, false);
          rows_acc(acc, C, row0, row1 + 1, t2, false);
          Task t = make_task(T_MROW);
          t.m = nb;
          t.n = w;
          t.k = h;
          t.alpha = 1.0;
          t.a = opnd(B_WS, Wp.at(row0, 0), na, OM_T);
          t.b = opnd(B_WS, C.at(row0, x0), na, OM_T);
          t.c = opnd(B_WS, Z.at(0, x0), TILE);
          t.aux[0] = B_WS;
          t.aux[1] = TILE;
          t.aux[2] = (int32_t)(uint32_t)(Tp.off & 0xffffffffLL);
          t.aux[3] = (int32_t)(Tp.off >> 32);
          S.gemm(t, kg(0, c, t2), acc);
        }
        for (int i = row0 / TILE; i <= row1 / TILE; i++) {
          const int rs = std::max(i * TILE, row0), re = std::min(i * TILE + TILE, row1 + 1);
          Task g = gemm(re - rs, w, nb, -1.0, opnd(B_WS, Wp.at(rs, 0), na), opnd(B_WS, Z.at(0, x0), TILE, OM_T), 1.0,
                        opnd(B_WS, C.at(rs, x0), na));
          S.submit(g, kg(i, c, t2 + 1), {Stf::W(C, i, t2), Stf::R(Wp, i, 0), Stf::R(Z, 0, t2)});
        }
      }
      c1 = c0;
    }
    // U22 = L22 (the last N2 rows of C)
    kg.step++;
    for (int j = 0; j < U22.ntc(); j++)
      for (int i = j; i < U22.ntr(); i++) {
        Task t = make_task(T_COPY);
        t.m = U22.th(i);
        t.n = U22.tw(j);
        t.aux[0] = (i == j) ? 1 : 0;
        t.a = opnd(B_WS, C.at(na - N2 + i * TILE, j * TILE), na);
        t.c = U22.op(i, j);
        std::vector<Stf::Acc> acc{Stf::W(U22, i, j)};
        rows_acc(acc, C, na - N2 + i * TILE, na - N2 + i * TILE + U22.th(i), j, false);
        S.submit(t, kg(i, c, j), acc);
      }
    // U21 := L22^{-T} U21; U11 -= U21^T U21
    const Mat M22 = S.mat(B_WS, alloc((int64_t)N2 * TILE), N2, N2, TILE);
    stf_diag_inverses(S, kg, U22, M22);
    if (N1 > 0) {
      stf_trsm_left(S, kg, U22, M22, U21, true);
      stf_syrk_t(S, kg, U21, U11, -1.0, 1.0);
    }
  }
  // U11 = L11 with U11 = L11^T L11: J U11 J = L' L'^T, L11 = J L'^T J
  if (N1 > 0) {
    const Mat R = S.mat(B_WS, alloc((int64_t)N1 * N1), N1, N1, N1);
    const Mat MR = S.mat(B_WS, alloc((int64_t)N1 * TILE), N1, N1, TILE);
    stf_antitranspose(S, kg, U11, R, N1);
    stf_potrf(S, kg, R, MR);
    stf_antitranspose(S, kg, R, U11, N1);
  }
  // join: the consumers of Vc see every write above
  kg.step++;
  std::vector<Stf::Acc> acc;
  Stf::all(acc, Vc, true, true);
  Stf::all(acc, U11, false, true);
  Stf::all(acc, U21, false);
  Stf::all(acc, U22, false, true);
  S.submit(make_task(T_NOP), kg(0, c, 0), acc, -1, 0.5);
  return 0;
}

}  // namespace chb
