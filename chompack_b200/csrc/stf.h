// Sequential task flow on top of DagBuilder: tasks are submitted in program
// order together with the 64x64 tiles they read and write, and the waits
// are inferred (read-after-write, write-after-write and write-after-read),
// so a sweep can be written as the reference's sequential BLAS script.
// Blocked dense routines (Cholesky, triangular solves, SYRK, inverse) are
// expressed as tile tasks through it.
#pragma once
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
      S.submit(t, kg(i, j, 0), acc);
    }
}

// M := L^{-1} (both n x n, lower tiles), from the diagonal-tile inverses.
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
  for (int c = 1; c < nb; c++) {
    kg.step++;
    for (int j = 0; j < c; j++) {
      Task t = make_task(T_MROW);
      t.m = L.tw(c);
      t.n = L.tw(j);
      t.k = (c - j) * TILE;
      t.alpha = -1.0;
      t.a = L.op(c, j);
      t.b = opnd(M.base, M.at(j * TILE, j * TILE), M.ld, OM_TRI_T, 0);
      t.c = M.op(c, j);
      const int64_t moff = Minv.at(c * TILE, 0);
      t.aux[0] = Minv.base;
      t.aux[1] = Minv.ld;
      t.aux[2] = (int32_t)(uint32_t)(moff & 0xffffffffLL);
      t.aux[3] = (int32_t)(moff >> 32);
      std::vector<Stf::Acc> acc{Stf::W(M, c, j), Stf::R(Minv, c, 0)};
      for (int l = j; l < c; l++) {
        acc.push_back(Stf::R(L, c, l));
        acc.push_back(Stf::R(M, l, j));
      }
      S.submit(t, kg(c, j, 1), acc);
    }
  }
}

}  // namespace chb
