/*
 * Oracle: plain-C restatement of the reference's multifrontal sweeps.
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  Each sweep follows the cited
 * reference file step by step over the same LIFO update stack; the dense
 * kernels below are straightforward textbook loops (no blocking, no BLAS),
 * so the oracle is slow but easy to audit.  Column-major storage throughout.
 */
#include "oracle.h"

#include <math.h>
#include <string.h>

#define A_(a, ld, i, j) ((a)[(int64_t)(j) * (ld) + (i)])

/* ---------------------------------------------------------------- dense */

/* lower Cholesky in place; returns 0 or the 1-based failing column */
static int potrf_l(int n, double* a, int lda) {
  for (int j = 0; j < n; j++) {
    double d = A_(a, lda, j, j);
    for (int l = 0; l < j; l++) d -= A_(a, lda, j, l) * A_(a, lda, j, l);
    if (!(d > 0.0)) return j + 1;
    d = sqrt(d);
    A_(a, lda, j, j) = d;
    for (int i = j + 1; i < n; i++) {
      double s = A_(a, lda, i, j);
      for (int l = 0; l < j; l++) s -= A_(a, lda, i, l) * A_(a, lda, j, l);
      A_(a, lda, i, j) = s / d;
    }
  }
  return 0;
}

/* B(m x n) := B * L^{-T}, L lower n x n (solve X L^T = B row by row) */
static void trsm_rltn(int m, int n, const double* L, int ldl, double* b, int ldb) {
  for (int i = 0; i < m; i++)
    for (int j = 0; j < n; j++) {
      double s = A_(b, ldb, i, j);
      for (int l = 0; l < j; l++) s -= A_(b, ldb, i, l) * A_(L, ldl, j, l);
      A_(b, ldb, i, j) = s / A_(L, ldl, j, j);
    }
}

/* B(m x n) := B * L^{-1}, L lower n x n (solve X L = B, last column first) */
static void trsm_rlnn(int m, int n, const double* L, int ldl, double* b, int ldb) {
  for (int i = 0; i < m; i++)
    for (int j = n - 1; j >= 0; j--) {
      double s = A_(b, ldb, i, j);
      for (int l = j + 1; l < n; l++) s -= A_(b, ldb, i, l) * A_(L, ldl, l, j);
      A_(b, ldb, i, j) = s / A_(L, ldl, j, j);
    }
}

/* C(n x n, lower) += alpha * A * A^T, A n x k */
static void syrk_ln(int n, int k, double alpha, const double* a, int lda, double* c, int ldc) {
  for (int j = 0; j < n; j++)
    for (int i = j; i < n; i++) {
      double s = 0.0;
      for (int l = 0; l < k; l++) s += A_(a, lda, i, l) * A_(a, lda, j, l);
      A_(c, ldc, i, j) += alpha * s;
    }
}

/* copy the lower trapezoid of an m x n block */
static void lacpy_l(int m, int n, const double* a, int lda, double* b, int ldb) {
  for (int j = 0; j < n; j++)
    for (int i = j; i < m; i++) A_(b, ldb, i, j) = A_(a, lda, i, j);
}

/* ----------------------------------------------------------- sweeps */

/* cholesky.c:3-84 */
int orc_cholesky(int64_t n, int64_t nsn, const int64_t* snpost, const int64_t* snptr, const int64_t* relptr,
                 const int64_t* relidx, const int64_t* chptr, const int64_t* chidx, const int64_t* blkptr,
                 double* blkval, double* fws, double* upd, int64_t* upd_size) {
  (void)n;
  double* U = upd;
  int64_t nup = 0;
  for (int64_t ki = 0; ki < nsn; ki++) {
    int64_t k = snpost[ki];
    int nn = (int)(snptr[k + 1] - snptr[k]);
    int na = (int)(relptr[k + 1] - relptr[k]);
    int nj = nn + na;
    /* frontal matrix: [blk, 0] (cholesky.c:33-38) */
    lacpy_l(nj, nn, blkval + blkptr[k], nj, fws, nj);
    for (int j = nn; j < nj; j++)
      for (int i = j; i < nj; i++) fws[(int64_t)nj * j + i] = 0.0;
    /* extend-add of the children's updates, popped off the stack (:41-52) */
    for (int64_t l = chptr[k + 1] - 1; l >= chptr[k]; l--) {
      nup--;
      U -= upd_size[nup] * upd_size[nup];
      int64_t off = relptr[chidx[l]];
      int N = (int)(relptr[chidx[l] + 1] - off);
      for (int j = 0; j < N; j++)
        for (int i = j; i < N; i++) fws[(int64_t)nj * relidx[off + j] + relidx[off + i]] += U[(int64_t)N * j + i];
    }
    /* L11 (:55-56) */
    int info = potrf_l(nn, fws, nj);
    if (info) return info;
    if (na > 0) {
      trsm_rltn(na, nn, fws, nj, fws + nn, nj);                   /* L21 (:61)   */
      syrk_ln(na, nn, -1.0, fws + nn, nj, fws + (int64_t)nn * nj + nn, nj);  /* (:64-69) */
      trsm_rlnn(na, nn, fws, nj, fws + nn, nj);                   /* (:72)       */
      upd_size[nup++] = na;                                        /* push (:75-77) */
      lacpy_l(na, na, fws + (int64_t)nn * nj + nn, nj, U, na);
      U += (int64_t)na * na;
    }
    lacpy_l(nj, nn, fws, nj, blkval + blkptr[k], nj);             /* (:81) */
  }
  return 0;
}
