/*
 * Oracle: plain-C restatement of the reference's multifrontal sweeps.
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  Each sweep follows the cited
 * reference file step by step over the same LIFO update stack; the dense
 * kernels below are straightforward textbook loops (no blocking, no BLAS),
 * so the oracle is slow but easy to audit.  Column-major storage throughout.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
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


/* ---- generic naive dense kernels (column-major; "lower" = lower triangle) */

/* element (i, j) of op(A) */
static double opel(const double* a, int lda, int trans, int i, int j) {
  return trans ? A_(a, lda, j, i) : A_(a, lda, i, j);
}

/* element (i, j) of the lower-triangular L (zero above the diagonal) */
static double trel(const double* l, int ldl, int i, int j) { return i >= j ? A_(l, ldl, i, j) : 0.0; }

/* C(m x n) = alpha op(A) op(B) + beta C; C is not read when beta == 0 */
static void gemm(int ta, int tb, int m, int n, int k, double alpha, const double* a, int lda, const double* b,
                 int ldb, double beta, double* c, int ldc) {
  for (int j = 0; j < n; j++)
    for (int i = 0; i < m; i++) {
      double s = 0.0;
      for (int l = 0; l < k; l++) s += opel(a, lda, ta, i, l) * opel(b, ldb, tb, l, j);
      A_(c, ldc, i, j) = alpha * s + (beta == 0.0 ? 0.0 : beta * A_(c, ldc, i, j));
    }
}

/* lower part of C(n x n) = alpha op(A) op(A)^T + beta C, op(A) n x k */
static void syrk_l(int trans, int n, int k, double alpha, const double* a, int lda, double beta, double* c,
                   int ldc) {
  for (int j = 0; j < n; j++)
    for (int i = j; i < n; i++) {
      double s = 0.0;
      for (int l = 0; l < k; l++) s += opel(a, lda, trans, i, l) * opel(a, lda, trans, j, l);
      A_(c, ldc, i, j) = alpha * s + (beta == 0.0 ? 0.0 : beta * A_(c, ldc, i, j));
    }
}

/* element (i, j) of the symmetric matrix whose lower triangle is stored */
static double syel(const double* s, int lds, int i, int j) { return i >= j ? A_(s, lds, i, j) : A_(s, lds, j, i); }

/* C(m x n) = alpha S B + beta C (right: alpha B S + beta C); S symmetric,
 * lower-stored, of order m (right: n) */
static void symm_l(int right, int m, int n, double alpha, const double* sy, int lds, const double* b, int ldb,
                   double beta, double* c, int ldc) {
  for (int j = 0; j < n; j++)
    for (int i = 0; i < m; i++) {
      double s = 0.0;
      if (!right)
        for (int l = 0; l < m; l++) s += syel(sy, lds, i, l) * A_(b, ldb, l, j);
      else
        for (int l = 0; l < n; l++) s += A_(b, ldb, i, l) * syel(sy, lds, l, j);
      A_(c, ldc, i, j) = alpha * s + (beta == 0.0 ? 0.0 : beta * A_(c, ldc, i, j));
    }
}

/* B(m x n) := op(L) B (right: B op(L)), L lower; through a copy of B */
static void trmm_l(int right, int trans, int m, int n, const double* l, int ldl, double* b, int ldb) {
  double* t = malloc(sizeof(double) * (size_t)m * n + 8);
  for (int j = 0; j < n; j++)
    for (int i = 0; i < m; i++) t[(int64_t)j * m + i] = A_(b, ldb, i, j);
  for (int j = 0; j < n; j++)
    for (int i = 0; i < m; i++) {
      double s = 0.0;
      if (!right)
        for (int q = 0; q < m; q++) s += (trans ? trel(l, ldl, q, i) : trel(l, ldl, i, q)) * t[(int64_t)j * m + q];
      else
        for (int q = 0; q < n; q++) s += t[(int64_t)q * m + i] * (trans ? trel(l, ldl, j, q) : trel(l, ldl, q, j));
      A_(b, ldb, i, j) = s;
    }
  free(t);
}

/* B(m x n) := op(L)^{-1} B (right: B op(L)^{-1}), L lower, by substitution.
 * Returns 0, or the 1-based index of a zero diagonal entry (dtrtrs). */
static int trsm_l(int right, int trans, int m, int n, const double* l, int ldl, double* b, int ldb) {
  const int o = right ? n : m;
  for (int d = 0; d < o; d++)
    if (A_(l, ldl, d, d) == 0.0) return d + 1;
  if (!right) {
    for (int j = 0; j < n; j++) {
      if (!trans) {   /* forward: L x = b */
        for (int i = 0; i < m; i++) {
          double s = A_(b, ldb, i, j);
          for (int q = 0; q < i; q++) s -= A_(l, ldl, i, q) * A_(b, ldb, q, j);
          A_(b, ldb, i, j) = s / A_(l, ldl, i, i);
        }
      } else {        /* backward: L^T x = b */
        for (int i = m - 1; i >= 0; i--) {
          double s = A_(b, ldb, i, j);
          for (int q = i + 1; q < m; q++) s -= A_(l, ldl, q, i) * A_(b, ldb, q, j);
          A_(b, ldb, i, j) = s / A_(l, ldl, i, i);
        }
      }
    }
  } else {
    for (int i = 0; i < m; i++) {
      if (!trans) {   /* x L = b: last column first */
        for (int j = n - 1; j >= 0; j--) {
          double s = A_(b, ldb, i, j);
          for (int q = j + 1; q < n; q++) s -= A_(b, ldb, i, q) * A_(l, ldl, q, j);
          A_(b, ldb, i, j) = s / A_(l, ldl, j, j);
        }
      } else {        /* x L^T = b: first column first */
        for (int j = 0; j < n; j++) {
          double s = A_(b, ldb, i, j);
          for (int q = 0; q < j; q++) s -= A_(b, ldb, i, q) * A_(l, ldl, j, q);
          A_(b, ldb, i, j) = s / A_(l, ldl, j, j);
        }
      }
    }
  }
  return 0;
}

/* L := L^{-1} in place (lower, non-unit); 1-based index of a zero pivot */
static int trtri_l(int n, double* l, int ldl) {
  for (int d = 0; d < n; d++)
    if (A_(l, ldl, d, d) == 0.0) return d + 1;
  double* x = malloc(sizeof(double) * (size_t)n * n + 8);
  for (int j = 0; j < n; j++)       /* column j of L^{-1}: L x = e_j */
    for (int i = 0; i < n; i++) {
      double s = (i == j) ? 1.0 : 0.0;
      for (int q = j; q < i; q++) s -= A_(l, ldl, i, q) * x[(int64_t)j * n + q];
      x[(int64_t)j * n + i] = (i < j) ? 0.0 : s / A_(l, ldl, i, i);
    }
  for (int j = 0; j < n; j++)
    for (int i = j; i < n; i++) A_(l, ldl, i, j) = x[(int64_t)j * n + i];
  free(x);
  return 0;
}

/* upper Cholesky A = U^T U in place (upper triangle); 1-based failing column */
static int potrf_u(int n, double* a, int lda) {
  for (int j = 0; j < n; j++) {
    double d = A_(a, lda, j, j);
    for (int q = 0; q < j; q++) d -= A_(a, lda, q, j) * A_(a, lda, q, j);
    if (!(d > 0.0)) return j + 1;
    d = sqrt(d);
    A_(a, lda, j, j) = d;
    for (int i = j + 1; i < n; i++) {
      double s = A_(a, lda, j, i);
      for (int q = 0; q < j; q++) s -= A_(a, lda, q, j) * A_(a, lda, q, i);
      A_(a, lda, j, i) = s / d;
    }
  }
  return 0;
}

/* zero the strict upper triangle of the n x n block */
static void zero_upper(int n, double* a, int lda) {
  for (int j = 1; j < n; j++)
    for (int i = 0; i < j; i++) A_(a, lda, i, j) = 0.0;
}

/* extend-add: F[r, r] += U (lower parts), U N x N */
static void extend_add(double* f, int ldf, const int64_t* r, int N, const double* u) {
  for (int j = 0; j < N; j++)
    for (int i = j; i < N; i++) f[(int64_t)ldf * r[j] + r[i]] += u[(int64_t)N * j + i];
}

/* U = F[r, r] (lower parts) */
static void extract(const double* f, int ldf, const int64_t* r, int N, double* u) {
  for (int j = 0; j < N; j++)
    for (int i = j; i < N; i++) u[(int64_t)N * j + i] = f[(int64_t)ldf * r[j] + r[i]];
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

/* llt.c:3-60: X = L L^T, postorder */
void orc_llt(int64_t n, int64_t nsn, const int64_t* snpost, const int64_t* snptr, const int64_t* relptr,
             const int64_t* relidx, const int64_t* chptr, const int64_t* chidx, const int64_t* blkptr,
             double* blkval, double* fws, double* upd, int64_t* upd_size) {
  (void)n;
  double* U = upd;
  int64_t nup = 0;
  for (int64_t ki = 0; ki < nsn; ki++) {
    const int64_t k = snpost[ki];
    const int nn = (int)(snptr[k + 1] - snptr[k]), na = (int)(relptr[k + 1] - relptr[k]), nj = nn + na;
    double* blk = blkval + blkptr[k];
    trmm_l(1, 0, na, nn, blk, nj, blk + nn, nj);          /* L21 := L21 L11 (:29)      */
    syrk_l(0, nj, nn, 1.0, blk, nj, 0.0, fws, nj);        /* F = [L11; L21][.]^T (:30) */
    for (int64_t l = chptr[k + 1] - 1; l >= chptr[k]; l--) { /* pop, extend-add (:33-43) */
      nup--;
      U -= upd_size[nup] * upd_size[nup];
      const int64_t off = relptr[chidx[l]];
      extend_add(fws, nj, relidx + off, (int)(relptr[chidx[l] + 1] - off), U);
    }
    if (na > 0) {                                          /* push (:46-50)             */
      upd_size[nup++] = na;
      lacpy_l(na, na, fws + (int64_t)nn * nj + nn, nj, U, na);
      U += (int64_t)na * na;
    }
    lacpy_l(nj, nn, fws, nj, blk, nj);                     /* (:53)                     */
  }
}

/* projected_inverse.c:3-75: Y = P(X^{-1}), reverse postorder */
int orc_projected_inverse(int64_t n, int64_t nsn, const int64_t* snpost, const int64_t* snptr,
                          const int64_t* relptr, const int64_t* relidx, const int64_t* chptr, const int64_t* chidx,
                          const int64_t* blkptr, double* blkval, double* fws, double* upd, int64_t* upd_size) {
  (void)n;
  double* U = upd;
  int64_t nup = 0;
  for (int64_t ki = nsn - 1; ki >= 0; ki--) {
    const int64_t k = snpost[ki];
    const int nn = (int)(snptr[k + 1] - snptr[k]), na = (int)(relptr[k + 1] - relptr[k]), nj = nn + na;
    double* blk = blkval + blkptr[k];
    const int info = trtri_l(nn, blk, nj);                 /* L11^{-1} (:33-34)         */
    if (info) return info;
    zero_upper(nn, blk, nj);                               /* (:36-38)                  */
    syrk_l(1, nn, nn, 1.0, blk, nj, 0.0, fws, nj);         /* F11 = L11^{-T} L11^{-1}   */
    if (na > 0) {
      nup--;                                               /* pop V_k (:45-48)          */
      U -= upd_size[nup] * upd_size[nup];
      lacpy_l(na, na, U, na, fws + (int64_t)nn * nj + nn, nj);
      /* F21 = -V_k L21 (:50-51); F11 -= F21^T L21 (:53-54) */
      symm_l(0, na, nn, -1.0, fws + (int64_t)nn * nj + nn, nj, blk + nn, nj, 0.0, fws + nn, nj);
      gemm(1, 0, nn, nn, na, -1.0, fws + nn, nj, blk + nn, nj, 1.0, fws, nj);
    }
    for (int64_t l = chptr[k]; l < chptr[k + 1]; l++) {    /* push children's (:58-70)  */
      const int64_t off = relptr[chidx[l]];
      const int N = (int)(relptr[chidx[l] + 1] - off);
      upd_size[nup++] = N;
      extract(fws, nj, relidx + off, N, U);
      U += (int64_t)N * N;
    }
    lacpy_l(nj, nn, fws, nj, blk, nj);                     /* (:73)                     */
  }
  return 0;
}

/* dlarfg (LAPACK): H [alpha; x] = [beta; 0], H = I - tau v v^T, v = [1; x'].
 * On exit alpha holds beta and x holds x'.  (The safe-minimum rescaling of
 * LAPACK is left out: it only acts when |beta| < 2^-1022.) */
static double larfg(int m, double* alpha, double* x) {
  if (m <= 1) return 0.0;
  double xn2 = 0.0;
  for (int i = 0; i < m - 1; i++) xn2 += x[i] * x[i];
  if (xn2 == 0.0) return 0.0;
  const double a = *alpha, xa = fabs(a), xb = sqrt(xn2);
  const double w = xa > xb ? xa : xb, z = xa > xb ? xb : xa;
  const double nrm = (z == 0.0) ? w : w * sqrt(1.0 + (z / w) * (z / w));   /* dlapy2 */
  const double beta = -copysign(nrm, a);
  const double tau = (beta - a) / beta, scal = 1.0 / (a - beta);
  for (int i = 0; i < m - 1; i++) x[i] *= scal;
  *alpha = beta;
  return tau;
}

/* update_factor.c:3-108.  Lower U_c (N x N, ld N) with U_c^T U_c = F[r, r]
 * for the front F (ld ldf, F22 = L_k with V_k = L_k^T L_k); C is scratch of
 * na x N2.  Returns 0 or an info code. */
static int update_factor_o(const int64_t* r, int nn, int na, double* u, int N, const double* f, int ldf,
                           double* C) {
  int N1 = 0;
  while (N1 < N && r[N1] < nn) N1++;
  const int N2 = N - N1;
  for (int j = 0; j < N1; j++)                              /* A and B (:24-28)           */
    for (int i = j; i < N; i++) u[(int64_t)N * j + i] = f[(int64_t)ldf * r[j] + r[i]];
  if (N2 > 0) {
    for (int j = 0; j < N2; j++) {                           /* C = L_k(:, r[N1:]) (:31-37) */
      const int jj = (int)r[N1 + j];
      for (int i = 0; i < na; i++) C[(int64_t)na * j + i] = (i + nn >= jj) ? f[(int64_t)ldf * jj + i + nn] : 0.0;
    }
    for (int j = 0; j < N2; j++) {                           /* QL by reflections (:39-47) */
      const int col = N2 - 1 - j, prow = na - 1 - j;
      const int x0 = (int)r[N1 + col] - nn;                  /* first nonzero row          */
      const int m = prow - x0 + 1;
      if (m <= 1) continue;
      double* cc = C + (int64_t)na * col;
      const double tau = larfg(m, cc + prow, cc + x0);
      if (tau == 0.0) continue;
      for (int q = 0; q < col; q++) {                        /* dlarfx on columns < col    */
        double* cq = C + (int64_t)na * q;
        double w = cq[prow];
        for (int i = x0; i < prow; i++) w += cc[i] * cq[i];
        w *= tau;
        cq[prow] -= w;
        for (int i = x0; i < prow; i++) cq[i] -= cc[i] * w;
      }
    }
    for (int j = 0; j < N2; j++)                             /* L22 (:50)                  */
      for (int i = j; i < N2; i++) u[(int64_t)N * (N1 + j) + N1 + i] = C[(int64_t)na * j + na - N2 + i];
    int info = trsm_l(0, 1, N2, N1, u + (int64_t)N1 * N + N1, N, u + N1, N);  /* (:52) */
    if (info) return info;
    syrk_l(1, N1, N2, -1.0, u + N1, N, 1.0, u, N);           /* A -= L21^T L21 (:54)       */
  }
  /* L11 with A = L11^T L11: reverse, upper Cholesky, reverse (:57-87) */
  double* t = malloc(sizeof(double) * (size_t)N1 * N1 + 8);
  for (int j = 0; j < N1; j++)
    for (int i = j; i < N1; i++) t[(int64_t)N1 * (N1 - 1 - j) + (N1 - 1 - i)] = u[(int64_t)N * j + i];
  const int info = potrf_u(N1, t, N1);
  if (!info)
    for (int j = 0; j < N1; j++)
      for (int i = j; i < N1; i++) u[(int64_t)N * j + i] = t[(int64_t)N1 * (N1 - 1 - j) + (N1 - 1 - i)];
  free(t);
  return info;
}

/* completion.c:3-120: the factor L of the max-det completion, reverse postorder */
int orc_completion(int64_t n, int64_t nsn, const int64_t* snpost, const int64_t* snptr, const int64_t* relptr,
                   const int64_t* relidx, const int64_t* chptr, const int64_t* chidx, const int64_t* blkptr,
                   double* blkval, double* fws, double* upd, int64_t* upd_size, int factored_updates) {
  (void)n;
  double* U = upd;
  int64_t nup = 0;
  for (int64_t ki = nsn - 1; ki >= 0; ki--) {
    const int64_t k = snpost[ki];
    const int nn = (int)(snptr[k + 1] - snptr[k]), na = (int)(relptr[k + 1] - relptr[k]), nj = nn + na;
    double* blk = blkval + blkptr[k];
    double* F22 = fws + (int64_t)nn * nj + nn;
    lacpy_l(nj, nn, blk, nj, fws, nj);                       /* (:29)                      */
    if (na > 0) {                                            /* pop V_k (:32-37)           */
      nup--;
      U -= upd_size[nup] * upd_size[nup];
      lacpy_l(na, na, U, na, F22, nj);
    }
    double* ws = (factored_updates && chptr[k + 1] > chptr[k]) ? malloc(sizeof(double) * ((size_t)na * nj + 8)) : NULL;
    for (int64_t l = chptr[k]; l < chptr[k + 1]; l++) {      /* children's updates (:44-66) */
      const int64_t off = relptr[chidx[l]];
      const int N = (int)(relptr[chidx[l] + 1] - off);
      upd_size[nup++] = N;
      if (factored_updates) {
        const int info = update_factor_o(relidx + off, nn, na, U, N, fws, nj, ws);
        if (info) {
          free(ws);
          return info;
        }
      } else {
        extract(fws, nj, relidx + off, N, U);
      }
      U += (int64_t)N * N;
    }
    free(ws);
    if (na > 0) {
      int t1 = 1, t2 = 0;                                    /* V_k = L^T L (factored)     */
      if (!factored_updates) {
        const int info = potrf_l(na, F22, nj);               /* V_k = L L^T (:79-82)       */
        if (info) return info;
        t1 = 0;
        t2 = 1;
      }
      int info = trsm_l(0, t1, na, nn, F22, nj, blk + nn, nj);  /* (:88)                 */
      if (info) return info;
      syrk_l(1, nn, na, -1.0, blk + nn, nj, 1.0, blk, nj);    /* (:90)                      */
      info = trsm_l(0, t2, na, nn, F22, nj, blk + nn, nj);     /* (:91)                      */
      if (info) return info;
      for (int j = 0; j < nn; j++)
        for (int i = nn; i < nj; i++) A_(blk, nj, i, j) = -A_(blk, nj, i, j);  /* (:94) */
    }
    /* inv(D) = R R^T by the reversed upper Cholesky; L = R^{-T} (:97-113) */
    for (int j = 0; j < nn; j++)
      for (int i = j; i < nn; i++) fws[(int64_t)nn * (nn - 1 - j) + (nn - 1 - i)] = A_(blk, nj, i, j);
    int info = potrf_u(nn, fws, nn);
    if (info) return info;
    for (int j = 0; j < nn; j++)
      for (int i = j; i < nn; i++) A_(blk, nj, i, j) = fws[(int64_t)nn * (nn - 1 - j) + (nn - 1 - i)];
    info = trtri_l(nn, blk, nj);
    if (info) return info;
  }
  return 0;
}

/* hessian.c:3-111 (_Y2K), postorder, one U */
static void y2k(int64_t nsn, const int64_t* snpost, const int64_t* snptr, const int64_t* relptr,
                const int64_t* relidx, const int64_t* chptr, const int64_t* chidx, const int64_t* blkptr,
                const double* lblk, double* ublk, double* fws, double** Up, int64_t* nup, int64_t* upd_size, int inv) {
  const double a = inv ? 1.0 : -1.0;
  for (int64_t ki = 0; ki < nsn; ki++) {
    const int64_t k = snpost[ki];
    const int nn = (int)(snptr[k + 1] - snptr[k]), na = (int)(relptr[k + 1] - relptr[k]), nj = nn + na;
    const double* L21 = lblk + blkptr[k] + nn;
    double* F22 = fws + (int64_t)nn * nj + nn;
    lacpy_l(nj, nn, ublk + blkptr[k], nj, fws, nj);
    for (int j = nn; j < nj; j++)
      for (int i = j; i < nj; i++) A_(fws, nj, i, j) = 0.0;
    for (int pass = 0; pass < 2; pass++) {
      if (pass == (inv ? 0 : 1)) {
        if (na > 0) {
          gemm(0, 1, na, na, nn, a, L21, nj, fws + nn, nj, 1.0, F22, nj);     /* :62-63 */
          symm_l(1, na, nn, a, fws, nj, L21, nj, 1.0, fws + nn, nj);          /* :65    */
          gemm(0, 1, na, na, nn, a, fws + nn, nj, L21, nj, 1.0, F22, nj);     /* :67    */
        }
        continue;
      }
      for (int64_t l = chptr[k + 1] - 1; l >= chptr[k]; l--) {              /* :44-58 / :70-84 */
        (*nup)--;
        *Up -= upd_size[*nup] * upd_size[*nup];
        const int64_t off = relptr[chidx[l]];
        extend_add(fws, nj, relidx + off, (int)(relptr[chidx[l] + 1] - off), *Up);
      }
    }
    if (na > 0) {
      upd_size[(*nup)++] = na;
      lacpy_l(na, na, F22, nj, *Up, na);
      *Up += (int64_t)na * na;
    }
    lacpy_l(nj, nn, fws, nj, ublk + blkptr[k], nj);
  }
}

/* hessian.c:114-197 (_M2T), reverse postorder, one U */
static void m2t(int64_t nsn, const int64_t* snpost, const int64_t* snptr, const int64_t* relptr,
                const int64_t* relidx, const int64_t* chptr, const int64_t* chidx, const int64_t* blkptr,
                const double* lblk, double* ublk, double* fws, double** Up, int64_t* nup, int64_t* upd_size, int inv) {
  const double a = inv ? 1.0 : -1.0;
  for (int64_t ki = nsn - 1; ki >= 0; ki--) {
    const int64_t k = snpost[ki];
    const int nn = (int)(snptr[k + 1] - snptr[k]), na = (int)(relptr[k + 1] - relptr[k]), nj = nn + na;
    const double* L21 = lblk + blkptr[k] + nn;
    double* F22 = fws + (int64_t)nn * nj + nn;
    lacpy_l(nj, nn, ublk + blkptr[k], nj, fws, nj);
    if (na > 0) {
      (*nup)--;
      *Up -= upd_size[*nup] * upd_size[*nup];
      lacpy_l(na, na, *Up, na, F22, nj);
    }
    for (int pass = 0; pass < 2; pass++) {
      if (pass == (inv ? 1 : 0)) {
        if (na > 0) {
          gemm(1, 0, nn, nn, na, a, fws + nn, nj, L21, nj, 1.0, fws, nj);     /* :168    */
          symm_l(0, na, nn, a, F22, nj, L21, nj, 1.0, fws + nn, nj);          /* :170    */
          gemm(1, 0, nn, nn, na, a, L21, nj, fws + nn, nj, 1.0, fws, nj);     /* :172    */
        }
        if (!inv) lacpy_l(nj, nn, fws, nj, ublk + blkptr[k], nj);           /* :176    */
        continue;
      }
      for (int64_t l = chptr[k]; l < chptr[k + 1]; l++) {                    /* :151-162 / :179-190 */
        const int64_t off = relptr[chidx[l]];
        const int N = (int)(relptr[chidx[l] + 1] - off);
        upd_size[(*nup)++] = N;
        extract(fws, nj, relidx + off, N, *Up);
        *Up += (int64_t)N * N;
      }
    }
    if (inv) lacpy_l(nj, nn, fws, nj, ublk + blkptr[k], nj);
  }
}

/* hessian.c:200-347 (_scale), reverse postorder, all U */
static int scale(int64_t nsn, const int64_t* snpost, const int64_t* snptr, const int64_t* relptr,
                 const int64_t* relidx, const int64_t* chptr, const int64_t* chidx, const int64_t* blkptr,
                 const double* lblk, const double* yblk, double** ublk, int nu, double* fws, double* upd,
                 int64_t* upd_size, int inv, int adj, int factored) {
  double* U = upd;
  int64_t nup = 0;
  for (int64_t ki = nsn - 1; ki >= 0; ki--) {
    const int64_t k = snpost[ki];
    const int nn = (int)(snptr[k + 1] - snptr[k]), na = (int)(relptr[k + 1] - relptr[k]), nj = nn + na;
    double* F22 = fws + (int64_t)nn * nj + nn;
    const double* L11 = lblk + blkptr[k];
    lacpy_l(nj, nn, yblk + blkptr[k], nj, fws, nj);
    for (int j = nn; j < nj; j++)
      for (int i = j; i < nj; i++) A_(fws, nj, i, j) = 0.0;
    if (na > 0) {
      nup--;
      U -= upd_size[nup] * upd_size[nup];
      lacpy_l(na, na, U, na, F22, nj);
    }
    double* ws = (factored && chptr[k + 1] > chptr[k]) ? malloc(sizeof(double) * ((size_t)na * nj + 8)) : NULL;
    for (int64_t l = chptr[k]; l < chptr[k + 1]; l++) {      /* :256-278 */
      const int64_t off = relptr[chidx[l]];
      const int N = (int)(relptr[chidx[l] + 1] - off);
      upd_size[nup++] = N;
      if (factored) {
        const int info = update_factor_o(relidx + off, nn, na, U, N, fws, nj, ws);
        if (info) {
          free(ws);
          return info;
        }
      } else {
        extract(fws, nj, relidx + off, N, U);
      }
      U += (int64_t)N * N;
    }
    free(ws);
    int t3 = 0;
    if (na > 0) {
      if (factored) {
        t3 = adj;                                            /* V_k = L^T L (:287-291) */
      } else {
        const int info = potrf_l(na, F22, nj);               /* V_k = L L^T (:293-298) */
        if (info) return info;
        t3 = !adj;
      }
    }
    const int t1 = !adj, t2 = adj;                           /* :302-309 */
    for (int u = 0; u < nu; u++) {
      double* ub = ublk[u] + blkptr[k];
      for (int j = 0; j < nn - 1; j++)                       /* symmetrise (:314-318) */
        for (int i = j + 1; i < nn; i++) A_(ub, nj, j, i) = A_(ub, nj, i, j);
      if (!inv) {                                            /* :321-330 */
        trsm_l(1, t1, nj, nn, L11, nj, ub, nj);
        trsm_l(0, t2, nn, nn, L11, nj, ub, nj);
        zero_upper(nn, ub, nj);
        if (na > 0) trmm_l(0, t3, na, nn, F22, nj, ub + nn, nj);
      } else {                                               /* :332-341 */
        trmm_l(1, t1, nj, nn, L11, nj, ub, nj);
        trmm_l(0, t2, nn, nn, L11, nj, ub, nj);
        zero_upper(nn, ub, nj);
        if (na > 0) trsm_l(0, t3, na, nn, F22, nj, ub + nn, nj);
      }
    }
  }
  return 0;
}

/* hessian.c:349-374 */
int orc_hessian(int64_t n, int64_t nsn, const int64_t* snpost, const int64_t* snptr, const int64_t* relptr,
                const int64_t* relidx, const int64_t* chptr, const int64_t* chidx, const int64_t* blkptr,
                const double* lblkval, const double* yblkval, double** ublkval, int64_t nu, double* fws,
                double* upd, int64_t* upd_size, int inv, int adj, int factored_updates) {
  (void)n;
  int info = 0;
  if (adj != inv)
    info = scale(nsn, snpost, snptr, relptr, relidx, chptr, chidx, blkptr, lblkval, yblkval, ublkval, (int)nu, fws,
                 upd, upd_size, inv, adj, factored_updates);
  for (int64_t u = 0; u < nu; u++) {
    double* Up = upd;
    int64_t nup = 0;
    if (adj)
      m2t(nsn, snpost, snptr, relptr, relidx, chptr, chidx, blkptr, lblkval, ublkval[u], fws, &Up, &nup, upd_size,
          inv);
    else
      y2k(nsn, snpost, snptr, relptr, relidx, chptr, chidx, blkptr, lblkval, ublkval[u], fws, &Up, &nup, upd_size,
          inv);
  }
  if (adj == inv)
    info = scale(nsn, snpost, snptr, relptr, relidx, chptr, chidx, blkptr, lblkval, yblkval, ublkval, (int)nu, fws,
                 upd, upd_size, inv, adj, factored_updates);
  return info;
}

/* trsm.c:3-139: B := alpha L^{-1} B ('N', postorder) or alpha L^{-T} B ('T',
 * reverse postorder); B column-major with leading dimension ldb, rows in the
 * original order (row p[snode[.]]).  fws: clique_number x nrhs; upd:
 * stack_solve x nrhs. */
void orc_trsm(char trans, int nrhs, double alpha, int64_t n, int64_t nsn, const int64_t* snpost,
              const int64_t* snptr, const int64_t* snode, const int64_t* relptr, const int64_t* relidx,
              const int64_t* chptr, const int64_t* chidx, const int64_t* blkptr, const int64_t* p,
              const double* blkval, double* b, int ldb, double* fws, double* upd, int64_t* upd_size) {
  (void)n;
  double* U = upd;
  int64_t nup = 0;
  const int tr = (trans == 'T');
  for (int64_t kk = 0; kk < nsn; kk++) {
    const int64_t k = tr ? snpost[nsn - 1 - kk] : snpost[kk];
    const int nn = (int)(snptr[k + 1] - snptr[k]), na = (int)(relptr[k + 1] - relptr[k]), nj = nn + na;
    const double* blk = blkval + blkptr[k];
    for (int j = 0; j < nrhs; j++) {                         /* gather x_k (:40-47 / :88-95) */
      for (int i = 0; i < nn; i++) fws[(int64_t)nj * j + i] = alpha * b[(int64_t)j * ldb + p[snode[snptr[k] + i]]];
      for (int i = nn; i < nj; i++) fws[(int64_t)nj * j + i] = 0.0;
    }
    if (!tr) {
      for (int64_t l = chptr[k + 1] - 1; l >= chptr[k]; l--) {  /* :50-59 */
        nup--;
        U -= upd_size[nup] * nrhs;
        const int64_t off = relptr[chidx[l]];
        const int N = (int)(relptr[chidx[l] + 1] - off);
        for (int j = 0; j < nrhs; j++)
          for (int i = 0; i < N; i++) fws[(int64_t)nj * j + relidx[off + i]] += U[(int64_t)N * j + i];
      }
      if (na > 0) {                                           /* :61-67 */
        gemm(0, 0, na, nrhs, nn, -1.0, blk + nn, nj, fws, nj, 1.0, fws + nn, nj);
        upd_size[nup++] = na;
        for (int j = 0; j < nrhs; j++)
          for (int i = 0; i < na; i++) U[(int64_t)na * j + i] = fws[(int64_t)nj * j + nn + i];
        U += (int64_t)na * nrhs;
      }
      trsm_l(0, 0, nn, nrhs, blk, nj, fws, nj);                /* :69 */
    } else {
      trsm_l(0, 1, nn, nrhs, blk, nj, fws, nj);                /* :97 */
      if (na > 0) {                                           /* :99-105 */
        nup--;
        U -= upd_size[nup] * nrhs;
        for (int j = 0; j < nrhs; j++)
          for (int i = 0; i < na; i++) fws[(int64_t)nj * j + nn + i] = U[(int64_t)na * j + i];
        gemm(1, 0, nn, nrhs, na, -1.0, blk + nn, nj, fws + nn, nj, 1.0, fws, nj);
      }
      for (int64_t l = chptr[k]; l < chptr[k + 1]; l++) {     /* :107-117 */
        const int64_t off = relptr[chidx[l]];
        const int N = (int)(relptr[chidx[l] + 1] - off);
        upd_size[nup++] = N;
        for (int j = 0; j < nrhs; j++)
          for (int i = 0; i < N; i++) U[(int64_t)N * j + i] = fws[(int64_t)nj * j + relidx[off + i]];
        U += (int64_t)N * nrhs;
      }
    }
    for (int j = 0; j < nrhs; j++)                           /* scatter x_k (:71-77 / :119-125) */
      for (int i = 0; i < nn; i++) b[(int64_t)j * ldb + p[snode[snptr[k] + i]]] = fws[(int64_t)nj * j + i];
  }
}

/* dot.c:3-23: <X, Y> = 2 * (sum over the lower trapezoids) - sum over diagonals */
double orc_dot(int64_t nsn, const int64_t* snptr, const int64_t* sncolptr, const int64_t* blkptr,
               const double* x, const double* y) {
  double val = 0.0;
  for (int64_t k = 0; k < nsn; k++) {
    const int nn = (int)(snptr[k + 1] - snptr[k]), nj = (int)(sncolptr[k + 1] - sncolptr[k]);
    for (int j = 0; j < nn; j++) {
      const int64_t d = blkptr[k] + (int64_t)j * nj + j;   /* diagonal entry of column j */
      double s = 0.0;
      for (int i = 0; i < nj - j; i++) s += x[d + i] * y[d + i];
      val += 2.0 * s - x[d] * y[d];
    }
  }
  return val;
}

/* update_factor (update_factor.c:3-108) on its own, for tests: r (N child
 * indices into the front), F (nj x nj, ld ldf), u (N x N); C scratch na x N */
int orc_update_factor(const int64_t* r, int nn, int na, double* u, int N, const double* f, int ldf, double* C) {
  return update_factor_o(r, nn, na, u, N, f, ldf, C);
}
