/*
 * Oracle: a plain-C restatement of the reference's numeric multifrontal
 * sweeps (chompack src/C/*.c), with its own naive dense kernels in place of
 * BLAS/LAPACK.  TEST INFRASTRUCTURE ONLY — the checker used by tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg; never linked into
 * or called by the product.
 *
 * Arguments follow the reference's C signatures (src/C/chompack.h:63-231):
 * int64 symbolic arrays, blkval in the reference block layout, caller-owned
 * workspaces sized from symb.memory.
 */
#ifndef CHB_ORACLE_H
#define CHB_ORACLE_H
#include <stdint.h>

int orc_cholesky(int64_t n, int64_t nsn, const int64_t* snpost, const int64_t* snptr, const int64_t* relptr,
                 const int64_t* relidx, const int64_t* chptr, const int64_t* chidx, const int64_t* blkptr,
                 double* blkval, double* fws, double* upd, int64_t* upd_size);

void orc_llt(int64_t n, int64_t nsn, const int64_t* snpost, const int64_t* snptr, const int64_t* relptr,
             const int64_t* relidx, const int64_t* chptr, const int64_t* chidx, const int64_t* blkptr,
             double* blkval, double* fws, double* upd, int64_t* upd_size);

int orc_projected_inverse(int64_t n, int64_t nsn, const int64_t* snpost, const int64_t* snptr,
                          const int64_t* relptr, const int64_t* relidx, const int64_t* chptr, const int64_t* chidx,
                          const int64_t* blkptr, double* blkval, double* fws, double* upd, int64_t* upd_size);

int orc_completion(int64_t n, int64_t nsn, const int64_t* snpost, const int64_t* snptr, const int64_t* relptr,
                   const int64_t* relidx, const int64_t* chptr, const int64_t* chidx, const int64_t* blkptr,
                   double* blkval, double* fws, double* upd, int64_t* upd_size, int factored_updates);

int orc_hessian(int64_t n, int64_t nsn, const int64_t* snpost, const int64_t* snptr, const int64_t* relptr,
                const int64_t* relidx, const int64_t* chptr, const int64_t* chidx, const int64_t* blkptr,
                const double* lblkval, const double* yblkval, double** ublkval, int64_t nu, double* fws,
                double* upd, int64_t* upd_size, int inv, int adj, int factored_updates);

void orc_trsm(char trans, int nrhs, double alpha, int64_t n, int64_t nsn, const int64_t* snpost,
              const int64_t* snptr, const int64_t* snode, const int64_t* relptr, const int64_t* relidx,
              const int64_t* chptr, const int64_t* chidx, const int64_t* blkptr, const int64_t* p,
              const double* blkval, double* b, int ldb, double* fws, double* upd, int64_t* upd_size);

int orc_update_factor(const int64_t* r, int nn, int na, double* u, int N, const double* f, int ldf, double* C);

double orc_dot(int64_t nsn, const int64_t* snptr, const int64_t* sncolptr, const int64_t* blkptr,
               const double* x, const double* y);

#endif
