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

#endif
