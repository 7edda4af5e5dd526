/*
 * chompack_b200 — C ABI of the B200 (sm_100a) multifrontal sweeps over a
 * supernodal clique tree.
 *
 * The boundary replaces the reference's CPython extension `chompack.cbase`
 * (src/C/cbase.c) and the plain-C kernels it wraps (src/C/chompack.h:63-231).
 * Every entry point takes plain pointers and sizes: int64 index arrays in the
 * reference's `symbolic` layout on the host, float64 `blkval` buffers in the
 * reference's block layout on the device, and a CUDA stream as `void*`.
 *
 * Return codes: 0 success; > 0 a LAPACK-style `info` from a device
 * factorisation (the reference raises ArithmeticError on it, cbase.c:281);
 * < 0 an argument, consistency or CUDA error (see chb_last_error()).
 */
#ifndef CHOMPACK_B200_H
#define CHOMPACK_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Host symbolic analysis (reference: src/python/symbolic.py).               */
/* Each function restates the named reference function over int64 arrays.   */
/* ------------------------------------------------------------------------ */

/* Merge decision callback: merge_fn(|J_parent|, |J_k|, |N_parent|, |N_k|)
 * returns non-zero to merge supernode k into its parent (symbolic.py:527). */
typedef int (*chb_merge_fn)(int64_t cp, int64_t ck, int64_t np, int64_t nk);

/* etree(A) — symbolic.py:49-72. cp/ri: CCS of the symmetric pattern. */
int chb_sym_etree(int64_t n, const int64_t* cp, const int64_t* ri, int64_t* parent);
/* post_order(parent) — symbolic.py:26-47. */
int chb_sym_post_order(int64_t n, const int64_t* parent, int64_t* post);
/* counts(A, parent, post) — symbolic.py:95-131. */
int chb_sym_counts(int64_t n, const int64_t* cp, const int64_t* ri, const int64_t* parent,
                   const int64_t* post, int64_t* colcount);
/* supernodes(par, post, colcount) incl. pothen_sun — symbolic.py:133-244. */
int chb_sym_supernodes(int64_t n, const int64_t* par, const int64_t* post, const int64_t* colcount,
                       int64_t* snode, int64_t* snptr, int64_t* snpar, int64_t* nsn);
/* amalgamate(...) with merge_size_fill(tsize, tfill) or merge_fn —
 * symbolic.py:246-326, :486-496. */
int chb_sym_amalgamate(int64_t n, int64_t* colcount, int64_t* snode, int64_t* snptr, int64_t* snpar,
                       const int64_t* snpost_in, int64_t* snpost_out, int64_t* nsn, int64_t tsize,
                       int64_t tfill, chb_merge_fn merge_fn);
/* embed(A, ...) — symbolic.py:328-384 (rowidx == NULL: only colptr). */
int chb_sym_embed(int64_t n, const int64_t* cp, const int64_t* ri, const int64_t* colcount,
                  const int64_t* snode, const int64_t* snptr, const int64_t* snpar, const int64_t* snpost,
                  int64_t nsn, int64_t* colptr, int64_t* rowidx);
/* relative_idx(colptr, rowidx, snptr, snpar) — symbolic.py:386-411. */
int chb_sym_relative_idx(int64_t nsn, const int64_t* colptr, const int64_t* rowidx, const int64_t* snptr,
                         const int64_t* snpar, int64_t* relptr, int64_t* relidx);
/* Approximate minimum degree ordering (stands in for cvxopt.amd.order,
 * called by symbolic.py:541-542). cp/ri: CCS of the symmetric pattern
 * (diagonal entries allowed); perm[n] receives the elimination order. */
int chb_amd_order(int64_t n, const int64_t* cp, const int64_t* ri, int64_t* perm);

/* ------------------------------------------------------------------------ */
/* Device plan: the symbolic arrays a sweep reads, uploaded once.            */
/* ------------------------------------------------------------------------ */

typedef struct chb_plan chb_plan;

/* Upload a symbolic factorisation (the attributes cbase.c:229-246 and
 * :1021-1042 read from `symb`) and build the level schedules.  All arrays are
 * host int64 in the reference's layout; snpost must be range(nsn) (the
 * reference renumbers supernodes in postorder, symbolic.py:564-575).  The plan
 * is bound to `device`; device < 0 gives a host-only plan that supports the
 * introspection calls only. */
int chb_plan_create(int64_t n, int64_t nsn, const int64_t* snptr, const int64_t* snpar,
                    const int64_t* relptr, const int64_t* relidx, const int64_t* chptr,
                    const int64_t* chidx, const int64_t* blkptr, const int64_t* snode, const int64_t* p,
                    int device, chb_plan** plan);
int chb_plan_destroy(chb_plan* plan);

/* Operation codes for workspace queries. */
enum chb_op {
  CHB_OP_CHOLESKY = 0,
  CHB_OP_LLT = 1,
  CHB_OP_PROJECTED_INVERSE = 2,
  CHB_OP_COMPLETION = 3,
  CHB_OP_HESSIAN = 4,
  CHB_OP_TRSM = 5,
  CHB_OP_DOT = 6,
  CHB_OP_TRMM = 7,
  CHB_OP_CONVENTIONAL = 8
};

/* Device workspace (bytes) an operation needs; `k` is nrhs for CHB_OP_TRSM
 * and CHB_OP_TRMM,
 * the number of U matrices for CHB_OP_HESSIAN and factored_updates for
 * CHB_OP_COMPLETION (ignored otherwise); `flags` is the hessian adj/inv
 * selector (adj | inv << 1 | factored_updates << 2), else 0.  This replaces
 * the per-call malloc of fws/upd/upd_size sized from symb.memory
 * (cbase.c:249-258, :1037-1039).  The caller owns the workspace, which must
 * be 256-byte aligned. */
int chb_workspace_size(const chb_plan* plan, int op, int64_t k, int flags, size_t* bytes);

/* Sweeps on values held in host memory.  The reference's cspmatrix keeps
 * its values on the host (cbase.c:176-284 reads and writes blkval in
 * place); these entry points keep that calling pattern without serialising
 * the copies.  The values are cut into at most 24 chunks at supernode
 * boundaries.  With host_in, chunk j is copied into dev_blkval while the
 * sweep runs and every task that touches it waits for its arrival; with
 * host_out, chunk j is copied back as soon as every task that writes it
 * has finished (outgoing chunks also cut large supernodes between 64-column
 * tiles).  Either may be NULL (values already on the device / result
 * left on the device); host buffers should be pinned for the copies to
 * overlap.  The workspace is the one chb_workspace_size gives for `flags`
 * = chb_io_flags(host_in != NULL, host_out != NULL).  The call returns when
 * everything is enqueued on `stream`; the stream's completion includes the
 * copies. */
int chb_io_flags(int host_in, int host_out);
/* 1 when the driver offers stream waits on device flags (the results then
 * stream out while the sweep runs), 0 when they are copied after it. */
int chb_io_overlap_available(void);
int chb_cholesky_io(chb_plan* plan, const double* host_in, double* host_out, double* dev_blkval, void* work,
                    size_t work_bytes, void* stream);
int chb_projected_inverse_io(chb_plan* plan, const double* host_in, double* host_out, double* dev_blkval,
                             void* work, size_t work_bytes, void* stream);
int chb_llt_io(chb_plan* plan, const double* host_in, double* host_out, double* dev_blkval, void* work,
               size_t work_bytes, void* stream);
/* Mixed precision (no counterpart in the reference).  Every GEMM task of
 * the sweep (Schur-complement updates, panel solves through the explicit
 * inverse of the diagonal tile, the products of the projected inverse)
 * runs on TF32 tensor cores with FP32 accumulation from the FP64 operands
 * (CHB_PREC_TF32: one product, about 11 bits per operand; CHB_PREC_TF32X3:
 * high/low splits and three products, about 22 bits); results are added in
 * FP64.  Diagonal-tile factorisations and inverses, the look-ahead steps,
 * split-K sums, assembly and extraction stay FP64.  host_in / host_out as
 * for chb_cholesky_io (NULL: device values only).  Workspace: the flags
 * chb_precision_flags(precision) | chb_io_flags(...). */
enum { CHB_PREC_FP64 = 0, CHB_PREC_TF32 = 1, CHB_PREC_TF32X3 = 2 };

/* y += alpha X x for the symmetric chordal matrix in blkval (FP64; the
 * residual of iterative refinement): x, y are n x nrhs column-major with
 * leading dimension ld, rows in the original order; sncolptr / snrowidx
 * are the symbolic's arrays on the device (int64).  No counterpart in the
 * reference's C code (its Python solves build the residual with cvxopt). */
int chb_symv(chb_plan* plan, const double* blkval, const int64_t* sncolptr, const int64_t* snrowidx, const double* x,
             double* y, int64_t nrhs, int64_t ld, double alpha, void* stream);
int chb_precision_flags(int precision);
int chb_cholesky_prec(chb_plan* plan, int precision, const double* host_in, double* host_out, double* dev_blkval,
                      void* work, size_t work_bytes, void* stream);
int chb_projected_inverse_prec(chb_plan* plan, int precision, const double* host_in, double* host_out,
                               double* dev_blkval, void* work, size_t work_bytes, void* stream);

/* Introspection of a streamed program: counts[0..1] = incoming and
 * outgoing chunks; the incoming chunks' value offsets (count + 1) and copy
 * order; the outgoing chunks' value offsets (count + 1) and the order in
 * which their signals are listed.  Array arguments may be NULL. */
int chb_program_io(chb_plan* plan, int op, int64_t k, int flags, int64_t* counts, int64_t* in_off,
                   int32_t* in_order, int64_t* out_off, int32_t* out_order);

/* Introspection of a compiled sweep (works on a host-only plan, device < 0):
 * info[0..7] = tasks, waits, counters, workspace doubles, workspace bytes,
 * byte offset of the doubles, doubles of update matrices, sizeof(task).
 * chb_program_export copies the task list, the (counter, target) waits and
 * the per-supernode descriptors into caller buffers of those sizes. */
int chb_program_info(chb_plan* plan, int op, int64_t k, int flags, int64_t* info);
int chb_program_export(chb_plan* plan, int op, int64_t k, int flags, void* tasks, void* waits, void* fronts);
/* The update-matrix pool of a compiled sweep under CHB_OPT_SCRATCH_LIMIT:
 * info[0..3] = the pool's bytes (-1: the program has no pool), the reuse
 * waits it added, the workspace bytes of the program, and the span (ns) of
 * the simulated list schedule that ordered its tasks (the planner's model,
 * not a measurement). */
int chb_program_pool(chb_plan* plan, int op, int64_t k, int flags, int64_t* info);
/* The dynamic-schedule data of a compiled sweep: sizes[0..5] = lengths of
 * the pending counts per task, the successor offsets per counter (counters
 * + 1), the successor list, the completion value per counter, the initial
 * ready bitmap and its summary (64-bit words).  Array arguments may be NULL
 * (sizes only). */
int chb_program_schedule(chb_plan* plan, int op, int64_t k, int flags, int64_t* sizes, int32_t* npend,
                         int32_t* succ_off, int32_t* succ, int32_t* ctarget, uint64_t* ready0, uint64_t* summ0);

/* ------------------------------------------------------------------------ */
/* Numeric sweeps.  All pointers are device pointers; calls are asynchronous */
/* on `stream` except that chb_info() synchronises to read the status.       */
/* ------------------------------------------------------------------------ */

/* cholesky — cholesky.c:3-84 (wrapper cbase.c:187-284).  In place on blkval. */
int chb_cholesky(chb_plan* plan, double* blkval, void* work, size_t work_bytes, void* stream);

/* llt — llt.c:3-60 (wrapper cbase.c:298-390).  In place on blkval. */
int chb_llt(chb_plan* plan, double* blkval, void* work, size_t work_bytes, void* stream);

/* projected_inverse — projected_inverse.c:3-75 (wrapper cbase.c:404-500). */
int chb_projected_inverse(chb_plan* plan, double* blkval, void* work, size_t work_bytes, void* stream);

/* completion — completion.c:3-120 + update_factor.c:3-108 (wrapper
 * cbase.c:521-621).  factored_updates as in the reference (default 1). */
int chb_completion(chb_plan* plan, double* blkval, int factored_updates, void* work, size_t work_bytes,
                   void* stream);

/* hessian — hessian.c:349-374 (_Y2K :3, _M2T :114, _scale :216; wrapper
 * cbase.c:675-857).  ublkval: host array of nu device pointers, each a U
 * blkval updated in place.  adj/inv as hessian.c; the reference's adj=None
 * (full Hessian) is two calls with adj toggled (cbase.c:833-841). */
int chb_hessian(chb_plan* plan, const double* lblkval, const double* yblkval, double* const* ublkval,
                int64_t nu, int adj, int inv, int factored_updates, void* work, size_t work_bytes,
                void* stream);

/* trsm — trsm.c:3-139 (wrapper cbase.c:965-1077).  B := alpha*L^{-1}B
 * (trans 'N') or alpha*L^{-T}B (trans 'T'); B is n x nrhs column-major with
 * leading dimension ldB, rows in the original (unpermuted) order. */
int chb_trsm(chb_plan* plan, char trans, int64_t nrhs, double alpha, const double* blkval, double* B,
             int64_t ldB, void* work, size_t work_bytes, void* stream);

/* trsm for repeated solves with one factor (no counterpart in the
 * reference; iterative refinement calls it twice per iteration).  A solve
 * computes, from L alone, the inverses of the diagonal tiles and their
 * coupling products into its workspace; with reuse != 0 they are taken
 * from `work` as an earlier call left them, which must have had the same
 * plan, trans, nrhs and unchanged blkval, with no other call using `work`
 * in between (the caller keeps one workspace per trans).  reuse == 0 is
 * chb_trsm. */
int chb_trsm_reuse(chb_plan* plan, char trans, int64_t nrhs, double alpha, const double* blkval, double* B,
                   int64_t ldB, void* work, size_t work_bytes, int reuse, void* stream);

/* trmm — pybase/trmm.py:4-116 (Python only in the reference).  B :=
 * alpha*L*B (trans 'N') or alpha*L^T*B (trans 'T') with the factor that
 * chb_cholesky leaves in blkval; B as for chb_trsm.  Workspace
 * chb_workspace_size(plan, CHB_OP_TRMM, nrhs, trans == 'T', ...). */
int chb_trmm(chb_plan* plan, char trans, int64_t nrhs, double alpha, const double* blkval, double* B,
             int64_t ldB, void* work, size_t work_bytes, void* stream);

/* Conventional factor — the block products of cspmatrix.spmatrix() on a
 * factor (symbolic.py:1052-1068): every off-diagonal block W = L_{Ak,Nk}
 * L_kk^{-1} that chb_cholesky leaves (cholesky.c:72) becomes W L_kk, in
 * place.  Workspace chb_workspace_size(plan, CHB_OP_CONVENTIONAL, 0, 0, ...). */
int chb_factor_conventional(chb_plan* plan, double* blkval, void* work, size_t work_bytes, void* stream);

/* Element-wise block operations (Python loops over supernodes in the
 * reference).  sncolptr / snrowidx are the symbolic's arrays (int64) in
 * device memory; all vectors and matrices are device memory.
 * chb_lower_ccs — the lower trapezoid of every block in compressed-column
 *   order (cspmatrix.spmatrix(), symbolic.py:1071-1098): colptr (n+1, column
 *   j of supernode k has nj - (j - snptr[k]) entries) gives where each column
 *   goes; values and, unless NULL, row indices (reordered numbering) are
 *   written.
 * chb_syr2 — X := alpha P(u v^T + v u^T) + beta X on the lower trapezoid of
 *   every block (base.py:28-67); u, v are n-vectors in the original
 *   numbering (gathered through p) unless `reordered`.
 * chb_add_projection — X := alpha P(A) + beta X for a dense column-major A
 *   (lda >= n) on every entry of every block (symbolic.py:1176-1210):
 *   symmetric_original != 0 reads the symmetric matrix of A's lower triangle
 *   through p (the reference's reordered=False), else A[r, c] in the
 *   reordered numbering.
 * chb_diag — the n diagonal entries in the reordered numbering
 *   (symbolic.py:1113-1128). */
int chb_lower_ccs(chb_plan* plan, const double* blkval, const int64_t* sncolptr, const int64_t* snrowidx,
                  const int64_t* colptr, double* values, int64_t* rowidx, void* stream);
int chb_syr2(chb_plan* plan, double* blkval, const int64_t* sncolptr, const int64_t* snrowidx, const double* u,
             const double* v, double alpha, double beta, int reordered, void* stream);
int chb_add_projection(chb_plan* plan, double* blkval, const int64_t* sncolptr, const int64_t* snrowidx,
                       const double* A, int64_t lda, double alpha, double beta, int symmetric_original,
                       void* stream);
int chb_diag(chb_plan* plan, const double* blkval, double* d, void* stream);

/* chb_add_sparse — X += alpha tril(P(symmetrize(A))) for a sparse A of order
 *   n given as nnz (I, J, V) triplets in device memory (cspmatrix +=
 *   spmatrix, symbolic.py:1138-1174): only A's lower entries (I >= J) are
 *   read; each is renumbered through p (unless `reordered`), swapped into the
 *   lower triangle and added into the block that holds it.  Triplets outside
 *   the chordal pattern or with an index outside [0, n) are skipped and
 *   counted in *bad (a device word, zeroed first); the caller reads it after
 *   the stream's work and raises, as the reference's lookup would.  Repeated
 *   triplets are summed. */
int chb_add_sparse(chb_plan* plan, double* blkval, const int64_t* sncolptr, const int64_t* snrowidx, int64_t nnz,
                   const int64_t* I, const int64_t* J, const double* V, double alpha, int reordered,
                   unsigned long long* bad, void* stream);

/* Product-form Cholesky factor of I + V diag(a) V^T = L_1...L_k L_k^T...L_1^T
 * (V n x k), each L_i held as column i of V, L and B (pfcholesky.c:52-136;
 * the reference's pfcholesky class composes them with the chordal factor,
 * pfcholesky.py:113-211).  All arrays are column-major device memory with
 * the given leading dimensions (>= max(1, n)).  Each call is one launch on
 * `stream` into a caller-provided workspace of chb_pf_workspace_size(n,
 * ncols) bytes (256-byte aligned; ncols = k for chb_pftrf, nrhs for the
 * others), and its status comes back from chb_pf_info(work, stream).
 *
 * chb_pftrf — dpftrf (pfcholesky.c:52-88, wrapper cbase.pfchol cbase.c:862-880):
 *   a (k device doubles), V overwritten as dpftrf does, L and B written.
 *   chb_pf_info returns -1 when 1 - alpha v^2 <= 0 for some row (the
 *   reference's return value; cbase raises ArithmeticError); the contents of
 *   V, L and B are then unspecified.
 * chb_pfsv — dpfsv (:90-112) on each of the nrhs columns of U (cbase.pftrsm
 *   cbase.c:885-911): U := (L_1...L_k)^{-1} U ('N') or (L_k^T...L_1^T)^{-1} U ('T').
 * chb_pfmv — dpfmv (:114-136) on each column of U (cbase.pftrmm
 *   cbase.c:916-942): U := L_1...L_k U ('N') or L_k^T...L_1^T U ('T'). */
int chb_pf_workspace_size(int64_t n, int64_t ncols, size_t* bytes);
int chb_pftrf(int64_t n, int64_t k, const double* a, double* V, int64_t ldv, double* L, int64_t ldl, double* B,
              int64_t ldb, void* work, size_t work_bytes, void* stream);
int chb_pfsv(int64_t n, int64_t k, char trans, const double* V, int64_t ldv, const double* L, int64_t ldl,
             const double* B, int64_t ldb, double* U, int64_t ldu, int64_t nrhs, void* work, size_t work_bytes,
             void* stream);
int chb_pfmv(int64_t n, int64_t k, char trans, const double* V, int64_t ldv, const double* L, int64_t ldl,
             const double* B, int64_t ldb, double* U, int64_t ldu, int64_t nrhs, void* work, size_t work_bytes,
             void* stream);
/* Synchronise `stream` and return the status of the last product-form call
 * that used `work`: 0, -1 (dpftrf: not positive definite), or -30 when a
 * grid-wide wait of the kernel ran out. */
int chb_pf_info(void* work, void* stream);

/* dot — dot.c:3-23 (wrapper cbase.c:106-174).  Writes <X,Y> to result (one
 * device double). */
int chb_dot(chb_plan* plan, const double* x, const double* y, double* result, void* work,
            size_t work_bytes, void* stream);

/* log det X from its factor L (the blkval chb_cholesky leaves):
 * 2 * sum of log L_kk(j, j) over the diagonal blocks, deterministic.  No
 * single reference routine: the reference's callers form it from the
 * factor's diagonal (L.diag(), symbolic.py:1113-1128).  Workspace as for
 * CHB_OP_DOT. */
int chb_logdet(chb_plan* plan, const double* l, double* result, void* work, size_t work_bytes, void* stream);

/* y = alpha * w .* x over the stored block entries, w = 2 below the
 * diagonal, 1 on it, 0 in the strict upper part of each diagonal block: maps
 * a chordal symmetric matrix to the gradient, with respect to the stored
 * entries, of <X, .> (the inner product of dot).  x and y may alias.  No
 * reference counterpart (used by the autograd layer). */
int chb_sym_weight(chb_plan* plan, const double* x, double* y, double alpha, void* stream);

/* Batches.  chb_plan_merge builds one plan over the disjoint union of the
 * given plans' clique trees (a forest): supernodes, columns, relative
 * indices and block values are concatenated in the order given, so a batch
 * of matrices, or of value sets on one pattern (the same plan repeated),
 * is factored by ONE launch of each sweep on the concatenated blkval.  The
 * inputs may be host-only plans (device < 0) and stay owned by the caller.
 * The batched counterpart the reference lacks (its wrapper takes one
 * cspmatrix per call, cbase.c:187-284). */
int chb_plan_merge(const chb_plan* const* plans, int count, int device, chb_plan** out);

/* The matrices of a (merged) plan: count, and their supernode ranges
 * seg[m] .. seg[m+1] (count + 1 entries; may be NULL). */
int chb_plan_batch_info(const chb_plan* plan, int64_t* count, int64_t* seg);

/* Per-matrix log det (from the factor) and <X, Y> of a merged plan:
 * results[m], m < count (device doubles).  Workspace as for CHB_OP_DOT. */
int chb_logdet_batch(chb_plan* plan, const double* l, double* results, void* work, size_t work_bytes,
                     void* stream);
int chb_dot_batch(chb_plan* plan, const double* x, const double* y, double* results, void* work,
                  size_t work_bytes, void* stream);

/* Profiling: when `buffer` (device memory, 32 bytes per task) is set, the
 * next sweeps whose task count fits `capacity_tasks` record per task the
 * global-timer ns at claim, start (dependencies met) and end, and the SM id
 * | task kind << 32.  Pass NULL to switch tracing off. */
int chb_set_trace(chb_plan* plan, void* buffer, int64_t capacity_tasks);

/* Task scheduling of the plan's sweeps: 0 dynamic (a finished task releases
 * its waiters; CTAs claim ready tasks near the lowest list positions), 1
 * static (CTAs take tasks in list order and wait for their dependencies),
 * -1 the default (CHB_SCHEDULE=static|dynamic from the environment, else
 * static for cholesky, llt and trsm, and for projected_inverse on a merged
 * plan, and dynamic for the others).  Both give
 * bit-identical results, except for the triangular solve unless
 * CHB_OPT_ORDERED_SUMS is set (its additions into vector blocks use atomics
 * by default). */
int chb_plan_set_schedule(chb_plan* plan, int mode);

/* Program-build options of the plan's sweeps (no counterpart in the
 * reference: they choose how a sweep is cut into tasks, not what it
 * computes).  value < 0 restores the default (the environment variable of
 * the same name, else the built-in value).  Setting an option drops the
 * plan's compiled programs, so call it only while no sweep of the plan is
 * in flight; the next sweeps rebuild them.
 *   CHB_OPT_SMALL_FRONT_NJ  largest front order run as one shared-memory
 *                           task (0..64, default 64)
 *   CHB_OPT_SUBTREES        small complete subtrees (fronts of order <= 32)
 *                           bundled four per task, one warp each (1/0)
 *   CHB_OPT_CHOL_KSPLIT     cholesky: K chunk of the split Schur-complement
 *                           tiles (multiple of 64, 0 = whole)
 *   CHB_OPT_PINV_KSPLIT     projected_inverse: K chunk of its long-K tiles
 *   CHB_OPT_FUSED_LA        cholesky: fused diagonal task (1/0)
 *   CHB_OPT_TF32_TCGEN05    mixed precision: TF32 tiles on tcgen05 with
 *                           tensor-memory accumulators (1) or warp-level
 *                           mma.sync (0, the default)
 *   CHB_OPT_ORDERED_SUMS    trsm: every addition into a vector block in a
 *                           fixed order (1: bit-reproducible, slower) or
 *                           with atomics as inputs arrive (0, the default)
 *   CHB_OPT_SCRATCH_LIMIT   cholesky and projected_inverse: bytes for the
 *                           update matrices of the fronts.  By default each
 *                           front's update matrix has memory of its own
 *                           (the sum over all fronts, several times the
 *                           factor).  With a limit they share a pool of at
 *                           most that size where the schedule allows: a
 *                           front that takes memory another one held waits
 *                           until that one's readers are done (memory the
 *                           reference's stack, symbolic.py:634-661, reuses
 *                           in postorder).  The pool grows past the limit
 *                           only where no memory can be shared; the
 *                           results are bit-identical to the unlimited
 *                           layout.  chb_workspace_size reports the total.
 * chb_plan_get_option gives the value the next program build uses. */
enum chb_option {
  CHB_OPT_SMALL_FRONT_NJ = 0,
  CHB_OPT_SUBTREES = 1,
  CHB_OPT_CHOL_KSPLIT = 2,
  CHB_OPT_PINV_KSPLIT = 3,
  CHB_OPT_FUSED_LA = 4,
  CHB_OPT_TF32_TCGEN05 = 5,
  CHB_OPT_ORDERED_SUMS = 6,
  CHB_OPT_SCRATCH_LIMIT = 7,
  CHB_OPT_COUNT = 8
};
int chb_plan_set_option(chb_plan* plan, int option, int64_t value);
int chb_plan_get_option(const chb_plan* plan, int option, int64_t* value);

/* Bound of every wait inside the plan's sweeps: a task's wait on its
 * dependencies, on an incoming chunk or for ready work gives up after
 * `polls` polls (with a back-off of up to ~1 us each); the sweep then ends
 * early and chb_info returns -30.  polls < 0 restores the default (about
 * 10 s of polling).  Small values are for tests of that failure path. */
int chb_plan_set_spin_limit(chb_plan* plan, int64_t polls);

/* Diagnostics: resident CTAs per SM of the persistent sweep kernel on the
 * current device, for the FP64 build of the kernel (tcgen05 = 0) or the one
 * with the TF32 tiles on tcgen05 (tcgen05 = 1); a sweep launches that many
 * per SM. */
int chb_engine_occupancy(int tcgen05, int* blocks_per_sm);

/* Allocation-free Cholesky.  No counterpart in the reference: an addition for
 * callers that cannot call cudaMalloc when they factor (frameworks whose
 * device memory all comes from their own pool and that forbid allocations
 * behind their back, processes that must not grow their device footprint
 * after start-up).  Same result as chb_cholesky, but all device scratch comes
 * from one static __device__ array of CHB_NOALLOC_SCRATCH_BYTES (32 MiB) that
 * every GPU which loads this library holds until the process exits; problems
 * that need more are rejected with error -40 and a message giving the size.
 * The plan may be host-only (device < 0).  The first call on a device looks
 * up the array's device address (cudaGetSymbolAddress) with that device
 * current.  The call is synchronous: it waits for the sweep on `stream` and
 * returns its status like chb_info.  It always runs the static list order
 * (chb_plan_set_schedule does not apply) and writes no trace (chb_set_trace
 * does not apply).  Every call shares the one array: calls from host threads
 * of one process take turns on an internal lock, but work of another stream
 * or process that overlaps a call on the GPU races with it: serialise it. */
#define CHB_NOALLOC_SCRATCH_BYTES (32u << 20)
int chb_cholesky_noalloc(chb_plan* plan, double* blkval, void* stream);

/* Synchronise `stream` and return the status of the last sweep run with this
 * workspace: 0, or the 1-based failing column of the first failing front
 * (LAPACK info convention), or < 0 on a device-side consistency error. */
int chb_info(chb_plan* plan, void* work, void* stream);

/* Text of the last host-side error on this thread. */
const char* chb_last_error(void);

/* Build/version string (compute capability the kernels were built for). */
const char* chb_version(void);

#ifdef __cplusplus
}
#endif

#endif /* CHOMPACK_B200_H */
