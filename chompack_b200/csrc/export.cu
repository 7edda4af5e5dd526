// Element-wise operations between a cspmatrix's blocks and ordinary arrays,
// on the device (reference: src/python/symbolic.py:1032-1128 and
// src/python/base.py:28-67, both Python loops over supernodes there):
//
// * lower_ccs  — the lower trapezoid of every block in compressed-column
//   order (cspmatrix.spmatrix(), symbolic.py:1071-1098): column j = col0 + i
//   of supernode k holds rows i..nj-1 of block column i, which are contiguous
//   in blkval, so each column is one contiguous copy; row indices come from
//   the clique's row list.
// * syr2       — X := alpha P(u v^T + v u^T) + beta X (base.py:28-67): the
//   lower trapezoid of each block, with u, v gathered through p unless the
//   vectors are already in the reordered numbering.
// * projection — X := alpha P(A) + beta X for a dense A (symbolic.py:1176-1210):
//   every entry of each block (the reference updates whole blocks).
// * diag       — the diagonal entries (symbolic.py:1113-1128).
// * add_sparse — X += alpha tril(P(symmetrize(A))) for a sparse A given as
//   (I, J, V) triplets in the original numbering (cspmatrix += spmatrix,
//   symbolic.py:1138-1174).
//
// The block kernels run one CTA per supernode block (grid-stride), columns
// across warps, rows across lanes: reads and writes of blkval are coalesced
// column segments.  add_sparse runs one thread per triplet.
#include <cuda_runtime.h>

#include "../../include/chompack_b200.h"
#include "engine.h"
#include "internal.h"
#include "plan.h"

namespace chb {
namespace {

constexpr int EX_THREADS = 256;
constexpr int EX_WARPS = EX_THREADS / 32;

__global__ void __launch_bounds__(EX_THREADS) lower_ccs_blocks(const double* __restrict__ blkval,
                                                               const FrontDesc* __restrict__ fronts, int nsn,
                                                               const int64_t* __restrict__ sncolptr,
                                                               const int64_t* __restrict__ snrowidx,
                                                               const int64_t* __restrict__ colptr,
                                                               double* __restrict__ vals, int64_t* __restrict__ rows) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = blockIdx.x; k < nsn; k += gridDim.x) {
    const FrontDesc f = fronts[k];
    const int64_t* __restrict__ ri = snrowidx + sncolptr[k];
    for (int i = warp; i < f.nn; i += EX_WARPS) {
      const int64_t dst = colptr[f.col0 + i];
      const double* __restrict__ src = blkval + f.blk + (int64_t)i * f.nj;
      for (int r = i + lane; r < f.nj; r += 32) {
        vals[dst + (r - i)] = src[r];
        if (rows) rows[dst + (r - i)] = ri[r];
      }
    }
  }
}

__global__ void __launch_bounds__(EX_THREADS) syr2_blocks(double* __restrict__ blkval,
                                                          const FrontDesc* __restrict__ fronts, int nsn,
                                                          const int64_t* __restrict__ sncolptr,
                                                          const int64_t* __restrict__ snrowidx,
                                                          const int64_t* __restrict__ perm,
                                                          const double* __restrict__ u, const double* __restrict__ v,
                                                          double alpha, double beta) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = blockIdx.x; k < nsn; k += gridDim.x) {
    const FrontDesc f = fronts[k];
    const int64_t* __restrict__ ri = snrowidx + sncolptr[k];
    for (int c = warp; c < f.nn; c += EX_WARPS) {
      const int64_t gc = perm ? perm[ri[c]] : ri[c];
      const double auc = alpha * u[gc], avc = alpha * v[gc];
      double* __restrict__ col = blkval + f.blk + (int64_t)c * f.nj;
      for (int r = c + lane; r < f.nj; r += 32) {
        const int64_t gr = perm ? perm[ri[r]] : ri[r];
        // the reference: dscal by beta, then u v^T and v u^T added
        double x = beta * col[r];
        x = fma(u[gr], avc, x);
        x = fma(v[gr], auc, x);
        col[r] = x;
      }
    }
  }
}

// mode 0: A[r, c] in the reordered numbering; mode 1: the symmetric matrix
// of A's lower triangle in the original numbering, A[max(p_r, p_c), min(p_r, p_c)]
__global__ void __launch_bounds__(EX_THREADS) projection_blocks(double* __restrict__ blkval,
                                                                const FrontDesc* __restrict__ fronts, int nsn,
                                                                const int64_t* __restrict__ sncolptr,
                                                                const int64_t* __restrict__ snrowidx,
                                                                const int64_t* __restrict__ perm,
                                                                const double* __restrict__ A, int64_t lda,
                                                                double alpha, double beta, int mode) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = blockIdx.x; k < nsn; k += gridDim.x) {
    const FrontDesc f = fronts[k];
    const int64_t* __restrict__ ri = snrowidx + sncolptr[k];
    for (int c = warp; c < f.nn; c += EX_WARPS) {
      const int64_t gc = mode ? perm[ri[c]] : ri[c];
      double* __restrict__ col = blkval + f.blk + (int64_t)c * f.nj;
      for (int r = lane; r < f.nj; r += 32) {
        const int64_t gr = mode ? perm[ri[r]] : ri[r];
        const int64_t i = mode ? (gr > gc ? gr : gc) : gr;
        const int64_t j = mode ? (gr > gc ? gc : gr) : gc;
        col[r] = fma(alpha, A[j * lda + i], beta * col[r]);
      }
    }
  }
}

__global__ void __launch_bounds__(EX_THREADS) diag_blocks(const double* __restrict__ blkval,
                                                          const FrontDesc* __restrict__ fronts, int nsn,
                                                          double* __restrict__ d) {
  for (int k = blockIdx.x; k < nsn; k += gridDim.x) {
    const FrontDesc f = fronts[k];
    for (int i = threadIdx.x; i < f.nn; i += EX_THREADS) d[f.col0 + i] = blkval[f.blk + (int64_t)i * f.nj + i];
  }
}

// One thread per triplet (grid-stride).  symmetrize() reads only the lower
// entries (i >= j) of A and mirrors them, perm() renumbers through p and
// tril() keeps the lower copy, so each lower entry of A lands once, at
// (max, min) of (ip[i], ip[j]).  The supernode holding column j is the last
// k with col0 <= j (binary search over the fronts, which are in column
// order), the row's position the index of i in the clique's ascending row
// list (binary search); the entry is added at
// blk + (j - col0) nj + position.  An entry whose row is not in the list
// (outside the chordal pattern) or whose index is out of range is counted
// in *bad and not written.  Values are added with atomics, so duplicated
// triplets are summed; a duplicate-free A (an spmatrix) adds each position
// once, alpha * v as the reference does.
__global__ void __launch_bounds__(EX_THREADS) add_sparse_entries(
    double* __restrict__ blkval, const FrontDesc* __restrict__ fronts, int nsn, int64_t n,
    const int64_t* __restrict__ sncolptr, const int64_t* __restrict__ snrowidx, const int64_t* __restrict__ iperm,
    int64_t nnz, const int64_t* __restrict__ I, const int64_t* __restrict__ J, const double* __restrict__ V,
    double alpha, unsigned long long* __restrict__ bad) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += stride) {
    int64_t i = I[e], j = J[e];
    if (i < 0 || j < 0 || i >= n || j >= n) {
      atomicAdd(bad, 1ull);
      continue;
    }
    if (i < j) continue;
    if (iperm) {
      i = iperm[i];
      j = iperm[j];
    }
    if (i < j) {
      const int64_t t = i;
      i = j;
      j = t;
    }
    int lo = 0, hi = nsn - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (fronts[mid].col0 <= j) lo = mid;
      else hi = mid - 1;
    }
    const int64_t col0 = fronts[lo].col0, blk = fronts[lo].blk;
    const int nj = fronts[lo].nj, nn = fronts[lo].nn;
    const int64_t* __restrict__ ri = snrowidx + sncolptr[lo];
    int a = 0, b = nj;
    while (a < b) {
      const int m = (a + b) >> 1;
      if (ri[m] < i) a = m + 1;
      else b = m;
    }
    if (j - col0 >= nn || a == nj || ri[a] != i) {
      atomicAdd(bad, 1ull);
      continue;
    }
    atomicAdd(blkval + blk + (j - col0) * nj + a, alpha * V[e]);
  }
}

int grid_for(int nsn) { return nsn < 8192 ? nsn : 8192; }

}  // namespace
}  // namespace chb

using namespace chb;

static int ex_check(chb_plan* plan) {
  if (!plan) return set_error(-1, "null plan");
  if (plan->device < 0 || !plan->d_fronts) return set_error(-2, "host-only plan: no device data");
  return 0;
}

static int ex_done(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(-100 - (int)e, "%s launch failed: %s", what, cudaGetErrorString(e));
  return 0;
}

extern "C" int chb_lower_ccs(chb_plan* plan, const double* blkval, const int64_t* sncolptr, const int64_t* snrowidx,
                             const int64_t* colptr, double* values, int64_t* rowidx, void* stream) {
  clear_error();
  int rc = ex_check(plan);
  if (rc) return rc;
  if (!blkval || !sncolptr || !snrowidx || !colptr || !values) return set_error(-1, "null argument");
  if (plan->nsn == 0) return 0;
  lower_ccs_blocks<<<grid_for((int)plan->nsn), EX_THREADS, 0, (cudaStream_t)stream>>>(
      blkval, plan->d_fronts, (int)plan->nsn, sncolptr, snrowidx, colptr, values, rowidx);
  return ex_done("lower_ccs");
}

extern "C" int chb_syr2(chb_plan* plan, double* blkval, const int64_t* sncolptr, const int64_t* snrowidx,
                        const double* u, const double* v, double alpha, double beta, int reordered, void* stream) {
  clear_error();
  int rc = ex_check(plan);
  if (rc) return rc;
  if (!blkval || !sncolptr || !snrowidx || !u || !v) return set_error(-1, "null argument");
  if (plan->nsn == 0) return 0;
  syr2_blocks<<<grid_for((int)plan->nsn), EX_THREADS, 0, (cudaStream_t)stream>>>(
      blkval, plan->d_fronts, (int)plan->nsn, sncolptr, snrowidx, reordered ? nullptr : plan->d_perm, u, v, alpha,
      beta);
  return ex_done("syr2");
}

extern "C" int chb_add_projection(chb_plan* plan, double* blkval, const int64_t* sncolptr, const int64_t* snrowidx,
                                  const double* A, int64_t lda, double alpha, double beta, int symmetric_original,
                                  void* stream) {
  clear_error();
  int rc = ex_check(plan);
  if (rc) return rc;
  if (!blkval || !sncolptr || !snrowidx || !A) return set_error(-1, "null argument");
  if (lda < (plan->n > 1 ? plan->n : 1)) return set_error(-1, "lda must be at least max(1, n)");
  if (plan->nsn == 0) return 0;
  projection_blocks<<<grid_for((int)plan->nsn), EX_THREADS, 0, (cudaStream_t)stream>>>(
      blkval, plan->d_fronts, (int)plan->nsn, sncolptr, snrowidx, plan->d_perm, A, lda, alpha, beta,
      symmetric_original ? 1 : 0);
  return ex_done("add_projection");
}

extern "C" int chb_diag(chb_plan* plan, const double* blkval, double* d, void* stream) {
  clear_error();
  int rc = ex_check(plan);
  if (rc) return rc;
  if (!blkval || !d) return set_error(-1, "null argument");
  if (plan->nsn == 0) return 0;
  diag_blocks<<<grid_for((int)plan->nsn), EX_THREADS, 0, (cudaStream_t)stream>>>(blkval, plan->d_fronts,
                                                                                   (int)plan->nsn, d);
  return ex_done("diag");
}

extern "C" int chb_add_sparse(chb_plan* plan, double* blkval, const int64_t* sncolptr, const int64_t* snrowidx,
                              int64_t nnz, const int64_t* I, const int64_t* J, const double* V, double alpha,
                              int reordered, unsigned long long* bad, void* stream) {
  clear_error();
  int rc = ex_check(plan);
  if (rc) return rc;
  if (nnz < 0) return set_error(-1, "negative nnz");
  if (!blkval || !sncolptr || !snrowidx || !bad || (nnz > 0 && (!I || !J || !V)))
    return set_error(-1, "null argument");
  if (cudaMemsetAsync(bad, 0, sizeof(unsigned long long), (cudaStream_t)stream) != cudaSuccess)
    return ex_done("add_sparse");
  if (nnz == 0 || plan->nsn == 0) return 0;
  const int64_t want = (nnz + EX_THREADS - 1) / EX_THREADS;
  const int grid = (int)(want < 148 * 64 ? want : 148 * 64);
  add_sparse_entries<<<grid, EX_THREADS, 0, (cudaStream_t)stream>>>(
      blkval, plan->d_fronts, (int)plan->nsn, plan->n, sncolptr, snrowidx, reordered ? nullptr : plan->d_iperm, nnz,
      I, J, V, alpha, bad);
  return ex_done("add_sparse");
}
