// Trace inner product <X, Y> of two chordal matrices on the same pattern
// (reference: dot.c:3-23): sum over the lower trapezoid of every supernode
// block, off-diagonal entries counted twice.  One CTA per supernode block
// writes a partial sum; a single CTA adds the partials in a fixed order, so
// the result is deterministic.
#include <cuda_runtime.h>

#include "engine.h"

namespace chb {

namespace {
constexpr int DOT_THREADS = 256;

__device__ double block_sum(double v, double* sh) {
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int s = DOT_THREADS / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  return sh[0];
}

__global__ void __launch_bounds__(DOT_THREADS) dot_blocks(const double* __restrict__ x, const double* __restrict__ y,
                                                          const FrontDesc* __restrict__ fronts, int nsn,
                                                          double* __restrict__ partial) {
  __shared__ double sh[DOT_THREADS];
  for (int k = blockIdx.x; k < nsn; k += gridDim.x) {
    const FrontDesc f = fronts[k];
    const int64_t total = (int64_t)f.nj * f.nn;
    double acc = 0.0;
    for (int64_t idx = threadIdx.x; idx < total; idx += DOT_THREADS) {
      const int r = (int)(idx % f.nj), c = (int)(idx / f.nj);
      if (r < c) continue;
      const double p = x[f.blk + idx] * y[f.blk + idx];
      acc += (r == c) ? p : 2.0 * p;
    }
    const double s = block_sum(acc, sh);
    if (threadIdx.x == 0) partial[k] = s;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(DOT_THREADS) dot_final(const double* __restrict__ partial, int n,
                                                         double* __restrict__ out) {
  __shared__ double sh[DOT_THREADS];
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += DOT_THREADS) acc += partial[i];
  const double s = block_sum(acc, sh);
  if (threadIdx.x == 0) *out = s;
}
// log det X = 2 * sum_k sum_j log L_kk(j, j) from the factor's diagonal
// blocks; one partial per supernode, added by dot_final.
__global__ void __launch_bounds__(DOT_THREADS) logdet_blocks(const double* __restrict__ l,
                                                             const FrontDesc* __restrict__ fronts, int nsn,
                                                             double* __restrict__ partial) {
  __shared__ double sh[DOT_THREADS];
  for (int k = blockIdx.x; k < nsn; k += gridDim.x) {
    const FrontDesc f = fronts[k];
    double acc = 0.0;
    for (int j = threadIdx.x; j < f.nn; j += DOT_THREADS) acc += 2.0 * log(l[f.blk + (int64_t)j * f.nj + j]);
    const double s = block_sum(acc, sh);
    if (threadIdx.x == 0) partial[k] = s;
    __syncthreads();
  }
}

// y = alpha * w .* x over the stored entries, w = 2 below the diagonal, 1 on
// it, 0 in the strict upper part of a diagonal block: the map from a
// chordal symmetric matrix to the gradient of a function of its stored
// entries (<A, B> = sum w a b).
__global__ void __launch_bounds__(DOT_THREADS) symw_blocks(const double* __restrict__ x, double* __restrict__ y,
                                                           double alpha, const FrontDesc* __restrict__ fronts,
                                                           int nsn) {
  for (int k = blockIdx.x; k < nsn; k += gridDim.x) {
    const FrontDesc f = fronts[k];
    const int64_t total = (int64_t)f.nj * f.nn;
    for (int64_t idx = threadIdx.x; idx < total; idx += DOT_THREADS) {
      const int r = (int)(idx % f.nj), c = (int)(idx / f.nj);
      const double w = (r > c) ? 2.0 : (r == c ? 1.0 : 0.0);
      y[f.blk + idx] = alpha * w * x[f.blk + idx];
    }
  }
}
// out[m] = sum of partial[seg[m] .. seg[m+1]) in a fixed order (one CTA per
// segment): the per-matrix results of a merged plan.
__global__ void __launch_bounds__(DOT_THREADS) seg_final(const double* __restrict__ partial,
                                                         const int64_t* __restrict__ seg, int count,
                                                         double* __restrict__ out) {
  __shared__ double sh[DOT_THREADS];
  for (int m = blockIdx.x; m < count; m += gridDim.x) {
    double acc = 0.0;
    for (int64_t i = seg[m] + threadIdx.x; i < seg[m + 1]; i += DOT_THREADS) acc += partial[i];
    const double s = block_sum(acc, sh);
    if (threadIdx.x == 0) out[m] = s;
    __syncthreads();
  }
}
// y += alpha X x for the symmetric chordal matrix X in blkval (lower
// trapezoid of each supernode block; both triangles applied), nrhs columns
// of leading dimension ld, rows in the original order through perm.
// One CTA per strip of 64 rows of a supernode block (items[] = (k, first
// row)); the strip is walked in 64 x 64 tiles of its stored lower part,
// staged in shared memory with coalesced loads, so every stored entry is
// read from memory once.  From each tile:
//   rows:    y[row i] += sum_j X(i, j) x[col j]   over stored j <= i,
//   columns: y[col j] += sum_i X(i, j) x[row i]   over stored i >  j,
// which together apply the symmetric matrix once.  Four threads share a
// row (or column) and reduce through shared memory; each strip adds its
// rows once and its columns once per right-hand side with atomics, so the
// last bits of y depend on the schedule.
constexpr int SYMV_RHS = 8;   // right-hand sides per pass
constexpr int SYMV_T = 64;    // strip height and tile width
constexpr int SYMV_LD = SYMV_T + 1;
__global__ void __launch_bounds__(DOT_THREADS) symv_strips(const double* __restrict__ blkval,
                                                           const FrontDesc* __restrict__ fronts,
                                                           const int2* __restrict__ items, int nitems,
                                                           const int64_t* __restrict__ sncolptr,
                                                           const int64_t* __restrict__ snrowidx,
                                                           const int64_t* __restrict__ perm, const double* __restrict__ x,
                                                           double* __restrict__ y, int nrhs, int64_t ld, double alpha) {
  // the tile, and (once its entries are consumed) the 4-way reductions
  __shared__ double tile[SYMV_T * SYMV_LD];
  __shared__ double xr[SYMV_RHS][SYMV_T];   // x at the strip's rows
  __shared__ double xc[SYMV_RHS][SYMV_T];   // x at the tile's columns
  static_assert(4 * SYMV_RHS * SYMV_T <= SYMV_T * SYMV_LD, "reduction buffer exceeds the tile");
  double (*red)[SYMV_RHS][SYMV_T] = reinterpret_cast<double (*)[SYMV_RHS][SYMV_T]>(tile);
  __shared__ int64_t grow[SYMV_T], gcol[SYMV_T];
  const int t = threadIdx.x, lr = t & (SYMV_T - 1), q = t >> 6;  // q = 0..3
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int2 w = items[it];
    const FrontDesc f = fronts[w.x];
    const int nn = f.nn, nj = f.nj, i0 = w.y;
    const int mi = min(SYMV_T, nj - i0);
    const int64_t* __restrict__ rows = snrowidx + sncolptr[w.x];
    const double* __restrict__ b = blkval + f.blk;
    const int jend = min(nn, i0 + mi);  // columns holding stored entries of the strip
    for (int r0 = 0; r0 < nrhs; r0 += SYMV_RHS) {
      const int nr = min(SYMV_RHS, nrhs - r0);
      __syncthreads();
      if (t < SYMV_T) grow[t] = t < mi ? perm[rows[i0 + t]] : 0;
      __syncthreads();
      for (int e = t; e < SYMV_RHS * SYMV_T; e += DOT_THREADS) {
        const int r = e / SYMV_T, ii = e % SYMV_T;
        xr[r][ii] = (r < nr && ii < mi) ? x[grow[ii] + (r0 + r) * ld] : 0.0;
      }
      double racc[SYMV_RHS];
#pragma unroll
      for (int r = 0; r < SYMV_RHS; r++) racc[r] = 0.0;
      for (int j0 = 0; j0 < jend; j0 += SYMV_T) {
        const int mj = min(SYMV_T, jend - j0);
        __syncthreads();
        if (t < SYMV_T) gcol[t] = t < mj ? perm[rows[j0 + t]] : 0;
        // tile(ii, jj) = X(i0 + ii, j0 + jj) where stored (row >= column)
        for (int c = q; c < SYMV_T; c += 4) {
          const int gi = i0 + lr, gj = j0 + c;
          tile[c * SYMV_LD + lr] = (lr < mi && c < mj && gi >= gj) ? b[(int64_t)gj * nj + gi] : 0.0;
        }
        __syncthreads();
        for (int e = t; e < SYMV_RHS * SYMV_T; e += DOT_THREADS) {
          const int r = e / SYMV_T, jj = e % SYMV_T;
          xc[r][jj] = (r < nr && jj < mj) ? x[gcol[jj] + (r0 + r) * ld] : 0.0;
        }
        __syncthreads();
        // rows: thread (row lr, columns c = q mod 4)
        for (int c = q; c < mj; c += 4) {
          const double v = tile[c * SYMV_LD + lr];
#pragma unroll
          for (int r = 0; r < SYMV_RHS; r++) racc[r] = fma(v, xc[r][c], racc[r]);
        }
        // columns: thread (column lr, rows ii = q mod 4), strictly below the diagonal
        double cacc[SYMV_RHS];
#pragma unroll
        for (int r = 0; r < SYMV_RHS; r++) cacc[r] = 0.0;
        for (int ii = q; ii < mi; ii += 4) {
          const double v = (i0 + ii > j0 + lr) ? tile[lr * SYMV_LD + ii] : 0.0;
#pragma unroll
          for (int r = 0; r < SYMV_RHS; r++) cacc[r] = fma(v, xr[r][ii], cacc[r]);
        }
        __syncthreads();  // every thread is done with the tile's entries
#pragma unroll
        for (int r = 0; r < SYMV_RHS; r++) red[q][r][lr] = cacc[r];
        __syncthreads();
        for (int e = t; e < SYMV_RHS * SYMV_T; e += DOT_THREADS) {
          const int r = e / SYMV_T, jj = e % SYMV_T;
          if (r < nr && jj < mj) {
            const double s = red[0][r][jj] + red[1][r][jj] + red[2][r][jj] + red[3][r][jj];
            if (s != 0.0) atomicAdd(y + gcol[jj] + (r0 + r) * ld, alpha * s);
          }
        }
      }
      __syncthreads();
#pragma unroll
      for (int r = 0; r < SYMV_RHS; r++) red[q][r][lr] = racc[r];
      __syncthreads();
      for (int e = t; e < SYMV_RHS * SYMV_T; e += DOT_THREADS) {
        const int r = e / SYMV_T, ii = e % SYMV_T;
        if (r < nr && ii < mi) {
          const double s = red[0][r][ii] + red[1][r][ii] + red[2][r][ii] + red[3][r][ii];
          atomicAdd(y + grow[ii] + (r0 + r) * ld, alpha * s);
        }
      }
    }
  }
}

}  // namespace

cudaError_t symv_launch(const double* blkval, const FrontDesc* fronts, const int2* items, int nitems,
                        const int64_t* sncolptr, const int64_t* snrowidx, const int64_t* perm, const double* x,
                        double* y, int nrhs, int64_t ld, double alpha, cudaStream_t stream) {
  if (nitems <= 0 || nrhs <= 0) return cudaSuccess;
  const int grid = nitems < 65535 ? nitems : 65535;
  symv_strips<<<grid, DOT_THREADS, 0, stream>>>(blkval, fronts, items, nitems, sncolptr, snrowidx, perm, x, y, nrhs,
                                                 ld, alpha);
  return cudaGetLastError();
}

cudaError_t segment_sums(const double* partial, const int64_t* seg, int count, double* out, cudaStream_t stream) {
  if (count > 0) seg_final<<<count < 4096 ? count : 4096, DOT_THREADS, 0, stream>>>(partial, seg, count, out);
  return cudaGetLastError();
}

cudaError_t logdet_partials(const double* l, const FrontDesc* fronts, int nsn, double* partial, cudaStream_t stream) {
  if (nsn > 0) logdet_blocks<<<nsn < 4096 ? nsn : 4096, DOT_THREADS, 0, stream>>>(l, fronts, nsn, partial);
  return cudaGetLastError();
}

cudaError_t dot_partials(const double* x, const double* y, const FrontDesc* fronts, int nsn, double* partial,
                         cudaStream_t stream) {
  if (nsn > 0) dot_blocks<<<nsn < 4096 ? nsn : 4096, DOT_THREADS, 0, stream>>>(x, y, fronts, nsn, partial);
  return cudaGetLastError();
}

cudaError_t logdet_launch(const double* l, const FrontDesc* fronts, int nsn, double* partial, double* out,
                          cudaStream_t stream) {
  if (nsn > 0) {
    int grid = nsn < 4096 ? nsn : 4096;
    logdet_blocks<<<grid, DOT_THREADS, 0, stream>>>(l, fronts, nsn, partial);
  }
  dot_final<<<1, DOT_THREADS, 0, stream>>>(partial, nsn, out);
  return cudaGetLastError();
}

cudaError_t symw_launch(const double* x, double* y, double alpha, const FrontDesc* fronts, int nsn,
                        cudaStream_t stream) {
  if (nsn > 0) {
    int grid = nsn < 4096 ? nsn : 4096;
    symw_blocks<<<grid, DOT_THREADS, 0, stream>>>(x, y, alpha, fronts, nsn);
  }
  return cudaGetLastError();
}

cudaError_t dot_launch(const double* x, const double* y, const FrontDesc* fronts, int nsn, double* partial,
                       double* out, cudaStream_t stream) {
  if (nsn > 0) {
    int grid = nsn < 4096 ? nsn : 4096;
    dot_blocks<<<grid, DOT_THREADS, 0, stream>>>(x, y, fronts, nsn, partial);
  }
  dot_final<<<1, DOT_THREADS, 0, stream>>>(partial, nsn, out);
  return cudaGetLastError();
}

}  // namespace chb
