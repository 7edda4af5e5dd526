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
// of leading dimension ld, rows in the original order through perm.  One
// CTA per supernode k (nn columns, nj rows):
//   rows: y[row i] += sum_j X(i, j) x[col j] with one thread per row (the
//         diagonal block read symmetrically), one atomic per row;
//   columns: y[col j] += sum_{i >= nn} X(i, j) x[row i] for the rows below
//         the diagonal block, one warp per column, one atomic per column.
// The atomics make the last bits of y depend on the schedule.
constexpr int SYMV_RHS = 8;  // right-hand sides per pass
__global__ void __launch_bounds__(DOT_THREADS) symv_blocks(const double* __restrict__ blkval,
                                                           const FrontDesc* __restrict__ fronts,
                                                           const int64_t* __restrict__ sncolptr,
                                                           const int64_t* __restrict__ snrowidx,
                                                           const int64_t* __restrict__ perm, const double* __restrict__ x,
                                                           double* __restrict__ y, int nsn, int nrhs, int64_t ld,
                                                           double alpha) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = blockIdx.x; k < nsn; k += gridDim.x) {
    const FrontDesc f = fronts[k];
    const int nn = f.nn, nj = f.nj;
    const int64_t* __restrict__ rows = snrowidx + sncolptr[k];
    const double* __restrict__ b = blkval + f.blk;
    for (int r0 = 0; r0 < nrhs; r0 += SYMV_RHS) {
      const int nr = min(SYMV_RHS, nrhs - r0);
      // rows
      for (int i = threadIdx.x; i < nj; i += DOT_THREADS) {
        double acc[SYMV_RHS];
#pragma unroll
        for (int r = 0; r < SYMV_RHS; r++) acc[r] = 0.0;
        for (int j = 0; j < nn; j++) {
          const double v = (i >= j) ? b[(int64_t)j * nj + i] : b[(int64_t)i * nj + j];
          const int64_t C = perm[rows[j]];
#pragma unroll
          for (int r = 0; r < SYMV_RHS; r++)
            if (r < nr) acc[r] = fma(v, x[C + (r0 + r) * ld], acc[r]);
        }
        const int64_t R = perm[rows[i]];
#pragma unroll
        for (int r = 0; r < SYMV_RHS; r++)
          if (r < nr) atomicAdd(y + R + (r0 + r) * ld, alpha * acc[r]);
      }
      // columns, from the rows below the diagonal block
      for (int j = warp; j < nn; j += DOT_THREADS / 32) {
        double acc[SYMV_RHS];
#pragma unroll
        for (int r = 0; r < SYMV_RHS; r++) acc[r] = 0.0;
        for (int i = nn + lane; i < nj; i += 32) {
          const double v = b[(int64_t)j * nj + i];
          const int64_t R = perm[rows[i]];
#pragma unroll
          for (int r = 0; r < SYMV_RHS; r++)
            if (r < nr) acc[r] = fma(v, x[R + (r0 + r) * ld], acc[r]);
        }
#pragma unroll
        for (int r = 0; r < SYMV_RHS; r++) {
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], o);
        }
        if (lane == 0) {
          const int64_t C = perm[rows[j]];
#pragma unroll
          for (int r = 0; r < SYMV_RHS; r++)
            if (r < nr) atomicAdd(y + C + (r0 + r) * ld, alpha * acc[r]);
        }
      }
    }
  }
}

}  // namespace

cudaError_t symv_launch(const double* blkval, const FrontDesc* fronts, const int64_t* sncolptr,
                        const int64_t* snrowidx, const int64_t* perm, const double* x, double* y, int nsn, int nrhs,
                        int64_t ld, double alpha, cudaStream_t stream) {
  if (nsn <= 0 || nrhs <= 0) return cudaSuccess;
  symv_blocks<<<nsn, DOT_THREADS, 0, stream>>>(blkval, fronts, sncolptr, snrowidx, perm, x, y, nsn, nrhs, ld, alpha);
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
