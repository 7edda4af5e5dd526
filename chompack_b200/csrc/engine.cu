// Persistent task-graph executor for the multifrontal sweeps (sm_100a).
//
// One kernel launch runs a whole sweep.  Each CTA (128 threads) loops:
// claim the next task index with an atomic counter, wait until the counters
// the task depends on reach their targets (bounded spin; on timeout the CTA
// records DE_TIMEOUT and leaves, so a planning error can never hang the
// GPU), execute the task, then publish its counter with release semantics.
//
// Dense FP64 tile arithmetic uses the double-precision tensor-core MMA
// (mma.sync m8n8k4 f64): a 64x64 C tile is split over 4 warps, 32x32 each.
// Operand tiles are staged through shared memory with L2-coherent loads
// (__ldcg), since tiles produced by other CTAs in the same launch must not be
// read from a stale L1 line.
#include <cuda_runtime.h>
#include <cstdint>

#include "engine.h"

namespace chb {

// ------------------------------------------------------------------ sync
__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void red_release_add(int* p, int v) {
  asm volatile("red.release.gpu.global.add.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ int ld_volatile(const int* p) { return *((const volatile int*)p); }

// ------------------------------------------------------------- operands
struct SmemLayout {
  double* A;   // [TILE][LDS]: A(r, k) stored at A[k*LDS + r]
  double* B;   // [TILE][LDS]
};

__device__ __forceinline__ const double* base_ptr(const RunArgs& ra, uint8_t b) { return ra.bases[b]; }

// Element (r, k) of an operand, already known to be inside [0,rows) x [0,K).
__device__ __forceinline__ double op_elem(const double* X, const Operand& o, int r, int k) {
  switch (o.mode) {
    case OM_N:
      return __ldcg(X + (int64_t)k * o.ld + r);
    case OM_T:
      return __ldcg(X + (int64_t)r * o.ld + k);
    case OM_TRI_N:
      return (r + o.diag >= k) ? __ldcg(X + (int64_t)k * o.ld + r) : 0.0;
    case OM_TRI_T:
      return (k + o.diag >= r) ? __ldcg(X + (int64_t)r * o.ld + k) : 0.0;
    default: {  // OM_SYM: element (r + diag, k + pad2) of a symmetric matrix
      int gr = r + o.diag, gc = k + o.pad2;
      return (gr >= gc) ? __ldcg(X + (int64_t)gc * o.ld + gr) : __ldcg(X + (int64_t)gr * o.ld + gc);
    }
  }
}

// Stage opX(r, k0 + kk) for r < 64, kk < KC into S[kk*LDS + r] (zero padded).
__device__ __forceinline__ void stage(const RunArgs& ra, const Operand& o, int rows, int k0, int K, double* S) {
  const double* X = base_ptr(ra, o.base) + o.off;
  const bool kfast = (o.mode == OM_T || o.mode == OM_TRI_T);
#pragma unroll 4
  for (int s = 0; s < (TILE * KC) / NTHREADS; s++) {
    int idx = threadIdx.x + s * NTHREADS;
    int r, kk;
    if (kfast) {
      kk = idx % KC;
      r = idx / KC;
    } else {
      r = idx % TILE;
      kk = idx / TILE;
    }
    int k = k0 + kk;
    double v = 0.0;
    if (r < rows && k < K) v = op_elem(X, o, r, k);
    S[kk * LDS + r] = v;
  }
}

__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

// acc += A(:, 0:kn) * B(:, 0:kn)^T from staged tiles (kn multiple of 4).
__device__ __forceinline__ void mma_block(const double* sA, const double* sB, int kn, double (&acc)[4][4][2]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, q = lane & 3;
  const int r0 = (warp >> 1) * 32 + g, c0 = (warp & 1) * 32 + g;
  for (int kk = 0; kk < kn; kk += 4) {
    double a[4], b[4];
#pragma unroll
    for (int i = 0; i < 4; i++) a[i] = sA[(kk + q) * LDS + r0 + 8 * i];
#pragma unroll
    for (int j = 0; j < 4; j++) b[j] = sB[(kk + q) * LDS + c0 + 8 * j];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) dmma(acc[i][j], a[i], b[j]);
  }
}

__device__ __forceinline__ void zero_acc(double (&acc)[4][4][2]) {
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j][0] = acc[i][j][1] = 0.0;
}

// acc = opA * opB^T over the full K range.
__device__ void gemm_acc(const RunArgs& ra, const Task& t, const SmemLayout& sm, double (&acc)[4][4][2]) {
  zero_acc(acc);
  for (int k0 = 0; k0 < t.k; k0 += KC) {
    stage(ra, t.a, t.m, k0, t.k, sm.A);
    stage(ra, t.b, t.n, k0, t.k, sm.B);
    __syncthreads();
    int kn = min(KC, t.k - k0);
    kn = (kn + 3) & ~3;
    mma_block(sm.A, sm.B, kn, acc);
    __syncthreads();
  }
}

// C = alpha*acc + beta*C (masked to m x n and, for CM_LOWER, to the lower
// triangle).
__device__ void store_acc(const RunArgs& ra, const Task& t, const Operand& co, double alpha, double beta,
                          const double (&acc)[4][4][2]) {
  double* C = ra.bases[co.base] + co.off;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, q = lane & 3;
  const int r0 = (warp >> 1) * 32 + g;
#pragma unroll
  for (int i = 0; i < 4; i++) {
    int r = r0 + 8 * i;
    if (r >= t.m) continue;
#pragma unroll
    for (int j = 0; j < 4; j++) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        int c = (warp & 1) * 32 + 8 * j + 2 * q + h;
        if (c >= t.n) continue;
        if (t.cmode == CM_LOWER && r + t.cdiag < c) continue;
        double* p = C + (int64_t)c * co.ld + r;
        double v = alpha * acc[i][j][h];
        if (beta != 0.0) v += beta * __ldcg(p);
        *p = v;
      }
    }
  }
}

// ------------------------------------------------------------------ GEMM
__device__ void run_gemm(const RunArgs& ra, const Task& t, const SmemLayout& sm) {
  double acc[4][4][2];
  gemm_acc(ra, t, sm, acc);
  store_acc(ra, t, t.c, t.alpha, t.beta, acc);
}

// C = alpha * M2 * (opA * opB^T), M2 = lower-triangular m x m tile (operand
// `c` of the task holds C; M2 is described by aux: base aux[0], ld aux[1],
// offset (aux[2] | aux[3] << 32)).
__device__ void run_mrow(const RunArgs& ra, const Task& t, const SmemLayout& sm) {
  double acc[4][4][2];
  gemm_acc(ra, t, sm, acc);
  // T = acc (m x n) into sm.B as B-stage layout: sB[k*LDS + n] = T(k, n)
  {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, q = lane & 3;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int j = 0; j < 4; j++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
          int r = (warp >> 1) * 32 + 8 * i + g;
          int c = (warp & 1) * 32 + 8 * j + 2 * q + h;
          sm.B[r * LDS + c] = acc[i][j][h];
        }
  }
  // sA[k*LDS + r] = M2(r, k) (lower triangle, zero padded)
  const int64_t moff = (int64_t)(uint32_t)t.aux[2] | ((int64_t)t.aux[3] << 32);
  const double* M2 = ra.bases[t.aux[0]] + moff;
  const int ldm = t.aux[1];
  for (int idx = threadIdx.x; idx < TILE * TILE; idx += NTHREADS) {
    int r = idx % TILE, k = idx / TILE;
    double v = 0.0;
    if (r < t.m && k < t.m && r >= k) v = __ldcg(M2 + (int64_t)k * ldm + r);
    sm.A[k * LDS + r] = v;
  }
  __syncthreads();
  zero_acc(acc);
  mma_block(sm.A, sm.B, (t.m + 3) & ~3, acc);
  __syncthreads();
  store_acc(ra, t, t.c, t.alpha, 0.0, acc);
}

// ----------------------------------------------------------------- POTRF
// Cholesky of the b x b diagonal tile (operand a, in place, lower part
// written back); if aux[1] != 0 also writes M = L^{-1} (full b x b with
// zeros above the diagonal) to operand c.  A non-positive pivot records the
// LAPACK-style info aux[0] + j + 1 in ctl[2] (first writer wins).
__device__ void run_potrf(const RunArgs& ra, const Task& t, double* smem) {
  const int b = t.m;
  const int LD = TILE + 1;
  double* sL = smem;            // [col][row], ld 65
  double* sM = smem + TILE * LD;
  double* X = ra.bases[t.a.base] + t.a.off;
  const int lda = t.a.ld;
  for (int idx = threadIdx.x; idx < b * b; idx += NTHREADS) {
    int r = idx % b, c = idx / b;
    sL[c * LD + r] = (r >= c) ? __ldcg(X + (int64_t)c * lda + r) : 0.0;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int j = 0; j < b; j++) {
    __syncthreads();  // trailing update of column j-1 complete
    double d = sL[j * LD + j];
    bool bad = !(d > 0.0);
    double piv = sqrt(bad ? 1.0 : d);
    double inv = 1.0 / piv;
    if (bad && threadIdx.x == 0) atomicCAS(&ra.ctl[2], 0, t.aux[0] + j + 1);
    for (int i = j + 1 + threadIdx.x; i < b; i += NTHREADS) sL[j * LD + i] *= inv;
    __syncthreads();  // column j scaled; nobody reads sL(j,j) below
    if (threadIdx.x == 0) sL[j * LD + j] = piv;
    for (int l = j + 1 + warp; l < b; l += NTHREADS / 32) {
      double ljl = sL[j * LD + l];
      for (int i = l + lane; i < b; i += 32) sL[l * LD + i] -= sL[j * LD + i] * ljl;
    }
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < b * b; idx += NTHREADS) {
    int r = idx % b, c = idx / b;
    if (r >= c) X[(int64_t)c * lda + r] = sL[c * LD + r];
  }
  if (t.aux[1]) {
    // column c of M = L^{-1}:  M(c,c) = 1/L(c,c);
    // M(i,c) = -(sum_{l=c}^{i-1} L(i,l) M(l,c)) / L(i,i)
    for (int c = threadIdx.x; c < b; c += NTHREADS) {
      sM[c * LD + c] = 1.0 / sL[c * LD + c];
      for (int i = c + 1; i < b; i++) {
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        int l = c;
        for (; l + 3 < i; l += 4) {
          s0 += sL[l * LD + i] * sM[c * LD + l];
          s1 += sL[(l + 1) * LD + i] * sM[c * LD + l + 1];
          s2 += sL[(l + 2) * LD + i] * sM[c * LD + l + 2];
          s3 += sL[(l + 3) * LD + i] * sM[c * LD + l + 3];
        }
        for (; l < i; l++) s0 += sL[l * LD + i] * sM[c * LD + l];
        sM[c * LD + i] = -((s0 + s1) + (s2 + s3)) / sL[i * LD + i];
      }
    }
    __syncthreads();
    double* M = ra.bases[t.c.base] + t.c.off;
    const int ldm = t.c.ld;
    for (int idx = threadIdx.x; idx < b * b; idx += NTHREADS) {
      int r = idx % b, c = idx / b;
      M[(int64_t)c * ldm + r] = (r >= c) ? sM[c * LD + r] : 0.0;
    }
  }
}

// ------------------------------------------------------------ assembly
// Extend-add for front k = aux[0], front columns [aux[1], aux[2]):
//   * zero the columns of the update block U_k that fall in the range
//     (if aux[3] & 1);
//   * for each child, last to first (the order the reference pops its update
//     stack, cholesky.c:41-52), add U_child(i, q) into F(r[i], r[q]) for the
//     child columns q whose relative index r[q] lies in the range.
// F(i, j) is blkval (front panel, ld nj) for j < nn, else U_k (ld na).
__device__ void run_asm(const RunArgs& ra, const Task& t) {
  const FrontDesc f = ra.fronts[t.aux[0]];
  const int j0 = t.aux[1], j1 = t.aux[2];
  double* P = ra.bases[B_X] + f.blk;
  double* Uk = ra.bases[B_WS] + f.upd;
  if (t.aux[3] & 1) {
    for (int j = max(j0, f.nn); j < j1; j++) {
      int jj = j - f.nn;
      for (int i = jj + threadIdx.x; i < f.na; i += NTHREADS) Uk[(int64_t)jj * f.na + i] = 0.0;
    }
  }
  __syncthreads();
  for (int l = f.chend - 1; l >= f.chbeg; l--) {
    const FrontDesc ch = ra.fronts[ra.chidx[l]];
    const int N = ch.na;
    const int32_t* r = ra.relidx + ch.relptr;
    const double* Uc = ra.bases[B_WS] + ch.upd;
    // child columns with r[q] in [j0, j1): r is strictly increasing
    int lo = 0, hi = N;
    while (lo < hi) { int mid = (lo + hi) >> 1; if (r[mid] < j0) lo = mid + 1; else hi = mid; }
    int q0 = lo;
    hi = N;
    while (lo < hi) { int mid = (lo + hi) >> 1; if (r[mid] < j1) lo = mid + 1; else hi = mid; }
    int q1 = lo;
    for (int q = q0; q < q1; q++) {
      const int col = r[q];
      for (int i = q + threadIdx.x; i < N; i += NTHREADS) {
        const int row = r[i];
        double v = __ldcg(Uc + (int64_t)q * N + i);
        if (col < f.nn) P[(int64_t)col * f.nj + row] += v;
        else Uk[(int64_t)(col - f.nn) * f.na + (row - f.nn)] += v;
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- kernel
__global__ void __launch_bounds__(NTHREADS, 3) engine_kernel(RunArgs ra) {
  extern __shared__ double smem[];
  __shared__ int s_task;
  __shared__ int s_abort;
  SmemLayout sm{smem, smem + TILE * LDS};
  for (;;) {
    if (threadIdx.x == 0) s_task = atomicAdd(&ra.ctl[0], 1);
    __syncthreads();
    const int ti = s_task;
    if (ti >= ra.ntasks) break;
    const Task& t = ra.tasks[ti];
    if (threadIdx.x == 0) {
      int abort = 0;
      for (int w = 0; w < t.nwait && !abort; w++) {
        const int2 wt = ra.waits[t.wait_off + w];
        int64_t spins = 0;
        unsigned ns = 32;
        while (ld_acquire(ra.counters + wt.x) < wt.y) {
          if (++spins > ra.spin_limit) {
            atomicCAS(&ra.ctl[1], 0, DE_TIMEOUT);
            atomicAdd(&ra.ctl[3], 1);
            abort = 1;
            break;
          }
          if ((spins & 15) == 0 && ld_volatile(&ra.ctl[1]) != 0) { abort = 1; break; }
          __nanosleep(ns);
          if (ns < 256) ns <<= 1;
        }
      }
      if (!abort && ld_volatile(&ra.ctl[1]) != 0) abort = 1;
      s_abort = abort;
    }
    __syncthreads();
    if (s_abort) break;
    switch (t.op) {
      case T_GEMM: run_gemm(ra, t, sm); break;
      case T_MROW: run_mrow(ra, t, sm); break;
      case T_POTRF: run_potrf(ra, t, smem); break;
      case T_ASM: run_asm(ra, t); break;
      default:
        if (threadIdx.x == 0) atomicCAS(&ra.ctl[1], 0, DE_BAD_TASK);
        break;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      red_release_add(ra.counters + ti, 1);
      if (t.group >= 0) red_release_add(ra.counters + t.group, 1);
    }
  }
}

size_t engine_smem_bytes() { return (size_t)2 * TILE * LDS * sizeof(double); }

// The dynamic shared-memory attribute must have been raised on the current
// device by engine_occupancy() (done when a plan is created).
cudaError_t engine_launch(const RunArgs& ra, int grid, cudaStream_t stream) {
  size_t smem = engine_smem_bytes();
  engine_kernel<<<grid, NTHREADS, smem, stream>>>(ra);
  return cudaGetLastError();
}

int engine_occupancy(int* blocks_per_sm) {
  size_t smem = engine_smem_bytes();
  cudaError_t e = cudaFuncSetAttribute(engine_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return -1;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, engine_kernel, NTHREADS, smem);
  return e == cudaSuccess ? 0 : -1;
}

}  // namespace chb
