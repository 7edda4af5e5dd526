// Product-form Cholesky factor of I + V diag(a) V^T (reference:
// src/C/pfcholesky.c; composed by src/python/pfcholesky.py:113-211):
//
//   I + V diag(a) V^T = L_1 L_2 ... L_k L_k^T ... L_2^T L_1^T,
//
// each L_i = diag(l_i) + strictly-lower(v_i b_i^T) stored as three n-vectors
// (column i of V, L and B).  The reference's kernels are first-order
// recurrences along the n rows:
//
//   dpftrf (pfcholesky.c:52-88), per factor i:
//     alpha_0 = -a_i, l_j = sqrt(1 - alpha_j v_j^2), b_j = -alpha_j v_j / l_j,
//     alpha_{j+1} = alpha_j + b_j^2; then every later column j > i of V is
//     solved with L_i (ddrsv 'N').
//   ddrsv (:4-25)  x_r := (x_r - p_r s_r) / l_r,  s_{r+1} = s_r + q_r x_r(new)
//   ddrmv (:27-50) x_r := l_r x_r + p_r s_r,       s_{r+1} = s_r + q_r x_r(old)
//   with (p, q) = (v, b) for 'N' (rows ascending) and (b, v) for 'T' (rows
//   descending); dpfsv / dpfmv (:90-136) apply the k factors in sequence.
//
// Here every recurrence is a scan over rows, so it runs in parallel:
// * the running sum s of ddrsv / ddrmv is an affine recurrence
//   s_{r+1} = a_r s_r + c_r (ddrsv: a_r = 1 - p_r q_r / l_r, c_r = q_r x_r / l_r;
//   ddrmv: a_r = 1, c_r = q_r x_r), a scan of affine maps;
// * alpha satisfies 1/alpha_{j+1} = 1/alpha_j - v_j^2 (substitute b_j), so
//   alpha_j = 1 / (1/alpha_0 - sum_{t<j} v_t^2) is a prefix sum.
//
// One persistent kernel (cooperative launch, so all CTAs are resident) runs
// a whole call.  The rows are split into one contiguous range per CTA.  Per
// step (one factor) a CTA first reduces its rows' maps to one aggregate per
// column, publishes it, waits until every CTA has published (a bounded wait
// on a counter in the workspace), composes its predecessors' aggregates into
// its carry-in and applies the scan to its rows.  Rows go through the CTA in
// sub-blocks of 2048 (8 per thread: sequential per thread, then a block scan
// of the per-thread maps).  dpftrf takes two such steps per factor (the
// alpha prefix sum, then the solves of the later columns).  Every wait is
// bounded in time; a wait that runs out records an error and the kernel
// returns.
#include <cuda_runtime.h>

#include <cstring>

#include "../../include/chompack_b200.h"
#include "internal.h"

namespace chb {
namespace {

constexpr int PF_THREADS = 256;
constexpr int PF_Q = 8;                       // rows per thread per sub-block
constexpr int PF_SB = PF_THREADS * PF_Q;      // rows per sub-block
constexpr int PF_WARPS = PF_THREADS / 32;
constexpr size_t PF_CTL_BYTES = 256;          // control words at the start of the workspace
constexpr unsigned long long PF_WAIT_NS = 4000000000ull;   // 4 s per wait

enum { PF_OP_TRF = 0, PF_OP_SV = 1, PF_OP_MV = 2 };
// ctl[0]: error (1 = a wait ran out), ctl[1]: info (-1: 1 - alpha v^2 <= 0),
// ctl[2]: arrival counter of the grid-wide waits
enum { C_ERR = 0, C_INFO = 1, C_BAR = 2 };

struct PfArgs {
  int op;
  int trans;                 // 0 'N', 1 'T'
  int64_t n;
  int k;
  int ncols;                 // right-hand sides (sv / mv)
  const double* a;
  double* V;
  int64_t ldv;
  double* L;
  int64_t ldl;
  double* B;
  int64_t ldb;
  double* U;
  int64_t ldu;
  int* ctl;
  double2* agg;              // [2][gridDim.x][agg_cols] per-CTA aggregates (A, C)
  int agg_cols;
  int64_t chunk;             // rows per CTA
};

// affine map s -> A s + C; compose(f, g) applies g first, then f
struct Aff {
  double A, C;
};
__device__ __forceinline__ Aff compose(Aff f, Aff g) { return {f.A * g.A, fma(f.A, g.C, f.C)}; }

__device__ __forceinline__ int ld_acquire_i(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Grid-wide wait number `phase` (0, 1, ...): every CTA arrives once per
// phase; returns false when a wait ran out (here or in another CTA).
__device__ bool grid_wait(int* ctl, int phase) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(&ctl[C_BAR], 1);
    const int target = (phase + 1) * (int)gridDim.x;
    const unsigned long long t0 = now_ns();
    unsigned ns = 32;
    int good = 1;
    while (ld_acquire_i(&ctl[C_BAR]) < target) {
      if (*((volatile int*)&ctl[C_ERR]) != 0) {
        good = 0;
        break;
      }
      if (now_ns() - t0 > PF_WAIT_NS) {
        atomicExch(&ctl[C_ERR], 1);
        good = 0;
        break;
      }
      __nanosleep(ns);
      if (ns < 512) ns <<= 1;
    }
    ok = good;
  }
  __syncthreads();
  return ok != 0;
}

// Exclusive block scan of per-thread maps in thread order; returns this
// thread's exclusive prefix and writes the block's total to *tot.
__device__ Aff block_scan(Aff m, Aff* tot) {
  __shared__ Aff warp_tot[PF_WARPS];
  __shared__ Aff warp_pre[PF_WARPS + 1];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  Aff inc = m;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    Aff o;
    o.A = __shfl_up_sync(0xffffffffu, inc.A, off);
    o.C = __shfl_up_sync(0xffffffffu, inc.C, off);
    if (lane >= off) inc = compose(inc, o);
  }
  Aff exc;
  exc.A = __shfl_up_sync(0xffffffffu, inc.A, 1);
  exc.C = __shfl_up_sync(0xffffffffu, inc.C, 1);
  if (lane == 0) exc = {1.0, 0.0};
  if (lane == 31) warp_tot[w] = inc;
  __syncthreads();
  if (threadIdx.x == 0) {
    Aff run = {1.0, 0.0};
    for (int i = 0; i < PF_WARPS; i++) {
      warp_pre[i] = run;
      run = compose(warp_tot[i], run);
    }
    warp_pre[PF_WARPS] = run;
  }
  __syncthreads();
  *tot = warp_pre[PF_WARPS];
  const Aff r = compose(exc, warp_pre[w]);
  __syncthreads();   // warp_tot / warp_pre are reused by the next call
  return r;
}

// One column of one step: the rows' recurrence kind and vectors.
//   kind 0: sum       s_{r+1} = s_r + x_r^2            (dpftrf's alpha scan)
//   kind 1: ddrsv     x_r := (x_r - p_r s_r)/l_r, a_r = 1 - p_r q_r/l_r, c_r = q_r x_r/l_r
//   kind 2: ddrmv     x_r := l_r x_r + p_r s_r,   a_r = 1,               c_r = q_r x_r
struct Col {
  int kind;
  double* x;
  const double* p;
  const double* q;
  const double* l;
};

__device__ __forceinline__ Aff row_map(const Col& c, int64_t i) {
  const double x = c.x[i];
  if (c.kind == 0) return {1.0, x * x};
  const double q = c.q[i];
  if (c.kind == 1) {
    const double l = c.l[i];
    return {1.0 - c.p[i] * q / l, q * x / l};
  }
  return {1.0, q * x};
}

__device__ __forceinline__ int64_t phys(const PfArgs& pa, int64_t r) { return pa.trans ? pa.n - 1 - r : r; }

// Aggregate of the CTA's rows [r0, r1) for one column.
__device__ Aff cta_aggregate(const PfArgs& pa, const Col& c, int64_t r0, int64_t r1) {
  Aff total = {1.0, 0.0};
  for (int64_t sb = r0; sb < r1; sb += PF_SB) {
    Aff m = {1.0, 0.0};
    const int64_t base = sb + (int64_t)threadIdx.x * PF_Q;
#pragma unroll
    for (int t = 0; t < PF_Q; t++) {
      const int64_t r = base + t;
      if (r < r1) m = compose(row_map(c, phys(pa, r)), m);
    }
    Aff tot;
    block_scan(m, &tot);
    total = compose(tot, total);
  }
  return total;
}

// Apply the recurrence to the CTA's rows with carry-in s.  For kind 0 the
// exclusive prefix sum P_r is handed to `alpha_rows` instead.
__device__ void cta_apply(const PfArgs& pa, const Col& c, int64_t r0, int64_t r1, double s, double* ldst,
                          double* bdst, double inv_alpha0, int* failed) {
  for (int64_t sb = r0; sb < r1; sb += PF_SB) {
    Aff m = {1.0, 0.0};
    const int64_t base = sb + (int64_t)threadIdx.x * PF_Q;
#pragma unroll
    for (int t = 0; t < PF_Q; t++) {
      const int64_t r = base + t;
      if (r < r1) m = compose(row_map(c, phys(pa, r)), m);
    }
    Aff tot;
    const Aff pre = block_scan(m, &tot);
    double st = fma(pre.A, s, pre.C);
#pragma unroll
    for (int t = 0; t < PF_Q; t++) {
      const int64_t r = base + t;
      if (r >= r1) break;
      const int64_t i = phys(pa, r);
      const Aff mr = row_map(c, i);
      const double x = c.x[i];
      if (c.kind == 0) {
        // dpftrf: alpha_j = 1 / (1/alpha_0 - sum_{t<j} v_t^2)
        const double alpha = 1.0 / (inv_alpha0 - st);
        const double tmp = 1.0 - alpha * x * x;
        if (!(tmp > 0.0)) *failed = 1;
        const double l = sqrt(tmp);
        ldst[i] = l;
        bdst[i] = -alpha * x / l;
      } else if (c.kind == 1) {
        c.x[i] = (x - c.p[i] * st) / c.l[i];
      } else {
        c.x[i] = fma(c.l[i], x, c.p[i] * st);
      }
      st = fma(mr.A, st, mr.C);
    }
    s = fma(tot.A, s, tot.C);
  }
}

// Carry-in of CTA g for column j: the predecessors' aggregates applied in
// order to s = 0.
__device__ double carry_in(const PfArgs& pa, const double2* agg, int j) {
  double s = 0.0;
  for (int g = 0; g < (int)blockIdx.x; g++) {
    const double2 m = __ldcg(agg + (size_t)g * pa.agg_cols + j);
    s = fma(m.x, s, m.y);
  }
  return s;
}

// One scan step over `ncol` columns given by colf(j): aggregates, the
// grid-wide wait, carry-ins, application.  Returns false on a failed wait.
template <class ColF, class Apply>
__device__ bool scan_step(const PfArgs& pa, int& phase, int ncol, ColF colf, Apply apply) {
  const int64_t r0 = (int64_t)blockIdx.x * pa.chunk;
  const int64_t r1 = r0 + pa.chunk < pa.n ? r0 + pa.chunk : pa.n;
  double2* agg = pa.agg + (size_t)(phase & 1) * gridDim.x * pa.agg_cols;
  double2* mine = agg + (size_t)blockIdx.x * pa.agg_cols;
  __shared__ double carry[PF_THREADS];
  for (int j = 0; j < ncol; j++) {
    const Aff t = cta_aggregate(pa, colf(j), r0, r1);
    if (threadIdx.x == 0) __stcg(mine + j, make_double2(t.A, t.C));
  }
  if (!grid_wait(pa.ctl, phase)) return false;
  phase++;
  for (int j0 = 0; j0 < ncol; j0 += PF_THREADS) {
    if (j0 + (int)threadIdx.x < ncol) carry[threadIdx.x] = carry_in(pa, agg, j0 + threadIdx.x);
    __syncthreads();
    const int jn = ncol - j0 < PF_THREADS ? ncol - j0 : PF_THREADS;
    for (int j = 0; j < jn; j++) apply(colf(j0 + j), r0, r1, carry[j]);
    __syncthreads();
  }
  return true;
}

__global__ void __launch_bounds__(PF_THREADS) pf_kernel(PfArgs pa) {
  int phase = 0;
  if (pa.op == PF_OP_TRF) {
    __shared__ int failed;
    for (int i = 0; i < pa.k; i++) {
      double* v = pa.V + (size_t)i * pa.ldv;
      double* l = pa.L + (size_t)i * pa.ldl;
      double* b = pa.B + (size_t)i * pa.ldb;
      const double inv_alpha0 = 1.0 / (-pa.a[i]);
      if (threadIdx.x == 0) failed = 0;
      // alpha: prefix sums of v_i^2 -> l_i, b_i on this CTA's rows
      if (!scan_step(
              pa, phase, 1, [&](int) { return Col{0, v, nullptr, nullptr, nullptr}; },
              [&](const Col& c, int64_t r0, int64_t r1, double s) {
                int f = 0;
                cta_apply(pa, c, r0, r1, s, l, b, inv_alpha0, &f);
                if (f) failed = 1;
              }))
        return;
      __syncthreads();
      if (threadIdx.x == 0 && failed) atomicExch(&pa.ctl[C_INFO], -1);
      // the later columns solved with L_i (ddrsv 'N'); a failure anywhere
      // is visible to every CTA after the step's wait
      const int nlater = pa.k - 1 - i;
      bool stop = false;
      if (!scan_step(
              pa, phase, nlater,
              [&](int j) { return Col{1, pa.V + (size_t)(i + 1 + j) * pa.ldv, v, b, l}; },
              [&](const Col& c, int64_t r0, int64_t r1, double s) {
                if (*((volatile int*)&pa.ctl[C_INFO]) != 0) {
                  stop = true;
                  return;
                }
                cta_apply(pa, c, r0, r1, s, nullptr, nullptr, 0.0, nullptr);
              }))
        return;
      if (stop || *((volatile int*)&pa.ctl[C_INFO]) != 0) return;
    }
    return;
  }
  // dpfsv / dpfmv over the right-hand sides: factor order per op and trans
  const bool forward = (pa.op == PF_OP_SV) == (pa.trans == 0);
  const int kind = pa.op == PF_OP_SV ? 1 : 2;
  for (int s = 0; s < pa.k; s++) {
    const int i = forward ? s : pa.k - 1 - s;
    const double* v = pa.V + (size_t)i * pa.ldv;
    const double* l = pa.L + (size_t)i * pa.ldl;
    const double* b = pa.B + (size_t)i * pa.ldb;
    const double* p = pa.trans ? b : v;
    const double* q = pa.trans ? v : b;
    if (!scan_step(
            pa, phase, pa.ncols, [&](int j) { return Col{kind, pa.U + (size_t)j * pa.ldu, p, q, l}; },
            [&](const Col& c, int64_t r0, int64_t r1, double s0) {
              cta_apply(pa, c, r0, r1, s0, nullptr, nullptr, 0.0, nullptr);
            }))
      return;
  }
}

// Launch shape: one CTA per `chunk` rows, at most the resident capacity.
int pf_capacity(int* cap) {
  int dev = 0, nsm = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return set_error(-3, "no current CUDA device");
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return set_error(-3, "cannot query the device");
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pf_kernel, PF_THREADS, 0) != cudaSuccess || per_sm < 1)
    return set_error(-12, "product-form kernel cannot be resident");
  *cap = nsm * per_sm;
  return 0;
}

size_t pf_work_bytes(int cap, int64_t ncols) {
  return PF_CTL_BYTES + 2 * (size_t)cap * (size_t)(ncols > 0 ? ncols : 1) * sizeof(double2);
}

int pf_launch(PfArgs pa, int64_t ncols_agg, void* work, size_t work_bytes, void* stream) {
  if (pa.n < 0 || pa.k < 0 || ncols_agg < 0) return set_error(-1, "negative size");
  if (pa.n == 0 || pa.k == 0) return 0;
  if (ncols_agg > (1 << 24)) return set_error(-1, "too many columns");
  int cap = 0;
  int rc = pf_capacity(&cap);
  if (rc) return rc;
  const size_t need = pf_work_bytes(cap, ncols_agg);
  if (!work || work_bytes < need)
    return set_error(-4, "workspace too small: %zu bytes given, %zu needed", work_bytes, need);
  if (((uintptr_t)work & 255) != 0) return set_error(-4, "workspace must be 256-byte aligned");
  int64_t grid = (pa.n + 255) / 256;
  if (grid > cap) grid = cap;
  pa.chunk = (pa.n + grid - 1) / grid;
  grid = (pa.n + pa.chunk - 1) / pa.chunk;
  pa.ctl = (int*)work;
  pa.agg = (double2*)((char*)work + PF_CTL_BYTES);
  pa.agg_cols = (int)(ncols_agg > 0 ? ncols_agg : 1);
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaMemsetAsync(work, 0, PF_CTL_BYTES, s);
  if (e == cudaSuccess) {
    void* args[] = {&pa};
    e = cudaLaunchCooperativeKernel((const void*)pf_kernel, dim3((unsigned)grid), dim3(PF_THREADS), args, 0, s);
  }
  if (e != cudaSuccess) return set_error(-100 - (int)e, "product-form launch failed: %s", cudaGetErrorString(e));
  return 0;
}

}  // namespace
}  // namespace chb

using namespace chb;

extern "C" int chb_pf_workspace_size(int64_t n, int64_t ncols, size_t* bytes) {
  clear_error();
  if (!bytes) return set_error(-1, "null argument");
  if (n < 0 || ncols < 0) return set_error(-1, "negative size");
  int cap = 0;
  int rc = pf_capacity(&cap);
  if (rc) return rc;
  *bytes = pf_work_bytes(cap, ncols);
  return 0;
}

extern "C" int chb_pftrf(int64_t n, int64_t k, const double* a, double* V, int64_t ldv, double* L, int64_t ldl,
                         double* B, int64_t ldb, void* work, size_t work_bytes, void* stream) {
  clear_error();
  if (n > 0 && k > 0 && (!a || !V || !L || !B)) return set_error(-1, "null argument");
  if (ldv < (n > 1 ? n : 1) || ldl < (n > 1 ? n : 1) || ldb < (n > 1 ? n : 1))
    return set_error(-1, "leading dimensions must be at least max(1, n)");
  if (k > (1 << 24)) return set_error(-1, "k too large");
  PfArgs pa;
  std::memset(&pa, 0, sizeof(pa));
  pa.op = PF_OP_TRF;
  pa.n = n;
  pa.k = (int)k;
  pa.a = a;
  pa.V = V;
  pa.ldv = ldv;
  pa.L = L;
  pa.ldl = ldl;
  pa.B = B;
  pa.ldb = ldb;
  return pf_launch(pa, k, work, work_bytes, stream);
}

static int pf_apply(int op, int64_t n, int64_t k, char trans, const double* V, int64_t ldv, const double* L,
                    int64_t ldl, const double* B, int64_t ldb, double* U, int64_t ldu, int64_t nrhs, void* work,
                    size_t work_bytes, void* stream) {
  clear_error();
  if (trans != 'N' && trans != 'T') return set_error(-1, "trans must be 'N' or 'T'");
  if (n > 0 && k > 0 && nrhs > 0 && (!V || !L || !B || !U)) return set_error(-1, "null argument");
  const int64_t lmin = n > 1 ? n : 1;
  if (ldv < lmin || ldl < lmin || ldb < lmin || ldu < lmin)
    return set_error(-1, "leading dimensions must be at least max(1, n)");
  if (k > (1 << 24) || nrhs > (1 << 24)) return set_error(-1, "size too large");
  if (nrhs == 0) return 0;
  PfArgs pa;
  std::memset(&pa, 0, sizeof(pa));
  pa.op = op;
  pa.trans = trans == 'T';
  pa.n = n;
  pa.k = (int)k;
  pa.ncols = (int)nrhs;
  pa.V = const_cast<double*>(V);
  pa.ldv = ldv;
  pa.L = const_cast<double*>(L);
  pa.ldl = ldl;
  pa.B = const_cast<double*>(B);
  pa.ldb = ldb;
  pa.U = U;
  pa.ldu = ldu;
  return pf_launch(pa, nrhs, work, work_bytes, stream);
}

extern "C" int chb_pfsv(int64_t n, int64_t k, char trans, const double* V, int64_t ldv, const double* L,
                        int64_t ldl, const double* B, int64_t ldb, double* U, int64_t ldu, int64_t nrhs, void* work,
                        size_t work_bytes, void* stream) {
  return pf_apply(PF_OP_SV, n, k, trans, V, ldv, L, ldl, B, ldb, U, ldu, nrhs, work, work_bytes, stream);
}

extern "C" int chb_pfmv(int64_t n, int64_t k, char trans, const double* V, int64_t ldv, const double* L,
                        int64_t ldl, const double* B, int64_t ldb, double* U, int64_t ldu, int64_t nrhs, void* work,
                        size_t work_bytes, void* stream) {
  return pf_apply(PF_OP_MV, n, k, trans, V, ldv, L, ldl, B, ldb, U, ldu, nrhs, work, work_bytes, stream);
}

extern "C" int chb_pf_info(void* work, void* stream) {
  clear_error();
  if (!work) return set_error(-1, "null workspace");
  cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
  if (e != cudaSuccess) return set_error(-100 - (int)e, "product-form sweep failed: %s", cudaGetErrorString(e));
  int ctl[4];
  e = cudaMemcpy(ctl, work, sizeof(ctl), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return set_error(-3, "cannot read the product-form status");
  if (ctl[C_ERR]) return set_error(-30, "a grid-wide wait of the product-form kernel timed out");
  return ctl[C_INFO];
}
