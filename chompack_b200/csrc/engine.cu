// Persistent task-graph executor for the multifrontal sweeps (sm_100a).
//
// One kernel launch runs a whole sweep, in one of two schedules.  Static:
// each CTA (128 threads) claims the next task index in list order with an
// atomic counter, waits until the counters the task depends on reach their
// targets (bounded spin; on timeout the CTA records DE_TIMEOUT and leaves,
// so a planning error can never hang the GPU), executes the task, then
// publishes its counter with release semantics.  Dynamic: a finished task
// releases its waiters itself and keeps one of them; idle CTAs claim the
// others from a ready bitmap (bounded polling, same timeout rule).
//
// Dense FP64 tile arithmetic uses the double-precision tensor-core MMA
// (mma.sync m16n8k4 f64): a 64x64 C tile is split over 4 warps, 32x32 each.
// GEMM operand tiles are staged through a ring of shared-memory K chunks by
// cp.async; tiles produced by other CTAs in the same launch are read only
// after an acquire that ordered their writes before the read.  The other
// tasks read with L2-coherent loads (__ldcg).
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

// Publication of a counter: every caller runs it from one thread right
// after a __syncthreads(), and the release is cumulative, so the CTA's
// writes before the barrier are visible (gpu scope) before the increment
// without a separate fence (measured: cholesky 6.48 -> 6.38 ms at 40^3
// without the __threadfence() that preceded it).
__device__ __forceinline__ void red_release_add(int* p, int v) {
  asm volatile("red.release.gpu.global.add.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ int ld_volatile(const int* p) { return *((const volatile int*)p); }

__device__ __forceinline__ int ld_acquire_sys(const int* p) {
  int v;
  asm volatile("ld.acquire.sys.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Waits until the copy of incoming chunk j has raised its flag (the host
// stream copies the chunk, then the flag).  Bounded like every wait: on
// timeout DE_TIMEOUT is recorded and the sweep leaves.
__device__ void wait_arrival(const RunArgs& ra, int j) {
  if (j < 0 || j >= ra.nio_in) {
    atomicCAS(&ra.ctl[1], 0, DE_BAD_TASK);
    return;
  }
  int64_t spins = 0;
  unsigned ns = 64;
  while (ld_acquire_sys(ra.io_in + j) == 0) {
    if (++spins > ra.spin_limit) {
      atomicCAS(&ra.ctl[1], 0, DE_TIMEOUT);
      atomicAdd(&ra.ctl[3], 1);
      return;
    }
    if ((spins & 15) == 0 && ld_volatile(&ra.ctl[1]) != 0) return;
    __nanosleep(ns);
    if (ns < 1024) ns <<= 1;
  }
}

// Host-visible flag: the CTA's earlier writes (ordered by the caller's
// __syncthreads) become visible to the copy engines before the flag.
__device__ __forceinline__ void raise_io_flag(int* p) {
  __threadfence_system();
  asm volatile("st.release.sys.global.b32 [%0], %1;" ::"l"(p), "r"(1) : "memory");
}

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// ------------------------------------------------------ dynamic schedule
// Ready tasks are bits of a bitmap (64 tasks per word, bit = list position)
// with a summary bitmap of the nonzero words.  ctl[5] is the finished
// frontier: every task in the words below it has finished, so no ready bit
// can appear there again; ctl[4] counts finished tasks.
//
// A finished task decrements the pending counts of its waiters (one lane of
// warp 0 per waiter, acq_rel).  Of the waiters it makes ready, the CTA keeps
// the one of lowest list position and runs it next, so a chain of dependent
// tasks never passes through the bitmap; the others are published with a
// release OR into the bitmap and claimed by idle CTAs with an acquire AND.
//
// Summary invariant: a word that turns nonzero has its summary bit set after
// it; a claimer that clears a summary bit re-reads the word after the clear
// and sets the bit again if the word is nonzero.  The fences between the word
// and summary accesses on both sides keep a nonzero word from ever losing its
// summary bit.
__device__ __forceinline__ int atom_add_acq_rel(int* p, int v) {
  int old;
  asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

__device__ __forceinline__ void red_or_release(unsigned long long* p, unsigned long long v) {
  asm volatile("red.release.gpu.global.or.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ unsigned long long atom_and_acquire(unsigned long long* p, unsigned long long v) {
  unsigned long long old;
  asm volatile("atom.acquire.gpu.global.and.b64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
  return old;
}

__device__ __forceinline__ unsigned long long atom_and_acq_rel(unsigned long long* p, unsigned long long v) {
  unsigned long long old;
  asm volatile("atom.acq_rel.gpu.global.and.b64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
  return old;
}

// Publishes ready task s: its bit (release: the waiter's inputs are visible
// to whoever acquires the bit), then its word's summary bit (release: after
// the word).  Neither waits for a reply.
__device__ __forceinline__ void publish_ready(const RunArgs& ra, int s) {
  red_or_release(ra.ready + (s >> 6), 1ull << (s & 63));
  red_or_release(ra.summ + (s >> 12), 1ull << ((s >> 6) & 63));
}

// Clears the summary bit of a word seen empty.  The acq_rel AND reads the
// summary after any publish that set the bit, so the word re-read below
// shows that publish's task (unless it was claimed since).
__device__ __forceinline__ void clear_summary(const RunArgs& ra, int wi) {
  const unsigned long long bit = 1ull << (wi & 63);
  atom_and_acq_rel(ra.summ + (wi >> 6), ~bit);
  if (ld_relaxed_u64(ra.ready + wi) != 0) red_or_release(ra.summ + (wi >> 6), bit);
}

__device__ __forceinline__ void cp_async4(void* smem_dst, const void* gmem_src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(gmem_src) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Releases the waiters listed in succ[b, e) (warp 0); the first 32 come
// from pre (shared memory) when it is given.  With handoff, the released
// waiter of lowest list position (below *next, the earlier candidate)
// becomes *next and is not published; the displaced candidate is.
__device__ __forceinline__ void release_list(const RunArgs& ra, int b, int e, const int* pre, bool handoff,
                                             int* next) {
  const int lane = threadIdx.x & 31;
  for (int i0 = b; i0 < e; i0 += 32) {
    int s = -1;
    if (i0 + lane < e) {
      s = (pre && i0 == b) ? pre[lane] : __ldg(ra.succ + i0 + lane);
      if (atom_add_acq_rel(ra.pend + s, -1) != 1) s = -1;
    }
    __syncwarp();  // orders every lane's acquire before the other lanes' publishes
    if (!handoff) {
      if (s >= 0) publish_ready(ra, s);
      continue;
    }
    int m = (s >= 0) ? s : 0x7fffffff;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = min(m, __shfl_xor_sync(0xffffffffu, m, o));
    const int prev = *next;
    const int keep = min(m, prev);
    if (s >= 0 && s != keep) publish_ready(ra, s);
    if (lane == 0 && prev != 0x7fffffff && prev != keep) publish_ready(ra, prev);
    *next = keep;
  }
}

// Advances the finished frontier over every word whose tasks have all
// finished.
__device__ __forceinline__ void advance_frontier(const RunArgs& ra) {
  __threadfence();
  int cur = ld_volatile(&ra.ctl[5]);
  while (cur < ra.nwords) {
    const int cnt = min(64, ra.ntasks - 64 * cur);
    if (ld_volatile(ra.wclaimed + cur) < cnt) break;
    const int prev = atomicCAS(&ra.ctl[5], cur, cur + 1);
    cur = (prev == cur) ? cur + 1 : prev;
  }
}

// Claims the word's set bit of rank (blockIdx.x mod its popcount), so that
// CTAs claiming at once spread over the word (lane 0).  Returns the task, or
// -1 when the word has emptied (then, for a word found through the summary,
// its summary bit is cleared).
__device__ __forceinline__ int claim_in_word(const RunArgs& ra, int wi, unsigned long long w, bool from_summary) {
  while (w) {
    const unsigned lo = (unsigned)w, hi = (unsigned)(w >> 32);
    const int plo = __popc(lo), r = (int)(blockIdx.x % (unsigned)(plo + __popc(hi)));
    const int pos = r < plo ? (int)__fns(lo, 0, r + 1) : 32 + (int)__fns(hi, 0, r - plo + 1);
    const unsigned long long bit = 1ull << pos;
    const unsigned long long old = atom_and_acquire(ra.ready + wi, ~bit);
    if (old & bit) return wi * 64 + pos;
    w = old;
  }
  if (from_summary) clear_summary(ra, wi);
  return -1;
}

// Claims a ready task for this CTA (warp 0; every lane returns it): first in
// the 32 bitmap words from the cached frontier *lo, then through the summary
// beyond them.  Returns ntasks when every task has finished, when a device
// error is set, or when nothing became ready within the spin limit
// (DE_TIMEOUT).
__device__ __forceinline__ int claim_task(const RunArgs& ra, int* lo) {
  const int lane = threadIdx.x & 31;
  int64_t spins = 0;
  unsigned ns = 64;
  for (;;) {
    const int wi = *lo + lane;
    const unsigned long long w = (wi < ra.nwords) ? ld_relaxed_u64(ra.ready + wi) : 0ull;
    int stop = 0, front = 0;
    if (lane == 0) {
      stop = ld_volatile(&ra.ctl[4]) >= ra.ntasks || ld_volatile(&ra.ctl[1]) != 0;
      front = ld_volatile(&ra.ctl[5]);
    }
    if (__shfl_sync(0xffffffffu, stop, 0)) return ra.ntasks;
    front = __shfl_sync(0xffffffffu, front, 0);
    unsigned bal = __ballot_sync(0xffffffffu, w != 0);
    while (bal) {
      const int src = __ffs(bal) - 1;
      bal &= bal - 1;
      const unsigned long long ww = __shfl_sync(0xffffffffu, w, src);
      int got = -1;
      if (lane == 0) got = claim_in_word(ra, *lo + src, ww, false);
      got = __shfl_sync(0xffffffffu, got, 0);
      if (got >= 0) return got;
    }
    if (front > *lo) {
      *lo = front;
      continue;
    }
    // beyond the window: summary words from the one holding word *lo + 32
    const int first = *lo + 32;
    for (int s0 = first >> 6; s0 < ra.nsumm; s0 += 32) {
      unsigned long long sw = (s0 + lane < ra.nsumm) ? ld_relaxed_u64(ra.summ + s0 + lane) : 0ull;
      if (s0 + lane == (first >> 6)) sw &= ~0ull << (first & 63);
      unsigned sb = __ballot_sync(0xffffffffu, sw != 0);
      while (sb) {
        const int src = __ffs(sb) - 1;
        sb &= sb - 1;
        unsigned long long bits = __shfl_sync(0xffffffffu, sw, src);
        int got = -1;
        if (lane == 0) {
          while (bits && got < 0) {
            const int wj = (s0 + src) * 64 + __ffsll((long long)bits) - 1;
            bits &= bits - 1;
            got = claim_in_word(ra, wj, ld_relaxed_u64(ra.ready + wj), true);
          }
        }
        got = __shfl_sync(0xffffffffu, got, 0);
        if (got >= 0) return got;
      }
    }
    if (++spins > ra.spin_limit) {
      if (lane == 0) {
        atomicCAS(&ra.ctl[1], 0, DE_TIMEOUT);
        atomicAdd(&ra.ctl[3], 1);
      }
      return ra.ntasks;
    }
    __nanosleep(ns);
    if (ns < 512) ns <<= 1;
  }
}

// After task ti (warp 0, the CTA's writes ordered before by __syncthreads):
// releases the waiters of the task (the first 32 prefetched into pre;
// already done mid task by a split task: own_released) and,
// when the task completes its group, of the group; counts the task into its
// bitmap word's finished tasks and the finished count.  Returns the released
// waiter this CTA runs next, or -1 (also when a device error is set).
__device__ __forceinline__ int finish_task(const RunArgs& ra, int ti, int group, int sb, int se, const int* pre,
                                           bool own_released) {
  const int lane = threadIdx.x & 31;
  int next = 0x7fffffff;
  int gdone = 0, filled = 0, err = 0;
  if (lane == 0 && group >= 0) gdone = atom_add_acq_rel(ra.counters + group, 1) + 1 == __ldg(ra.ctarget + group);
  if (lane == 1) filled = atomicAdd(ra.wclaimed + (ti >> 6), 1) + 1 == min(64, ra.ntasks - (ti & ~63));
  if (lane == 2) err = ld_volatile(&ra.ctl[1]);
  if (lane == 3) red_release_add(ra.counters + ti, 1);  // for the mid waits of split tasks
  cp_async_wait_all();
  if (!own_released) release_list(ra, sb, se, pre, true, &next);
  if (__shfl_sync(0xffffffffu, gdone, 0))
    release_list(ra, __ldg(ra.succ_off + group), __ldg(ra.succ_off + group + 1), nullptr, true, &next);
  if (lane == 1 && filled) advance_frontier(ra);
  if (lane == 0) red_release_add(&ra.ctl[4], 1);
  if (__shfl_sync(0xffffffffu, err, 2) != 0 && next != 0x7fffffff) {
    if (lane == 0) publish_ready(ra, next);  // left for the exit path; nothing runs after an error
    next = 0x7fffffff;
  }
  return next == 0x7fffffff ? -1 : next;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned sm_id() {
  unsigned r;
  asm volatile("mov.u32 %0, %%smid;" : "=r"(r));
  return r;
}

// ------------------------------------------------------------- operands
struct SmemLayout {
  double* A;   // [TILE][LDS]: A(r, k) stored at A[k*LDS + r]
  double* B;   // [TILE][LDS]
};

constexpr int PER_THREAD = (TILE * KC) / NTHREADS;  // staged elements per thread

// Address of element (r, k) of an operand; ok is cleared outside the
// triangle of OM_TRI_* operands (the caller sets it from the bounds).
template <int MODE>
__device__ __forceinline__ const double* op_addr(const double* X, int ld, int diag, int koff, int r, int k, bool& ok) {
  if (MODE == OM_N) return X + (int64_t)k * ld + r;
  if (MODE == OM_T) return X + (int64_t)r * ld + k;
  if (MODE == OM_TRI_N) {
    ok = ok && r + diag >= k;
    return X + (int64_t)k * ld + r;
  }
  if (MODE == OM_TRI_T) {
    ok = ok && k + diag >= r;
    return X + (int64_t)r * ld + k;
  }
  // OM_SYM: element (r + diag, k + koff) of a symmetric matrix stored lower
  const int gr = r + diag, gc = k + koff;
  return gr >= gc ? X + (int64_t)gc * ld + gr : X + (int64_t)gr * ld + gc;
}

// 8-byte asynchronous copy global -> shared; zeros when !ok (nothing is read).
// Tiles written by other CTAs of the launch are read only after an acquire
// that ordered their writes before this copy, so the L1-allocating form
// sees them.
__device__ __forceinline__ void cp_async8_zfill(double* dst, const double* src, bool ok) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(ok ? 8 : 0) : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Coordinates of the s-th staged element of this thread.  Operands read
// along k (OM_T, OM_TRI_T) give consecutive threads consecutive k so that
// global reads stay coalesced; the others give consecutive threads
// consecutive rows.
template <int MODE>
__device__ __forceinline__ void stage_coord(int s, int& r, int& kk) {
  const int idx = threadIdx.x + s * NTHREADS;
  if (MODE == OM_T || MODE == OM_TRI_T) {
    kk = idx % KC;
    r = idx / KC;
  } else {
    r = idx % TILE;
    kk = idx / TILE;
  }
}

// Issues the copies of the operand's K chunk [k0, k0 + KC) into a stage:
// S[kk*LDS + r] = op(r, k0 + kk), zero outside [0,rows) x [0,K).  For the
// plain and triangular modes a thread's elements lie at fixed strides from
// one base pointer (the coordinates of stage_coord with the thread count a
// multiple of TILE and of KC), which saves the per-element address
// arithmetic.
static_assert(NTHREADS % TILE == 0 && NTHREADS % KC == 0, "stage coordinates assume whole rows / columns");
template <int MODE>
__device__ __forceinline__ void issue_chunk_t(const double* __restrict__ X, int ld, int diag, int koff, int rows,
                                              int k0, int K, double* S) {
  const int tid = threadIdx.x;
  if (MODE == OM_N || MODE == OM_TRI_N) {
    constexpr int KSTEP = NTHREADS / TILE;  // k rows per element step
    const int r = tid % TILE, kb = tid / TILE;
    const double* p = X + (int64_t)(k0 + kb) * ld + r;
#pragma unroll
    for (int s = 0; s < PER_THREAD; s++) {
      const int kk = kb + KSTEP * s, k = k0 + kk;
      const bool ok = r < rows && k < K && (MODE == OM_N || r + diag >= k);
      cp_async8_zfill(S + kk * LDS + r, ok ? p + (int64_t)(KSTEP * s) * ld : X, ok);
    }
  } else if (MODE == OM_T || MODE == OM_TRI_T) {
    constexpr int RSTEP = NTHREADS / KC;  // rows per element step
    const int kk = tid % KC, rb = tid / KC, k = k0 + kk;
    const double* p = X + (int64_t)rb * ld + k;
#pragma unroll
    for (int s = 0; s < PER_THREAD; s++) {
      const int r = rb + RSTEP * s;
      const bool ok = r < rows && k < K && (MODE == OM_T || k + diag >= r);
      cp_async8_zfill(S + kk * LDS + r, ok ? p + (int64_t)(RSTEP * s) * ld : X, ok);
    }
  } else {
#pragma unroll
    for (int s = 0; s < PER_THREAD; s++) {
      int r, kk;
      stage_coord<MODE>(s, r, kk);
      const int k = k0 + kk;
      bool ok = r < rows && k < K;
      const double* src = op_addr<MODE>(X, ld, diag, koff, r, k, ok);
      cp_async8_zfill(S + kk * LDS + r, ok ? src : X, ok);
    }
  }
}

// Operand held in registers for the duration of a task.
struct Opnd {
  const double* X;
  int ld, diag, koff, mode;
};

__device__ __forceinline__ Opnd make_opnd(const RunArgs& ra, const Operand& o) {
  Opnd p;
  p.X = ra.bases[o.base] + o.off;
  p.ld = o.ld;
  p.diag = o.diag;
  p.koff = o.pad2;
  p.mode = o.mode;
  return p;
}

__device__ __forceinline__ void issue_chunk(const Opnd& o, int rows, int k0, int K, double* S) {
  switch (o.mode) {
    case OM_N: issue_chunk_t<OM_N>(o.X, o.ld, o.diag, o.koff, rows, k0, K, S); break;
    case OM_T: issue_chunk_t<OM_T>(o.X, o.ld, o.diag, o.koff, rows, k0, K, S); break;
    case OM_TRI_N: issue_chunk_t<OM_TRI_N>(o.X, o.ld, o.diag, o.koff, rows, k0, K, S); break;
    case OM_TRI_T: issue_chunk_t<OM_TRI_T>(o.X, o.ld, o.diag, o.koff, rows, k0, K, S); break;
    default: issue_chunk_t<OM_SYM>(o.X, o.ld, o.diag, o.koff, rows, k0, K, S); break;
  }
}

// Double-precision tensor-core MMA, m16n8k4 (sm_90+):
//   A 16x4 row-major: a0 = A(g, q), a1 = A(g + 8, q)
//   B 4x8 col-major:  b0 = B(q, g)
//   C 16x8:           c0,c1 = C(g, 2q + {0,1}), c2,c3 = C(g + 8, 2q + {0,1})
// with g = lane / 4, q = lane % 4.  A warp owns a 32x32 C sub-tile: two m16
// rows x four n8 columns.
__device__ __forceinline__ void dmma16(double (&c)[4], double a0, double a1, double b) {
  asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
               : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
               : "d"(a0), "d"(a1), "d"(b));
}

// Accumulator layout: acc[i][j][h] with i in 0..1 (m16 tile), j in 0..3 (n8
// tile), h in 0..3 (c0..c3).
typedef double Acc[2][4][4];

// Tile coordinates of acc[i][j][h] inside the 64x64 C tile.
__device__ __forceinline__ void acc_coord(int i, int j, int h, int& r, int& c) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, q = lane & 3;
  r = (warp >> 1) * 32 + 16 * i + g + ((h & 2) ? 8 : 0);
  c = (warp & 1) * 32 + 8 * j + 2 * q + (h & 1);
}

// acc += A(:, 0:kn) * B(:, 0:kn)^T from tiles in shared memory, A(r, k) at
// sA[k*LA + r] and B(c, k) at sB[k*LB + c] (kn multiple of 4).
template <int LA, int LB>
__device__ __forceinline__ void mma_block_ld(const double* sA, const double* sB, int kn, Acc& acc) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, q = lane & 3;
  const int r0 = (warp >> 1) * 32 + g, c0 = (warp & 1) * 32 + g;
#pragma unroll 4
  for (int kk = 0; kk < kn; kk += 4) {
    double a[2][2], b[4];
    const double* ak = sA + (kk + q) * LA + r0;
    const double* bk = sB + (kk + q) * LB + c0;
#pragma unroll
    for (int i = 0; i < 2; i++) {
      a[i][0] = ak[16 * i];
      a[i][1] = ak[16 * i + 8];
    }
#pragma unroll
    for (int j = 0; j < 4; j++) b[j] = bk[8 * j];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) dmma16(acc[i][j], a[i][0], a[i][1], b[j]);
  }
}

// The GEMM stages (leading dimension LDS).
__device__ __forceinline__ void mma_block(const double* sA, const double* sB, int kn, Acc& acc) {
  mma_block_ld<LDS, LDS>(sA, sB, kn, acc);
}

// The m16 and n8 tiles of the calling warp's 32x32 sub-tile that meet an
// m x n product (warp-uniform): mi in 0..2, nj in 0..4.
__device__ __forceinline__ void warp_tiles(int m, int n, int& mi, int& nj) {
  const int warp = threadIdx.x >> 5;
  const int r = m - (warp >> 1) * 32, c = n - (warp & 1) * 32;
  mi = r <= 0 ? 0 : (r >= 32 ? 2 : (r + 15) >> 4);
  nj = c <= 0 ? 0 : (c >= 32 ? 4 : (c + 7) >> 3);
}

// mma_block for a partial tile: only the warp's first mi m16 and nj n8
// tiles are multiplied (the others hold rows or columns outside the
// product, which the epilogue does not store).  A narrow product (a few
// right-hand sides, the edge tiles of a front) then issues a fraction of
// the MMAs of a full 64x64 tile.
__device__ __forceinline__ void mma_block_part(const double* sA, const double* sB, int kn, Acc& acc, int mi,
                                               int nj) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, q = lane & 3;
  const int r0 = (warp >> 1) * 32 + g, c0 = (warp & 1) * 32 + g;
#pragma unroll 2
  for (int kk = 0; kk < kn; kk += 4) {
    double a[2][2], b[4];
    const double* ak = sA + (kk + q) * LDS + r0;
    const double* bk = sB + (kk + q) * LDS + c0;
#pragma unroll
    for (int i = 0; i < 2; i++) {
      a[i][0] = i < mi ? ak[16 * i] : 0.0;
      a[i][1] = i < mi ? ak[16 * i + 8] : 0.0;
    }
#pragma unroll
    for (int j = 0; j < 4; j++) b[j] = j < nj ? bk[8 * j] : 0.0;
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 4; j++)
        if (i < mi && j < nj) dmma16(acc[i][j], a[i][0], a[i][1], b[j]);
  }
}

__device__ __forceinline__ void zero_acc(Acc& acc) {
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int h = 0; h < 4; h++) acc[i][j][h] = 0.0;
}

// ------------------------------------------------------------ TF32 path
__device__ __forceinline__ uint32_t to_tf32(float f) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(f));
  return r;
}

// TF32 MMA m16n8k8 with FP32 accumulation:
//   A 16x8 row-major: a0 = A(g, q), a1 = A(g+8, q), a2 = A(g, q+4), a3 = A(g+8, q+4)
//   B 8x8 col-major:  b0 = B(q, g), b1 = B(q+4, g)
//   C 16x8: as the FP64 MMA (c0,c1 row g, c2,c3 row g+8; columns 2q, 2q+1)
__device__ __forceinline__ void mma_tf32(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
               : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
               : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

typedef float AccF[2][4][4];

// High and low TF32 parts of an FP64 value (x ~ hi + lo to about 22 bits).
__device__ __forceinline__ void split_tf32(double x, uint32_t& hi, uint32_t& lo) {
  const float f = (float)x;
  hi = to_tf32(f);
  lo = to_tf32((float)(x - (double)__uint_as_float(hi)));
}

// accf += A(:, 0:kn) B(:, 0:kn)^T from FP64 stages (kn a multiple of 8; the
// stage is zero past K).  X3: three products (hi*hi + hi*lo + lo*hi).
template <bool X3>
__device__ __forceinline__ void mma_block_tf32(const double* sA, const double* sB, int kn, AccF& acc) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, q = lane & 3;
  const int r0 = (warp >> 1) * 32 + g, c0 = (warp & 1) * 32 + g;
#pragma unroll 2
  for (int kk = 0; kk < kn; kk += 8) {
    uint32_t ah[2][4], al[2][4], bh[4][2], bl[4][2];
    const double* ak0 = sA + (kk + q) * LDS + r0;
    const double* ak4 = sA + (kk + q + 4) * LDS + r0;
    const double* bk0 = sB + (kk + q) * LDS + c0;
    const double* bk4 = sB + (kk + q + 4) * LDS + c0;
#pragma unroll
    for (int i = 0; i < 2; i++) {
      const double v[4] = {ak0[16 * i], ak0[16 * i + 8], ak4[16 * i], ak4[16 * i + 8]};
#pragma unroll
      for (int e = 0; e < 4; e++) {
        if (X3) split_tf32(v[e], ah[i][e], al[i][e]);
        else ah[i][e] = to_tf32((float)v[e]);
      }
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const double v0 = bk0[8 * j], v1 = bk4[8 * j];
      if (X3) {
        split_tf32(v0, bh[j][0], bl[j][0]);
        split_tf32(v1, bh[j][1], bl[j][1]);
      } else {
        bh[j][0] = to_tf32((float)v0);
        bh[j][1] = to_tf32((float)v1);
      }
    }
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) {
        if (X3) {
          mma_tf32(acc[i][j], al[i], bh[j][0], bh[j][1]);
          mma_tf32(acc[i][j], ah[i], bl[j][0], bl[j][1]);
        }
        mma_tf32(acc[i][j], ah[i], bh[j][0], bh[j][1]);
      }
  }
}

// acc = opA * opB^T over K through a GEMM_STAGES-deep ring of K chunks in
// shared memory: the copies of chunk c + GEMM_STAGES - 1 are in flight while
// chunk c is multiplied; one barrier per chunk.
constexpr int GEMM_STAGES = 4;
constexpr int STAGE_DOUBLES = 2 * KC * LDS;  // A chunk, then B chunk

template <int PREC>
__device__ void gemm_acc_p(const Opnd& A, const Opnd& B, int m, int n, int K, const SmemLayout& sm, Acc& acc) {
  AccF accf;
  if (PREC != PREC_FP64) {
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 4; j++)
#pragma unroll
        for (int h = 0; h < 4; h++) accf[i][j][h] = 0.f;
  }
  zero_acc(acc);
  const int nch = (K + KC - 1) / KC;
  double* const ring = sm.A;
  int wmi, wnj;
  warp_tiles(m, n, wmi, wnj);
  const bool full = wmi == 2 && wnj == 4;
#pragma unroll
  for (int c = 0; c < GEMM_STAGES - 1; c++) {
    if (c < nch) {
      issue_chunk(A, m, c * KC, K, ring + c * STAGE_DOUBLES);
      issue_chunk(B, n, c * KC, K, ring + c * STAGE_DOUBLES + KC * LDS);
    }
    cp_async_commit();
  }
  for (int c = 0; c < nch; c++) {
    cp_async_wait_group<GEMM_STAGES - 2>();  // this thread's copies of chunk c
    __syncthreads();                         // everyone's; and chunk c - 1 is consumed
    const int cn = c + GEMM_STAGES - 1;
    if (cn < nch) {
      double* d = ring + (cn % GEMM_STAGES) * STAGE_DOUBLES;
      issue_chunk(A, m, cn * KC, K, d);
      issue_chunk(B, n, cn * KC, K, d + KC * LDS);
    }
    cp_async_commit();
    const double* st = ring + (c % GEMM_STAGES) * STAGE_DOUBLES;
    int kn = min(KC, K - c * KC);
    if (PREC == PREC_FP64) {
      kn = (kn + 3) & ~3;
      if (full) mma_block(st, st + KC * LDS, kn, acc);
      else if (wmi > 0 && wnj > 0) mma_block_part(st, st + KC * LDS, kn, acc, wmi, wnj);
    } else {
      kn = (kn + 7) & ~7;
      mma_block_tf32<PREC == PREC_TF32X3>(st, st + KC * LDS, kn, accf);
    }
  }
  cp_async_wait_group<0>();
  __syncthreads();
  if (PREC != PREC_FP64) {
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 4; j++)
#pragma unroll
        for (int h = 0; h < 4; h++) acc[i][j][h] = (double)accf[i][j][h];
  }
}

// ------------------------------------------------------ tcgen05 TF32 tiles
// TF32 GEMM tiles of the mixed-precision sweeps on the fifth-generation
// tensor cores: tcgen05.mma.cta_group::1.kind::tf32 with M = N = 64 and
// K = 8 per instruction, FP32 accumulators in tensor memory (64 columns per
// CTA, allocated once per launch when the program has such tiles).  K goes
// through the FP64 cp.async ring as for the other tiles (three stages here);
// per chunk of KC = 16 the 128 threads round the stage to TF32 (cvt.rna, as
// the mma.sync tiles do) into one of two shared-memory buffers in the
// canonical K-major layout without swizzle: core matrices of 8 rows x 16
// bytes, element (r, k) of the chunk at byte ((r/8)*4 + k/4)*128 + (r%8)*16 +
// (k%4)*4, so the next 4 columns start 128 bytes on (leading byte offset) and
// the next 8 rows 512 bytes on (stride byte offset).  One thread issues the
// chunk's two MMAs and commits them to the buffer's mbarrier; a buffer is
// refilled once its last commit has arrived.  The epilogue reads the
// accumulator with tcgen05.ld (for M = 64, row 16w + i lives in TMEM lane
// 32w + i, so warp w reads its own sub-partition's lanes 0..15) and adds
// alpha*acc + beta*C in FP64.
constexpr int TC_STAGES = 3;                       // FP64 ring stages of a tcgen05 tile
constexpr int TC_STAGE_FLOATS = 2 * TILE * KC;     // A then B of one chunk, TF32
// instruction descriptor: F32 accumulator (bits 4-5 = 1), A and B TF32
// (bits 7-9, 10-12 = 2), both K-major, N >> 3 (bits 17-22), M >> 4 (bits 24-28)
constexpr uint32_t TC_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TILE >> 3) << 17) |
                              ((uint32_t)(TILE >> 4) << 24);
static_assert(TC_STAGES * STAGE_DOUBLES * 8 + 2 * TC_STAGE_FLOATS * 4 <= ENGINE_SMEM_BASE_DOUBLES * 8,
              "tcgen05 staging exceeds the engine's shared memory");

struct TcState {
  uint32_t tmem;        // accumulator: TMEM lane 0, first allocated column
  uint64_t* mbar;       // two mbarriers in shared memory
  uint32_t ncommit[2];  // commits issued to each mbarrier (same in every thread)
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: start address >> 4 (bits 0-13), leading
// byte offset 128 >> 4 (bits 16-29), stride byte offset 512 >> 4 (bits
// 32-45), descriptor version 1 (bits 46-47), no swizzle (bits 61-63 = 0)
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) | ((uint64_t)(512u >> 4) << 32) |
         (1ull << 46);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
      "l"(adesc), "l"(bdesc), "r"(TC_IDESC), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void tc_commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_init(uint64_t* m) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(m)) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* m, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(m)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the completion of the phase with the given parity (an
// MMA chunk takes well under a microsecond; each try_wait may suspend the
// thread for a while, so the bound is time, 2 s); a wait that runs out
// records DE_TIMEOUT and returns false.
__device__ bool mbar_wait(const RunArgs& ra, uint64_t* m, uint32_t parity) {
  if (mbar_test(m, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_test(m, parity)) {
    if (global_ns() - t0 > 2000000000ull) {
      atomicCAS(&ra.ctl[1], 0, DE_TIMEOUT);
      return false;
    }
  }
  return true;
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// One FP64 stage (A(r, k) at st[k*LDS + r], B at st + KC*LDS) rounded to
// TF32 into a staging buffer in the canonical K-major layout; each thread
// writes 16-byte rows of core matrices.
__device__ __forceinline__ void tc_stage(const double* st, float* S) {
#pragma unroll
  for (int it = 0; it < 4; it++) {
    const int idx = threadIdx.x + it * NTHREADS;  // (operand, 4-column group, row)
    const int op = idx >> 8, q = (idx >> 6) & 3, r = idx & 63;
    const double* src = st + op * KC * LDS + 4 * q * LDS + r;
    float4 v;
    v.x = __uint_as_float(to_tf32((float)src[0]));
    v.y = __uint_as_float(to_tf32((float)src[LDS]));
    v.z = __uint_as_float(to_tf32((float)src[2 * LDS]));
    v.w = __uint_as_float(to_tf32((float)src[3 * LDS]));
    *reinterpret_cast<float4*>(S + op * TILE * KC + ((r >> 3) * 4 + q) * 32 + (r & 7) * 4) = v;
  }
}

// C = alpha * opA * opB^T + beta * C for an m x n tile (masked to r + cdiag
// >= c when lower) with TF32 products on tcgen05 and FP32 accumulation.
__device__ void gemm_tc_tf32(const RunArgs& ra, const Opnd& A, const Opnd& B, int m, int n, int K,
                             const SmemLayout& sm, TcState& ts, double* __restrict__ C, int ldc, bool lower,
                             int cdiag, double alpha, double beta) {
  const int nch = (K + KC - 1) / KC;
  double* const ring = sm.A;
  float* const stg = reinterpret_cast<float*>(ring + TC_STAGES * STAGE_DOUBLES);
#pragma unroll
  for (int c = 0; c < TC_STAGES - 1; c++) {
    if (c < nch) {
      issue_chunk(A, m, c * KC, K, ring + c * STAGE_DOUBLES);
      issue_chunk(B, n, c * KC, K, ring + c * STAGE_DOUBLES + KC * LDS);
    }
    cp_async_commit();
  }
  for (int c = 0; c < nch; c++) {
    cp_async_wait_group<TC_STAGES - 2>();  // this thread's copies of chunk c
    __syncthreads();                       // everyone's; and chunk c - 1 is converted
    const int cn = c + TC_STAGES - 1;
    if (cn < nch) {
      double* d = ring + (cn % TC_STAGES) * STAGE_DOUBLES;
      issue_chunk(A, m, cn * KC, K, d);
      issue_chunk(B, n, cn * KC, K, d + KC * LDS);
    }
    cp_async_commit();
    const int buf = c & 1;
    if (c >= 2) mbar_wait(ra, ts.mbar + buf, (ts.ncommit[buf] - 1) & 1);  // chunk c - 2 has read it
    float* S = stg + buf * TC_STAGE_FLOATS;
    tc_stage(ring + (c % TC_STAGES) * STAGE_DOUBLES, S);
    fence_proxy_async();
    __syncthreads();
    if (threadIdx.x == 0) {
      tc_fence_after();
      const uint32_t sa = smem_u32(S), sb = smem_u32(S + TILE * KC);
      tc_mma(ts.tmem, tc_desc(sa), tc_desc(sb), c > 0 ? 1u : 0u);
      tc_mma(ts.tmem, tc_desc(sa + 256), tc_desc(sb + 256), 1u);
      tc_commit(ts.mbar + buf);
    }
    ts.ncommit[buf]++;
  }
  cp_async_wait_group<0>();
  // the last commit covers every MMA of the tile
  const int lb = (nch - 1) & 1;
  mbar_wait(ra, ts.mbar + lb, (ts.ncommit[lb] - 1) & 1);
  tc_fence_after();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r = warp * 16 + lane;
  const uint32_t taddr = ts.tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
  for (int c0 = 0; c0 < TILE; c0 += 16) {
    uint32_t v[16];
    tmem_ld16(taddr + c0, v);
    if (lane < 16 && r < m) {
      double old[16];
#pragma unroll
      for (int j = 0; j < 16; j++) {
        const int c = c0 + j;
        const bool ok = c < n && !(lower && r + cdiag < c);
        old[j] = (beta != 0.0 && ok) ? __ldcg(C + (int64_t)c * ldc + r) : 0.0;
      }
#pragma unroll
      for (int j = 0; j < 16; j++) {
        const int c = c0 + j;
        if (c >= n || (lower && r + cdiag < c)) continue;
        double x = alpha * (double)__uint_as_float(v[j]);
        if (beta != 0.0) x += beta * old[j];
        C[(int64_t)c * ldc + r] = x;
      }
    }
  }
  tc_fence_before();
  __syncthreads();
}

__device__ __forceinline__ void gemm_acc(const Opnd& A, const Opnd& B, int m, int n, int K, const SmemLayout& sm,
                                         Acc& acc) {
  gemm_acc_p<PREC_FP64>(A, B, m, n, K, sm, acc);
}

// C = alpha*acc + beta*C (masked to m x n and, for lower, to r + cdiag >= c).
// All old values are fetched before the first store so that the loads are
// in flight together (the compiler cannot reorder them across stores to C).
// C += alpha acc with atomic adds (CM_ATOMIC).
__device__ void store_acc_atomic(double* __restrict__ C, int ldc, int m, int n, double alpha, const Acc& acc) {
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int h = 0; h < 4; h++) {
        int r, c;
        acc_coord(i, j, h, r, c);
        if (r < m && c < n) atomicAdd(C + (int64_t)c * ldc + r, alpha * acc[i][j][h]);
      }
}

__device__ void store_acc(double* __restrict__ C, int ldc, int m, int n, bool lower, int cdiag, double alpha,
                          double beta, const Acc& acc) {
  double old[2][4][4];
  if (beta != 0.0) {
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 4; j++)
#pragma unroll
        for (int h = 0; h < 4; h++) {
          int r, c;
          acc_coord(i, j, h, r, c);
          const bool ok = r < m && c < n && !(lower && r + cdiag < c);
          old[i][j][h] = ok ? __ldcg(C + (int64_t)c * ldc + r) : 0.0;
        }
  }
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int h = 0; h < 4; h++) {
        int r, c;
        acc_coord(i, j, h, r, c);
        if (r >= m || c >= n) continue;
        if (lower && r + cdiag < c) continue;
        double v = alpha * acc[i][j][h];
        if (beta != 0.0) v += beta * old[i][j][h];
        C[(int64_t)c * ldc + r] = v;
      }
}

// ------------------------------------------------------------------ GEMM
// GEMM task (T_GEMM), and the look-ahead step of the blocked Cholesky
// (T_LA) as two passes through the same code.  T_LA, with the next diagonal
// tile D (operand c, m x m, lower part), the tile A below the current
// diagonal block (operand a, m x n, overwritten) and M = L_cc^{-1} (operand
// b, read as lower-triangular):
//   pass 0: L = A M^T -> A;  early signal (aux[3] - 1, when aux[3] > 0)
//   pass 1: D -= L L^T (lower part), L read back from L2
// Both passes share one inlined copy of the GEMM code: a second copy (or a
// call) makes the persistent kernel spill.
template <bool TC>
__device__ void run_gemm_or_la(const RunArgs& ra, const Task& t, const SmemLayout& sm, TcState& ts) {
  const bool la = t.op == T_LA;
  const int passes = la ? 2 : 1;
  for (int ph = 0; ph < passes; ph++) {
    const Operand& ob = (la && ph == 1) ? t.a : t.b;
    const Operand& oc = (la && ph == 0) ? t.a : t.c;
    const Opnd A = make_opnd(ra, t.a), B = make_opnd(ra, ob);
    const int m = t.m, n = (la && ph == 1) ? t.m : t.n, K = (la && ph == 1) ? t.n : t.k;
    const bool lower = la ? ph == 1 : t.cmode == CM_LOWER;
    const int cdiag = la ? 0 : t.cdiag;
    const double alpha = la ? (ph == 0 ? 1.0 : -1.0) : t.alpha;
    const double beta = la ? (ph == 0 ? 0.0 : 1.0) : t.beta;
    if (TC && !la && t.c.prec == PREC_TF32) {
      gemm_tc_tf32(ra, A, B, m, n, K, sm, ts, ra.bases[oc.base] + oc.off, oc.ld, lower, cdiag, alpha, beta);
      continue;
    }
    Acc acc;
    if (la || t.c.prec == PREC_FP64) gemm_acc_p<PREC_FP64>(A, B, m, n, K, sm, acc);
    else if (t.c.prec == PREC_TF32) gemm_acc_p<PREC_TF32>(A, B, m, n, K, sm, acc);
    else gemm_acc_p<PREC_TF32X3>(A, B, m, n, K, sm, acc);
    if (!la && t.cmode == CM_ATOMIC) store_acc_atomic(ra.bases[oc.base] + oc.off, oc.ld, m, n, alpha, acc);
    else store_acc(ra.bases[oc.base] + oc.off, oc.ld, m, n, lower, cdiag, alpha, beta, acc);
    if (la && ph == 0) {
      __syncthreads();
      if (t.aux[3] > 0) {
        if (ra.dynamic) {
          const int c = t.aux[3] - 1;
          if (threadIdx.x < 32)
            release_list(ra, __ldg(ra.succ_off + c), __ldg(ra.succ_off + c + 1), nullptr, false, nullptr);
        } else if (threadIdx.x == 0) {
          red_release_add(ra.counters + (t.aux[3] - 1), 1);
        }
      }
    }
  }
}

// Reduction of split-K partial products (T_SUM): C = alpha * sum_q P_q +
// beta * C over the m x n tile (masked to r + cdiag >= c when cmode is
// CM_LOWER), P_q at a.off + q * aux[1] (ld a.ld), q = 0 .. aux[0]-1 added in
// order, so the result does not depend on the schedule.
__device__ void run_sum(const RunArgs& ra, const Task& t) {
  const double* __restrict__ P = ra.bases[t.a.base] + t.a.off;
  double* __restrict__ C = ra.bases[t.c.base] + t.c.off;
  const int ldp = t.a.ld, ldc = t.c.ld, m = t.m, n = t.n, np = t.aux[0];
  const int64_t stride = (int64_t)(uint32_t)t.aux[1];
  const bool lower = t.cmode == CM_LOWER;
  constexpr int NQ = 4;                            // quarters of the tile
  constexpr int E = TILE * TILE / NTHREADS / NQ;  // elements per thread and quarter
  constexpr int U = 4;                            // partials loaded together
  // a thread's elements of U partials are loaded together (up to U E loads
  // in flight), then added partial after partial in index order; quarters
  // keep the registers in check
#pragma unroll 1
  for (int qt = 0; qt < NQ; qt++) {
    if (qt * E * NTHREADS / TILE >= n) break;  // the quarter's columns start at or after n
    double acc[E];
#pragma unroll
    for (int e = 0; e < E; e++) acc[e] = 0.0;
    for (int q0 = 0; q0 < np; q0 += U) {
      double v[U][E];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const double* Pq = P + (q0 + u) * stride;
#pragma unroll
        for (int e = 0; e < E; e++) {
          const int idx = threadIdx.x + (qt * E + e) * NTHREADS, r = idx % TILE, c = idx / TILE;
          v[u][e] = (q0 + u < np && r < m && c < n) ? __ldcg(Pq + (int64_t)c * ldp + r) : 0.0;
        }
      }
#pragma unroll
      for (int u = 0; u < U; u++)
#pragma unroll
        for (int e = 0; e < E; e++)
          if (q0 + u < np) acc[e] += v[u][e];
    }
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int idx = threadIdx.x + (qt * E + e) * NTHREADS, r = idx % TILE, c = idx / TILE;
      if (r >= m || c >= n || (lower && r + t.cdiag < c)) continue;
      double v = t.alpha * acc[e];
      if (t.beta != 0.0) v += t.beta * __ldcg(C + (int64_t)c * ldc + r);
      C[(int64_t)c * ldc + r] = v;
    }
  }
}

// C = alpha * M2 * (opA * opB^T), M2 = lower-triangular m x m tile (operand
// `c` of the task holds C; M2 is described by aux: base aux[0], ld aux[1],
// offset (aux[2] | aux[3] << 32)).
// One step of a block substitution (the triangular solves):
// C (m x n) = alpha A (m x K) B (K x n) + beta C, m <= 64, K <= TRSV_KMAX,
// with A a step operand computed before the sweep's chain ([-G_c | M_c] or
// [M_c; -H_c] stored transposed) and B adjacent x tiles, C one of them.
// A's copies into shared memory (sA[k*TRSV_LA + r], zero outside m x K) are
// issued before the task's mid waits [cdiag, nwait) (the x tiles it reads,
// written by the chain), so that they overlap the wait; then B is read in
// groups of 8 right-hand sides (sB[k*8 + j]) and each warp multiplies its
// 16 rows with FP64 MMAs.  A wait that runs out sets the timeout status
// and returns once the copies have landed.
__device__ void run_trsv(const RunArgs& ra, const Task& t, double* smem) {
  __shared__ int s_trsv_abort;
  constexpr int LA = TRSV_LA;
  double* sA = smem;
  double* sB = smem + TRSV_KMAX * LA;
  const int m = t.m, n = t.n, K = t.k, K4 = (K + 3) & ~3;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, q = lane & 3;
  {
    const double* __restrict__ X = ra.bases[t.a.base] + t.a.off;
    const int ld = t.a.ld;
    if (t.a.mode == OM_T) {
      // A(r, k) = X[r*ld + k]: consecutive threads take consecutive k
      for (int idx = tid; idx < TILE * K4; idx += NTHREADS) {
        const int k = idx % K4, r = idx / K4;
        const bool ok = r < m && k < K;
        cp_async8_zfill(sA + k * LA + r, ok ? X + (int64_t)r * ld + k : X, ok);
      }
    } else {
      for (int idx = tid; idx < TILE * K4; idx += NTHREADS) {
        const int r = idx % TILE, k = idx / TILE;
        const bool ok = r < m && k < K;
        cp_async8_zfill(sA + k * LA + r, ok ? X + (int64_t)k * ld + r : X, ok);
      }
    }
    cp_async_commit();
  }
  if (tid == 0) {
    int abort = 0;
    for (int w = t.cdiag; w < t.nwait && !abort; w++) {
      const int2 wt = ra.waits[t.wait_off + w];
      int64_t spins = 0;
      unsigned ns = 16;
      while (ld_acquire(ra.counters + wt.x) < wt.y) {
        if (++spins > ra.spin_limit) {
          atomicCAS(&ra.ctl[1], 0, DE_TIMEOUT);
          atomicAdd(&ra.ctl[3], 1);
          abort = 1;
          break;
        }
        if ((spins & 15) == 0 && ld_volatile(&ra.ctl[1]) != 0) { abort = 1; break; }
        __nanosleep(ns);
        if (ns < 128) ns <<= 1;
      }
    }
    s_trsv_abort = abort;
  }
  __syncthreads();
  if (s_trsv_abort) {
    cp_async_wait_all();
    return;
  }
  const double* __restrict__ Xb = ra.bases[t.b.base] + t.b.off;
  const int ldb = t.b.ld;  // B(j, k) = Xb[j*ldb + k] (x tiles, operand mode OM_T)
  double* __restrict__ C = ra.bases[t.c.base] + t.c.off;
  const int ldc = t.c.ld;
  for (int j0 = 0; j0 < n; j0 += 8) {
    const int nb = min(8, n - j0);
    for (int base = 0; base < K4 * 8; base += 4 * NTHREADS) {
      double v[4];
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int idx = base + tid + e * NTHREADS, k = idx % K4, j = idx / K4;
        v[e] = (idx < K4 * 8 && k < K && j < nb) ? __ldcg(Xb + (int64_t)(j0 + j) * ldb + k) : 0.0;
      }
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int idx = base + tid + e * NTHREADS, k = idx % K4, j = idx / K4;
        if (idx < K4 * 8) sB[k * 8 + j] = v[e];
      }
    }
    if (j0 == 0) cp_async_wait_all();
    __syncthreads();
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (16 * warp < m) {
      const double* ar = sA + 16 * warp + g;
#pragma unroll 4
      for (int k = 0; k < K4; k += 4) dmma16(acc, ar[(k + q) * LA], ar[(k + q) * LA + 8], sB[(k + q) * 8 + g]);
    }
#pragma unroll
    for (int h = 0; h < 4; h++) {
      const int r = 16 * warp + g + ((h & 2) ? 8 : 0), j = 2 * q + (h & 1);
      if (r < m && j < nb) {
        double* cp = C + (int64_t)(j0 + j) * ldc + r;
        double val = t.alpha * acc[h];
        if (t.beta != 0.0) val += t.beta * __ldcg(cp);
        *cp = val;
      }
    }
    __syncthreads();
  }
}

__device__ void run_mrow(const RunArgs& ra, const Task& t, const SmemLayout& sm) {
  const Opnd A = make_opnd(ra, t.a), B = make_opnd(ra, t.b);
  double* C = ra.bases[t.c.base] + t.c.off;
  const int ldc = t.c.ld, m = t.m, n = t.n, K = t.k;
  const double alpha = t.alpha;
  const int64_t moff = (int64_t)(uint32_t)t.aux[2] | ((int64_t)t.aux[3] << 32);
  const double* __restrict__ M2 = ra.bases[t.aux[0]] + moff;
  const int ldm = t.aux[1];
  Acc acc;
  gemm_acc(A, B, m, n, K, sm, acc);
  // T = acc (m x n) into sm.B in B-stage layout: sB[k*LDS + n] = T(k, n)
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int h = 0; h < 4; h++) {
        int r, c;
        acc_coord(i, j, h, r, c);
        sm.B[r * LDS + c] = acc[i][j][h];
      }
  // sA[k*LDS + r] = M2(r, k) (lower triangle, zero padded), 32 loads in
  // flight per thread
  {
    double v[TILE * TILE / NTHREADS];
#pragma unroll
    for (int s2 = 0; s2 < TILE * TILE / NTHREADS; s2++) {
      const int idx = threadIdx.x + s2 * NTHREADS;
      const int r = idx % TILE, k = idx / TILE;
      v[s2] = (r < m && k < m && r >= k) ? __ldcg(M2 + (int64_t)k * ldm + r) : 0.0;
    }
#pragma unroll
    for (int s2 = 0; s2 < TILE * TILE / NTHREADS; s2++) {
      const int idx = threadIdx.x + s2 * NTHREADS;
      sm.A[(idx / TILE) * LDS + idx % TILE] = v[s2];
    }
  }
  __syncthreads();
  zero_acc(acc);
  mma_block(sm.A, sm.B, (m + 3) & ~3, acc);
  __syncthreads();
  store_acc(C, ldc, m, n, false, 0, alpha, 0.0, acc);
}

// ----------------------------------------------------------------- POTRF
// Cholesky of the b x b diagonal tile (operand a, in place, lower part
// written back); if aux[1] != 0 also writes M = L^{-1} (full b x b with
// zeros above the diagonal) to operand c.  A non-positive pivot records the
// LAPACK-style info aux[0] + j + 1 in ctl[2] (first writer wins).
//
// The tile is padded to 64 x 64 with an identity block (which factors and
// inverts to itself and does not couple to the leading b x b part), then
// processed in four 16-column blocks J:
//   (a) the 16x16 diagonal block is factored in registers (lane i holds
//       row i, right-looking) and inverted (lane c holds column c of
//       Minv_JJ);
//   (b) panel below: L(r, J) = A(r, J) Minv_JJ^T            (DMMA)
//   (c) trailing lower triangle: A(r, c) -= L(r, J) L(c, J)^T (DMMA)
// and the inverse of the whole tile block row by block row:
//   M(I, :I) = -Minv_II (L(I, :I) M(:I, :I))                (DMMA)
// Warp 0 carries the dependent chain: in step J it computes the panel rows
// of block J (from block J-1), updates the diagonal block J, factors and
// inverts it.  Warps 1-3 meanwhile compute the other panel rows, update the
// trailing rows below block J (after a named barrier on warp 0's panel
// rows) and assemble block row J-1 of the inverse.  One block-wide barrier
// per step; only block row 3 of the inverse follows the last step.
constexpr int POTRF_LD = TILE + 1;
// sL, sM, 1 / L(j, j), the pivot-column broadcast (2 x 16), per-warp 16 x 8
// staging of the inverse assembly (16 x 64 in all)
constexpr int POTRF_SMEM_DOUBLES = 2 * TILE * POTRF_LD + TILE + 32 + 16 * TILE;

// Phase timing for development builds (-DCHB_PROFILE_POTRF); compiled out
// otherwise.  Cycles per phase summed over tasks (thread 0's view):
// diagonal task 0 tile load, 1 panel rows and diagonal-block update,
// 2 16x16 factor, 3 16x16 inverse, 4 end-of-step barrier, 5 L store,
// 6 last inverse block row, 7 M store, 8 first-part publish; look-ahead
// 16 mid waits, 17 tile load, 18 L' product, 19 L' store, 20 early signal,
// 21 L'L'^T product, 22 D update.  Task counts at 12 and 24.
#ifdef CHB_PROFILE_POTRF
__device__ unsigned long long g_potrf_phase[32];
#define POTRF_STAMP(i)                                                    \
  do {                                                                    \
    long long now_ = clock64();                                           \
    if (threadIdx.x == 0) atomicAdd(&g_potrf_phase[i], now_ - stamp_);    \
    stamp_ = now_;                                                        \
  } while (0)
#define POTRF_COUNT(i)                                        \
  do {                                                        \
    if (threadIdx.x == 0) atomicAdd(&g_potrf_phase[i], 1ull); \
  } while (0)
#define POTRF_CLOCK_START long long stamp_ = clock64()
#else
#define POTRF_STAMP(i) \
  do {                 \
  } while (0)
#define POTRF_COUNT(i) \
  do {                 \
  } while (0)
#define POTRF_CLOCK_START \
  do {                    \
  } while (0)
#endif

// acc += A(16 x K) B(K x 8) with A(r, k) = pa[r + k*lda] and
// B(k, n) = pb[k*ksb + n*nsb] in shared memory (K a multiple of 4).
__device__ __forceinline__ void warp_mma_16x8(double (&acc)[4], const double* pa, int lda, const double* pb,
                                              int ksb, int nsb, int K, bool negate) {
  const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  const double sgn = negate ? -1.0 : 1.0;
#pragma unroll 4
  for (int k = 0; k < K; k += 4) {
    const double a0 = sgn * pa[g + (k + q) * lda];
    const double a1 = sgn * pa[g + 8 + (k + q) * lda];
    const double b0 = pb[(k + q) * ksb + g * nsb];
    dmma16(acc, a0, a1, b0);
  }
}

// Named barriers (id 0 is __syncthreads): bar.arrive publishes the
// caller's shared-memory writes to the threads that bar.sync on the id.
__device__ __forceinline__ void named_bar_arrive(int id, int nthreads) {
  asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}
__device__ __forceinline__ void named_bar_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// Panel rows [r0, r0 + 16) of the 16-column block at jp, in place:
// L(r, jp + n) = sum_k A(r, jp + k) Minv(n, k), both 16x8 halves by the
// calling warp (sL, sM: [col][row], leading dimension POTRF_LD).
__device__ __forceinline__ void potrf_panel_rows(double* sL, const double* sM, int jp, int r0) {
  constexpr int LD = POTRF_LD;
  const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  double a0[4] = {0.0, 0.0, 0.0, 0.0}, a1[4] = {0.0, 0.0, 0.0, 0.0};
  warp_mma_16x8(a0, sL + jp * LD + r0, LD, sM + jp * LD + jp, LD, 1, 16, false);
  warp_mma_16x8(a1, sL + jp * LD + r0, LD, sM + jp * LD + jp + 8, LD, 1, 16, false);
  __syncwarp();
  const int r = r0 + g, c0 = jp + 2 * q, c1 = c0 + 8;
  sL[c0 * LD + r] = a0[0];
  sL[(c0 + 1) * LD + r] = a0[1];
  sL[c0 * LD + r + 8] = a0[2];
  sL[(c0 + 1) * LD + r + 8] = a0[3];
  sL[c1 * LD + r] = a1[0];
  sL[(c1 + 1) * LD + r] = a1[1];
  sL[c1 * LD + r + 8] = a1[2];
  sL[(c1 + 1) * LD + r + 8] = a1[3];
  __syncwarp();
}

// Lower-triangle part of the 16x8 tile at (r0, c0) minus the rank-16
// product of the panel block at jp: A(r, c) -= sum_k L(r, jp + k) L(c, jp + k).
__device__ __forceinline__ void potrf_syrk_tile(double* sL, int jp, int r0, int c0) {
  constexpr int LD = POTRF_LD;
  const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  const int r = r0 + g, c = c0 + 2 * q;
  double ac[4] = {sL[c * LD + r], sL[(c + 1) * LD + r], sL[c * LD + r + 8], sL[(c + 1) * LD + r + 8]};
  warp_mma_16x8(ac, sL + jp * LD + r0, LD, sL + jp * LD + c0, LD, 1, 16, true);
  if (r >= c) sL[c * LD + r] = ac[0];
  if (r >= c + 1) sL[(c + 1) * LD + r] = ac[1];
  if (r + 8 >= c) sL[c * LD + r + 8] = ac[2];
  if (r + 8 >= c + 1) sL[(c + 1) * LD + r + 8] = ac[3];
}

// Block row I of the inverse, column tiles tj = first, first + stride, ...
// of 8 columns: T = L(I, :I) M(:I, :I) (K = 16 I) staged in the warp's own
// 16x8 area sTw, then M(I, tile) = -Minv_II T.
__device__ __forceinline__ void potrf_inv_row(const double* sL, double* sM, double* sTw, int I, int first,
                                              int stride) {
  constexpr int LD = POTRF_LD;
  const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  const int i0 = 16 * I, ntj = i0 / 8;
  for (int tj = first; tj < ntj; tj += stride) {
    double ac[4] = {0.0, 0.0, 0.0, 0.0};
    warp_mma_16x8(ac, sL + i0, LD, sM + (8 * tj) * LD, 1, LD, i0, false);
    const int c = 2 * q;
    sTw[g + 16 * c] = ac[0];
    sTw[g + 16 * (c + 1)] = ac[1];
    sTw[g + 8 + 16 * c] = ac[2];
    sTw[g + 8 + 16 * (c + 1)] = ac[3];
    __syncwarp();
    double am[4] = {0.0, 0.0, 0.0, 0.0};
    warp_mma_16x8(am, sM + i0 * LD + i0, LD, sTw, 1, 16, 16, true);
    __syncwarp();
    const int c0 = 8 * tj + 2 * q, r0 = i0 + g;
    sM[c0 * LD + r0] = am[0];
    sM[(c0 + 1) * LD + r0] = am[1];
    sM[c0 * LD + r0 + 8] = am[2];
    sM[(c0 + 1) * LD + r0 + 8] = am[3];
  }
}

// acc[j] += A(16w : 16w + 16, :) B(8j : 8j + 8, :)^T for the calling warp w
// (rows of the 64x64 product by 16-row block, all eight 8-column tiles),
// A(r, k) at sA[k * POTRF_LD + r], B(c, k) at sB[k * POTRF_LD + c], B lower
// triangular: tile j takes only k < 8 (j + 1), so every warp issues 72 of
// the 128 MMAs of a full 64-deep product.
__device__ __forceinline__ void mma_rows_lower_b(const double* sA, const double* sB, double (&acc)[8][4]) {
  constexpr int LD = POTRF_LD;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, q = lane & 3;
  const int r0 = 16 * warp + g;
#pragma unroll 1
  for (int kb = 0; kb < TILE / 8; kb++) {
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int k = 8 * kb + 4 * h + q;
      const double a0 = sA[k * LD + r0], a1 = sA[k * LD + r0 + 8];
#pragma unroll
      for (int j = 0; j < TILE / 8; j++)
        if (j >= kb) dmma16(acc[j], a0, a1, sB[k * LD + 8 * j + g]);
    }
  }
}

// The 20 16x8 tiles on or below the diagonal of a 64x64 product, five per
// warp: tile t lies in 16-row block rb and 8-column block j, listed by row
// block 3, 2, 1, 0 (8, 6, 4 and 2 tiles).
__device__ __forceinline__ void lower_tile(int t, int& rb, int& j) {
  rb = t < 8 ? 3 : (t < 14 ? 2 : (t < 18 ? 1 : 0));
  j = t - (t < 8 ? 0 : (t < 14 ? 8 : (t < 18 ? 14 : 18)));
}

// acc[i] += A(rows of tile i) A(columns of tile i)^T over k < kn for the
// calling warp's five lower tiles (tile 5 w + i), A(r, k) at
// sA[k * POTRF_LD + r]: 80 MMAs per warp instead of 128 for the full square.
__device__ __forceinline__ void mma_lower_tiles(const double* sA, int kn, double (&acc)[5][4]) {
  constexpr int LD = POTRF_LD;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, q = lane & 3;
  int ro[5], co[5];
#pragma unroll
  for (int i = 0; i < 5; i++) {
    int rb, j;
    lower_tile(5 * warp + i, rb, j);
    ro[i] = 16 * rb + g;
    co[i] = 8 * j + g;
  }
#pragma unroll 4
  for (int kk = 0; kk < kn; kk += 4) {
    const double* ak = sA + (kk + q) * LD;
#pragma unroll
    for (int i = 0; i < 5; i++) dmma16(acc[i], ak[ro[i]], ak[ro[i] + 8], ak[co[i]]);
  }
}

// Look-ahead part of a fused diagonal task (T_POTRF with k = m2 > 0, run
// after the factorisation of the b = 64 tile; sL holds L_cc and sM holds
// M = L_cc^{-1}, both with leading dimension POTRF_LD):
//   1. wait for the task's mid waits (waits [cdiag, nwait): the updates of
//      tiles (c+1, c) and (c+1, c+1) from the previous column block);
//   2. L' = A(c+1, c) M^T  (m2 x b; A staged into sL), stored in place and
//      kept in sL;
//   3. early signal aux[3] - 1 (the readers of L');
//   4. A(c+1, c+1) -= L' L'^T (lower part, m2 x m2).
// The tiles lie at a.off + b (panel) and a.off + b*lda + b (diagonal).
__device__ __forceinline__ void potrf_lookahead(const RunArgs& ra, const Task& t, double* smem) {
  __shared__ int s_la_abort;
  constexpr int LD = POTRF_LD;
  double* sL = smem;
  const double* sM = smem + TILE * LD;
  const int b = t.m, m2 = t.k, lda = t.a.ld;
  double* __restrict__ X = ra.bases[t.a.base] + t.a.off;
  double* __restrict__ P = X + b;
  double* __restrict__ D = X + (int64_t)b * lda + b;
  const int tid = threadIdx.x;
  POTRF_CLOCK_START;
  POTRF_COUNT(24);
  __syncthreads();
  if (tid == 0) {
    int abort = 0;
    for (int w = t.cdiag; w < t.nwait && !abort; w++) {
      const int2 wt = ra.waits[t.wait_off + w];
      int64_t spins = 0;
      unsigned ns = 16;
      while (ld_acquire(ra.counters + wt.x) < wt.y) {
        if (++spins > ra.spin_limit) {
          atomicCAS(&ra.ctl[1], 0, DE_TIMEOUT);
          atomicAdd(&ra.ctl[3], 1);
          abort = 1;
          break;
        }
        if ((spins & 15) == 0 && ld_volatile(&ra.ctl[1]) != 0) { abort = 1; break; }
        __nanosleep(ns);
        if (ns < 128) ns <<= 1;
      }
    }
    s_la_abort = abort;
  }
  __syncthreads();
  if (s_la_abort) return;
  POTRF_STAMP(16);
  // A(c+1, c) into sL (rows >= m2 zero)
  {
    double v[TILE * TILE / NTHREADS];
#pragma unroll
    for (int s2 = 0; s2 < TILE * TILE / NTHREADS; s2++) {
      const int idx = tid + s2 * NTHREADS;
      const int r = idx % TILE, c = idx / TILE;
      v[s2] = (r < m2 && c < b) ? __ldcg(P + (int64_t)c * lda + r) : 0.0;
    }
#pragma unroll
    for (int s2 = 0; s2 < TILE * TILE / NTHREADS; s2++) {
      const int idx = tid + s2 * NTHREADS;
      sL[(idx / TILE) * LD + idx % TILE] = v[s2];
    }
  }
  __syncthreads();
  POTRF_STAMP(17);
  const int lane = tid & 31, warp = tid >> 5, g = lane >> 2, q = lane & 3;
  {
    double acc[TILE / 8][4];
#pragma unroll
    for (int j = 0; j < TILE / 8; j++) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0;
    mma_rows_lower_b(sL, sM, acc);  // b = TILE: only the last block column of a front has b < TILE
    __syncthreads();
    POTRF_STAMP(18);
    // L' into sL and in place
#pragma unroll
    for (int j = 0; j < TILE / 8; j++)
#pragma unroll
      for (int h = 0; h < 4; h++) {
        const int r = 16 * warp + g + ((h & 2) ? 8 : 0), c = 8 * j + 2 * q + (h & 1);
        const double v = (r < m2) ? acc[j][h] : 0.0;
        sL[c * LD + r] = v;
        if (r < m2 && c < b) P[(int64_t)c * lda + r] = v;
      }
  }
  __syncthreads();
  POTRF_STAMP(19);
  if (t.aux[3] > 0) {
    if (ra.dynamic) {
      const int c = t.aux[3] - 1;
      if (tid < 32) release_list(ra, __ldg(ra.succ_off + c), __ldg(ra.succ_off + c + 1), nullptr, false, nullptr);
    } else if (tid == 0) {
      red_release_add(ra.counters + (t.aux[3] - 1), 1);
    }
  }
  POTRF_STAMP(20);
  // D -= L' L'^T on and below the diagonal
  double acc[5][4];
#pragma unroll
  for (int i = 0; i < 5; i++) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.0;
  mma_lower_tiles(sL, b, acc);
  POTRF_STAMP(21);
  double old[5][4];
#pragma unroll
  for (int i = 0; i < 5; i++) {
    int rb, j;
    lower_tile(5 * warp + i, rb, j);
#pragma unroll
    for (int h = 0; h < 4; h++) {
      const int r = 16 * rb + g + ((h & 2) ? 8 : 0), c = 8 * j + 2 * q + (h & 1);
      old[i][h] = (r < m2 && r >= c) ? __ldcg(D + (int64_t)c * lda + r) : 0.0;
    }
  }
#pragma unroll
  for (int i = 0; i < 5; i++) {
    int rb, j;
    lower_tile(5 * warp + i, rb, j);
#pragma unroll
    for (int h = 0; h < 4; h++) {
      const int r = 16 * rb + g + ((h & 2) ? 8 : 0), c = 8 * j + 2 * q + (h & 1);
      if (r < m2 && r >= c) D[(int64_t)c * lda + r] = old[i][h] - acc[i][h];
    }
  }
  POTRF_STAMP(22);
}

__device__ void run_potrf(const RunArgs& ra, const Task& t, double* smem, int ti) {
  const int b = t.m;
  const int LD = POTRF_LD;
  double* sL = smem;               // [col][row], lower; upper part zero
  double* sM = sL + TILE * LD;     // inverse, upper part zero
  double* rdiag = sM + TILE * LD;  // 1 / L(j,j)
  double* colb = rdiag + TILE;     // pivot-column broadcast, 2 x 16
  double* sT = colb + 32;          // per-warp 16 x 8 staging (warp w at 128 w)
  double* __restrict__ X = ra.bases[t.a.base] + t.a.off;
  const int lda = t.a.ld;
  const int info_base = t.aux[0];
  const bool want_inv = t.aux[1] != 0;
  const bool factor = t.aux[2] == 0;  // aux[2] != 0: the tile already holds L; invert only
  double* __restrict__ Mout = want_inv ? ra.bases[t.c.base] + t.c.off : nullptr;
  const int ldm = t.c.ld;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  POTRF_CLOCK_START;
  POTRF_COUNT(12);
  {
    double v[TILE * TILE / NTHREADS];
#pragma unroll
    for (int s2 = 0; s2 < TILE * TILE / NTHREADS; s2++) {
      const int idx = tid + s2 * NTHREADS;
      const int r = idx % TILE, c = idx / TILE;
      v[s2] = (r < b && c < b && r >= c) ? __ldcg(X + (int64_t)c * lda + r) : (r == c ? 1.0 : 0.0);
    }
#pragma unroll
    for (int s2 = 0; s2 < TILE * TILE / NTHREADS; s2++) {
      const int idx = tid + s2 * NTHREADS;
      sL[(idx / TILE) * LD + idx % TILE] = (idx % TILE >= idx / TILE) ? v[s2] : 0.0;
      sM[(idx / TILE) * LD + idx % TILE] = 0.0;
    }
  }
  __syncthreads();
  POTRF_STAMP(0);
  // only the 16-column blocks that meet the b x b tile (the padding is the
  // identity and is neither factored nor inverted)
  const int NJ = (b + 15) >> 4, NB = 16 * NJ;
#pragma unroll 1
  for (int J = 0; J < NJ; J++) {
    const int j0 = 16 * J, j1 = j0 + 16, jp = j0 - 16;
    const bool panel = factor && J > 0;     // panel of block J-1 and the updates it feeds
    const bool below = panel && J < NJ - 1; // rows below block J to update
    if (warp == 0) {
      if (panel) {
        potrf_panel_rows(sL, sM, jp, j0);
        if (below) named_bar_arrive(1, NTHREADS);
        potrf_syrk_tile(sL, jp, j0, j0);
        potrf_syrk_tile(sL, jp, j0, j0 + 8);
        __syncwarp();
      }
      POTRF_STAMP(1);
      if (!factor) {
        // invert-only: reciprocals of the diagonal (a zero pivot is singular)
        const int il = lane & 15;
        const double d = sL[(j0 + il) * LD + j0 + il];
        if (lane < 16) {
          if (d == 0.0 && j0 + il < b) atomicCAS(&ra.ctl[2], 0, info_base + j0 + il + 1);
          rdiag[j0 + il] = 1.0 / (d == 0.0 ? 1.0 : d);
        }
        __syncwarp();
      }
      {
        // (a) factor the 16x16 diagonal block in registers: lane i < 16 row i
        const int il = lane & 15;
        if (factor) {
        double a[16];
#pragma unroll
        for (int c = 0; c < 16; c++) a[c] = sL[(j0 + c) * LD + j0 + il];
        // The pivot column goes to the other lanes through shared memory (one
        // store per lane, then broadcast loads): fifteen double shuffles per
        // pivot are throughput-bound and cost 2.5x more on this part.
        // The next pivot, a(jj+1, jj+1) - l(jj+1, jj)^2, is formed by lane
        // jj+1 from its own values right after its multiplier, so the chain
        // from pivot to pivot is shuffle -> rsqrt -> multiply -> FMA and the
        // broadcast and the other updates run beside it.
        double dn = a[0];
        int first_bad = -1;  // first non-positive pivot, reported once after the loop
#pragma unroll
        for (int jj = 0; jj < 16; jj++) {
          const double d = __shfl_sync(0xffffffffu, dn, jj);
          const bool bad = !(d > 0.0);
          first_bad = (bad && first_bad < 0) ? jj : first_bad;
          const double x = bad ? 1.0 : d;
          const double rs = rsqrt(x);
          const double l = (il == jj) ? x * rs : a[jj] * rs;
          a[jj] = (il >= jj) ? l : a[jj];
          if (jj + 1 < 16) dn = fma(-l, l, a[jj + 1]);
          if (lane == jj) rdiag[j0 + jj] = rs;
          if (lane < 16) colb[16 * (jj & 1) + il] = l;
          __syncwarp();
#pragma unroll
          for (int kk = jj + 1; kk < 16; kk++) {
            const double lkj = colb[16 * (jj & 1) + kk];
            if (il >= kk) a[kk] = fma(-l, lkj, a[kk]);
          }
        }
        if (lane == 0 && first_bad >= 0 && j0 + first_bad < b) atomicCAS(&ra.ctl[2], 0, info_base + j0 + first_bad + 1);
        if (lane < 16) {
#pragma unroll
          for (int c = 0; c < 16; c++)
            if (c <= il) sL[(j0 + c) * LD + j0 + il] = a[c];
        }
        }
        __syncwarp();
        POTRF_STAMP(2);
        // inverse of the block: lane c < 16 holds column c,
        // M(r, c) = -rd(r) sum_{l<r} L(r, l) M(l, c) for r > c, M(c, c) = rd(c),
        // right-looking: as soon as M(l, c) is known it is added into the
        // partial sums of all later rows, so the dependent chain per row is
        // one multiply and one FMA (FP64 latency, not the row's dot product)
        double m[16], sacc[16];
#pragma unroll
        for (int r = 0; r < 16; r++) sacc[r] = 0.0;
#pragma unroll
        for (int l = 0; l < 16; l++) {
          const double rd = rdiag[j0 + l];
          m[l] = (l == il) ? rd : ((l > il) ? -rd * sacc[l] : 0.0);
#pragma unroll
          for (int r = l + 1; r < 16; r++) sacc[r] = fma(sL[(j0 + l) * LD + j0 + r], m[l], sacc[r]);
        }
        if (lane < 16) {
#pragma unroll
          for (int r = 0; r < 16; r++)
            if (r >= il) sM[(j0 + il) * LD + j0 + r] = m[r];
        }
        POTRF_STAMP(3);
      }
    } else {
      if (below) {
        const int rb = j0 + 16 * warp;  // warps 1, 2: the panel rows below block J
        if (rb < NB) potrf_panel_rows(sL, sM, jp, rb);
        named_bar_sync(1, NTHREADS);
        // rows >= j1, columns >= j0, lower part, from the panel of block J-1
        const int nti = (NB - j1) / 16, ntj = (NB - j0) / 8;
        for (int tt = warp - 1; tt < nti * ntj; tt += NTHREADS / 32 - 1) {
          const int r0 = j1 + 16 * (tt / ntj), c0 = j0 + 8 * (tt % ntj);
          if (c0 <= r0 + 15) potrf_syrk_tile(sL, jp, r0, c0);
        }
      }
      if (want_inv && J >= 2) potrf_inv_row(sL, sM, sT + 128 * warp, J - 1, warp - 1, NTHREADS / 32 - 1);
    }
    __syncthreads();
    POTRF_STAMP(4);
  }
  if (factor) {
#pragma unroll 8
    for (int s2 = 0; s2 < TILE * TILE / NTHREADS; s2++) {
      const int idx = tid + s2 * NTHREADS;
      const int r = idx % TILE, c = idx / TILE;
      if (r < b && c < b && r >= c) X[(int64_t)c * lda + r] = sL[c * LD + r];
    }
  }
  POTRF_STAMP(5);
  if (!want_inv) return;
  // the last block row of the inverse (rows 1 .. NJ-2 were assembled above)
  if (NJ >= 2) potrf_inv_row(sL, sM, sT + 128 * warp, NJ - 1, warp, NTHREADS / 32);
  __syncthreads();
  POTRF_STAMP(6);
#pragma unroll 8
  for (int s2 = 0; s2 < TILE * TILE / NTHREADS; s2++) {
    const int idx = tid + s2 * NTHREADS;
    const int r = idx % TILE, cc = idx / TILE;
    if (r < b && cc < b) Mout[(int64_t)cc * ldm + r] = sM[cc * LD + r];
  }
  POTRF_STAMP(7);
  if (t.k > 0) {
    // first part done: L_cc and M_cc are stored; the task's own waiters go
    __syncthreads();
    if (ra.dynamic) {
      if (tid < 32) release_list(ra, __ldg(ra.succ_off + ti), __ldg(ra.succ_off + ti + 1), nullptr, false, nullptr);
    } else if (tid == 0) {
      red_release_add(ra.counters + ti, 1);
    }
    POTRF_STAMP(8);
    potrf_lookahead(ra, t, smem);
  }
}

// ------------------------------------------------------------ assembly
// Extend-add for front k = aux[0], front columns [aux[1], aux[2]):
//   * zero the columns of the update block U_k that fall in the range
//     (if aux[3] & 1);
//   * for each child, last to first (the order the reference pops its update
//     stack, cholesky.c:41-52), add U_child(i, q) into F(r[i], r[q]) for the
//     child columns q whose relative index r[q] lies in the range.
// F(i, j) is the front panel (operand a: nj rows, ld a.ld) for j < nn, else
// the update block U_k (operand c, ld c.ld).  One warp per child column;
// children are applied one after the other.
// A child's relative indices, staged in shared memory once per child when
// they fit (one coalesced pass), so that each scattered access costs one
// round trip instead of two; otherwise read from global memory.
constexpr int RIDX_SMEM_MAX = ENGINE_SMEM_BASE_DOUBLES * 2;  // int32 entries in the base shared memory
__device__ __forceinline__ const int32_t* stage_ridx(const int32_t* __restrict__ r, int N, double* smem) {
  if (N > RIDX_SMEM_MAX) return r;
  int32_t* sr = reinterpret_cast<int32_t*>(smem);
  for (int i = threadIdx.x; i < N; i += NTHREADS) sr[i] = __ldg(r + i);
  __syncthreads();
  return sr;
}

constexpr int GATHER_INFLIGHT = 8;  // scattered elements in flight per lane

__device__ void run_asm(const RunArgs& ra, const Task& t, double* smem) {
  const FrontDesc f = ra.fronts[t.aux[0]];
  const int j0 = t.aux[1], j1 = t.aux[2];
  const bool zero_u = (t.aux[3] & 1) != 0;
  double* __restrict__ P = ra.bases[t.a.base] + t.a.off;
  const int ldp = t.a.ld;
  double* __restrict__ Uk = ra.bases[t.c.base] + t.c.off;
  const int ldu = t.c.ld;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (zero_u) {
    for (int j = max(j0, f.nn) + warp; j < j1; j += NTHREADS / 32) {
      const int jj = j - f.nn;
      for (int i = jj + lane; i < f.na; i += 32) Uk[(int64_t)jj * ldu + i] = 0.0;
    }
  }
  __syncthreads();
  for (int l = f.chend - 1; l >= f.chbeg; l--) {
    const FrontDesc ch = ra.fronts[ra.chidx[l]];
    const int N = ch.na;
    const int32_t* r = stage_ridx(ra.relidx + ch.relptr, N, smem);
    const double* __restrict__ Uc = ra.bases[B_WS] + t.off2 + ch.upd;
    // child columns with r[q] in [j0, j1): r is strictly increasing
    int lo = 0, hi = N;
    while (lo < hi) { int mid = (lo + hi) >> 1; if (r[mid] < j0) lo = mid + 1; else hi = mid; }
    const int q0 = lo;
    hi = N;
    while (lo < hi) { int mid = (lo + hi) >> 1; if (r[mid] < j1) lo = mid + 1; else hi = mid; }
    const int q1 = lo;
    for (int q = q0 + warp; q < q1; q += NTHREADS / 32) {
      const int col = r[q];
      double* __restrict__ dst =
          (col < f.nn) ? P + (int64_t)col * ldp : Uk + (int64_t)(col - f.nn) * ldu - f.nn;
      const double* __restrict__ src = Uc + (int64_t)q * N;
      for (int i0 = q; i0 < N; i0 += GATHER_INFLIGHT * 32) {
        int ri[GATHER_INFLIGHT];
        double u[GATHER_INFLIGHT], d[GATHER_INFLIGHT];
#pragma unroll
        for (int e = 0; e < GATHER_INFLIGHT; e++) {
          const int i = i0 + lane + 32 * e;
          ri[e] = (i < N) ? r[i] : -1;
          u[e] = (i < N) ? __ldcg(src + i) : 0.0;
          d[e] = (i < N) ? __ldcg(dst + ri[e]) : 0.0;
        }
#pragma unroll
        for (int e = 0; e < GATHER_INFLIGHT; e++)
          if (ri[e] >= 0) dst[ri[e]] = d[e] + u[e];
      }
    }
    __syncthreads();
  }
}

// A whole small cholesky front (T_FRONT, nj <= TILE; cholesky.c:33-72 for
// one node) in shared memory, F(r, c) at F[c*FLD + r], lower part:
//   1. F = the block's lower trapezoid (columns < nn), zero elsewhere;
//   2. the children's update matrices added, last child first;
//   3. the first nn columns eliminated (right-looking: pivot, column scaled,
//      trailing lower part updated, a warp per column), which leaves L11,
//      L21 and the Schur complement F22 - L21 L21^T;
//   4. the rows below replaced by W = L21 L11^{-1} (the reference's layout
//      of the off-diagonal block), one row per thread;
//   5. the block and the update matrix (operand c) written back.
// A non-positive pivot records ctl[2] = j + 1 and continues with 1.
constexpr int FLD = TILE + 1;
static_assert(2 * TILE * FLD + TILE / 2 <= ENGINE_SMEM_BASE_DOUBLES, "small fronts exceed the engine's shared memory");

__device__ void run_front(const RunArgs& ra, const Task& t, double* smem) {
  const FrontDesc f = ra.fronts[t.aux[0]];
  const int nn = f.nn, na = f.na, nj = f.nj;
  double* F = smem;
  double* __restrict__ X = ra.bases[t.a.base] + t.a.off;
  double* __restrict__ U = ra.bases[t.c.base] + t.c.off;
  const int ldu = t.c.ld;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int NW = NTHREADS / 32;
  for (int c = warp; c < nj; c += NW)
    for (int r = lane; r < nj; r += 32)
      F[c * FLD + r] = (c < nn && r >= c) ? __ldcg(X + (int64_t)c * nj + r) : 0.0;
  __syncthreads();
  // the children's update matrices, last child first: its relative indices
  // staged in shared memory, then the lower triangle of U_c flattened over
  // the threads with FRONT_E loads in flight per thread (a child's entries
  // land on distinct front entries)
  constexpr int FRONT_E = 8;
  int* sr = reinterpret_cast<int*>(F + TILE * FLD + 2 * TILE);
  for (int l = f.chend - 1; l >= f.chbeg; l--) {
    const FrontDesc ch = ra.fronts[ra.chidx[l]];
    const int Nc = ch.na, tot = Nc * Nc;
    const int32_t* __restrict__ rr = ra.relidx + ch.relptr;
    const double* __restrict__ Uc = ra.bases[B_WS] + t.off2 + ch.upd;
    if (tid < Nc) sr[tid] = __ldg(rr + tid);
    __syncthreads();
    for (int base = 0; base < tot; base += FRONT_E * NTHREADS) {
      double v[FRONT_E];
      int dst[FRONT_E];
#pragma unroll
      for (int e = 0; e < FRONT_E; e++) {
        const int idx = base + tid + e * NTHREADS, q = idx / Nc, i = idx - q * Nc;
        const bool ok = idx < tot && i >= q;
        v[e] = ok ? __ldcg(Uc + idx) : 0.0;
        dst[e] = ok ? sr[q] * FLD + sr[i] : -1;
      }
#pragma unroll
      for (int e = 0; e < FRONT_E; e++)
        if (dst[e] >= 0) F[dst[e]] += v[e];
    }
    __syncthreads();
  }
  // Pivots with one barrier each: pivot j updates the trailing part with
  // its unscaled column, F(i, c) -= F(i, j) F(c, j) / d_j, and the column
  // itself is scaled by 1 / L(j, j) in the next pivot's phase (nobody reads
  // it then); 1 / L(j, j) = rsqrt(d_j), kept for the solve below.
  // The diagonal entries L(j, j) = d_j / sqrt(d_j) are written after the
  // loop (every thread reads d_j in pivot j's phase).
  double* rl = F + TILE * FLD;  // 1 / L(j, j)
  double* lj = rl + TILE;       // L(j, j)
  int first_bad = -1;
  for (int j = 0; j < nn; j++) {
    const double d = F[j * FLD + j];
    const bool bad = !(d > 0.0);
    if (bad && first_bad < 0) first_bad = j;
    const double rs = rsqrt(bad ? 1.0 : d), rd = rs * rs;
    if (j > 0) {
      const double rp = rl[j - 1];
      for (int i = j + tid; i < nj; i += NTHREADS) F[(j - 1) * FLD + i] *= rp;
    }
    if (tid == 0) {
      rl[j] = rs;  // read from the next phase on
      lj[j] = (bad ? 1.0 : d) * rs;
    }
    for (int c = j + 1 + warp; c < nj; c += NW) {
      const double fc = F[j * FLD + c] * rd;
      for (int i = c + lane; i < nj; i += 32) F[c * FLD + i] -= F[j * FLD + i] * fc;
    }
    __syncthreads();
  }
  if (nn > 0)
    for (int i = nn + tid; i < nj; i += NTHREADS) F[(nn - 1) * FLD + i] *= rl[nn - 1];
  for (int j = tid; j < nn; j += NTHREADS) F[j * FLD + j] = lj[j];
  if (tid == 0 && first_bad >= 0) atomicCAS(&ra.ctl[2], 0, first_bad + 1);
  __syncthreads();
  // W = L21 L11^{-1}, one row per thread, right-looking: w_j = t_j / L(j, j),
  // then t_j' -= w_j L(j, j') for j' < j (independent updates)
  for (int i = nn + tid; i < nj; i += NTHREADS)
    for (int j = nn - 1; j >= 0; j--) {
      const double v = F[j * FLD + i] * rl[j];
      F[j * FLD + i] = v;
      for (int l2 = 0; l2 < j; l2++) F[l2 * FLD + i] -= v * F[l2 * FLD + j];
    }
  __syncthreads();
  for (int c = warp; c < nn; c += NW)
    for (int r = c + lane; r < nj; r += 32) X[(int64_t)c * nj + r] = F[c * FLD + r];
  for (int q = warp; q < na; q += NW)
    for (int i = q + lane; i < na; i += 32) U[(int64_t)q * ldu + i] = F[(nn + q) * FLD + nn + i];
}

// A whole small projected-inverse front (T_PFRONT, nj <= TILE;
// projected_inverse.c:33-73 for one node) in two shared-memory buffers of
// leading dimension FLD: G holds L11, then M = L11^{-1} (inverted in place,
// columns last to first, as LAPACK's unblocked triangular inverse does),
// then S21; F holds the front: W and V_k (operand c) first, then
// [Y11; S21 | V_k].
//   Y11 = M^T M;  S21 = -V_k W;  Y11 -= S21^T W;
//   U_c = F(r_c, r_c) for every child c (lower parts);
//   the block <- [Y11 (strict upper part zeroed); S21].
// A zero diagonal entry records ctl[2] = j + 1 and is taken as 1.
__device__ void run_pfront(const RunArgs& ra, const Task& t, double* smem) {
  const FrontDesc f = ra.fronts[t.aux[0]];
  const int nn = f.nn, na = f.na, nj = f.nj;
  double* G = smem;
  double* F = smem + TILE * FLD;
  double* __restrict__ X = ra.bases[t.a.base] + t.a.off;
  const double* __restrict__ V = ra.bases[t.c.base] + t.c.off;
  const int ldv = t.c.ld;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int NW = NTHREADS / 32;
  for (int c = warp; c < nn; c += NW)
    for (int r = lane; r < nj; r += 32) {
      const double v = __ldcg(X + (int64_t)c * nj + r);
      if (r < nn) G[c * FLD + r] = (r >= c) ? v : 0.0;
      else F[c * FLD + r] = v;
    }
  for (int q = warp; q < na; q += NW)
    for (int i = q + lane; i < na; i += 32) F[(nn + q) * FLD + nn + i] = __ldcg(V + (int64_t)q * ldv + i);
  __syncthreads();
  int first_bad = -1;
  for (int j = nn - 1; j >= 0; j--) {
    const double d = G[j * FLD + j];
    if (d == 0.0 && first_bad < 0) first_bad = j;
    const double ajj = 1.0 / (d == 0.0 ? 1.0 : d);
    const int i = j + 1 + tid;
    double ti = 0.0;
    if (i < nn)
      for (int l = j + 1; l <= i; l++) ti = fma(G[l * FLD + i], G[j * FLD + l], ti);
    __syncthreads();
    if (i < nn) G[j * FLD + i] = -ajj * ti;
    if (tid == 0) G[j * FLD + j] = ajj;
    __syncthreads();
  }
  if (tid == 0 && first_bad >= 0) atomicCAS(&ra.ctl[2], 0, first_bad + 1);
  for (int j = warp; j < nn; j += NW)
    for (int i = j + lane; i < nn; i += 32) {
      double v = 0.0;
      for (int l = i; l < nn; l++) v = fma(G[i * FLD + l], G[j * FLD + l], v);
      F[j * FLD + i] = v;
    }
  __syncthreads();
  if (na > 0) {
    for (int j = warp; j < nn; j += NW)
      for (int i = lane; i < na; i += 32) {
        double v = 0.0;
        for (int l = 0; l < na; l++) {
          const double vil = (i >= l) ? F[(nn + l) * FLD + nn + i] : F[(nn + i) * FLD + nn + l];
          v = fma(vil, F[j * FLD + nn + l], v);
        }
        G[j * FLD + i] = -v;
      }
    __syncthreads();
    for (int j = warp; j < nn; j += NW)
      for (int i = j + lane; i < nn; i += 32) {
        double v = 0.0;
        for (int l = 0; l < na; l++) v = fma(G[i * FLD + l], F[j * FLD + nn + l], v);
        F[j * FLD + i] -= v;
      }
    __syncthreads();
    for (int j = warp; j < nn; j += NW)
      for (int i = lane; i < na; i += 32) F[j * FLD + nn + i] = G[j * FLD + i];
    __syncthreads();
  }
  // the children's updates V_c = F(r_c, r_c), lower triangle, the relative
  // indices staged in shared memory per child
  int* sr = reinterpret_cast<int*>(smem + 2 * TILE * FLD);
  for (int l = f.chbeg; l < f.chend; l++) {
    const FrontDesc ch = ra.fronts[ra.chidx[l]];
    const int Nc = ch.na, tot = Nc * Nc;
    const int32_t* __restrict__ rr = ra.relidx + ch.relptr;
    double* __restrict__ Uc = ra.bases[B_WS] + t.off2 + ch.upd;
    if (tid < Nc) sr[tid] = __ldg(rr + tid);
    __syncthreads();
    for (int idx = tid; idx < tot; idx += NTHREADS) {
      const int q = idx / Nc, i = idx - q * Nc;
      if (i >= q) Uc[idx] = F[sr[q] * FLD + sr[i]];
    }
    __syncthreads();
  }
  for (int c = warp; c < nn; c += NW)
    for (int r = lane; r < nj; r += 32)
      X[(int64_t)c * nj + r] = (r < nn && r < c) ? 0.0 : F[c * FLD + r];
}

// Gather of a child's update matrix out of its parent's front
// (projected_inverse.c:62-71, completion.c:61-66): for child c = aux[0] and
// child columns q in [aux[1], aux[2]), U_c(i, q) = F(r[i], r[q]) for i >= q,
// where F(row, col) (col <= row) is read from
//   operand a (rows < nn, ld a.ld) when row < nn,
//   operand b (rows >= nn, row nn at offset 0, ld b.ld) when col < nn <= row,
//   operand c (update block, ld c.ld) when col >= nn.
__device__ void run_extract(const RunArgs& ra, const Task& t, double* smem) {
  const FrontDesc ch = ra.fronts[t.aux[0]];
  const FrontDesc f = ra.fronts[ch.parent];
  const int q0 = t.aux[1], q1 = t.aux[2];
  const int N = ch.na, nn = f.nn;
  const int32_t* r = stage_ridx(ra.relidx + ch.relptr, N, smem);
  const double* __restrict__ F11 = ra.bases[t.a.base] + t.a.off;
  const double* __restrict__ F21 = ra.bases[t.b.base] + t.b.off;
  const double* __restrict__ F22 = ra.bases[t.c.base] + t.c.off;
  const int ld11 = t.a.ld, ld21 = t.b.ld, ld22 = t.c.ld;
  double* __restrict__ Uc = ra.bases[B_WS] + t.off2 + ch.upd;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int q = q0 + warp; q < q1; q += NTHREADS / 32) {
    const int col = r[q];
    for (int i0 = q; i0 < N; i0 += GATHER_INFLIGHT * 32) {
      double v[GATHER_INFLIGHT];
#pragma unroll
      for (int e = 0; e < GATHER_INFLIGHT; e++) {
        const int i = i0 + lane + 32 * e;
        const int row = (i < N) ? r[i] : 0;
        const double* src;
        if (col >= nn) src = F22 + (int64_t)(col - nn) * ld22 + (row - nn);
        else if (row >= nn) src = F21 + (int64_t)col * ld21 + (row - nn);
        else src = F11 + (int64_t)col * ld11 + row;
        v[e] = (i < N) ? __ldcg(src) : 0.0;
      }
#pragma unroll
      for (int e = 0; e < GATHER_INFLIGHT; e++) {
        const int i = i0 + lane + 32 * e;
        if (i < N) Uc[(int64_t)q * N + i] = v[e];
      }
    }
  }
}

// Tile copy C = alpha * A (m x n).  aux[0] bit 0: copy only the lower
// triangle (r >= c); bit 1: write zeros above the diagonal; bit 2: write
// zeros everywhere (A is not read).  Bit 3: anti-transpose inside an
// aux[1] x aux[1] matrix: operands a and c are the matrices' origins and the
// tile has origin (aux[2], aux[3]) in C; C(i, j) = A(n-1-j, n-1-i) for the
// lower entries i >= j (with J the order reversal, C = J A^T J).  Bit 4:
// transpose, C(r, c) = A(c, r); bit 5 with it: only entries above the
// diagonal of the tile (r < c), used to symmetrise a diagonal block.
__device__ void run_copy(const RunArgs& ra, const Task& t) {
  if (t.aux[0] & 16) {
    const double* __restrict__ A = ra.bases[t.a.base] + t.a.off;
    double* __restrict__ C = ra.bases[t.c.base] + t.c.off;
    const int lda = t.a.ld, ldc = t.c.ld, m = t.m, n = t.n;
    const bool upper = (t.aux[0] & 32) != 0;
    for (int base = 0; base < m * n; base += 8 * NTHREADS) {
      double v[8];
#pragma unroll
      for (int e = 0; e < 8; e++) {
        const int idx = base + threadIdx.x + e * NTHREADS;
        const int r = idx % m, c = idx / m;
        v[e] = (idx < m * n && (!upper || r < c)) ? __ldcg(A + (int64_t)r * lda + c) : 0.0;
      }
#pragma unroll
      for (int e = 0; e < 8; e++) {
        const int idx = base + threadIdx.x + e * NTHREADS;
        const int r = idx % m, c = idx / m;
        if (idx < m * n && (!upper || r < c)) C[(int64_t)c * ldc + r] = t.alpha * v[e];
      }
    }
    return;
  }
  if (t.aux[0] & 8) {
    const double* __restrict__ A = ra.bases[t.a.base] + t.a.off;
    double* __restrict__ C = ra.bases[t.c.base] + t.c.off;
    const int lda = t.a.ld, ldc = t.c.ld, m = t.m, n = t.n, nn = t.aux[1], i0 = t.aux[2], j0 = t.aux[3];
    for (int base = 0; base < m * n; base += 8 * NTHREADS) {
      double v[8];
#pragma unroll
      for (int e = 0; e < 8; e++) {
        const int idx = base + threadIdx.x + e * NTHREADS;
        const int gi = i0 + idx % m, gj = j0 + idx / m;
        v[e] = (idx < m * n && gi >= gj) ? __ldcg(A + (int64_t)(nn - 1 - gi) * lda + (nn - 1 - gj)) : 0.0;
      }
#pragma unroll
      for (int e = 0; e < 8; e++) {
        const int idx = base + threadIdx.x + e * NTHREADS;
        const int gi = i0 + idx % m, gj = j0 + idx / m;
        if (idx < m * n && gi >= gj) C[(int64_t)gj * ldc + gi] = v[e];
      }
    }
    return;
  }
  const double* __restrict__ A = ra.bases[t.a.base] + t.a.off;
  double* __restrict__ C = ra.bases[t.c.base] + t.c.off;
  const int lda = t.a.ld, ldc = t.c.ld, m = t.m, n = t.n;
  const bool lower = (t.aux[0] & 1) != 0, zup = (t.aux[0] & 2) != 0, zall = (t.aux[0] & 4) != 0;
  const double alpha = t.alpha;
  for (int base = 0; base < m * n; base += 8 * NTHREADS) {
    double v[8];
#pragma unroll
    for (int e = 0; e < 8; e++) {
      const int idx = base + threadIdx.x + e * NTHREADS;
      const int r = idx % m, c = idx / m;
      v[e] = (!zall && idx < m * n && (!lower || r >= c)) ? __ldcg(A + (int64_t)c * lda + r) : 0.0;
    }
#pragma unroll
    for (int e = 0; e < 8; e++) {
      const int idx = base + threadIdx.x + e * NTHREADS;
      const int r = idx % m, c = idx / m;
      if (idx >= m * n) continue;
      if (r >= c || !lower) C[(int64_t)c * ldc + r] = alpha * v[e];
      else if (zup) C[(int64_t)c * ldc + r] = 0.0;
    }
  }
}

// ------------------------------------------------------ update_factor
__device__ __forceinline__ double block_reduce_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
#pragma unroll
  for (int w = 0; w < NTHREADS / 32; w++) s += red[w];
  return s;
}

// Blocked Householder QL of a factored update (update_factor.c:29-47).
// For child c = aux[0] of front k, with V_k = L_k^T L_k (L_k lower, the
// parent's update block, operand a of QL_GATHER) and the child's relative
// indices r split as r[:N1] < nn <= r[N1:], the N2 columns
// C(:, j) = L_k(:, jj_j), jj_j = r[N1 + j] - nn, are reduced to [0; L22] by
// reflections applied last column first.  The reflection of column j acts on
// rows [jj_j, prow_j], prow_j = na - N2 + j, with LAPACK's dlarfg/dlarfx
// conventions: alpha = C(prow_j, j), x = C(jj_j:prow_j, j),
// beta = -sign(alpha) * hypot(alpha, ||x||), tau = (beta - alpha) / beta,
// v = [x / (alpha - beta); 1]; tau = 0 when x is empty or zero.
//
// A QL_PANEL task factors columns [c0, c1) inside shared memory (rows
// [row0, row1] = [jj_c0, prow_{c1-1}], the rows its reflections touch),
// applying each reflection to the panel's remaining columns only, and
// writes, for the columns to its left (updated by MROW/GEMM tasks):
//   W' (operand b): column c0 + i = reflector i, i = c1 - 1 - j (the order
//     they are applied), explicit over rows [row0, row1];
//   T  (operand c, nb x nb lower, ld c.ld): H_{c0} ... H_{c1-1} = I - W' T W'^T
//     (LAPACK dlarft 'B','C': T(i,i) = tau_i,
//      T(i+1:, i) = -tau_i T(i+1:, i+1:) W'(:, i+1:)^T w'_i).
// Phase timing for development builds (-DCHB_PROFILE_QL); compiled out
// otherwise.
#ifdef CHB_PROFILE_QL
__device__ unsigned long long g_ql_phase[12];
#define QL_STAMP(i)                                                  \
  do {                                                               \
    __syncthreads();                                                 \
    long long now_ = clock64();                                      \
    if (threadIdx.x == 0) atomicAdd(&g_ql_phase[i], now_ - qstamp_); \
    qstamp_ = now_;                                                  \
  } while (0)
#else
#define QL_STAMP(i) \
  do {              \
  } while (0)
#endif

__device__ void run_ql(const RunArgs& ra, const Task& t, double* smem) {
#ifdef CHB_PROFILE_QL
  long long qstamp_ = clock64();
#endif
  const FrontDesc ch = ra.fronts[t.aux[0]];
  const FrontDesc f = ra.fronts[ch.parent];
  const int N = ch.na, nn = f.nn, na = f.na;
  const int32_t* __restrict__ r = ra.relidx + ch.relptr;
  int lo = 0, hi = N;
  while (lo < hi) { int mid = (lo + hi) >> 1; if (__ldg(r + mid) < nn) lo = mid + 1; else hi = mid; }
  const int N1 = lo, N2 = N - N1;
  const int c0 = t.aux[1], c1 = t.aux[2];
  const int tid = threadIdx.x;
  if (t.aux[3] == QL_GATHER) {
    const double* __restrict__ Lk = ra.bases[t.a.base] + t.a.off;
    double* __restrict__ C = ra.bases[t.c.base] + t.c.off;
    const int ldl = t.a.ld, ldc = t.c.ld;
    for (int j = c0; j < c1; j++) {
      const int jj = __ldg(r + N1 + j) - nn;
      for (int i = tid; i < na; i += NTHREADS)
        C[(int64_t)j * ldc + i] = (i >= jj) ? __ldcg(Lk + (int64_t)jj * ldl + i) : 0.0;
    }
    return;
  }
  double* __restrict__ C = ra.bases[t.a.base] + t.a.off;
  double* __restrict__ W = ra.bases[t.b.base] + t.b.off;
  double* __restrict__ Tg = ra.bases[t.c.base] + t.c.off;
  const int ldc = t.a.ld, ldw = t.b.ld, ldt = t.c.ld;
  const int nb = c1 - c0;
  const int row0 = __ldg(r + N1 + c0) - nn, row1 = na - N2 + c1 - 1;
  const int h = row1 - row0 + 1;
  if (nb <= 0 || h <= 0 || ql_panel_doubles(h, nb) > ra.smem_doubles) {
    if (tid == 0) atomicCAS(&ra.ctl[1], DE_NONE, DE_BAD_TASK);
    return;
  }
  double* P = smem;                  // panel, column-major, ld h
  double* G = smem + h * nb;         // nb x nb, ld nb (after the panel is out)
  double* red = G + nb * nb;         // reduction scratch (32)
  double* taus = red + 32;           // nb <= 64 (tau of reflector i)
  int* lr0s = reinterpret_cast<int*>(taus + 64);   // 2 x 64 ints: support of reflector i
  // load the panel
  for (int idx = tid; idx < h * nb; idx += NTHREADS) {
    const int q = idx % h, pc = idx / h;
    P[idx] = __ldcg(C + (int64_t)(c0 + pc) * ldc + row0 + q);
  }
  __syncthreads();
  QL_STAMP(0);
  for (int i = 0; i < nb; i++) {
    const int col = c1 - 1 - i, pc = col - c0;
    const int lr0 = __ldg(r + N1 + col) - nn - row0;   // first row of x (local)
    const int lp = na - N2 + col - row0;               // pivot row (local)
    double* pv = P + pc * h;
    double tau = 0.0;
    if (lp > lr0) {
      double part = 0.0;
      for (int q = lr0 + tid; q < lp; q += NTHREADS) part += pv[q] * pv[q];
      const double xn2 = block_reduce_sum(part, red);
      QL_STAMP(5);
      if (xn2 != 0.0) {
        const double alpha = pv[lp];
        // dlapy2(alpha, ||x||)
        const double xa = fabs(alpha), xb = sqrt(xn2);
        const double w = fmax(xa, xb), z = fmin(xa, xb);
        const double nrm = (z == 0.0) ? w : w * sqrt(1.0 + (z / w) * (z / w));
        const double beta = -copysign(nrm, alpha);
        tau = (beta - alpha) / beta;
        const double scal = 1.0 / (alpha - beta);
        __syncthreads();  // everyone has read pv[lp] and the norm
        for (int q = lr0 + tid; q < lp; q += NTHREADS) pv[q] *= scal;
        __syncthreads();
        QL_STAMP(6);
        // H = I - tau v v^T on the panel columns to the left, rows [lr0, lp]:
        // w_q = tau v^T C(:, q) with a group of tpc threads per column (row
        // slices, two partial sums, shuffle reduction inside the group), then
        // C -= v w^T over all (row, column) pairs
        double* wq = G;  // G is unused until the reflections are done
        int tpc = 32;
        while (tpc > 1 && tpc * pc > NTHREADS) tpc >>= 1;
        {
          const int q2 = tid / tpc, sub = tid % tpc;
          double s0 = 0.0, s1 = 0.0;
          if (q2 < pc) {
            const double* cq = P + q2 * h;
            int q = lr0 + sub;
            for (; q + tpc < lp; q += 2 * tpc) {
              s0 = fma(pv[q], cq[q], s0);
              s1 = fma(pv[q + tpc], cq[q + tpc], s1);
            }
            if (q < lp) s0 = fma(pv[q], cq[q], s0);
            if (sub == 0) s1 += cq[lp];
          }
          double s = s0 + s1;
          for (int o = tpc >> 1; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
          if (q2 < pc && sub == 0) wq[q2] = tau * s;
        }
        __syncthreads();
        QL_STAMP(7);
        // rows on R lanes (the smallest power of two covering the reflector),
        // columns on NTHREADS / R groups: no division per element
        const int len = lp - lr0 + 1;
        int R = 1;
        while (R < len && R < NTHREADS) R <<= 1;
        {
          const int rl = tid % R, cg = tid / R, ncg = NTHREADS / R;
          for (int q = lr0 + rl; q <= lp; q += R) {
            const double vq = (q == lp) ? 1.0 : pv[q];
#pragma unroll 4
            for (int q2 = cg; q2 < pc; q2 += ncg) P[q2 * h + q] = fma(-vq, wq[q2], P[q2 * h + q]);
          }
        }
        __syncthreads();
        QL_STAMP(8);
        if (tid == 0) pv[lp] = beta;
      }
    }
    if (tid == 0) {
      taus[i] = tau;
      lr0s[i] = lr0;
      lr0s[64 + i] = lp;
    }
    __syncthreads();
  }
  QL_STAMP(1);
  // the panel back to C, then W' (explicit reflectors) in its place
  for (int idx = tid; idx < h * nb; idx += NTHREADS) {
    const int q = idx % h, pc = idx / h;
    C[(int64_t)(c0 + pc) * ldc + row0 + q] = P[idx];
  }
  __syncthreads();
  for (int idx = tid; idx < h * nb; idx += NTHREADS) {
    const int q = idx % h, pc = idx / h;
    const int i = c1 - 1 - (c0 + pc);
    const int a = lr0s[i], b = lr0s[64 + i];
    const double v = (q < a || q > b) ? 0.0 : (q == b ? 1.0 : P[idx]);
    P[idx] = v;
    W[(int64_t)(c0 + i) * ldw + row0 + q] = v;
  }
  __syncthreads();
  QL_STAMP(2);
  // G(a, b) = w'_a^T w'_b for a > b (w'_i is panel column nb - 1 - i):
  // each thread a 4 x 4 block of G over all rows (8 loads feed 16 FMAs, no
  // cross-lane reductions)
  {
    const int nbb = (nb + 3) >> 2;
    for (int blk = tid; blk < nbb * (nbb + 1) / 2; blk += NTHREADS) {
      int bi = 0;
      while ((bi + 1) * (bi + 2) / 2 <= blk) bi++;
      const int bj = blk - bi * (bi + 1) / 2;
      const double* wa[4];
      const double* wb[4];
#pragma unroll
      for (int x = 0; x < 4; x++) {
        wa[x] = P + (nb - 1 - min(4 * bi + x, nb - 1)) * h;
        wb[x] = P + (nb - 1 - min(4 * bj + x, nb - 1)) * h;
      }
      double acc[4][4];
#pragma unroll
      for (int x = 0; x < 4; x++)
#pragma unroll
        for (int y = 0; y < 4; y++) acc[x][y] = 0.0;
      for (int q = 0; q < h; q++) {
        double va[4], vb[4];
#pragma unroll
        for (int x = 0; x < 4; x++) {
          va[x] = wa[x][q];
          vb[x] = wb[x][q];
        }
#pragma unroll
        for (int x = 0; x < 4; x++)
#pragma unroll
          for (int y = 0; y < 4; y++) acc[x][y] = fma(va[x], vb[y], acc[x][y]);
      }
#pragma unroll
      for (int x = 0; x < 4; x++)
#pragma unroll
        for (int y = 0; y < 4; y++) {
          const int a = 4 * bi + x, b2 = 4 * bj + y;
          if (a < nb && b2 < a) G[b2 * nb + a] = acc[x][y];
        }
    }
  }
  __syncthreads();
  QL_STAMP(3);
  // T in place of G's lower part, last column first
  for (int i = nb - 1; i >= 0; i--) {
    double v = 0.0;
    const int rr = i + 1 + tid;
    if (rr < nb) {  // two partial sums: the chain is half as long
      double v1 = 0.0;
      int s2 = i + 1;
      for (; s2 + 1 <= rr; s2 += 2) {
        v = fma(G[s2 * nb + rr], G[i * nb + s2], v);
        v1 = fma(G[(s2 + 1) * nb + rr], G[i * nb + s2 + 1], v1);
      }
      if (s2 <= rr) v = fma(G[s2 * nb + rr], G[i * nb + s2], v);
      v = -taus[i] * (v + v1);
    }
    __syncthreads();
    if (rr < nb) G[i * nb + rr] = v;
    if (tid == 0) G[i * nb + i] = taus[i];
    __syncthreads();
  }
  for (int idx = tid; idx < nb * nb; idx += NTHREADS) {
    const int a = idx % nb, b = idx / nb;
    Tg[(int64_t)b * ldt + a] = (a >= b) ? G[idx] : 0.0;
  }
  QL_STAMP(4);
}

// ------------------------------------------------------- solve vectors
// Vector operations of the triangular solve sweep (T_VEC, sub-operation
// aux[0], nrhs = t.n right-hand sides).  Bp / x_k live at operand a or c
// with leading dimension n; the per-front vector updates u_k (na x nrhs,
// ld na) start at WS + b.off + vpos[k] * nrhs.
__device__ void run_vec(const RunArgs& ra, const Task& t, double* smem) {
  const int mode = t.aux[0], nrhs = t.n;
  if (mode == VEC_GATHER || mode == VEC_SCATTER) {
    const int r0 = t.aux[1], r1 = t.aux[2];
    double* __restrict__ Bp = ra.bases[t.c.base] + t.c.off;
    const int ldp = t.c.ld;
    double* __restrict__ Bu = ra.bases[B_RHS];
    const int64_t ldb = ra.ldb;
    const int rows = r1 - r0;
    for (int base = 0; base < rows * nrhs; base += 4 * NTHREADS) {
      double v[4];
      int64_t src[4];
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int idx = base + threadIdx.x + e * NTHREADS;
        const int i = r0 + idx % max(rows, 1), j = idx / max(rows, 1);
        src[e] = (idx < rows * nrhs) ? __ldg(ra.perm + i) + (int64_t)j * ldb : -1;
        if (mode == VEC_GATHER) v[e] = (src[e] >= 0) ? ra.alpha * __ldcg(Bu + src[e]) : 0.0;
        else v[e] = (src[e] >= 0) ? __ldcg(Bp + i + (int64_t)j * ldp) : 0.0;
      }
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int idx = base + threadIdx.x + e * NTHREADS;
        const int i = r0 + idx % max(rows, 1), j = idx / max(rows, 1);
        if (src[e] < 0) continue;
        if (mode == VEC_GATHER) Bp[i + (int64_t)j * ldp] = v[e];
        else Bu[src[e]] = v[e];
      }
    }
    return;
  }
  double* __restrict__ WS = ra.bases[B_WS];
  const int64_t vbase = t.b.off;
  // right-hand-side columns [j0, j1) of this task (aux[3] == 0: all)
  const int j0 = t.aux[2], j1 = t.aux[3] > 0 ? t.aux[3] : nrhs, nc = j1 - j0;
  constexpr int E = 8;  // elements per thread with their loads in flight together
  if (mode == VEC_ASM) {
    const FrontDesc f = ra.fronts[t.aux[1]];
    double* __restrict__ xk = ra.bases[t.a.base] + t.a.off;
    const int ldx = t.a.ld;
    double* __restrict__ uk = ra.bases[t.c.base] + t.c.off;
    const int nj = f.nj;
    if ((int64_t)nj * nc <= ENGINE_SMEM_BASE_DOUBLES) {
      // [x_k; u_k] columns staged in shared memory (u_k part zero), the
      // children added there, the result stored once
      for (int base = 0; base < nj * nc; base += E * NTHREADS) {
        double v[E];
#pragma unroll
        for (int e = 0; e < E; e++) {
          const int idx = base + threadIdx.x + e * NTHREADS;
          const int i = idx % nj, j = j0 + idx / nj;
          v[e] = (idx < nj * nc && i < f.nn) ? __ldcg(xk + i + (int64_t)j * ldx) : 0.0;
        }
#pragma unroll
        for (int e = 0; e < E; e++) {
          const int idx = base + threadIdx.x + e * NTHREADS;
          if (idx < nj * nc) smem[idx] = v[e];
        }
      }
      __syncthreads();
      for (int l = f.chend - 1; l >= f.chbeg; l--) {
        const FrontDesc ch = ra.fronts[ra.chidx[l]];
        const int Nc = ch.na, tot = Nc * nc;
        const int32_t* __restrict__ r = ra.relidx + ch.relptr;
        const double* __restrict__ uc = WS + vbase + ch.vpos * nrhs + (int64_t)j0 * Nc;
        for (int base = 0; base < tot; base += E * NTHREADS) {
          int dst[E];
          double v[E];
#pragma unroll
          for (int e = 0; e < E; e++) {
            const int idx = base + threadIdx.x + e * NTHREADS;
            const int i = idx % max(Nc, 1), j = idx / max(Nc, 1);
            dst[e] = (idx < tot) ? __ldg(r + i) + j * nj : -1;
            v[e] = (idx < tot) ? __ldcg(uc + idx) : 0.0;
          }
          // a child's relative indices are distinct: no two elements of one
          // pass meet in shared memory
#pragma unroll
          for (int e = 0; e < E; e++)
            if (dst[e] >= 0) smem[dst[e]] += v[e];
        }
        __syncthreads();
      }
      for (int idx = threadIdx.x; idx < nj * nc; idx += NTHREADS) {
        const int i = idx % nj, j = j0 + idx / nj;
        if (i < f.nn) xk[i + (int64_t)j * ldx] = smem[idx];
        else uk[(i - f.nn) + (int64_t)j * f.na] = smem[idx];
      }
      return;
    }
    // too tall for shared memory: zero u_k's columns, add in global memory
    for (int idx = threadIdx.x; idx < f.na * nc; idx += NTHREADS)
      uk[(idx % f.na) + (int64_t)(j0 + idx / f.na) * f.na] = 0.0;
    __syncthreads();
    for (int l = f.chend - 1; l >= f.chbeg; l--) {
      const FrontDesc ch = ra.fronts[ra.chidx[l]];
      const int Nc = ch.na, tot = Nc * nc;
      const int32_t* __restrict__ r = ra.relidx + ch.relptr;
      const double* __restrict__ uc = WS + vbase + ch.vpos * nrhs + (int64_t)j0 * Nc;
      for (int base = 0; base < tot; base += E * NTHREADS) {
        double* dst[E];
        double v[E], old[E];
#pragma unroll
        for (int e = 0; e < E; e++) {
          const int idx = base + threadIdx.x + e * NTHREADS;
          const int i = idx % max(Nc, 1), j = j0 + idx / max(Nc, 1);
          dst[e] = nullptr;
          v[e] = 0.0;
          if (idx < tot) {
            const int row = __ldg(r + i);
            dst[e] = (row < f.nn) ? xk + row + (int64_t)j * ldx : uk + (row - f.nn) + (int64_t)j * f.na;
            v[e] = __ldcg(uc + idx);
          }
        }
#pragma unroll
        for (int e = 0; e < E; e++) old[e] = dst[e] ? __ldcg(dst[e]) : 0.0;
#pragma unroll
        for (int e = 0; e < E; e++)
          if (dst[e]) *dst[e] = old[e] + v[e];
      }
      __syncthreads();
    }
    return;
  }
  if (mode == VEC_ZERO) {
    double* __restrict__ z = ra.bases[t.c.base] + t.c.off;
    const int64_t cnt = (int64_t)t.m * t.n;
    for (int64_t i = threadIdx.x; i < cnt; i += NTHREADS) z[i] = 0.0;
    return;
  }
  // VEC_EXTRACT / VEC_ADD for child aux1 of the front p described by
  // operands a (x_p) and c (u_p): rows [i0, i1) of u_c, columns [j0, j1)
  const FrontDesc ch = ra.fronts[t.aux[1]];
  const FrontDesc f = ra.fronts[ch.parent];
  double* __restrict__ xp = ra.bases[t.a.base] + t.a.off;
  const int ldx = t.a.ld;
  double* __restrict__ up = ra.bases[t.c.base] + t.c.off;
  const int Nc = ch.na;
  const int i0 = t.m, i1 = t.k > 0 ? t.k : Nc, ni = max(i1 - i0, 0), tot = ni * nc;
  const int32_t* __restrict__ r = ra.relidx + ch.relptr;
  double* __restrict__ uc = WS + vbase + ch.vpos * nrhs;
  for (int base = 0; base < tot; base += E * NTHREADS) {
    int row[E], ui[E];
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int idx = base + threadIdx.x + e * NTHREADS;
      const int i = i0 + idx % max(ni, 1), j = j0 + idx / max(ni, 1);
      row[e] = (idx < tot) ? __ldg(r + i) : -1;
      ui[e] = i + j * Nc;
    }
    if (mode == VEC_ADD) {
      // rows of one child are distinct, but other children add into the
      // same rows at the same time: atomic adds
      double v[E];
#pragma unroll
      for (int e = 0; e < E; e++) v[e] = row[e] >= 0 ? __ldcg(uc + ui[e]) : 0.0;
#pragma unroll
      for (int e = 0; e < E; e++) {
        if (row[e] < 0) continue;
        const int j = j0 + (base + threadIdx.x + e * NTHREADS) / max(ni, 1);
        double* dst = row[e] < f.nn ? xp + row[e] + (int64_t)j * ldx : up + (row[e] - f.nn) + (int64_t)j * f.na;
        atomicAdd(dst, v[e]);
      }
      continue;
    }
    double v[E];
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int j = j0 + (base + threadIdx.x + e * NTHREADS) / max(ni, 1);
      v[e] = row[e] < 0 ? 0.0
                        : (row[e] < f.nn ? __ldcg(xp + row[e] + (int64_t)j * ldx)
                                         : __ldcg(up + (row[e] - f.nn) + (int64_t)j * f.na));
    }
#pragma unroll
    for (int e = 0; e < E; e++)
      if (row[e] >= 0) uc[ui[e]] = v[e];
  }
}

// ---------------------------------------------------------------- kernel
// ------------------------------------------------------------ bundles
// Small-subtree bundles.  A T_SUBTREE / T_PSUBTREE task carries up to four
// ranges of supernodes, one per warp: warp w owns [aux[w], bundle_last(t, w)]
// (aux[w] < 0: idle).  Each range is a union of complete subtrees,
// contiguous in postorder, whose fronts all have nj <= SUB_NJ, so a range
// needs nothing from outside but, for projected_inverse, its roots' V_k.
// The warp processes its fronts alone (cholesky in postorder, projected
// inverse parents first), one row of the front per lane, in its own
// shared-memory matrices (row-major, stride SUB_LD).  The update matrices
// inside a range pass through the workspace at their usual offsets and are
// written and read by the same warp (ordered by __syncwarp); the parents of
// a range's roots wait on the whole task.  Arithmetic and summation orders
// are those of the one-front tasks (T_FRONT / T_PFRONT).
__device__ __forceinline__ int bundle_last(const Task& t, int w) {
  return w == 0 ? t.m : w == 1 ? t.n : w == 2 ? t.k : t.cdiag;
}

// cholesky.c:33-72 for one front of at most SUB_NJ rows, by one warp.
__device__ void chol_front_warp(const RunArgs& ra, int k, double* F, int lane) {
  const FrontDesc f = ra.fronts[k];
  const int nn = f.nn, na = f.na, nj = f.nj;
  double* __restrict__ X = ra.bases[B_X] + f.blk;
  double* __restrict__ W = ra.bases[B_WS];
  double* row = F + lane * SUB_LD;
  if (lane < nj)
    for (int c = 0; c < nj; c++) row[c] = (c < nn && lane >= c) ? __ldcg(X + (int64_t)c * nj + lane) : 0.0;
  __syncwarp();
  // extend-add, children last to first (the reference's stack order)
  for (int l = f.chend - 1; l >= f.chbeg; l--) {
    const FrontDesc ch = ra.fronts[ra.chidx[l]];
    const int Nc = ch.na;
    const int32_t* __restrict__ rr = ra.relidx + ch.relptr;
    const double* __restrict__ Uc = W + ch.upd;
    if (lane < Nc) {
      double* dst = F + __ldg(rr + lane) * SUB_LD;
      for (int q = 0; q <= lane; q++) dst[__ldg(rr + q)] += __ldcg(Uc + (int64_t)q * Nc + lane);
    }
    __syncwarp();
  }
  // partial Cholesky of the nn pivot columns; the trailing block becomes U_k
  int first_bad = -1;
  for (int j = 0; j < nn; j++) {
    const double d = F[j * SUB_LD + j];
    const bool bad = !(d > 0.0);
    if (bad && first_bad < 0) first_bad = j;
    const double lj = sqrt(bad ? 1.0 : d), rl = 1.0 / lj;
    double a = 0.0;
    if (lane > j && lane < nj) {
      a = row[j] * rl;
      row[j] = a;
    }
    __syncwarp();
    if (lane == j) row[j] = lj;
    if (lane > j && lane < nj)
      for (int c = j + 1; c <= lane; c++) row[c] -= a * F[c * SUB_LD + j];
    __syncwarp();
  }
  if (lane == 0 && first_bad >= 0) atomicCAS(&ra.ctl[2], 0, first_bad + 1);
  // separator rows: L21 L11^{-1}, the reference's off-diagonal layout (:72)
  if (lane >= nn && lane < nj)
    for (int j = nn - 1; j >= 0; j--) {
      double v = row[j];
      for (int l2 = j + 1; l2 < nn; l2++) v -= row[l2] * F[l2 * SUB_LD + j];
      row[j] = v / F[j * SUB_LD + j];
    }
  __syncwarp();
  for (int c = 0; c < nn; c++)
    if (lane >= c && lane < nj) X[(int64_t)c * nj + lane] = row[c];
  double* __restrict__ U = W + f.upd;
  for (int q = 0; q < na; q++)
    if (lane >= nn + q && lane < nj) U[(int64_t)q * na + (lane - nn)] = row[nn + q];
  __syncwarp();
}

// projected_inverse.c:33-73 for one front of at most SUB_NJ rows, by one
// warp: G holds L11, then M = L11^{-1}, then S21; F holds [W, V_k], then
// [Y11; S21 | V_k].
__device__ void pinv_front_warp(const RunArgs& ra, int k, double* G, double* F, int lane) {
  const FrontDesc f = ra.fronts[k];
  const int nn = f.nn, na = f.na, nj = f.nj;
  double* __restrict__ X = ra.bases[B_X] + f.blk;
  double* __restrict__ W = ra.bases[B_WS];
  const double* __restrict__ V = W + f.upd;
  if (lane < nj)
    for (int c = 0; c < nn; c++) {
      const double v = __ldcg(X + (int64_t)c * nj + lane);
      if (lane < nn) G[lane * SUB_LD + c] = (lane >= c) ? v : 0.0;
      else F[lane * SUB_LD + c] = v;
    }
  if (lane < na)
    for (int q = 0; q <= lane; q++) F[(nn + lane) * SUB_LD + nn + q] = __ldcg(V + (int64_t)q * na + lane);
  __syncwarp();
  // M = L11^{-1} in place, columns last to first
  int first_bad = -1;
  for (int j = nn - 1; j >= 0; j--) {
    const double d = G[j * SUB_LD + j];
    if (d == 0.0 && first_bad < 0) first_bad = j;
    const double ajj = 1.0 / (d == 0.0 ? 1.0 : d);
    double ti = 0.0;
    if (lane > j && lane < nn)
      for (int l = j + 1; l <= lane; l++) ti = fma(G[lane * SUB_LD + l], G[l * SUB_LD + j], ti);
    __syncwarp();
    if (lane > j && lane < nn) G[lane * SUB_LD + j] = -ajj * ti;
    if (lane == j) G[j * SUB_LD + j] = ajj;
    __syncwarp();
  }
  if (lane == 0 && first_bad >= 0) atomicCAS(&ra.ctl[2], 0, first_bad + 1);
  // Y11 = M^T M (lower part), rows < nn of F
  if (lane < nn)
    for (int j = 0; j <= lane; j++) {
      double v = 0.0;
      for (int l = lane; l < nn; l++) v = fma(G[l * SUB_LD + lane], G[l * SUB_LD + j], v);
      F[lane * SUB_LD + j] = v;
    }
  __syncwarp();
  if (na > 0) {
    // S21 = -V_k W (V_k read as symmetric from its lower part) into G
    if (lane < na)
      for (int j = 0; j < nn; j++) {
        double v = 0.0;
        for (int l = 0; l < na; l++) {
          const double vil = (lane >= l) ? F[(nn + lane) * SUB_LD + nn + l] : F[(nn + l) * SUB_LD + nn + lane];
          v = fma(vil, F[(nn + l) * SUB_LD + j], v);
        }
        G[lane * SUB_LD + j] = -v;
      }
    __syncwarp();
    // Y11 -= S21^T W
    if (lane < nn)
      for (int j = 0; j <= lane; j++) {
        double v = 0.0;
        for (int l = 0; l < na; l++) v = fma(G[l * SUB_LD + lane], F[(nn + l) * SUB_LD + j], v);
        F[lane * SUB_LD + j] -= v;
      }
    __syncwarp();
    if (lane < na)
      for (int j = 0; j < nn; j++) F[(nn + lane) * SUB_LD + j] = G[lane * SUB_LD + j];
    __syncwarp();
  }
  // the children's updates F(r_c, r_c), lower parts
  for (int l = f.chbeg; l < f.chend; l++) {
    const FrontDesc ch = ra.fronts[ra.chidx[l]];
    const int Nc = ch.na;
    const int32_t* __restrict__ rr = ra.relidx + ch.relptr;
    double* __restrict__ Uc = W + ch.upd;
    if (lane < Nc) {
      const double* src = F + __ldg(rr + lane) * SUB_LD;
      for (int q = 0; q <= lane; q++) Uc[(int64_t)q * Nc + lane] = src[__ldg(rr + q)];
    }
  }
  for (int c = 0; c < nn; c++)
    if (lane < nj) X[(int64_t)c * nj + lane] = (lane < nn && lane < c) ? 0.0 : F[lane * SUB_LD + c];
  __syncwarp();
}

__device__ void run_subtrees(const RunArgs& ra, const Task& t, double* smem) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int lo = t.aux[warp];
  if (lo < 0) return;
  const int hi = bundle_last(t, warp);
  if (t.op == T_SUBTREE) {
    double* F = smem + warp * SUB_NJ * SUB_LD;
    for (int k = lo; k <= hi; k++) chol_front_warp(ra, k, F, lane);
  } else {
    double* G = smem + warp * 2 * SUB_NJ * SUB_LD;
    for (int k = hi; k >= lo; k--) pinv_front_warp(ra, k, G, G + SUB_NJ * SUB_LD, lane);
  }
}

static_assert(NTHREADS == 128, "a bundle has one range per warp of a 4-warp CTA");
static_assert(8 * SUB_NJ * SUB_LD <= ENGINE_SMEM_BASE_DOUBLES, "bundle fronts exceed the engine's shared memory");

// TC: the instantiation launched for programs with TF32 tiles, which run on
// tcgen05 with tensor memory; the other one contains no tcgen05 code at all
// (with that code present, a launch of the FP64 sweeps measured 17-60 %
// slower at 40^3, although no tcgen05 instruction ran).
template <bool TC>
__global__ void __launch_bounds__(NTHREADS, 2) engine_kernel(RunArgs ra) {
  extern __shared__ double smem[];
  __shared__ int s_task;
  __shared__ int s_abort;
  __shared__ int s_next;      // dynamic: the waiter this CTA released and runs next, or -1
  __shared__ int s_succ[2];   // dynamic: waiter range of the current task
  __shared__ int s_pre[32];   // dynamic: its first 32 waiters (cp.async during the task)
  __shared__ __align__(16) Task s_t;
  static_assert(sizeof(Task) == 36 * 4, "task record is 36 words");
  SmemLayout sm{smem, smem + TILE * LDS};
  __shared__ int s_lo;        // dynamic: this CTA's copy of the finished frontier
  __shared__ uint32_t s_tmem;                 // tensor-memory base of the TF32 tiles
  __shared__ __align__(8) uint64_t s_mbar[2]; // their MMA-completion barriers
  if (threadIdx.x == 0) {
    s_next = -1;
    s_lo = 0;
  }
  TcState ts;
  ts.mbar = s_mbar;
  ts.ncommit[0] = ts.ncommit[1] = 0;
  ts.tmem = 0;
  if (TC) {
    // 64 columns of tensor memory (a 64 x 64 FP32 accumulator) for the
    // whole launch: two CTAs per SM take 128 of the 512 columns
    if (threadIdx.x < 32) {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 64;" ::"r"(smem_u32(&s_tmem))
                   : "memory");
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
      mbar_init(&s_mbar[0]);
      mbar_init(&s_mbar[1]);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    ts.tmem = s_tmem;
  }
  for (;;) {
    if (ra.dynamic) {
      // warp 0: the next task (handed over by the last one, or claimed), its
      // record and waiter range in one round of loads, its first waiters
      // prefetched asynchronously
      if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        __syncwarp();
        const unsigned long long t0 = ra.trace ? global_ns() : 0ull;
        int c = s_next;
        if (c < 0) c = claim_task(ra, &s_lo);
        if (c < ra.ntasks) {
          const uint32_t* src = reinterpret_cast<const uint32_t*>(ra.tasks + c);
          uint32_t* dst = reinterpret_cast<uint32_t*>(&s_t);
          const uint32_t v0 = __ldg(src + lane);
          const uint32_t v1 = lane < 4 ? __ldg(src + 32 + lane) : 0u;
          const int so = (lane == 4 || lane == 5) ? __ldg(ra.succ_off + c + lane - 4) : 0;
          dst[lane] = v0;
          if (lane < 4) dst[32 + lane] = v1;
          const int b = __shfl_sync(0xffffffffu, so, 4), e = __shfl_sync(0xffffffffu, so, 5);
          if (lane == 0) {
            s_succ[0] = b;
            s_succ[1] = e;
          }
          if (lane < e - b) cp_async4(&s_pre[lane], ra.succ + b + lane);
          cp_async_commit();
          if (lane == 0 && ra.trace) {
            ra.trace[4 * (int64_t)c] = t0;
            ra.trace[4 * (int64_t)c + 1] = global_ns();
          }
        }
        if (lane == 0) s_task = c;
      }
      __syncthreads();
      if (s_task >= ra.ntasks) break;
    } else {
      if (threadIdx.x == 0) s_task = atomicAdd(&ra.ctl[0], 1);
      __syncthreads();
      const int ti = s_task;
      if (ti >= ra.ntasks) break;
      {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(ra.tasks + ti);
        uint32_t* dst = reinterpret_cast<uint32_t*>(&s_t);
        for (int w = threadIdx.x; w < 36; w += NTHREADS) dst[w] = __ldg(src + w);
      }
      __syncthreads();
      if (threadIdx.x < 32) {
        // the task's waits, one per lane of warp 0 (32 at a time), so that
        // the wait records and the counters are read in one round each
        const int lane = threadIdx.x;
        if (lane == 0 && ra.trace) ra.trace[4 * (int64_t)ti] = global_ns();
        int abort = 0, timed_out = 0;
        const int npre = ((s_t.op == T_POTRF && s_t.k > 0) || s_t.op == T_TRSV) ? (int)s_t.cdiag : (int)s_t.nwait;
        for (int w0 = 0; w0 < npre; w0 += 32) {
          if (w0 + lane < npre) {
            const int2 wt = ra.waits[s_t.wait_off + w0 + lane];
            int64_t spins = 0;
            unsigned ns = 16;
            while (ld_acquire(ra.counters + wt.x) < wt.y) {
              if (++spins > ra.spin_limit) {
                atomicCAS(&ra.ctl[1], 0, DE_TIMEOUT);
                abort = timed_out = 1;
                break;
              }
              if ((spins & 15) == 0 && ld_volatile(&ra.ctl[1]) != 0) { abort = 1; break; }
              __nanosleep(ns);
              if (ns < 128) ns <<= 1;
            }
          }
          if (__any_sync(0xffffffffu, abort)) {
            abort = 1;
            break;
          }
        }
        timed_out = __any_sync(0xffffffffu, timed_out);
        if (lane == 0) {
          if (timed_out) atomicAdd(&ra.ctl[3], 1);  // CTAs whose wait ran out
          if (!abort && ld_volatile(&ra.ctl[1]) != 0) abort = 1;
          s_abort = abort;
          if (ra.trace) ra.trace[4 * (int64_t)ti + 1] = global_ns();
        }
      }
      __syncthreads();
      if (s_abort) break;
    }
    const int ti = s_task;
    const Task& t = s_t;
    switch (t.op) {
      case T_GEMM:
      case T_LA: run_gemm_or_la<TC>(ra, t, sm, ts); break;
      case T_MROW: run_mrow(ra, t, sm); break;
      case T_POTRF: run_potrf(ra, t, smem, ti); break;
      case T_ASM: run_asm(ra, t, smem); break;
      case T_FRONT: run_front(ra, t, smem); break;
      case T_PFRONT: run_pfront(ra, t, smem); break;
      case T_SUBTREE:
      case T_PSUBTREE: run_subtrees(ra, t, smem); break;
      case T_EXTRACT: run_extract(ra, t, smem); break;
      case T_COPY: run_copy(ra, t); break;
      case T_VEC: run_vec(ra, t, smem); break;
      case T_TRSV: run_trsv(ra, t, smem); break;
      case T_QL: run_ql(ra, t, smem); break;
      case T_NOP: break;
      case T_SUM: run_sum(ra, t); break;
      case T_SIGNAL:
        if (threadIdx.x == 0 && t.aux[0] >= 0 && t.aux[0] < ra.nio_out) raise_io_flag(ra.io_out + t.aux[0]);
        break;
      case T_ARRIVAL:
        if (threadIdx.x == 0) wait_arrival(ra, t.aux[0]);
        break;
      default:
        if (threadIdx.x == 0) atomicCAS(&ra.ctl[1], 0, DE_BAD_TASK);
        break;
    }
    __syncthreads();
    if (threadIdx.x == 0 && ra.trace) {
      ra.trace[4 * (int64_t)ti + 2] = global_ns();
      ra.trace[4 * (int64_t)ti + 3] = (unsigned long long)sm_id() | ((unsigned long long)t.op << 32);
    }
    if (!ra.dynamic) {
      if (threadIdx.x == 0) {
        red_release_add(ra.counters + ti, 1);
        if (t.group >= 0) red_release_add(ra.counters + t.group, 1);
      }
    } else if (threadIdx.x < 32) {
      const int nx = finish_task(ra, ti, t.group, s_succ[0], s_succ[1], s_pre, t.op == T_POTRF && t.k > 0);
      if (threadIdx.x == 0) s_next = nx;
    }
  }
  if (ra.nio_out > 0) {
    // the last CTA to leave raises every output flag (already raised after a
    // complete sweep; after an aborted one the waiting copies still proceed)
    __syncthreads();
    if (threadIdx.x == 0 && atomicAdd(&ra.ctl[6], 1) == (int)gridDim.x - 1)
      for (int j = 0; j < ra.nio_out; j++) raise_io_flag(ra.io_out + j);
  }
  if (TC) {
    // every tile waited for its last commit, so no MMA is in flight
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (threadIdx.x < 32)
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 64;" ::"r"(ts.tmem) : "memory");
  }
}

static_assert(2 * TILE * LDS <= ENGINE_SMEM_BASE_DOUBLES, "GEMM staging exceeds the engine's shared memory");
static_assert(GEMM_STAGES * STAGE_DOUBLES <= ENGINE_SMEM_BASE_DOUBLES, "GEMM ring exceeds the engine's shared memory");
static_assert(POTRF_SMEM_DOUBLES <= ENGINE_SMEM_BASE_DOUBLES, "POTRF exceeds the engine's shared memory");

#ifdef CHB_PROFILE_POTRF
// Development builds only: copies out (and optionally clears) the diagonal
// task's phase counters.
extern "C" int chb_dev_potrf_phase(unsigned long long* out, int clear) {
  cudaError_t e = cudaMemcpyFromSymbol(out, g_potrf_phase, sizeof(g_potrf_phase));
  if (e == cudaSuccess && clear) {
    static const unsigned long long zero[32] = {};
    e = cudaMemcpyToSymbol(g_potrf_phase, zero, sizeof(zero));
  }
  return (int)e;
}
#endif

size_t engine_smem_bytes() { return (size_t)ENGINE_SMEM_DOUBLES * sizeof(double); }

// The dynamic shared-memory attribute must have been raised on the current
// device by engine_occupancy() (done when a plan is created).  The launch
// uses ra.smem_doubles (at least the GEMM/POTRF staging).
cudaError_t engine_launch(const RunArgs& ra, int grid, cudaStream_t stream) {
  if (ra.smem_doubles < ENGINE_SMEM_BASE_DOUBLES || ra.smem_doubles > ENGINE_SMEM_DOUBLES) return cudaErrorInvalidValue;
  // the tcgen05 build is sized (engine_occupancy) for the base staging only
  if (ra.tmem && ra.smem_doubles != ENGINE_SMEM_BASE_DOUBLES) return cudaErrorInvalidValue;
  size_t smem = (size_t)ra.smem_doubles * sizeof(double);
  if (ra.tmem) engine_kernel<true><<<grid, NTHREADS, smem, stream>>>(ra);
  else engine_kernel<false><<<grid, NTHREADS, smem, stream>>>(ra);
  return cudaGetLastError();
}

// Resident CTAs per SM of one instantiation (tc: the tcgen05 one).  The
// dynamic shared-memory attribute is raised on both.  The FP64 build is
// sized for the largest staging (Householder panels, solve steps); the
// tcgen05 build only runs the TF32 sweeps, which launch with the base
// staging, and is queried at that size (the query still reports one CTA per
// SM for it; the plan launches it as wide as the FP64 build, see
// upload_plan).
int engine_occupancy(int* blocks_per_sm, bool tc) {
  size_t smem = engine_smem_bytes();
  cudaError_t e = cudaFuncSetAttribute(engine_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(engine_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return -1;
  const size_t smem_tc = (size_t)ENGINE_SMEM_BASE_DOUBLES * sizeof(double);
  e = tc ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, engine_kernel<true>, NTHREADS, smem_tc)
         : cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, engine_kernel<false>, NTHREADS, smem);
  return e == cudaSuccess ? 0 : -1;
}

}  // namespace chb
