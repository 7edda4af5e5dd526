// Task-graph engine shared by the host planner (plan.cpp) and the device
// executor (engine.cu).
//
// Every numeric sweep is compiled on the host into a list of tile tasks in a
// topological order.  One persistent kernel executes the list: each CTA
// claims the next task with an atomic counter, waits (bounded) until the
// tasks it depends on have signalled, runs it, and signals.  A task only
// ever waits on tasks that come earlier in the list, so the smallest
// unfinished claimed task can always run: the schedule cannot deadlock,
// whatever the number of resident CTAs.
#pragma once
#include <cstdint>

#include <vector_types.h>  // int2

#ifdef __CUDACC__
#define CHB_HD __host__ __device__
#else
#define CHB_HD
#endif

namespace chb {

constexpr int TILE = 64;          // tile edge (rows/cols of a C tile)
constexpr int NTHREADS = 128;     // threads per CTA (4 warps)
// Fronts of a small-subtree bundle (T_SUBTREE / T_PSUBTREE) have at most
// SUB_NJ rows: one row per lane of the warp that owns the range.
constexpr int SUB_NJ = 32;
constexpr int SUB_LD = SUB_NJ + 1;     // row stride of a warp's shared-memory front
constexpr int KC = 16;            // K chunk staged through shared memory
constexpr int LDS = TILE + 4;     // padded leading dimension of staged tiles
constexpr int MAX_BASES = 64;     // base-pointer slots (see Base below)
// Dynamic shared memory of the persistent kernel (doubles).  GEMM and POTRF
// tasks need ENGINE_SMEM_BASE_DOUBLES (74 KB); programs with Householder
// panels launch with ENGINE_SMEM_DOUBLES (112 KB, so that two CTAs still fit
// an SM: 228 KB, 1 KB reserved per CTA).  The others keep the smaller
// carve-out, which leaves more L1 for the register spills.
constexpr int ENGINE_SMEM_BASE_DOUBLES = 9472;
constexpr int ENGINE_SMEM_DOUBLES = 14336;
// T_TRSV: the largest K, and the leading dimension of its staged operand;
// programs with such steps launch with ENGINE_SMEM_DOUBLES
constexpr int TRSV_KMAX = 192;
constexpr int TRSV_LA = TILE + 2;
static_assert(TRSV_KMAX * TRSV_LA + TRSV_KMAX * 8 <= ENGINE_SMEM_DOUBLES, "T_TRSV staging exceeds shared memory");
// Shared-memory doubles a Householder panel of h rows and nb columns needs
// (panel, then its nb x nb T factor, plus scalars).
CHB_HD constexpr int ql_panel_doubles(int h, int nb) { return h * nb + nb * nb + 192; }

// Base-pointer slots a task operand refers to.
enum Base : uint8_t {
  B_X = 0,      // the cspmatrix values being transformed in place
  B_WS = 1,     // the double-precision workspace
  B_L = 2,      // factor values (hessian)
  B_Y = 3,      // projected-inverse values (hessian)
  B_RHS = 4,    // dense right-hand sides (trsm)
  B_U0 = 5      // first of the U matrices (hessian): slot B_U0 + u
};

// How a GEMM operand is read.  A tile operand maps tile coordinates (r, k),
// r in [0, 64), k in [0, K), to an element of a column-major matrix with
// origin `off` and leading dimension `ld`.
enum OpMode : uint8_t {
  OM_N = 0,      // X[k*ld + r]
  OM_T = 1,      // X[r*ld + k]
  OM_TRI_N = 2,  // lower-triangular X read as OM_N: zero unless r + diag >= k
  OM_TRI_T = 3,  // lower-triangular X read as OM_T: zero unless k + diag >= r
  OM_SYM = 4     // symmetric X stored in its lower triangle: element (r+diag, k)
};

enum CMode : uint8_t {
  CM_FULL = 0,   // write the whole m x n tile
  CM_LOWER = 1,  // write only entries with r + cdiag >= c (lower triangle)
  CM_ATOMIC = 2  // C += alpha op(A) op(B)^T with atomic adds (beta is 1): tiles that several
                 // tasks update at once, in any order
};

enum TaskOp : uint8_t {
  T_GEMM = 0,     // C = alpha * opA * opB^T + beta * C
  T_POTRF = 1,    // Cholesky of a diagonal tile; optionally its inverse
  T_ASM = 2,      // extend-add of child update matrices into a front
  T_MROW = 3,     // C = alpha * M2 * (opA * opB^T); M2 lower-triangular tile
  T_EXTRACT = 4,  // gather a child's update matrix out of its parent front
  T_COPY = 5,     // strided copy / scale / zero of a tile
  T_INV = 6,      // inverse of a lower-triangular diagonal tile
  T_RPOTRF = 7,   // "reverse" Cholesky: S = L^T L with L lower (diag tile)
  T_QL = 8,       // blocked Householder QL of update_factor (sub-op aux[3])
  T_VEC = 9,      // vector ops for the triangular solve sweep
  T_NOP = 10,     // no work: joins dependencies
  T_LA = 11,      // Cholesky look-ahead: L = A21 M^T (early signal), A22 -= L L^T
  T_SUM = 12,     // C = alpha * sum of aux[0] partial tiles (stride aux[1]) + beta * C
  T_SIGNAL = 13,  // host-visible flag io_out[aux[0]] = 1 (a chunk of the values is final)
  T_ARRIVAL = 14, // waits (bounded) until the host's copy raised io_in[aux[0]] (a chunk arrived)
  T_FRONT = 15,   // a whole small cholesky front (nj <= TILE) in shared memory (front aux[0])
  T_PFRONT = 16,  // a whole small projected-inverse front (nj <= TILE) in shared memory (front aux[0])
  T_SUBTREE = 17, // cholesky of up to four ranges of small complete subtrees, one per warp (see bundle_last)
  T_PSUBTREE = 18, // projected_inverse of such ranges, one per warp, parents first
  T_TRSV = 19     // a block-substitution step C = alpha opA opB^T (+ beta C), m <= 64, K <= TRSV_KMAX:
                  // opA (independent of the chain) staged before the mid waits [cdiag, nwait)
};

// Sub-operations of T_QL (child aux[0], columns [aux[1], aux[2]) of the
// parent-update columns C = L_k(:, r[N1:] - nn)).
enum QlOp : int {
  QL_GATHER = 0,  // C(:, j) = L_k(:, jj_j), zero above row jj_j
  QL_PANEL = 1    // Householder reflections of the panel; W' and T factor
};

// Product precision of a GEMM task (its C operand's prec): FP64 tensor
// cores, or TF32 tensor cores with FP32 accumulation from the FP64 operands
// (one product, or three with a high/low split of each operand, which
// carries about 22 bits); the result is added to C in FP64.
enum Precision : int16_t { PREC_FP64 = 0, PREC_TF32 = 1, PREC_TF32X3 = 2 };

struct Operand {
  int64_t off;    // element offset from the base pointer
  int32_t ld;     // leading dimension
  uint8_t base;   // Base slot
  uint8_t mode;   // OpMode
  int16_t prec;   // C operand of T_GEMM: product precision (Precision); else 0
  int32_t diag;   // diagonal offset for OM_TRI_* / OM_SYM
  int32_t pad2;   // OM_SYM: column offset of k = 0
};

struct Task {
  uint8_t op;       // TaskOp
  uint8_t cmode;    // CMode (GEMM / MROW)
  uint16_t nwait;   // number of (counter, target) waits
  int32_t wait_off; // first wait in the waits array
  int32_t group;    // extra counter signalled on completion (-1: none)
  int32_t m, n, k;  // C tile extent and inner dimension
  int32_t cdiag;    // diagonal offset for CM_LOWER
  int32_t aux[4];   // op-specific integers (front id, column range, ...)
  double alpha, beta;
  Operand a, b, c;
  int64_t off2;     // op-specific offset (base of the update-matrix region for
                    // T_ASM / T_EXTRACT)
};

// Per-supernode description used by the gather/scatter tasks.
struct FrontDesc {
  int32_t nn, na, nj;   // |N_k|, |A_k|, nn + na
  int32_t relptr;       // first relative index of this supernode
  int32_t chbeg, chend; // children are chidx[chbeg:chend]
  int32_t parent;       // snpar
  int32_t level;        // height in the supernodal tree
  int64_t blk;          // blkptr[k]
  int64_t upd;          // offset (doubles) of the update matrix in the workspace
  int64_t col0;         // snptr[k]: first (reordered) column of the supernode
  int64_t vpos;         // sum of na over the preceding supernodes (vector updates)
};

// Device-side run description (passed by value to the persistent kernel).
struct RunArgs {
  const Task* tasks;
  int32_t ntasks;
  int32_t smem_doubles;   // dynamic shared memory of this launch (doubles)
  const int2* waits;
  int* counters;          // ntasks task counters, then group counters
  int* ctl;               // [0] queue head, [1] error code, [2] info, [3] timeouts
  double* bases[MAX_BASES];  // device base pointers, indexed by Base
  const FrontDesc* fronts;
  const int32_t* relidx;
  const int32_t* chidx;
  int64_t spin_limit;     // polls before a wait gives up
  const int64_t* perm;    // p (trsm gather/scatter)
  int64_t ldb;            // leading dimension of the right-hand sides (trsm)
  double alpha;           // scale applied by the trsm gather
  unsigned long long* trace;  // optional: 4 words per task (claim, start, end, sm | op << 32)
  // Dynamic scheduling (dynamic != 0): a finished task decrements the
  // pending counts of its successors (CSR succ_off / succ per counter) and
  // sets the ready bits of those that reach zero; CTAs claim the ready task
  // of lowest list position.  ctl[4] counts finished tasks, ctl[5] is the
  // first word of the ready bitmap that may hold an unclaimed task.
  int dynamic;
  int nwords;                     // ready-bitmap words (64 tasks each)
  int nsumm;                      // summary words (64 bitmap words each)
  int tmem;                       // 1: TF32 GEMM tiles run on tcgen05 (tensor memory allocated per CTA)
  int* pend;                      // unmet dependencies per task
  unsigned long long* ready;      // ready, unclaimed tasks
  unsigned long long* summ;       // nonzero ready words
  int* wclaimed;                  // claimed tasks per bitmap word
  const int* succ_off;            // ncounters + 1
  const int* succ;
  const int* ctarget;             // value at which a counter is complete
  // Streamed output: T_SIGNAL raises io_out[chunk] (system scope) when a
  // chunk of the values is final; the last CTA to leave raises all nio_out
  // flags, so that copies waiting on them never wait on an aborted sweep.
  int* io_out;
  int nio_out;
  int nio_in;
  int* io_in;    // arrival flags, raised by the copies of the incoming chunks
};

// Sub-operations of T_VEC (triangular solve sweep).
enum VecOp : int {
  VEC_GATHER = 0,   // Bp[i, :] = alpha * B[p[i], :] for i in [aux1, aux2)
  VEC_SCATTER = 1,  // B[p[i], :] = Bp[i, :]
  VEC_ASM = 2,      // front aux1: zero u_k, add the children's updates into x_k / u_k
  VEC_EXTRACT = 3,  // child aux1: u_c = [x_p; u_p](r_c), rows [m, k) of u_c (k == 0: all)
  VEC_ADD = 4,      // child aux1: [x_p; u_p](r_c) += u_c with atomic adds, rows [m, k) of u_c
  VEC_ZERO = 5      // operand c: m * n doubles set to zero
};
// VEC_ASM, VEC_EXTRACT and VEC_ADD take the right-hand-side columns
// [aux2, aux3) (aux3 == 0: all n).

// Error codes written to ctl[1].
enum DeviceError : int {
  DE_NONE = 0,
  DE_TIMEOUT = 1,
  DE_BAD_TASK = 2
};

}  // namespace chb
