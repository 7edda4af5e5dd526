// Host-side plan: uploaded symbolic data, workspace layout and the compiled
// task programs of each sweep.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>

#include "../../include/chompack_b200.h"
#include <memory>
#include <vector>

#include "engine.h"

struct chb_plan;

namespace chb {

// Streaming of the values between host and device while a sweep runs.
// With `in`, the values are copied in chunks of whole supernodes, and every
// task that touches incoming chunk j waits for a T_ARRIVAL task that waits
// for the flag the copy stream raises after the chunk's copy.  With `out`, a
// T_SIGNAL task per outgoing chunk raises a host-visible flag once every
// task whose writes overlap the chunk has finished; outgoing chunks may cut
// a large supernode between tile columns, so that its leading columns go
// out while the rest is still being computed.
struct IoSpec {
  bool in = false, out = false;
  std::vector<int64_t> in_off;    // value offsets of the incoming chunks (chunks + 1): whole supernodes
  std::vector<double> arrive_us;  // estimated arrival of each incoming chunk (list order only)
  std::vector<int64_t> out_off;   // outgoing chunks: large supernodes split at 64-column boundaries
  std::vector<int> in_order;      // order of the incoming copies (set by DagBuilder::finish)
};

struct Program {
  std::vector<Task> tasks;
  std::vector<int2> waits;
  int64_t ncounters = 0;   // tasks + groups
  int64_t ws_doubles = 0;  // doubles of workspace (update matrices + scratch)
  int smem_doubles = ENGINE_SMEM_BASE_DOUBLES;  // dynamic shared memory per CTA
  bool static_default = false;  // list order unless the plan asks otherwise
  bool tf32_tiles = false;      // some GEMM tile computes in TF32 (one product)
  IoSpec io;                    // streaming of the values (set before building)
  std::vector<int> out_order;   // chunks in the list order of their signals
  // Own layout of the update matrices (a scratch limit): the supernode
  // descriptors with this program's update-matrix offsets (empty: the
  // plan's), the pool's size and the reuse waits it took.
  std::vector<FrontDesc> fronts;
  FrontDesc* d_fronts = nullptr;
  int64_t pool_doubles = 0;
  int64_t pool_waits = 0;
  double sim_span_us = 0.0;  // span of the simulated list schedule that ordered the tasks
  Task* d_tasks = nullptr;
  int2* d_waits = nullptr;
  // dynamic scheduling data (filled by DagBuilder::finish)
  std::vector<int> npend;                 // waits per task
  std::vector<int> succ_off, succ;        // waiters per counter (CSR)
  std::vector<int> ctarget;               // completion value per counter
  std::vector<unsigned long long> ready0, summ0;  // initially ready tasks
  int* d_npend = nullptr;
  int* d_succ_off = nullptr;
  int* d_succ = nullptr;
  int* d_ctarget = nullptr;
  unsigned long long* d_ready0 = nullptr;
  unsigned long long* d_summ0 = nullptr;
  ~Program();
};

// Byte layout of a caller workspace for one program:
//   [0, 256)                 control words (queue head, error, info, ...)
//   [256, counters_end)      task / group counters (int32)
//   [dbl_off, ...)           doubles: update matrices, then program scratch
struct WsLayout {
  size_t counters_off;
  size_t pend_off, ready_off, summ_off, wcl_off;  // dynamic scheduling state
  size_t dbl_off;
  size_t total;
};
WsLayout ws_layout(const Program& p);

// Key of a program in the plan's cache.
struct ProgKey {
  int op;
  int64_t k;
  int flags;
  bool operator<(const ProgKey& o) const {
    if (op != o.op) return op < o.op;
    if (k != o.k) return k < o.k;
    return flags < o.flags;
  }
};

}  // namespace chb

struct chb_plan {
  int device = 0;
  int64_t n = 0, nsn = 0;
  std::vector<chb::FrontDesc> fronts;  // host copy (upd = offset of U_k)
  std::vector<int32_t> relidx, chidx, snpar, level;
  std::vector<int64_t> snptr, snode, perm;
  int64_t blk_total = 0;
  int64_t upd_total = 0;   // sum of na^2
  int nlevels = 0;
  chb::FrontDesc* d_fronts = nullptr;
  int32_t* d_relidx = nullptr;
  int32_t* d_chidx = nullptr;
  int64_t* d_perm = nullptr;    // p (trsm row gather)
  int64_t* d_iperm = nullptr;   // inverse of p (sparse assembly)
  std::vector<int64_t> seg;     // matrices of a merged plan: supernodes [seg[m], seg[m+1])
  int64_t* d_seg = nullptr;
  int2* d_symv_items = nullptr;  // 64-row strips of the supernode blocks (supernode, first row)
  int n_symv_items = 0;
  int grid = 0;                 // persistent grid size (the FP64 instantiation)
  int grid_tc = 0;              // persistent grid size of the tcgen05 instantiation
  int schedule = -1;            // -1 default (CHB_SCHEDULE, else per sweep), 0 dynamic, 1 static list order
  int64_t spin_limit = -1;      // polls before a wait gives up; -1: the default (kDefaultSpinLimit)
  int64_t opt[CHB_OPT_COUNT] = {-1, -1, -1, -1, -1, -1, -1, -1};  // program-build options (-1: default)
  unsigned long long* trace = nullptr;  // optional per-task timing buffer (device)
  int64_t trace_cap = 0;                // tasks it can hold
  std::map<chb::ProgKey, std::unique_ptr<chb::Program>> progs;
  // streaming of the values to and from host memory (created on first use);
  // outgoing chunks go round-robin over several streams, so that a chunk
  // that finishes later than predicted holds up only its own stream
  static constexpr int IO_OUT_STREAMS = 4;
  cudaStream_t io_in = nullptr, io_out[IO_OUT_STREAMS] = {};
  cudaEvent_t ev_start = nullptr, ev_in = nullptr, ev_out[IO_OUT_STREAMS] = {};
  int* h_one = nullptr;  // pinned 1, copied into an arrival counter after its chunk
};

namespace chb {
// Build (or fetch) the program of an operation.  Returns nullptr and sets
// the error text on failure.
Program* get_program(chb_plan* plan, int op, int64_t k, int flags);
// Host side only (no device upload).
Program* build_host_program(chb_plan* plan, int op, int64_t k, int flags);

// Host buffers of a streamed run (see IoSpec): host_in is copied into the
// values (bases[B_X]) chunk by chunk while the sweep runs, and each chunk
// of the result is copied to host_out as soon as it is final.
struct HostIo {
  const double* host_in = nullptr;
  double* host_out = nullptr;
};

// Program flags selecting the streamed variants (bits above the sweeps' own
// flags).
// Polls of a task's wait (with a back-off of up to ~1 us) before it gives
// up and the sweep ends with status -30: about 10 s.
constexpr int64_t kDefaultSpinLimit = 40000000LL;
constexpr int PF_IO_IN = 1 << 16;
constexpr int PF_IO_OUT = 1 << 17;
// Program flags selecting the mixed-precision variants of cholesky and
// projected_inverse: every GEMM task's product in TF32 (or 3xTF32) with
// FP32 accumulation; diagonal tiles, look-ahead steps and sums stay FP64.
constexpr int PF_TF32 = 1 << 18;
constexpr int PF_TF32X3 = 1 << 19;

// Launch a program.  bases: MAX_BASES device pointers (unused slots null).
int run_program(chb_plan* plan, Program* prog, void* work, size_t work_bytes, double* const* bases, int nbases,
                cudaStream_t stream, int64_t run_ldb = 0, double run_alpha = 1.0, const HostIo* io = nullptr);

// Device entry points implemented in engine.cu.
size_t engine_smem_bytes();
cudaError_t engine_launch(const RunArgs& ra, int grid, cudaStream_t stream);
int engine_occupancy(int* blocks_per_sm, bool tc = false);
cudaError_t logdet_launch(const double* l, const FrontDesc* fronts, int nsn, double* partial, double* out,
                          cudaStream_t stream);
cudaError_t symw_launch(const double* x, double* y, double alpha, const FrontDesc* fronts, int nsn,
                        cudaStream_t stream);
cudaError_t segment_sums(const double* partial, const int64_t* seg, int count, double* out, cudaStream_t stream);
cudaError_t symv_launch(const double* blkval, const FrontDesc* fronts, const int2* items, int nitems,
                        const int64_t* sncolptr, const int64_t* snrowidx, const int64_t* perm, const double* x,
                        double* y, int nrhs, int64_t ld, double alpha, cudaStream_t stream);
cudaError_t logdet_partials(const double* l, const FrontDesc* fronts, int nsn, double* partial, cudaStream_t stream);
cudaError_t dot_partials(const double* x, const double* y, const FrontDesc* fronts, int nsn, double* partial,
                         cudaStream_t stream);
cudaError_t dot_launch(const double* x, const double* y, const FrontDesc* fronts, int nsn, double* partial,
                       double* out, cudaStream_t stream);

// Program builders (one per sweep), in build_*.cpp.
int build_cholesky(const chb_plan& P, Program& prog);
int build_projected_inverse(const chb_plan& P, Program& prog);
int build_llt(const chb_plan& P, Program& prog);
int build_conventional(const chb_plan& P, Program& prog);
int build_completion(const chb_plan& P, Program& prog, bool factored);
// trsm flags: 1 trans 'T', 2 the step operands are already in the workspace
int build_trsm(const chb_plan& P, Program& prog, int64_t nrhs, bool trans, bool reuse = false);
int build_trmm(const chb_plan& P, Program& prog, int64_t nrhs, bool trans);
// flags: adj | inv << 1 | factored_updates << 2; nu U matrices in base slots
// B_U0 .. B_U0 + nu - 1.
int build_hessian(const chb_plan& P, Program& prog, int nu, int flags);
}  // namespace chb
