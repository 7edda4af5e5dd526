// Plan creation (symbolic upload), program cache and program launch.
#include "plan.h"
#include "dag.h"

#include <cstdlib>

#include <algorithm>
#include <cstring>

#include "../../include/chompack_b200.h"
#include "internal.h"

namespace chb {

Program::~Program() {
  if (d_tasks) cudaFree(d_tasks);
  if (d_waits) cudaFree(d_waits);
  if (d_npend) cudaFree(d_npend);
  if (d_succ_off) cudaFree(d_succ_off);
  if (d_succ) cudaFree(d_succ);
  if (d_ctarget) cudaFree(d_ctarget);
  if (d_ready0) cudaFree(d_ready0);
  if (d_summ0) cudaFree(d_summ0);
  if (d_fronts) cudaFree(d_fronts);
}

static size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

WsLayout ws_layout(const Program& p) {
  WsLayout L;
  L.counters_off = 256;
  const size_t nt = p.tasks.size(), nw = p.ready0.size(), ns = p.summ0.size();
  L.pend_off = round_up(L.counters_off + (size_t)p.ncounters * sizeof(int), 256);
  L.ready_off = round_up(L.pend_off + nt * sizeof(int), 256);
  L.summ_off = round_up(L.ready_off + nw * sizeof(unsigned long long), 256);
  L.wcl_off = round_up(L.summ_off + ns * sizeof(unsigned long long), 256);
  L.dbl_off = round_up(L.wcl_off + nw * sizeof(int), 256);
  L.total = L.dbl_off + (size_t)p.ws_doubles * sizeof(double);
  return L;
}

#define CUDA_TRY(x)                                                                          \
  do {                                                                                       \
    cudaError_t e_ = (x);                                                                    \
    if (e_ != cudaSuccess) return set_error(-100 - (int)e_, "%s: %s", #x, cudaGetErrorString(e_)); \
  } while (0)

static int upload_program(Program& prog) {
  if (!prog.tasks.empty()) {
    CUDA_TRY(cudaMalloc(&prog.d_tasks, prog.tasks.size() * sizeof(Task)));
    CUDA_TRY(cudaMemcpy(prog.d_tasks, prog.tasks.data(), prog.tasks.size() * sizeof(Task), cudaMemcpyHostToDevice));
  }
  if (!prog.waits.empty()) {
    CUDA_TRY(cudaMalloc(&prog.d_waits, prog.waits.size() * sizeof(int2)));
    CUDA_TRY(cudaMemcpy(prog.d_waits, prog.waits.data(), prog.waits.size() * sizeof(int2), cudaMemcpyHostToDevice));
  }
  auto up = [](auto** dst, const auto& v) -> int {
    if (v.empty()) return 0;
    const size_t bytes = v.size() * sizeof(v[0]);
    CUDA_TRY(cudaMalloc((void**)dst, bytes));
    CUDA_TRY(cudaMemcpy(*dst, v.data(), bytes, cudaMemcpyHostToDevice));
    return 0;
  };
  int rc = up(&prog.d_npend, prog.npend);
  if (!rc) rc = up(&prog.d_fronts, prog.fronts);
  if (!rc) rc = up(&prog.d_succ_off, prog.succ_off);
  if (!rc) rc = up(&prog.d_succ, prog.succ);
  if (!rc) rc = up(&prog.d_ctarget, prog.ctarget);
  if (!rc) rc = up(&prog.d_ready0, prog.ready0);
  if (!rc) rc = up(&prog.d_summ0, prog.summ0);
  return rc;
}

// Builds the host side of a program only (no device upload); used by the
// introspection entry points, which must work without a GPU.
// Chunks of the values for streaming (at most 24 each way: the arrival
// flags are control words 8..31, the output flags 32..55).  Incoming: cut at
// the first supernode boundary after 1/24 of the values.  Outgoing: the
// same, and a supernode larger than that is cut between 64-column tiles
// (its block is column-major, so column ranges are contiguous).
static IoSpec make_io_spec(const chb_plan& plan, bool in, bool out) {
  IoSpec io;
  io.in = in;
  io.out = out;
  const int64_t total = plan.blk_total;
  auto cut = [&](int64_t target, bool split, std::vector<int64_t>& off) {
    off.assign(1, 0);
    for (int64_t k = 0; k < plan.nsn; k++) {
      const chb::FrontDesc& f = plan.fronts[k];
      const int64_t beg = f.blk, end = (k + 1 < plan.nsn) ? plan.fronts[k + 1].blk : total;
      if (split && end - beg > target && f.nj > 0) {
        const int64_t cols = std::max<int64_t>(64, (target / f.nj) / 64 * 64);
        for (int64_t c = cols; c < f.nn; c += cols) {
          const int64_t o = beg + c * f.nj;
          if (o - off.back() >= target / 2) off.push_back(o);
        }
      }
      if (end - off.back() >= target && end < total) off.push_back(end);
    }
    off.push_back(total);
  };
  const int64_t t0 = std::max<int64_t>(total / 24, 1);
  cut(t0, false, io.in_off);
  for (int64_t t = t0;; t += t0 / 4 + 1) {
    cut(t, true, io.out_off);
    if (io.out_off.size() <= 25) break;
  }
  // arrival estimates at ~50 GB/s (only the list order uses them)
  for (size_t j = 0; j + 1 < io.in_off.size(); j++) io.arrive_us.push_back(io.in_off[j + 1] * 8.0 / 5e4);
  return io;
}

Program* build_host_program(chb_plan* plan, int op, int64_t k, int flags) {
  ProgKey key{op, k, flags};
  auto it = plan->progs.find(key);
  if (it != plan->progs.end()) return it->second.get();
  std::unique_ptr<Program> prog(new Program());
  const int io = flags & (PF_IO_IN | PF_IO_OUT);
  if (io) {
    if (op != CHB_OP_CHOLESKY && op != CHB_OP_PROJECTED_INVERSE && op != CHB_OP_LLT) {
      set_error(-2, "streamed values are available for cholesky, projected_inverse and llt");
      return nullptr;
    }
    if (plan->blk_total <= 0) {
      set_error(-2, "streamed values: empty factorisation");
      return nullptr;
    }
    prog->io = make_io_spec(*plan, (io & PF_IO_IN) != 0, (io & PF_IO_OUT) != 0);
    flags &= ~(PF_IO_IN | PF_IO_OUT);
  }
  const int16_t prec = (flags & PF_TF32X3) ? PREC_TF32X3 : (flags & PF_TF32) ? PREC_TF32 : PREC_FP64;
  if (prec != PREC_FP64) {
    if (op != CHB_OP_CHOLESKY && op != CHB_OP_PROJECTED_INVERSE) {
      set_error(-2, "mixed precision is available for cholesky and projected_inverse");
      return nullptr;
    }
    flags &= ~(PF_TF32 | PF_TF32X3);
  }
  int rc;
  switch (op) {
    case CHB_OP_CHOLESKY: rc = build_cholesky(*plan, *prog); break;
    case CHB_OP_PROJECTED_INVERSE: rc = build_projected_inverse(*plan, *prog); break;
    case CHB_OP_LLT: rc = build_llt(*plan, *prog); break;
    case CHB_OP_COMPLETION: rc = build_completion(*plan, *prog, k != 0); break;
    case CHB_OP_TRSM: rc = build_trsm(*plan, *prog, k, (flags & 1) != 0, (flags & 2) != 0); break;
    case CHB_OP_TRMM: rc = build_trmm(*plan, *prog, k, flags != 0); break;
    case CHB_OP_HESSIAN: rc = build_hessian(*plan, *prog, (int)k, flags); break;
    case CHB_OP_CONVENTIONAL: rc = build_conventional(*plan, *prog); break;
    default: rc = set_error(-2, "operation %d is not available", op); break;
  }
  if (rc != 0) return nullptr;
  if (prec != PREC_FP64)
    for (Task& t : prog->tasks)
      if (t.op == T_GEMM) t.c.prec = prec;
  prog->tf32_tiles = prec == PREC_TF32;
  for (const Task& t : prog->tasks)
    if (t.op == T_QL || t.op == T_TRSV) prog->smem_doubles = ENGINE_SMEM_DOUBLES;  // Householder panels, step operands
  // Default schedule per sweep, by measurement on a 3-D grid of 64,000
  // unknowns: the chains of small dependent tasks of cholesky, llt and trsm
  // run faster in static list order (a CTA already waits on the next task;
  // trmm has the solve's structure and takes its schedule);
  // the other sweeps gain from running whichever task is ready.  On a
  // merged plan (a batch of matrices or value sets) projected_inverse also
  // runs faster in list order: 256 uneven 2-D grids 36.5 -> 28.0 ms, and the
  // autotuner picked the static order for both batch workloads of the bench.
  const bool merged = plan->seg.size() > 2;
  prog->static_default = op == CHB_OP_CHOLESKY || op == CHB_OP_LLT || op == CHB_OP_TRSM || op == CHB_OP_TRMM ||
                         op == CHB_OP_CONVENTIONAL || (merged && op == CHB_OP_PROJECTED_INVERSE);
  Program* p = prog.get();
  plan->progs[key] = std::move(prog);
  return p;
}

Program* get_program(chb_plan* plan, int op, int64_t k, int flags) {
  Program* p = build_host_program(plan, op, k, flags);
  if (!p) return nullptr;
  if (!p->tasks.empty() && !p->d_tasks) {
    if (cudaSetDevice(plan->device) != cudaSuccess) {
      set_error(-3, "cudaSetDevice(%d) failed", plan->device);
      return nullptr;
    }
    if (upload_program(*p) != 0) return nullptr;
  }
  return p;
}

// cuStreamWaitValue32 through the runtime's driver entry point (no link
// against the driver library); null where the driver does not offer it.
typedef int (*WaitValue32Fn)(cudaStream_t, void*, unsigned int, unsigned int);
static WaitValue32Fn wait_value32() {
  static WaitValue32Fn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuStreamWaitValue32", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return (WaitValue32Fn)p;
  }();
  return fn;
}

extern "C" int chb_io_overlap_available() { return wait_value32() != nullptr; }

static int ensure_io_streams(chb_plan* plan) {
  if (plan->io_in) return 0;
  CUDA_TRY(cudaStreamCreateWithFlags(&plan->io_in, cudaStreamNonBlocking));
  CUDA_TRY(cudaEventCreateWithFlags(&plan->ev_start, cudaEventDisableTiming));
  CUDA_TRY(cudaEventCreateWithFlags(&plan->ev_in, cudaEventDisableTiming));
  for (int q = 0; q < chb_plan::IO_OUT_STREAMS; q++) {
    CUDA_TRY(cudaStreamCreateWithFlags(&plan->io_out[q], cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreateWithFlags(&plan->ev_out[q], cudaEventDisableTiming));
  }
  CUDA_TRY(cudaMallocHost(&plan->h_one, sizeof(int)));
  *plan->h_one = 1;
  return 0;
}

int run_program(chb_plan* plan, Program* prog, void* work, size_t work_bytes, double* const* bases, int nbases,
                cudaStream_t stream, int64_t run_ldb, double run_alpha, const HostIo* io) {
  const bool io_in = prog->io.in, io_out = prog->io.out;
  if ((io_in || io_out) != (io != nullptr) || (io && (io_in != (io->host_in != nullptr) ||
                                                     io_out != (io->host_out != nullptr))))
    return set_error(-6, "streamed program and host buffers do not match");
  WsLayout L = ws_layout(*prog);
  if (work_bytes < L.total || (L.total > 0 && !work))
    return set_error(-4, "workspace too small: %zu bytes given, %zu needed", work_bytes, L.total);
  if (((uintptr_t)work) % 256 != 0) return set_error(-5, "workspace must be 256-byte aligned");
  char* w = (char*)work;
  CUDA_TRY(cudaMemsetAsync(w, 0, L.dbl_off, stream));
  if (prog->tasks.empty()) return 0;
  RunArgs ra;
  std::memset(&ra, 0, sizeof(ra));
  ra.tasks = prog->d_tasks;
  ra.ntasks = (int32_t)prog->tasks.size();
  ra.smem_doubles = prog->smem_doubles;
  ra.waits = prog->d_waits;
  ra.ctl = (int*)w;
  ra.counters = (int*)(w + L.counters_off);
  for (int i = 0; i < nbases && i < MAX_BASES; i++) ra.bases[i] = bases[i];
  ra.bases[B_WS] = (double*)(w + L.dbl_off);
  ra.fronts = prog->d_fronts ? prog->d_fronts : plan->d_fronts;
  ra.relidx = plan->d_relidx;
  ra.chidx = plan->d_chidx;
  ra.spin_limit = plan->spin_limit >= 0 ? plan->spin_limit : kDefaultSpinLimit;
  ra.trace = (plan->trace && plan->trace_cap >= (int64_t)prog->tasks.size()) ? plan->trace : nullptr;
  ra.perm = plan->d_perm;
  // TF32 tiles as warp-level mma.sync, or on tcgen05 with tensor-memory
  // accumulators when the plan asks for it
  ra.tmem = prog->tf32_tiles && tf32_tcgen05(*plan) ? 1 : 0;
  ra.ldb = run_ldb;
  ra.alpha = run_alpha;
  // The plan's schedule, else CHB_SCHEDULE (static | dynamic), else the
  // sweep's default.
  static const char* sched = std::getenv("CHB_SCHEDULE");
  bool want_static = prog->static_default;
  if (sched && std::strcmp(sched, "static") == 0) want_static = true;
  if (sched && std::strcmp(sched, "dynamic") == 0) want_static = false;
  if (plan->schedule >= 0) want_static = plan->schedule == 1;
  const bool dynamic = !want_static && prog->d_npend && prog->d_ready0;
  if (dynamic) {
    ra.dynamic = 1;
    ra.nwords = (int)prog->ready0.size();
    ra.nsumm = (int)prog->summ0.size();
    ra.pend = (int*)(w + L.pend_off);
    ra.ready = (unsigned long long*)(w + L.ready_off);
    ra.summ = (unsigned long long*)(w + L.summ_off);
    ra.wclaimed = (int*)(w + L.wcl_off);
    ra.succ_off = prog->d_succ_off;
    ra.succ = prog->d_succ;
    ra.ctarget = prog->d_ctarget;
    CUDA_TRY(cudaMemcpyAsync(ra.pend, prog->d_npend, prog->npend.size() * sizeof(int), cudaMemcpyDeviceToDevice,
                             stream));
    CUDA_TRY(cudaMemcpyAsync(ra.ready, prog->d_ready0, prog->ready0.size() * sizeof(unsigned long long),
                             cudaMemcpyDeviceToDevice, stream));
    CUDA_TRY(cudaMemcpyAsync(ra.summ, prog->d_summ0, prog->summ0.size() * sizeof(unsigned long long),
                             cudaMemcpyDeviceToDevice, stream));
  }
  const int nin = (int)prog->io.in_off.size() - 1, nout = (int)prog->io.out_off.size() - 1;
  if (io_in) {
    ra.io_in = ra.ctl + 8;
    ra.nio_in = nin;
  }
  if (io_out) {
    ra.io_out = ra.ctl + 32;
    ra.nio_out = nout;
  }
  double* x = bases[B_X];
  if (io) {
    const int rs = ensure_io_streams(plan);
    if (rs) return rs;
    CUDA_TRY(cudaEventRecord(plan->ev_start, stream));
  }
  int grid = std::min<int64_t>(ra.tmem ? plan->grid_tc : plan->grid, (int64_t)prog->tasks.size());
  CUDA_TRY(engine_launch(ra, grid, stream));
  if (!io) return 0;
  if (io_in) {
    // chunk j, then its arrival flag (copies on one stream run in order), in
    // the order the task graph needs them
    const std::vector<int64_t>& off = prog->io.in_off;
    CUDA_TRY(cudaStreamWaitEvent(plan->io_in, plan->ev_start, 0));
    for (int j : prog->io.in_order) {
      CUDA_TRY(cudaMemcpyAsync(x + off[j], io->host_in + off[j], (off[j + 1] - off[j]) * sizeof(double),
                               cudaMemcpyHostToDevice, plan->io_in));
      CUDA_TRY(cudaMemcpyAsync(ra.io_in + j, plan->h_one, sizeof(int), cudaMemcpyHostToDevice, plan->io_in));
    }
    CUDA_TRY(cudaEventRecord(plan->ev_in, plan->io_in));
    CUDA_TRY(cudaStreamWaitEvent(stream, plan->ev_in, 0));
  }
  if (io_out) {
    const std::vector<int64_t>& off = prog->io.out_off;
    WaitValue32Fn wv = wait_value32();
    if (wv) {
      // each chunk as soon as its flag is up, dealt over the output streams
      // in the order the list finishes them
      const int nq = std::min<int>(chb_plan::IO_OUT_STREAMS, nout);
      for (int q = 0; q < nq; q++) CUDA_TRY(cudaStreamWaitEvent(plan->io_out[q], plan->ev_start, 0));
      for (size_t i = 0; i < prog->out_order.size(); i++) {
        const int j = prog->out_order[i];
        cudaStream_t sq = plan->io_out[i % nq];
        if (wv(sq, ra.io_out + j, 1u, 0u /* GEQ */) != 0) return set_error(-7, "cuStreamWaitValue32 failed");
        CUDA_TRY(cudaMemcpyAsync(io->host_out + off[j], x + off[j], (off[j + 1] - off[j]) * sizeof(double),
                                 cudaMemcpyDeviceToHost, sq));
      }
      for (int q = 0; q < nq; q++) {
        CUDA_TRY(cudaEventRecord(plan->ev_out[q], plan->io_out[q]));
        CUDA_TRY(cudaStreamWaitEvent(stream, plan->ev_out[q], 0));
      }
    } else {
      // no stream waits on this driver: copy after the sweep
      CUDA_TRY(cudaMemcpyAsync(io->host_out, x, off[nout] * sizeof(double), cudaMemcpyDeviceToHost, stream));
    }
  }
  return 0;
}

}  // namespace chb

using namespace chb;

// Device copies of the plan's symbolic data (skipped with device < 0: a
// host-only plan for introspection) and the persistent grid size.
static int upload_plan(chb_plan* P) {
  const int device = P->device;
  if (device < 0) return 0;
  const int64_t nsn = P->nsn, n = P->n, nrel = (int64_t)P->relidx.size();
  CUDA_TRY(cudaSetDevice(device));
  if (nsn > 0) {
    CUDA_TRY(cudaMalloc(&P->d_fronts, nsn * sizeof(FrontDesc)));
    CUDA_TRY(cudaMemcpy(P->d_fronts, P->fronts.data(), nsn * sizeof(FrontDesc), cudaMemcpyHostToDevice));
  }
  if (nrel > 0) {
    CUDA_TRY(cudaMalloc(&P->d_relidx, nrel * sizeof(int32_t)));
    CUDA_TRY(cudaMemcpy(P->d_relidx, P->relidx.data(), nrel * sizeof(int32_t), cudaMemcpyHostToDevice));
  }
  if (!P->chidx.empty()) {
    CUDA_TRY(cudaMalloc(&P->d_chidx, P->chidx.size() * sizeof(int32_t)));
    CUDA_TRY(cudaMemcpy(P->d_chidx, P->chidx.data(), P->chidx.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  }
  if (n > 0) {
    CUDA_TRY(cudaMalloc(&P->d_perm, n * sizeof(int64_t)));
    CUDA_TRY(cudaMemcpy(P->d_perm, P->perm.data(), n * sizeof(int64_t), cudaMemcpyHostToDevice));
    std::vector<int64_t> ip(n);
    for (int64_t i = 0; i < n; i++) ip[P->perm[i]] = i;
    CUDA_TRY(cudaMalloc(&P->d_iperm, n * sizeof(int64_t)));
    CUDA_TRY(cudaMemcpy(P->d_iperm, ip.data(), n * sizeof(int64_t), cudaMemcpyHostToDevice));
  }
  {
    // the strips of the chordal SYMV (chb_symv): 64 rows of a block each
    std::vector<int2> items;
    for (int64_t k = 0; k < P->nsn; k++)
      for (int i0 = 0; i0 < P->fronts[k].nj; i0 += 64) items.push_back(make_int2((int)k, i0));
    P->n_symv_items = (int)items.size();
    if (!items.empty()) {
      CUDA_TRY(cudaMalloc(&P->d_symv_items, items.size() * sizeof(int2)));
      CUDA_TRY(cudaMemcpy(P->d_symv_items, items.data(), items.size() * sizeof(int2), cudaMemcpyHostToDevice));
    }
  }
  CUDA_TRY(cudaMalloc(&P->d_seg, P->seg.size() * sizeof(int64_t)));
  CUDA_TRY(cudaMemcpy(P->d_seg, P->seg.data(), P->seg.size() * sizeof(int64_t), cudaMemcpyHostToDevice));
  int per_sm = 0, nsm = 0;
  if (engine_occupancy(&per_sm) != 0 || per_sm <= 0) return set_error(-12, "engine kernel cannot be resident");
  CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
  P->grid = per_sm * nsm;
  // The tcgen05 build has the FP64 build's registers and (at the base
  // staging its TF32 sweeps use) shared memory; the occupancy query reports
  // one CTA per SM for it, but two run side by side: launched with two per
  // SM, the 48^3 TF32 sweeps on tcgen05 took 16.5 / 20.5 ms against 26.3 /
  // 34.0 ms with one.  A CTA that is not resident claims nothing until it
  // is, so the wider grid is safe either way.
  int per_sm_tc = 0;
  if (engine_occupancy(&per_sm_tc, true) != 0 || per_sm_tc <= 0) return set_error(-12, "engine kernel cannot be resident");
  P->grid_tc = std::max(per_sm_tc, per_sm) * nsm;
  return 0;
}

extern "C" int chb_plan_create(int64_t n, int64_t nsn, const int64_t* snptr, const int64_t* snpar,
                               const int64_t* relptr, const int64_t* relidx, const int64_t* chptr,
                               const int64_t* chidx, const int64_t* blkptr, const int64_t* snode, const int64_t* p,
                               int device, chb_plan** out) {
  clear_error();
  if (!out) return set_error(-1, "null output pointer");
  *out = nullptr;
  if (n < 0 || nsn < 0) return set_error(-1, "negative size");
  std::unique_ptr<chb_plan> P(new chb_plan());
  P->device = device;
  P->n = n;
  P->nsn = nsn;
  P->fronts.resize(nsn);
  P->snpar.resize(nsn);
  P->level.assign(nsn, 0);
  P->snptr.assign(snptr, snptr + nsn + 1);
  P->snode.assign(snode, snode + n);
  P->perm.assign(p, p + n);
  {
    std::vector<char> seen(n, 0);
    for (int64_t i = 0; i < n; i++) {
      const int64_t v = P->perm[i];
      if (v < 0 || v >= n || seen[v]) return set_error(-5, "p is not a permutation of 0..n-1");
      seen[v] = 1;
    }
  }
  const int64_t nrel = relptr[nsn];
  P->relidx.resize(nrel);
  for (int64_t i = 0; i < nrel; i++) {
    if (relidx[i] < 0 || relidx[i] > INT32_MAX) return set_error(-6, "relidx out of range");
    P->relidx[i] = (int32_t)relidx[i];
  }
  P->chidx.resize(chptr[nsn]);
  for (int64_t i = 0; i < chptr[nsn]; i++) P->chidx[i] = (int32_t)chidx[i];
  int64_t upd = 0, vpos = 0;
  for (int64_t k = 0; k < nsn; k++) {
    FrontDesc& f = P->fronts[k];
    std::memset(&f, 0, sizeof(f));
    int64_t nn = snptr[k + 1] - snptr[k];
    int64_t na = relptr[k + 1] - relptr[k];
    if (nn <= 0 || na < 0 || nn + na > INT32_MAX / 2) return set_error(-7, "invalid supernode %lld", (long long)k);
    if (blkptr[k + 1] - blkptr[k] != nn * (nn + na)) return set_error(-8, "blkptr inconsistent at %lld", (long long)k);
    f.nn = (int32_t)nn;
    f.na = (int32_t)na;
    f.nj = (int32_t)(nn + na);
    f.relptr = (int32_t)relptr[k];
    f.chbeg = (int32_t)chptr[k];
    f.chend = (int32_t)chptr[k + 1];
    f.parent = (int32_t)snpar[k];
    f.blk = blkptr[k];
    f.upd = upd;
    f.col0 = snptr[k];
    f.vpos = vpos;
    upd += na * na;
    vpos += na;
    P->snpar[k] = (int32_t)snpar[k];
    if (snpar[k] < k || snpar[k] >= nsn) return set_error(-9, "snpar must point to a later supernode or itself");
    if ((snpar[k] == k) != (na == 0)) return set_error(-10, "root / separator mismatch at %lld", (long long)k);
    for (int64_t i = 0; i < na; i++) {
      int64_t r = relidx[relptr[k] + i];
      if (snpar[k] != k) {
        int64_t njp = (snptr[snpar[k] + 1] - snptr[snpar[k]]) + (relptr[snpar[k] + 1] - relptr[snpar[k]]);
        if (r >= njp || (i > 0 && r <= relidx[relptr[k] + i - 1]))
          return set_error(-11, "relidx of supernode %lld not increasing / in range", (long long)k);
      }
    }
  }
  P->upd_total = upd;
  P->blk_total = blkptr[nsn];
  // heights (children precede parents)
  int maxlv = 0;
  for (int64_t k = 0; k < nsn; k++) {
    if (snpar[k] != k) P->level[snpar[k]] = std::max(P->level[snpar[k]], P->level[k] + 1);
  }
  for (int64_t k = 0; k < nsn; k++) {
    P->fronts[k].level = P->level[k];
    maxlv = std::max(maxlv, P->level[k]);
  }
  P->nlevels = nsn ? maxlv + 1 : 0;

  P->seg.assign({0, nsn});
  int rc = upload_plan(P.get());
  if (rc) return rc;
  *out = P.release();
  return 0;
}

extern "C" int chb_plan_merge(const chb_plan* const* plans, int count, int device, chb_plan** out) {
  clear_error();
  if (!out) return set_error(-1, "null output pointer");
  *out = nullptr;
  if (count <= 0 || !plans) return set_error(-1, "merge: no plans");
  std::unique_ptr<chb_plan> P(new chb_plan());
  P->device = device;
  P->seg.push_back(0);
  int64_t n_off = 0, nsn_off = 0, rel_off = 0, ch_off = 0, blk_off = 0, upd = 0, vpos = 0;
  for (int m = 0; m < count; m++) {
    const chb_plan* Q = plans[m];
    if (!Q) return set_error(-1, "merge: null plan %d", m);
    for (int64_t k = 0; k < Q->nsn; k++) {
      FrontDesc f = Q->fronts[k];
      f.relptr += (int32_t)rel_off;
      f.chbeg += (int32_t)ch_off;
      f.chend += (int32_t)ch_off;
      f.parent += (int32_t)nsn_off;
      f.blk += blk_off;
      f.upd = upd;
      f.col0 += n_off;
      f.vpos = vpos;
      upd += (int64_t)f.na * f.na;
      vpos += f.na;
      P->fronts.push_back(f);
      P->snpar.push_back(Q->snpar[k] + (int32_t)nsn_off);
      P->level.push_back(Q->level[k]);
      P->snptr.push_back(Q->snptr[k] + n_off);
    }
    for (int32_t r : Q->relidx) P->relidx.push_back(r);
    for (int32_t c : Q->chidx) P->chidx.push_back(c + (int32_t)nsn_off);
    for (int64_t v : Q->snode) P->snode.push_back(v + n_off);
    for (int64_t v : Q->perm) P->perm.push_back(v + n_off);
    P->nlevels = std::max(P->nlevels, Q->nlevels);
    n_off += Q->n;
    nsn_off += Q->nsn;
    rel_off += (int64_t)Q->relidx.size();
    ch_off += (int64_t)Q->chidx.size();
    blk_off += Q->blk_total;
    P->seg.push_back(nsn_off);
    if (nsn_off > INT32_MAX / 2 || rel_off > INT32_MAX || ch_off > INT32_MAX)
      return set_error(-7, "merge: the batch exceeds the 32-bit index range");
  }
  P->snptr.push_back(n_off);
  P->n = n_off;
  P->nsn = nsn_off;
  P->blk_total = blk_off;
  P->upd_total = upd;
  int rc = upload_plan(P.get());
  if (rc) return rc;
  *out = P.release();
  return 0;
}

extern "C" int chb_plan_destroy(chb_plan* plan) {
  if (!plan) return 0;
  if (plan->device >= 0) cudaSetDevice(plan->device);
  plan->progs.clear();
  if (plan->io_in) cudaStreamDestroy(plan->io_in);
  if (plan->ev_start) cudaEventDestroy(plan->ev_start);
  if (plan->ev_in) cudaEventDestroy(plan->ev_in);
  for (int q = 0; q < chb_plan::IO_OUT_STREAMS; q++) {
    if (plan->io_out[q]) cudaStreamDestroy(plan->io_out[q]);
    if (plan->ev_out[q]) cudaEventDestroy(plan->ev_out[q]);
  }
  if (plan->h_one) cudaFreeHost(plan->h_one);
  if (plan->d_fronts) cudaFree(plan->d_fronts);
  if (plan->d_relidx) cudaFree(plan->d_relidx);
  if (plan->d_chidx) cudaFree(plan->d_chidx);
  if (plan->d_perm) cudaFree(plan->d_perm);
  if (plan->d_iperm) cudaFree(plan->d_iperm);
  if (plan->d_seg) cudaFree(plan->d_seg);
  if (plan->d_symv_items) cudaFree(plan->d_symv_items);
  delete plan;
  return 0;
}

extern "C" int chb_workspace_size(const chb_plan* plan_c, int op, int64_t k, int flags, size_t* bytes) {
  clear_error();
  chb_plan* plan = const_cast<chb_plan*>(plan_c);
  if (!plan || !bytes) return set_error(-1, "null argument");
  if (op == CHB_OP_DOT) {  // per-supernode partial sums
    *bytes = 256 + (size_t)(plan->nsn + 1) * sizeof(double);
    return 0;
  }
  Program* p = build_host_program(plan, op, k, flags);
  if (!p) return -2;
  *bytes = ws_layout(*p).total;
  return 0;
}

extern "C" int chb_program_info(chb_plan* plan, int op, int64_t k, int flags, int64_t* info) {
  clear_error();
  if (!plan || !info) return set_error(-1, "null argument");
  Program* p = build_host_program(plan, op, k, flags);
  if (!p) return -2;
  WsLayout L = ws_layout(*p);
  info[0] = (int64_t)p->tasks.size();
  info[1] = (int64_t)p->waits.size();
  info[2] = p->ncounters;
  info[3] = p->ws_doubles;
  info[4] = (int64_t)L.total;
  info[5] = (int64_t)L.dbl_off;
  info[6] = plan->upd_total;
  info[7] = (int64_t)sizeof(Task);
  return 0;
}

extern "C" int chb_program_pool(chb_plan* plan, int op, int64_t k, int flags, int64_t* info) {
  clear_error();
  if (!plan || !info) return set_error(-1, "null argument");
  Program* p = build_host_program(plan, op, k, flags);
  if (!p) return -2;
  info[0] = p->fronts.empty() ? -1 : p->pool_doubles * (int64_t)sizeof(double);
  info[1] = p->pool_waits;
  info[2] = (int64_t)ws_layout(*p).total;
  info[3] = (int64_t)(p->sim_span_us * 1000.0);
  return 0;
}

extern "C" int chb_program_export(chb_plan* plan, int op, int64_t k, int flags, void* tasks, void* waits,
                                  void* fronts) {
  clear_error();
  if (!plan) return set_error(-1, "null argument");
  Program* p = build_host_program(plan, op, k, flags);
  if (!p) return -2;
  if (tasks) std::memcpy(tasks, p->tasks.data(), p->tasks.size() * sizeof(Task));
  if (waits) std::memcpy(waits, p->waits.data(), p->waits.size() * sizeof(int2));
  const std::vector<FrontDesc>& fr = p->fronts.empty() ? plan->fronts : p->fronts;
  if (fronts) std::memcpy(fronts, fr.data(), fr.size() * sizeof(FrontDesc));
  return 0;
}

extern "C" int chb_program_schedule(chb_plan* plan, int op, int64_t k, int flags, int64_t* sizes, int32_t* npend,
                                    int32_t* succ_off, int32_t* succ, int32_t* ctarget, uint64_t* ready0,
                                    uint64_t* summ0) {
  clear_error();
  if (!plan || !sizes) return set_error(-1, "null argument");
  Program* p = build_host_program(plan, op, k, flags);
  if (!p) return -2;
  sizes[0] = (int64_t)p->npend.size();
  sizes[1] = (int64_t)p->succ_off.size();
  sizes[2] = (int64_t)p->succ.size();
  sizes[3] = (int64_t)p->ctarget.size();
  sizes[4] = (int64_t)p->ready0.size();
  sizes[5] = (int64_t)p->summ0.size();
  auto cp = [](void* dst, const auto& v) {
    if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
  };
  cp(npend, p->npend);
  cp(succ_off, p->succ_off);
  cp(succ, p->succ);
  cp(ctarget, p->ctarget);
  cp(ready0, p->ready0);
  cp(summ0, p->summ0);
  return 0;
}

extern "C" int chb_program_io(chb_plan* plan, int op, int64_t k, int flags, int64_t* counts, int64_t* in_off,
                              int32_t* in_order, int64_t* out_off, int32_t* out_order) {
  clear_error();
  if (!plan || !counts) return set_error(-1, "null argument");
  Program* p = build_host_program(plan, op, k, flags);
  if (!p) return -2;
  const int64_t nin = p->io.in ? (int64_t)p->io.in_off.size() - 1 : 0;
  const int64_t nout = p->io.out ? (int64_t)p->io.out_off.size() - 1 : 0;
  counts[0] = nin;
  counts[1] = nout;
  if (in_off && nin) std::memcpy(in_off, p->io.in_off.data(), (nin + 1) * sizeof(int64_t));
  if (in_order && nin) std::memcpy(in_order, p->io.in_order.data(), nin * sizeof(int));
  if (out_off && nout) std::memcpy(out_off, p->io.out_off.data(), (nout + 1) * sizeof(int64_t));
  if (out_order && !p->out_order.empty()) std::memcpy(out_order, p->out_order.data(), p->out_order.size() * sizeof(int));
  return 0;
}

extern "C" int chb_plan_set_schedule(chb_plan* plan, int mode) {
  clear_error();
  if (!plan) return set_error(-1, "null plan");
  if (mode < -1 || mode > 1) return set_error(-2, "schedule mode must be -1, 0 or 1");
  plan->schedule = mode;
  return 0;
}

extern "C" int chb_plan_set_option(chb_plan* plan, int option, int64_t value) {
  clear_error();
  if (!plan) return set_error(-1, "null plan");
  if (option < 0 || option >= CHB_OPT_COUNT) return set_error(-2, "unknown option %d", option);
  const int64_t v = value < 0 ? -1 : value;
  if (plan->opt[option] != v) {
    plan->opt[option] = v;
    plan->progs.clear();  // rebuilt with the new option by the next sweeps
  }
  return 0;
}

extern "C" int chb_plan_get_option(const chb_plan* plan, int option, int64_t* value) {
  clear_error();
  if (!plan || !value) return set_error(-1, "null argument");
  switch (option) {
    case CHB_OPT_SMALL_FRONT_NJ: *value = small_front_nj(*plan); break;
    case CHB_OPT_SUBTREES: *value = subtrees_on(*plan) ? 1 : 0; break;
    case CHB_OPT_CHOL_KSPLIT: *value = chol_ksplit(*plan); break;
    case CHB_OPT_PINV_KSPLIT: *value = pinv_ksplit(*plan); break;
    case CHB_OPT_FUSED_LA: *value = fused_la_allowed(*plan) ? 1 : 0; break;
    case CHB_OPT_TF32_TCGEN05: *value = tf32_tcgen05(*plan) ? 1 : 0; break;
    case CHB_OPT_ORDERED_SUMS: *value = ordered_sums(*plan) ? 1 : 0; break;
    case CHB_OPT_SCRATCH_LIMIT: *value = scratch_limit_bytes(*plan); break;
    default: return set_error(-2, "unknown option %d", option);
  }
  return 0;
}

extern "C" int chb_engine_occupancy(int tcgen05, int* blocks_per_sm) {
  clear_error();
  if (!blocks_per_sm) return set_error(-1, "null argument");
  if (engine_occupancy(blocks_per_sm, tcgen05 != 0) != 0) return set_error(-12, "occupancy query failed");
  return 0;
}

extern "C" int chb_plan_set_spin_limit(chb_plan* plan, int64_t polls) {
  clear_error();
  if (!plan) return set_error(-1, "null plan");
  plan->spin_limit = polls < 0 ? -1 : polls;
  return 0;
}

extern "C" int chb_set_trace(chb_plan* plan, void* buffer, int64_t capacity_tasks) {
  clear_error();
  if (!plan) return set_error(-1, "null plan");
  plan->trace = (unsigned long long*)buffer;
  plan->trace_cap = buffer ? capacity_tasks : 0;
  return 0;
}
