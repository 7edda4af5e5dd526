// Allocation-free variant of the Cholesky sweep.
//
// Some callers cannot call cudaMalloc at the point where they need a
// factorisation: a framework whose device memory all comes from its own pool
// and that forbids allocations behind its back, or a host process that must
// not grow its device footprint after start-up (a fixed memory budget agreed
// with the other jobs on the GPU).  chb_cholesky_noalloc serves them:
// everything the sweep needs on the device besides the caller's values
// (control words, task counters, the uploaded symbolic data, the task program
// and the workspace) lives in one file-scope __device__ array of
// CHB_NOALLOC_SCRATCH_BYTES, which every GPU that loads this library holds
// until the process exits.  The call is synchronous: it waits for the sweep
// and reads its status back, as chb_cholesky followed by chb_info does.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/chompack_b200.h"
#include "internal.h"
#include "plan.h"

namespace chb {

static __device__ __align__(256) unsigned char g_noalloc_scratch[CHB_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int MAX_DEVICES = 64;
unsigned char* g_scratch_addr[MAX_DEVICES];  // device address of the array, per device
int g_scratch_grid[MAX_DEVICES];
// Held for the whole of every call: host threads of one process that call
// concurrently take turns instead of interleaving their staging copies into
// the shared array.  Other processes, and other streams of this process that
// launch work which overlaps a call, are not covered.
std::mutex g_scratch_mu;

// Once per device, with that device current and g_scratch_mu held: look up
// the array's device address (the host-side symbol is only a stand-in) and
// prepare the kernel's launch shape.  Nothing here allocates.
int setup_device(int dev) {
  if (g_scratch_addr[dev]) return 0;
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p)
    return set_error(-41, "cudaGetSymbolAddress of the static scratch failed: %s", cudaGetErrorString(e));
  int per_sm = 0, nsm = 0;
  if (engine_occupancy(&per_sm) != 0 || per_sm <= 0) return set_error(-12, "engine kernel cannot be resident");
  e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return set_error(-42, "cudaDeviceGetAttribute failed: %s", cudaGetErrorString(e));
  g_scratch_grid[dev] = per_sm * nsm;
  g_scratch_addr[dev] = (unsigned char*)p;
  return 0;
}

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

}  // namespace
}  // namespace chb

using namespace chb;

extern "C" int chb_cholesky_noalloc(chb_plan* plan, double* blkval, void* stream_v) {
  clear_error();
  if (!plan) return set_error(-1, "null plan");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return set_error(-3, "no current CUDA device");
  if (dev < 0 || dev >= MAX_DEVICES) return set_error(-3, "device %d out of range", dev);
  if (plan->device >= 0 && plan->device != dev)
    return set_error(-3, "plan is bound to device %d but device %d is current", plan->device, dev);
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  int rc = setup_device(dev);
  if (rc) return rc;
  Program* prog = build_host_program(plan, CHB_OP_CHOLESKY, 0, 0);
  if (!prog) return -2;
  // the program's own update-matrix offsets under a scratch limit
  const std::vector<FrontDesc>& fronts = prog->fronts.empty() ? plan->fronts : prog->fronts;

  // layout inside the static array
  const size_t ctl_off = 0;
  const size_t cnt_off = 256;
  const size_t fr_off = align256(cnt_off + (size_t)prog->ncounters * sizeof(int));
  const size_t rel_off = align256(fr_off + fronts.size() * sizeof(FrontDesc));
  const size_t ch_off = align256(rel_off + plan->relidx.size() * sizeof(int32_t));
  const size_t tk_off = align256(ch_off + plan->chidx.size() * sizeof(int32_t));
  const size_t wt_off = align256(tk_off + prog->tasks.size() * sizeof(Task));
  const size_t db_off = align256(wt_off + prog->waits.size() * sizeof(int2));
  const size_t total = db_off + (size_t)prog->ws_doubles * sizeof(double);
  if (total > (size_t)CHB_NOALLOC_SCRATCH_BYTES)
    return set_error(-40,
                     "chb_cholesky_noalloc: this factorisation needs %zu bytes of device scratch; the "
                     "allocation-free entry point is limited to %zu bytes (use chb_cholesky with a "
                     "caller-provided workspace)",
                     total, (size_t)CHB_NOALLOC_SCRATCH_BYTES);

  cudaStream_t stream = (cudaStream_t)stream_v;
  unsigned char* base = g_scratch_addr[dev];
  cudaError_t e = cudaMemsetAsync(base + ctl_off, 0, fr_off - ctl_off, stream);
  if (e == cudaSuccess && !fronts.empty())
    e = cudaMemcpyAsync(base + fr_off, fronts.data(), fronts.size() * sizeof(FrontDesc), cudaMemcpyHostToDevice,
                        stream);
  if (e == cudaSuccess && !plan->relidx.empty())
    e = cudaMemcpyAsync(base + rel_off, plan->relidx.data(), plan->relidx.size() * sizeof(int32_t),
                        cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess && !plan->chidx.empty())
    e = cudaMemcpyAsync(base + ch_off, plan->chidx.data(), plan->chidx.size() * sizeof(int32_t),
                        cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess && !prog->tasks.empty())
    e = cudaMemcpyAsync(base + tk_off, prog->tasks.data(), prog->tasks.size() * sizeof(Task),
                        cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess && !prog->waits.empty())
    e = cudaMemcpyAsync(base + wt_off, prog->waits.data(), prog->waits.size() * sizeof(int2),
                        cudaMemcpyHostToDevice, stream);
  if (e != cudaSuccess) return set_error(-100 - (int)e, "staging into the static scratch failed: %s",
                                         cudaGetErrorString(e));
  if (!prog->tasks.empty()) {
    RunArgs ra;
    std::memset(&ra, 0, sizeof(ra));
    ra.tasks = (const Task*)(base + tk_off);
    ra.ntasks = (int32_t)prog->tasks.size();
    ra.smem_doubles = prog->smem_doubles;
    ra.waits = (const int2*)(base + wt_off);
    ra.ctl = (int*)(base + ctl_off);
    ra.counters = (int*)(base + cnt_off);
    ra.bases[B_X] = blkval;
    ra.bases[B_WS] = (double*)(base + db_off);
    ra.fronts = (const FrontDesc*)(base + fr_off);
    ra.relidx = (const int32_t*)(base + rel_off);
    ra.chidx = (const int32_t*)(base + ch_off);
    ra.spin_limit = 40000000LL;
    int grid = g_scratch_grid[dev];
    if ((int64_t)grid > (int64_t)prog->tasks.size()) grid = (int)prog->tasks.size();
    e = engine_launch(ra, grid, stream);
    if (e != cudaSuccess) return set_error(-100 - (int)e, "launch failed: %s", cudaGetErrorString(e));
  }
  // synchronous, like the reference: read the sweep status
  e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return set_error(-100 - (int)e, "sweep failed: %s", cudaGetErrorString(e));
  int ctl[4];
  e = cudaMemcpy(ctl, base + ctl_off, sizeof(ctl), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return set_error(-3, "cannot read the sweep status");
  if (ctl[1] == DE_TIMEOUT) return set_error(-30, "a task wait timed out (%d CTAs)", ctl[3]);
  if (ctl[1] != 0) return set_error(-31, "device error %d", ctl[1]);
  return ctl[2];
}
