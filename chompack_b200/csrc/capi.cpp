// C ABI entry points of the numeric sweeps (include/chompack_b200.h).
#include <cuda_runtime.h>

#include <cstring>

#include "../../include/chompack_b200.h"
#include "internal.h"
#include "plan.h"

using namespace chb;

namespace {

int check_plan(chb_plan* plan) {
  if (!plan) return set_error(-1, "null plan");
  if (plan->device < 0) return set_error(-1, "plan was created without a device");
  if (cudaSetDevice(plan->device) != cudaSuccess) return set_error(-3, "cudaSetDevice(%d) failed", plan->device);
  return 0;
}

int run_op(chb_plan* plan, int op, int64_t k, int flags, double* const* bases, int nbases, void* work,
           size_t work_bytes, void* stream, int64_t ldb = 0, double alpha = 1.0) {
  clear_error();
  int rc = check_plan(plan);
  if (rc) return rc;
  Program* prog = get_program(plan, op, k, flags);
  if (!prog) return -2;
  return run_program(plan, prog, work, work_bytes, bases, nbases, (cudaStream_t)stream, ldb, alpha);
}

int precision_flags(int precision) {
  return precision == CHB_PREC_TF32 ? PF_TF32 : precision == CHB_PREC_TF32X3 ? PF_TF32X3 : 0;
}

// A sweep on values held in host memory (see chb_cholesky_io).
int run_io(chb_plan* plan, int op, const double* host_in, double* host_out, double* dev_blkval, void* work,
           size_t work_bytes, void* stream, int precision = CHB_PREC_FP64) {
  clear_error();
  int rc = check_plan(plan);
  if (rc) return rc;
  if (!dev_blkval) return set_error(-1, "null device values");
  if (precision < CHB_PREC_FP64 || precision > CHB_PREC_TF32X3) return set_error(-1, "unknown precision %d", precision);
  const int flags = (host_in ? PF_IO_IN : 0) | (host_out ? PF_IO_OUT : 0) | precision_flags(precision);
  Program* prog = get_program(plan, op, 0, flags);
  if (!prog) return -2;
  double* bases[1] = {dev_blkval};
  if (!host_in && !host_out) return run_program(plan, prog, work, work_bytes, bases, 1, (cudaStream_t)stream);
  HostIo io;
  io.host_in = host_in;
  io.host_out = host_out;
  return run_program(plan, prog, work, work_bytes, bases, 1, (cudaStream_t)stream, 0, 1.0, &io);
}

}  // namespace

extern "C" int chb_io_flags(int host_in, int host_out) {
  return (host_in ? PF_IO_IN : 0) | (host_out ? PF_IO_OUT : 0);
}

extern "C" int chb_cholesky_io(chb_plan* plan, const double* host_in, double* host_out, double* dev_blkval,
                               void* work, size_t work_bytes, void* stream) {
  return run_io(plan, CHB_OP_CHOLESKY, host_in, host_out, dev_blkval, work, work_bytes, stream);
}

extern "C" int chb_projected_inverse_io(chb_plan* plan, const double* host_in, double* host_out,
                                        double* dev_blkval, void* work, size_t work_bytes, void* stream) {
  return run_io(plan, CHB_OP_PROJECTED_INVERSE, host_in, host_out, dev_blkval, work, work_bytes, stream);
}

extern "C" int chb_llt_io(chb_plan* plan, const double* host_in, double* host_out, double* dev_blkval, void* work,
                          size_t work_bytes, void* stream) {
  return run_io(plan, CHB_OP_LLT, host_in, host_out, dev_blkval, work, work_bytes, stream);
}

extern "C" int chb_precision_flags(int precision) { return precision_flags(precision); }

extern "C" int chb_cholesky_prec(chb_plan* plan, int precision, const double* host_in, double* host_out,
                                 double* dev_blkval, void* work, size_t work_bytes, void* stream) {
  return run_io(plan, CHB_OP_CHOLESKY, host_in, host_out, dev_blkval, work, work_bytes, stream, precision);
}

extern "C" int chb_projected_inverse_prec(chb_plan* plan, int precision, const double* host_in, double* host_out,
                                          double* dev_blkval, void* work, size_t work_bytes, void* stream) {
  return run_io(plan, CHB_OP_PROJECTED_INVERSE, host_in, host_out, dev_blkval, work, work_bytes, stream, precision);
}

extern "C" int chb_cholesky(chb_plan* plan, double* blkval, void* work, size_t work_bytes, void* stream) {
  double* bases[1] = {blkval};
  return run_op(plan, CHB_OP_CHOLESKY, 0, 0, bases, 1, work, work_bytes, stream);
}

extern "C" int chb_factor_conventional(chb_plan* plan, double* blkval, void* work, size_t work_bytes,
                                       void* stream) {
  double* bases[1] = {blkval};
  return run_op(plan, CHB_OP_CONVENTIONAL, 0, 0, bases, 1, work, work_bytes, stream);
}

extern "C" int chb_projected_inverse(chb_plan* plan, double* blkval, void* work, size_t work_bytes, void* stream) {
  double* bases[1] = {blkval};
  return run_op(plan, CHB_OP_PROJECTED_INVERSE, 0, 0, bases, 1, work, work_bytes, stream);
}

extern "C" int chb_llt(chb_plan* plan, double* blkval, void* work, size_t work_bytes, void* stream) {
  double* bases[1] = {blkval};
  return run_op(plan, CHB_OP_LLT, 0, 0, bases, 1, work, work_bytes, stream);
}

extern "C" int chb_completion(chb_plan* plan, double* blkval, int factored_updates, void* work, size_t work_bytes,
                              void* stream) {
  double* bases[1] = {blkval};
  return run_op(plan, CHB_OP_COMPLETION, factored_updates ? 1 : 0, 0, bases, 1, work, work_bytes, stream);
}

extern "C" int chb_hessian(chb_plan* plan, const double* lblkval, const double* yblkval, double* const* ublkval,
                           int64_t nu, int adj, int inv, int factored_updates, void* work, size_t work_bytes,
                           void* stream) {
  if (nu < 1 || nu > MAX_BASES - B_U0)
    return set_error(-1, "hessian: between 1 and %d U matrices per call, %lld given", MAX_BASES - B_U0, (long long)nu);
  if (!ublkval) return set_error(-1, "hessian: null U array");
  double* bases[MAX_BASES] = {};
  bases[B_L] = const_cast<double*>(lblkval);
  bases[B_Y] = const_cast<double*>(yblkval);
  for (int64_t u = 0; u < nu; u++) bases[B_U0 + u] = ublkval[u];
  const int flags = (adj ? 1 : 0) | (inv ? 2 : 0) | (factored_updates ? 4 : 0);
  return run_op(plan, CHB_OP_HESSIAN, nu, flags, bases, (int)(B_U0 + nu), work, work_bytes, stream);
}

extern "C" int chb_trsm(chb_plan* plan, char trans, int64_t nrhs, double alpha, const double* blkval, double* B,
                        int64_t ldB, void* work, size_t work_bytes, void* stream) {
  if (trans != 'N' && trans != 'T') return set_error(-1, "trans must be 'N' or 'T'");
  if (nrhs < 0 || (plan && ldB < plan->n)) return set_error(-1, "invalid nrhs or ldB");
  double* bases[B_RHS + 1] = {const_cast<double*>(blkval), nullptr, nullptr, nullptr, B};
  return run_op(plan, CHB_OP_TRSM, nrhs, trans == 'T' ? 1 : 0, bases, B_RHS + 1, work, work_bytes, stream, ldB,
                alpha);
}

extern "C" int chb_trsm_reuse(chb_plan* plan, char trans, int64_t nrhs, double alpha, const double* blkval,
                              double* B, int64_t ldB, void* work, size_t work_bytes, int reuse, void* stream) {
  if (trans != 'N' && trans != 'T') return set_error(-1, "trans must be 'N' or 'T'");
  if (nrhs < 0 || (plan && ldB < plan->n)) return set_error(-1, "invalid nrhs or ldB");
  double* bases[B_RHS + 1] = {const_cast<double*>(blkval), nullptr, nullptr, nullptr, B};
  const int flags = (trans == 'T' ? 1 : 0) | (reuse ? 2 : 0);
  return run_op(plan, CHB_OP_TRSM, nrhs, flags, bases, B_RHS + 1, work, work_bytes, stream, ldB, alpha);
}

extern "C" int chb_trmm(chb_plan* plan, char trans, int64_t nrhs, double alpha, const double* blkval, double* B,
                        int64_t ldB, void* work, size_t work_bytes, void* stream) {
  if (trans != 'N' && trans != 'T') return set_error(-1, "trans must be 'N' or 'T'");
  if (nrhs < 0 || (plan && ldB < plan->n)) return set_error(-1, "invalid nrhs or ldB");
  double* bases[B_RHS + 1] = {const_cast<double*>(blkval), nullptr, nullptr, nullptr, B};
  return run_op(plan, CHB_OP_TRMM, nrhs, trans == 'T' ? 1 : 0, bases, B_RHS + 1, work, work_bytes, stream, ldB,
                alpha);
}

extern "C" int chb_dot(chb_plan* plan, const double* x, const double* y, double* result, void* work,
                       size_t work_bytes, void* stream) {
  clear_error();
  int rc = check_plan(plan);
  if (rc) return rc;
  const size_t need = 256 + (size_t)(plan->nsn + 1) * sizeof(double);
  if (work_bytes < need || !work) return set_error(-4, "workspace too small: %zu bytes given, %zu needed", work_bytes, need);
  double* partial = (double*)((char*)work + 256);
  cudaError_t e = dot_launch(x, y, plan->d_fronts, (int)plan->nsn, partial, result, (cudaStream_t)stream);
  if (e != cudaSuccess) return set_error(-100 - (int)e, "dot launch failed: %s", cudaGetErrorString(e));
  return 0;
}

extern "C" int chb_logdet(chb_plan* plan, const double* l, double* result, void* work, size_t work_bytes,
                          void* stream) {
  clear_error();
  int rc = check_plan(plan);
  if (rc) return rc;
  const size_t need = 256 + (size_t)(plan->nsn + 1) * sizeof(double);
  if (work_bytes < need || !work) return set_error(-4, "workspace too small: %zu bytes given, %zu needed", work_bytes, need);
  double* partial = (double*)((char*)work + 256);
  cudaError_t e = logdet_launch(l, plan->d_fronts, (int)plan->nsn, partial, result, (cudaStream_t)stream);
  if (e != cudaSuccess) return set_error(-100 - (int)e, "logdet launch failed: %s", cudaGetErrorString(e));
  return 0;
}

// Per-matrix reductions of a merged plan (chb_plan_merge): results[m] for
// each of its matrices (a plan from chb_plan_create has one).
static int batch_reduce(chb_plan* plan, const double* a, const double* b, bool logdet, double* results, void* work,
                        size_t work_bytes, void* stream) {
  clear_error();
  int rc = check_plan(plan);
  if (rc) return rc;
  const size_t need = 256 + (size_t)(plan->nsn + 1) * sizeof(double);
  if (work_bytes < need || !work) return set_error(-4, "workspace too small: %zu bytes given, %zu needed", work_bytes, need);
  double* partial = (double*)((char*)work + 256);
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = logdet ? logdet_partials(a, plan->d_fronts, (int)plan->nsn, partial, st)
                         : dot_partials(a, b, plan->d_fronts, (int)plan->nsn, partial, st);
  if (e == cudaSuccess) e = segment_sums(partial, plan->d_seg, (int)plan->seg.size() - 1, results, st);
  if (e != cudaSuccess) return set_error(-100 - (int)e, "reduction launch failed: %s", cudaGetErrorString(e));
  return 0;
}

extern "C" int chb_logdet_batch(chb_plan* plan, const double* l, double* results, void* work, size_t work_bytes,
                                void* stream) {
  return batch_reduce(plan, l, nullptr, true, results, work, work_bytes, stream);
}

extern "C" int chb_dot_batch(chb_plan* plan, const double* x, const double* y, double* results, void* work,
                             size_t work_bytes, void* stream) {
  return batch_reduce(plan, x, y, false, results, work, work_bytes, stream);
}

extern "C" int chb_plan_batch_info(const chb_plan* plan, int64_t* count, int64_t* seg_out) {
  clear_error();
  if (!plan) return set_error(-1, "null plan");
  if (count) *count = (int64_t)plan->seg.size() - 1;
  if (seg_out)
    for (size_t i = 0; i < plan->seg.size(); i++) seg_out[i] = plan->seg[i];
  return 0;
}

extern "C" int chb_sym_weight(chb_plan* plan, const double* x, double* y, double alpha, void* stream) {
  clear_error();
  int rc = check_plan(plan);
  if (rc) return rc;
  cudaError_t e = symw_launch(x, y, alpha, plan->d_fronts, (int)plan->nsn, (cudaStream_t)stream);
  if (e != cudaSuccess) return set_error(-100 - (int)e, "sym_weight launch failed: %s", cudaGetErrorString(e));
  return 0;
}

extern "C" int chb_symv(chb_plan* plan, const double* blkval, const int64_t* sncolptr, const int64_t* snrowidx,
                        const double* x, double* y, int64_t nrhs, int64_t ld, double alpha, void* stream) {
  clear_error();
  int rc = check_plan(plan);
  if (rc) return rc;
  if (!blkval || !sncolptr || !snrowidx || !x || !y) return set_error(-1, "null argument");
  if (nrhs < 0 || ld < plan->n) return set_error(-1, "symv: nrhs >= 0 and ld >= n required");
  cudaError_t e = symv_launch(blkval, plan->d_fronts, plan->d_symv_items, plan->n_symv_items, sncolptr, snrowidx,
                              plan->d_perm, x, y, (int)nrhs, ld, alpha, (cudaStream_t)stream);
  if (e != cudaSuccess) return set_error(-100 - (int)e, "symv launch failed: %s", cudaGetErrorString(e));
  return 0;
}

extern "C" int chb_info(chb_plan* plan, void* work, void* stream) {
  clear_error();
  int rc = check_plan(plan);
  if (rc) return rc;
  if (cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) {
    cudaError_t e = cudaGetLastError();
    return set_error(-100 - (int)e, "stream synchronisation failed: %s", cudaGetErrorString(e));
  }
  int ctl[4];
  if (cudaMemcpy(ctl, work, sizeof(ctl), cudaMemcpyDeviceToHost) != cudaSuccess)
    return set_error(-3, "cannot read the sweep status");
  if (ctl[1] == DE_TIMEOUT) return set_error(-30, "a task wait timed out (%d CTAs)", ctl[3]);
  if (ctl[1] != 0) return set_error(-31, "device error %d", ctl[1]);
  return ctl[2];
}
