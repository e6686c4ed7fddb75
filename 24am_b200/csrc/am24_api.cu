// Host side of the C ABI (include/am24.h): handles, resident matrices, batch
// stepping and the denseDataSolver drivers (batch and on-the-fly modes).
//
// The drivers restate c++/src/gpower/sparse_PCA_solver.h:36-243 around the
// device step of am24_kernels.cu: the same settings mutation, batch-global or
// per-start termination, best-start choice and final normalisation.  All
// arithmetic of the AM step runs on the GPU; the host only decides control
// flow from a few scalars it reads back per iteration.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <string>
#include <unordered_map>
#include <vector>

#include <cudaTypedefs.h>

#include "am24.h"
#include "am24_internal.h"
#include "am24_host.h"

using namespace am24;
using namespace am24host;

namespace am24host {
thread_local std::string g_last_error;
}  // namespace am24host

namespace am24host {

// K-major FP32 operand [rows][ld], loaded as bk x box_rows tiles; the swizzle
// matches the row length (bk * 4 bytes) and the GEMM's smem descriptors.
am24_status make_map(am24_handle h, CUtensorMap *map, const float *base, int K, int rows, int ld,
                     int box_rows, int bk) {
  cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)ld * sizeof(float)};
  cuuint32_t box[2] = {(cuuint32_t)bk, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = h->encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(base), dims,
                         strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         bk == 32 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return fail(AM24_ERR_CUDA, "cuTensorMapEncodeTiled failed with code " + std::to_string((int)r));
  return AM24_OK;
}

// K-major 16-bit operand [rows][ld] (ld in elements; BF16, or FP16 when
// fp16), loaded as 32 x box_rows tiles (64-byte rows, 64-byte swizzle), as the
// 16-bit pair GEMMs read them.
am24_status make_map_bf16(am24_handle h, CUtensorMap *map, const uint16_t *base, int K, int rows,
                          int ld, int box_rows, bool fp16) {
  cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)ld * sizeof(uint16_t)};
  cuuint32_t box[2] = {(cuuint32_t)PAIR_BK_BF16, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = h->encode(map, fp16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16,
                         2, const_cast<uint16_t *>(base),
                         dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return fail(AM24_ERR_CUDA, "cuTensorMapEncodeTiled (BF16) failed with code " +
                                   std::to_string((int)r));
  return AM24_OK;
}

// The matrix's BF16 planes of B (made on first use): `planes` = 1 for b0
// alone (the single-pass BF16 product of MIXED), 3 for the exact split.  A
// matrix holding one plane that is asked for three gets a new buffer of three.
am24_status ensure_bf16_planes(am24_handle h, am24_matrix mat, int planes) {
  MatrixDev &M = mat->d;
  if (M.Bc_b3 && M.bf16_planes >= planes) return AM24_OK;
  const size_t plane = (size_t)M.n * M.ldm;
  uint16_t *p = nullptr;
  AM24_TRY(mat->mem.get(&p, (size_t)planes * plane));
  AM24_CUDA(cudaMemsetAsync(p, 0, sizeof(uint16_t) * planes * plane, h->stream));
  uint16_t *old = M.Bc_b3;
  const int old_planes = M.bf16_planes;
  M.Bc_b3 = p;
  M.bf16_planes = planes;
  cudaError_t e = launch_prep_bf16x3(M, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) {
    M.Bc_b3 = old;
    M.bf16_planes = old_planes;
    return fail(AM24_ERR_CUDA, std::string("BF16 planes: ") + cudaGetErrorString(e));
  }
  return AM24_OK;
}

// The matrix's TF32 hi/lo planes of B and B^T (made once, on first use).
am24_status ensure_tf32_planes(am24_handle h, am24_matrix mat) {
  MatrixDev &M = mat->d;
  if (M.Bc_hi) return AM24_OK;
  const size_t c_elems = (size_t)M.n * M.ldm, t_elems = (size_t)M.m * M.ldn;
  float *p[4] = {nullptr, nullptr, nullptr, nullptr};
  AM24_TRY(mat->mem.get(&p[0], c_elems));
  AM24_TRY(mat->mem.get(&p[1], c_elems));
  AM24_TRY(mat->mem.get(&p[2], t_elems));
  AM24_TRY(mat->mem.get(&p[3], t_elems));
  for (int i = 0; i < 4; i++)
    AM24_CUDA(cudaMemsetAsync(p[i], 0, sizeof(float) * (i < 2 ? c_elems : t_elems), h->stream));
  M.Bc_hi = p[0];
  M.Bc_lo = p[1];
  M.Bt_hi = p[2];
  M.Bt_lo = p[3];
  cudaError_t e = launch_prep_tf32_planes(M, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) {
    M.Bc_hi = M.Bc_lo = M.Bt_hi = M.Bt_lo = nullptr;
    return fail(AM24_ERR_CUDA, std::string("TF32 planes: ") + cudaGetErrorString(e));
  }
  return AM24_OK;
}

// The matrix's two scaled FP16 planes of B and their row scales (made once, on
// first use).
am24_status ensure_fp16_planes(am24_handle h, am24_matrix mat) {
  MatrixDev &M = mat->d;
  if (M.Bc_h2) return AM24_OK;
  const size_t plane = (size_t)M.n * M.ldm;
  uint16_t *p = nullptr;
  float *rs = nullptr;
  AM24_TRY(mat->mem.get(&p, 2 * plane));
  AM24_TRY(mat->mem.get(&rs, (size_t)M.n));
  if (M.ldm > M.m)  // the pad rows of both planes (2n columns)
    AM24_CUDA(cudaMemset2DAsync(p + M.m, sizeof(uint16_t) * M.ldm, 0,
                                sizeof(uint16_t) * (M.ldm - M.m), 2 * (size_t)M.n, h->stream));
  M.Bc_h2 = p;
  M.row_scale = rs;
  cudaError_t e = launch_prep_fp16x2(M, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) {
    M.Bc_h2 = nullptr;
    M.row_scale = nullptr;
    return fail(AM24_ERR_CUDA, std::string("FP16 planes: ") + cudaGetErrorString(e));
  }
  return AM24_OK;
}

// The matrix's two scaled FP16 planes of B^T and their row scales (made once,
// on first use).
am24_status ensure_bt_fp16_planes(am24_handle h, am24_matrix mat) {
  MatrixDev &M = mat->d;
  if (M.Bt_h2) return AM24_OK;
  const size_t plane = (size_t)M.m * M.ldn;
  uint16_t *p = nullptr;
  float *rs = nullptr;
  uint32_t *key = nullptr;
  AM24_TRY(mat->mem.get(&p, 2 * plane));
  AM24_TRY(mat->mem.get(&rs, (size_t)M.m));
  AM24_TRY(mat->mem.get(&key, (size_t)M.m));
  if (M.ldn > M.n)  // the pad columns of both planes (2m rows)
    AM24_CUDA(cudaMemset2DAsync(p + M.n, sizeof(uint16_t) * M.ldn, 0,
                                sizeof(uint16_t) * (M.ldn - M.n), 2 * (size_t)M.m, h->stream));
  M.Bt_h2 = p;
  M.bt_row_scale = rs;
  cudaError_t e = launch_prep_bt_fp16x2(M, key, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) {
    M.Bt_h2 = nullptr;
    M.bt_row_scale = nullptr;
    return fail(AM24_ERR_CUDA, std::string("FP16 planes of B^T: ") + cudaGetErrorString(e));
  }
  return AM24_OK;
}

// The phase word a MIXED batch starts in: the FP32 lead-in when it has one
// (lead + 1: that many accurate steps left, plus one), else the single-pass phase 0.
uint32_t mixed_first_phase(uint32_t lead) { return lead > 0 ? lead + 1u : 0u; }

// MIXED: back to the first phase with no start counted stable (a new batch).
cudaError_t reset_mixed(const BatchDev &d, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(d.stable, 0, sizeof(uint32_t) * d.k, st);
  const uint32_t words[4] = {mixed_first_phase(d.lead), 0u, 0u, 0u};
  // pageable source: staged before the call returns
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d.phase, words, sizeof words, cudaMemcpyHostToDevice, st);
  return e;
}

}  // namespace am24host

// The starting points staged in b's Vraw (all batch_size columns) become the
// batch's loadings: values and masks, dense-step gate, no select hints, and
// ValueCoordinateHolder::reset (c++/src/utils/various.h:33-38).
static am24_status load_from_vraw(am24_handle h, am24_batch b) {
  const MatrixDev &M = b->mat->d;
  const int k = b->d.k;
  AM24_CUDA(launch_load_columns(b->d.Vraw, M.ldn, M.n, k, b->d.Vx, M.ldn, b->d.vmask, h->stream));
  AM24_CUDA(cudaMemsetAsync(b->d.max_nnz, 0xFF, sizeof(uint32_t), h->stream));  // dense starts
  AM24_CUDA(cudaMemsetAsync(b->d.planes_nnz, 0, sizeof(uint32_t), h->stream));  // stale planes
  AM24_CUDA(cudaMemsetAsync(b->d.sel_hint, 0, sizeof(float) * k, h->stream));      // no hints
  AM24_CUDA(cudaMemsetAsync(b->d.val, 0, sizeof(float) * k, h->stream));
  AM24_CUDA(cudaMemsetAsync(b->d.err, 0, sizeof(float) * k, h->stream));
  AM24_CUDA(cudaMemsetAsync(b->d.ctl, 0, sizeof(uint32_t) * CTL_WORDS, h->stream));
  if (b->d.mixed) AM24_CUDA(reset_mixed(b->d, h->stream));
  return AM24_OK;
}

namespace am24host {

// Split-K factor for Z = B V: minimise rounds * (K blocks per unit + fixed
// per-unit cost) over the persistent grid.
void choose_splits(int tiles, int kb_total, int sms, int *splits, int *kbps) {
  double best_cost = 1e300;
  *splits = 1;
  *kbps = kb_total;
  for (int s = 1; s <= std::min(kb_total, 64); s++) {
    const int per = (kb_total + s - 1) / s;
    if (per < 4 && s > 1) break;
    const int s_eff = (kb_total + per - 1) / per;
    const long units = (long)tiles * s_eff;
    const long rounds = (units + sms - 1) / sms;
    const double cost = (double)rounds * (per + 8.0);
    if (cost < best_cost - 1e-9) {
      best_cost = cost;
      *splits = s_eff;
      *kbps = per;
    }
  }
}

am24_status validate_settings(const am24_settings *s) {
  if (!s) return fail(AM24_ERR_INVALID_ARG, "settings is NULL");
  if (s->formulation < 0 || s->formulation > 7)
    return fail(AM24_ERR_INVALID_ARG, "formulation must be 0..7");
  if (s->max_iter < 0) return fail(AM24_ERR_INVALID_ARG, "max_iter must be >= 0");
  if (s->total_starts < 1 && s->batch_size < 1)
    return fail(AM24_ERR_INVALID_ARG, "total_starts and batch_size cannot both be < 1");
  if (s->batch_size < 0) return fail(AM24_ERR_INVALID_ARG, "batch_size must be >= 0");
  if (is_constrained(s->formulation) && s->constraint < 1)
    return fail(AM24_ERR_INVALID_ARG, "constraint (s) must be >= 1 for constrained formulations");
  if (s->start_mode != AM24_START_REFERENCE && s->start_mode != AM24_START_INJECTED &&
      s->start_mode != AM24_START_DEVICE_UNIFORM)
    return fail(AM24_ERR_INVALID_ARG, "unknown start_mode");
  if (s->start_mode == AM24_START_DEVICE_UNIFORM && s->use_otf)
    return fail(AM24_ERR_INVALID_ARG, "device starts need batch mode (use_otf = 0)");
  if (s->l1_mode != AM24_L1_REFERENCE_SCAN && s->l1_mode != AM24_L1_EXACT)
    return fail(AM24_ERR_INVALID_ARG, "unknown l1_mode");
  if (s->precision != AM24_PRECISION_FP32 && s->precision != AM24_PRECISION_MIXED)
    return fail(AM24_ERR_INVALID_ARG, "unknown precision");
  if (s->precision == AM24_PRECISION_MIXED && !(s->stable_share > 0.f && s->stable_share <= 1.f))
    return fail(AM24_ERR_INVALID_ARG, "stable_share must be in (0, 1]");
  return AM24_OK;
}

StepParams step_params(const am24_settings &s, int it, int shift) {
  StepParams p;
  p.formulation = s.formulation;
  p.constraint = s.constraint;
  p.penalty = s.penalty;
  p.tolerance = s.tolerance;
  p.use_sort_hard = s.use_sort_hard;
  p.l1_mode = s.l1_mode;
  p.store_all = s.store_all;
  p.it = it;
  p.log_shift = shift;
  p.timeout_ns = (unsigned long long)(s.timeout_ms ? s.timeout_ms : 5000u) * 1000000ull;
  return p;
}

am24_status check_device_status(am24_batch b) {
  int st = 0;
  AM24_CUDA(cudaMemcpy(&st, b->d.status, sizeof(int), cudaMemcpyDeviceToHost));
  if (st != 0) {
    char buf[96];
    snprintf(buf, sizeof buf, "device-side wait timed out (code 0x%x)", st);
    return fail(AM24_ERR_DEVICE_TIMEOUT, buf);
  }
  return AM24_OK;
}

// What a batch loop ran: its steps, how many of them in the BF16 phase
// (MIXED), and the last step's largest change.
struct BatchRun {
  int steps = 0;
  uint32_t low_steps = 0;
  float max_err = 0.f;
};

// The reference's batch loop (sparse_PCA_solver.h:192-212) over the loaded
// batch: steps it = 0, 1, ... until one with it > 0, in the refinement phase,
// leaves the batch's largest change below the tolerance, or max_iter steps.
// The test runs on the device at the end of each step (finalize), which then
// sets the batch's stop word; steps stay queued up to AHEAD ahead of the
// host's look at that word, and the ones queued past the stop return at once.
am24_status run_batch_steps(am24_handle h, am24_batch b, const am24_settings &s, int shift,
                            BatchRun *out) {
  constexpr int AHEAD = am24_handle_s::AHEAD;
  const BatchDev &d = b->d;
  for (int it = 0; it < s.max_iter; it++) {
    StepParams p = step_params(s, it, shift);
    p.stop_check = 1;
    AM24_CUDA(launch_am_step(b->mat->d, b->d, b->tm, p, h->stream, &b->launches));
    AM24_CUDA(cudaMemcpyAsync(&h->flags[it % AHEAD], d.ctl + CTL_STOP, sizeof(uint32_t),
                              cudaMemcpyDeviceToHost, h->stream));
    AM24_CUDA(cudaEventRecord(h->run_ev[it % AHEAD], h->stream));
    const int probe = it - (AHEAD - 1);  // the oldest step still unread
    if (probe >= 0) {
      AM24_CUDA(cudaEventSynchronize(h->run_ev[probe % AHEAD]));
      if (h->flags[probe % AHEAD]) break;
    }
  }
  uint32_t c[CTL_WORDS];
  AM24_CUDA(cudaMemcpyAsync(c, d.ctl, sizeof c, cudaMemcpyDeviceToHost, h->stream));
  AM24_CUDA(cudaStreamSynchronize(h->stream));
  AM24_TRY(check_device_status(b));
  out->steps = (int)c[CTL_STEPS];
  out->low_steps = c[CTL_LOW_STEPS];
  memcpy(&out->max_err, &c[CTL_MAX_ERR], sizeof(float));
  return AM24_OK;
}

// getSignleStartingPoint (c++/src/gpower/gpower_commons.h:22-47) for global
// start index g, into a zeroed column x of length n, with the reference's
// float arithmetic: constrained forms draw s (index, value) pairs from rand_r
// seeded with g and scale by 1/sqrt(sum value^2); penalized forms draw
// U[-1, 1] entries and do not normalise.
void reference_start(float *x, unsigned n, bool constrained, unsigned s, unsigned g) {
  unsigned seed = g;
  if (constrained) {
    float norm = 0.f;
    for (unsigned i = 0; i < s; i++) {
      unsigned idx = (unsigned)(int)((float)n * (float)rand_r(&seed) / (float)RAND_MAX);
      if (idx == n) idx--;
      const float tmp = (float)rand_r(&seed) / (float)RAND_MAX;
      x[idx] = tmp;
      norm += tmp * tmp;
    }
    const float f = 1.0f / std::sqrt(norm);
    for (unsigned i = 0; i < n; i++) x[i] *= f;
  } else {
    for (unsigned i = 0; i < n; i++) {
      float tmp = (float)rand_r(&seed) / (float)RAND_MAX;
      tmp = -1.0f + 2.0f * tmp;
      x[i] = tmp;
    }
  }
}

// Fills `cols` starting-point columns (global indices first..) into host
// staging (n x cols, leading dimension n) from the caller's matrix or the
// reference generator.
void host_starts(const am24_settings &s, unsigned n, const float *start_points,
                 const unsigned *global_idx, int cols, std::vector<float> &out) {
  out.assign((size_t)n * cols, 0.f);
  for (int c = 0; c < cols; c++) {
    float *dst = &out[(size_t)c * n];
    if (s.start_mode == AM24_START_INJECTED)
      std::memcpy(dst, start_points + (size_t)global_idx[c] * n, sizeof(float) * n);
    else
      reference_start(dst, n, is_constrained(s.formulation), s.constraint, global_idx[c]);
  }
}

am24_status upload_columns(am24_handle h, am24_batch b, const float *host, int cols,
                           const int *slots) {
  const MatrixDev &M = b->mat->d;
  // stage through Vraw (raw GEMM output, free between steps), then split
  for (int c = 0; c < cols; c++) {
    AM24_CUDA(cudaMemcpyAsync(b->d.Vraw + (size_t)slots[c] * M.ldn, host + (size_t)c * M.n,
                              sizeof(float) * M.n, cudaMemcpyHostToDevice, h->stream));
    AM24_CUDA(launch_load_columns(b->d.Vraw + (size_t)slots[c] * M.ldn, M.ldn, M.n, 1,
                                  b->d.Vx + (size_t)slots[c] * M.ldn, M.ldn,
                                  b->d.vmask + (size_t)slots[c] * (M.ldn / 32), h->stream));
    AM24_CUDA(cudaMemsetAsync(b->d.sel_hint + slots[c], 0, sizeof(float), h->stream));
  }
  // new starts are dense: the next Z = B V runs on the tensor cores
  AM24_CUDA(cudaMemsetAsync(b->d.max_nnz, 0xFF, sizeof(uint32_t), h->stream));
  AM24_CUDA(cudaMemsetAsync(b->d.planes_nnz, 0, sizeof(uint32_t), h->stream));  // stale planes
  return AM24_OK;
}

}  // namespace am24host

// ============================================================== library
extern "C" {

uint32_t am24_abi_version(void) { return AM24_ABI_VERSION; }

const char *am24_last_error(void) { return g_last_error.c_str(); }

const char *am24_status_string(am24_status s) {
  switch (s) {
    case AM24_OK: return "ok";
    case AM24_ERR_INVALID_ARG: return "invalid argument";
    case AM24_ERR_OOM: return "out of device memory";
    case AM24_ERR_CUDA: return "CUDA error";
    case AM24_ERR_DEVICE_TIMEOUT: return "device-side wait timed out";
    case AM24_ERR_UNSUPPORTED: return "unsupported";
    case AM24_ERR_DEGENERATE: return "degenerate start (NaN objective)";
    case AM24_ERR_ADMISSION_REJECTED: return "admission rejected (HBM budget)";
  }
  return "unknown status";
}

// OptimizationSettings() defaults (c++/src/class/optimization_settings.h:101-123).
void am24_default_settings(am24_settings *s) {
  if (!s) return;
  std::memset(s, 0, sizeof *s);
  s->formulation = AM24_L0_CONSTRAINED_L2_PCA;
  s->tolerance = 0.01;
  s->constraint = 10;
  s->penalty = 0;
  s->total_starts = 64;
  s->batch_size = 64;
  s->use_sort_hard = 0;
  s->use_otf = 0;
  s->max_iter = 20;
  s->store_all = 0;
  s->start_mode = AM24_START_REFERENCE;
  s->l1_mode = AM24_L1_REFERENCE_SCAN;
  s->timeout_ms = 5000;
  s->precision = AM24_PRECISION_FP32;
  s->stable_iterations = 5;
  s->stable_share = 1.0f;
}

// chceckInputAndModifyIt (c++/src/class/optimization_settings.h:156-168).
am24_status am24_check_input(am24_settings *s, uint32_t n) {
  if (!s) return fail(AM24_ERR_INVALID_ARG, "settings is NULL");
  if (s->constraint > n) s->constraint = n;
  if (s->batch_size == 0) s->batch_size = s->total_starts;
  if (s->batch_size <= 0) return fail(AM24_ERR_INVALID_ARG, "batch_size must be positive");
  s->total_batches = (uint32_t)(s->total_starts / s->batch_size);
  if (s->total_batches * (uint32_t)s->batch_size < (uint32_t)std::max(s->total_starts, 0))
    s->total_batches++;
  s->total_starts = (int32_t)(s->total_batches * (uint32_t)s->batch_size);
  return AM24_OK;
}

am24_status am24_create(am24_handle *out, int device) {
  if (!out) return fail(AM24_ERR_INVALID_ARG, "handle pointer is NULL");
  *out = nullptr;
  int count = 0;
  AM24_CUDA(cudaGetDeviceCount(&count));
  if (device < 0 || device >= count)
    return fail(AM24_ERR_INVALID_ARG, "device index out of range");
  AM24_CUDA(cudaSetDevice(device));
  cudaDeviceProp prop;
  AM24_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10)
    return fail(AM24_ERR_UNSUPPORTED, std::string("needs an sm_100 (B200-class) GPU, found ") +
                                          prop.name);
  // Stream-ordered allocations (batches, one-call matrices, temporaries) come
  // from the device's default pool; keep what they free there for reuse
  // instead of returning it to the driver at every synchronization, which makes
  // the next allocation map the memory again.
  cudaMemPool_t pool;
  AM24_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
  uint64_t keep = UINT64_MAX;
  AM24_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
  auto *h = new am24_handle_s();
  h->device = device;
  cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) {
    e = cudaStreamCreateWithFlags(&h->copy, cudaStreamNonBlocking);
    if (e != cudaSuccess) cudaStreamDestroy(h->stream);
  }
  if (e != cudaSuccess) {
    delete h;
    return fail(AM24_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
  }
  void *fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
  if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn) {
    cudaStreamDestroy(h->stream);
    cudaStreamDestroy(h->copy);
    delete h;
    return fail(AM24_ERR_CUDA, "cuTensorMapEncodeTiled entry point not available");
  }
  h->encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  am24_status st = h->scratch.get(&h->ev_out, 1);
  if (st == AM24_OK && cudaMallocHost(reinterpret_cast<void **>(&h->flags),
                                      sizeof(uint32_t) * am24_handle_s::AHEAD) != cudaSuccess)
    st = fail(AM24_ERR_CUDA, "cudaMallocHost failed");
  for (int i = 0; st == AM24_OK && i < am24_handle_s::AHEAD; i++)
    if (cudaEventCreateWithFlags(&h->run_ev[i], cudaEventDisableTiming) != cudaSuccess)
      st = fail(AM24_ERR_CUDA, "cudaEventCreate failed");
  if (st != AM24_OK) {
    for (int i = 0; i < am24_handle_s::AHEAD; i++)
      if (h->run_ev[i]) cudaEventDestroy(h->run_ev[i]);
    if (h->flags) cudaFreeHost(h->flags);
    cudaStreamDestroy(h->stream);
    cudaStreamDestroy(h->copy);
    delete h;
    return st;
  }
  *out = h;
  return AM24_OK;
}

am24_status am24_destroy(am24_handle h) {
  if (!h) return AM24_OK;
  cudaSetDevice(h->device);
  cudaStreamSynchronize(h->copy);
  cudaStreamSynchronize(h->stream);
  for (int i = 0; i < am24_handle_s::AHEAD; i++) cudaEventDestroy(h->run_ev[i]);
  cudaFreeHost(h->flags);
  cudaStreamDestroy(h->copy);
  cudaStreamDestroy(h->stream);
  delete h;
  return AM24_OK;
}

am24_status am24_selftest_bounded_wait(am24_handle h, uint32_t timeout_us) {
  if (!h) return fail(AM24_ERR_INVALID_ARG, "NULL handle");
  AM24_CUDA(cudaSetDevice(h->device));
  int *status = nullptr;
  Allocs local(h->stream);
  AM24_TRY(local.get(&status, 1));
  AM24_CUDA(cudaMemsetAsync(status, 0, sizeof(int), h->stream));
  AM24_CUDA(launch_bounded_wait_probe((unsigned long long)timeout_us * 1000ull, status,
                                      h->stream));
  int code = 0;
  AM24_CUDA(cudaMemcpyAsync(&code, status, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  AM24_CUDA(cudaStreamSynchronize(h->stream));
  if (code != 0) {
    char buf[96];
    snprintf(buf, sizeof buf, "device-side wait timed out (code 0x%x)", code);
    return fail(AM24_ERR_DEVICE_TIMEOUT, buf);
  }
  return fail(AM24_ERR_CUDA, "the bounded-wait probe returned without giving up");
}

am24_status am24_sync(am24_handle h) {
  if (!h) return fail(AM24_ERR_INVALID_ARG, "handle is NULL");
  AM24_CUDA(cudaStreamSynchronize(h->stream));
  return AM24_OK;
}

// ============================================================== matrices
}  // extern "C"

// `ordered`: the matrix is private to the handle's stream (the one-call
// solves), so its memory is stream-ordered too.
static am24_status create_matrix(am24_handle h, const float *B, int32_t ldB, uint32_t m,
                                 uint32_t n, int32_t on_device, bool ordered, am24_matrix *out) {
  if (!h || !B || !out) return fail(AM24_ERR_INVALID_ARG, "NULL argument");
  *out = nullptr;
  if (m == 0 || n == 0) return fail(AM24_ERR_INVALID_ARG, "m and n must be positive");
  if (ldB < (int32_t)m) return fail(AM24_ERR_INVALID_ARG, "ldB must be >= m");
  if (m > (1u << 30) || n > (1u << 30)) return fail(AM24_ERR_INVALID_ARG, "matrix too large");
  AM24_CUDA(cudaSetDevice(h->device));
  auto *mat = new am24_matrix_s();
  if (ordered) {
    mat->mem.stream = h->stream;
    mat->mem.ordered = true;
  }
  MatrixDev &M = mat->d;
  M.m = (int)m;
  M.n = (int)n;
  M.ldm = round_up((int)m, 32);
  M.ldn = round_up((int)n, 32);
  am24_status st;
  const size_t c_elems = (size_t)n * M.ldm;
  if ((st = mat->mem.get(&M.Bc, c_elems)) != AM24_OK) {
    delete mat;
    return st;
  }
  // one 2-D copy straight into Bc's layout (host or device source), pad rows
  // zeroed; the other layouts are made from Bc when a batch first needs them
  cudaError_t e = cudaSuccess;
  if (M.ldm > (int)m)
    e = cudaMemset2DAsync(M.Bc + m, sizeof(float) * M.ldm, 0, sizeof(float) * (M.ldm - m), n,
                          h->stream);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(M.Bc, sizeof(float) * M.ldm, B, sizeof(float) * (size_t)ldB,
                          sizeof(float) * m, n,
                          on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                          h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) {
    delete mat;
    return fail(e == cudaErrorMemoryAllocation ? AM24_ERR_OOM : AM24_ERR_CUDA,
                std::string("matrix upload: ") + cudaGetErrorString(e));
  }
  *out = mat;
  return AM24_OK;
}

extern "C" {

am24_status am24_matrix_create_f32(am24_handle h, const float *B, int32_t ldB, uint32_t m,
                                   uint32_t n, int32_t on_device, am24_matrix *out) {
  return create_matrix(h, B, ldB, m, n, on_device, false, out);
}

am24_status am24_matrix_create_csc_f32(am24_handle h, const float *vals, const int32_t *row_ind,
                                       const int32_t *col_ptr, uint32_t m, uint32_t n,
                                       const float *means, const float *row_means,
                                       am24_matrix *out) {
  if (!col_ptr || !out) return fail(AM24_ERR_INVALID_ARG, "NULL argument");
  *out = nullptr;
  // the arrays are checked on the host first (no handle or device needed),
  // before any device write can use an index
  AM24_TRY(validate_csc(vals, row_ind, col_ptr, m, n));
  const size_t nnz = (size_t)col_ptr[n];
  if (!h) return fail(AM24_ERR_INVALID_ARG, "NULL handle");
  AM24_CUDA(cudaSetDevice(h->device));
  auto *mat = new am24_matrix_s();
  MatrixDev &M = mat->d;
  M.m = (int)m;
  M.n = (int)n;
  M.ldm = round_up((int)m, 32);
  M.ldn = round_up((int)n, 32);
  am24_status st = mat->mem.get(&M.Bc, (size_t)n * M.ldm);
  if (st != AM24_OK) {
    delete mat;
    return st;
  }
  Allocs local(h->stream);
  float *dv = nullptr, *dmean = nullptr, *drmean = nullptr;
  int32_t *dri = nullptr, *dcp = nullptr;
  cudaError_t e = cudaSuccess;
  if ((st = local.get(&dcp, (size_t)n + 1)) || (nnz && (st = local.get(&dv, nnz))) ||
      (nnz && (st = local.get(&dri, nnz))) || (means && (st = local.get(&dmean, (size_t)n))) ||
      (row_means && (st = local.get(&drmean, (size_t)m)))) {
    delete mat;
    return st;
  }
  e = cudaMemsetAsync(M.Bc, 0, sizeof(float) * (size_t)n * M.ldm, h->stream);
  if (!e) e = cudaMemcpyAsync(dcp, col_ptr, sizeof(int32_t) * (n + 1), cudaMemcpyHostToDevice,
                              h->stream);
  if (!e && nnz)
    e = cudaMemcpyAsync(dv, vals, sizeof(float) * nnz, cudaMemcpyHostToDevice, h->stream);
  if (!e && nnz)
    e = cudaMemcpyAsync(dri, row_ind, sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, h->stream);
  if (!e && means)
    e = cudaMemcpyAsync(dmean, means, sizeof(float) * n, cudaMemcpyHostToDevice, h->stream);
  if (!e && row_means)
    e = cudaMemcpyAsync(drmean, row_means, sizeof(float) * m, cudaMemcpyHostToDevice, h->stream);
  if (!e) e = launch_csc_to_dense(M, dv, dri, dcp, dmean, drmean, h->stream);
  if (!e) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) {
    delete mat;
    return fail(e == cudaErrorMemoryAllocation ? AM24_ERR_OOM : AM24_ERR_CUDA,
                std::string("sparse matrix upload: ") + cudaGetErrorString(e));
  }
  *out = mat;
  return AM24_OK;
}

am24_status am24_matrix_deflate(am24_handle h, am24_matrix mat, const float *x,
                                int32_t on_device) {
  if (!h || !mat || !x) return fail(AM24_ERR_INVALID_ARG, "NULL argument");
  if (mat->sparse) return deflate_sparse(h, mat, x, on_device);
  AM24_CUDA(cudaSetDevice(h->device));
  MatrixDev &M = mat->d;
  Allocs local(h->stream);
  float *xd = nullptr;
  double *partial = nullptr, *y = nullptr;
  AM24_TRY(local.get(&xd, (size_t)M.n));
  AM24_TRY(local.get(&partial, ev_partial_len(M)));
  AM24_TRY(local.get(&y, (size_t)M.m));
  AM24_CUDA(cudaMemcpyAsync(xd, x, sizeof(float) * M.n,
                            on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                            h->stream));
  AM24_CUDA(launch_deflate(M, xd, partial, y, h->stream));
  // every layout made so far is rebuilt from the new B, in place
  if (M.Bc_h2) AM24_CUDA(launch_prep_fp16x2(M, h->stream));
  if (M.Bt_h2) {
    uint32_t *key = nullptr;
    AM24_TRY(local.get(&key, (size_t)M.m));
    AM24_CUDA(launch_prep_bt_fp16x2(M, key, h->stream));
  }
  if (M.Bc_hi) AM24_CUDA(launch_prep_tf32_planes(M, h->stream));
  if (M.Bc_b3) AM24_CUDA(launch_prep_bf16x3(M, h->stream));
  AM24_CUDA(cudaStreamSynchronize(h->stream));
  return AM24_OK;
}

am24_status am24_matrix_read_f32(am24_handle h, am24_matrix mat, float *B, int32_t ldB) {
  if (!h || !mat || !B) return fail(AM24_ERR_INVALID_ARG, "NULL argument");
  if (mat->sparse) return fail(AM24_ERR_UNSUPPORTED, "a sparse-resident matrix has no dense copy");
  const MatrixDev &M = mat->d;
  if (ldB < M.m) return fail(AM24_ERR_INVALID_ARG, "ldB must be >= m");
  AM24_CUDA(cudaSetDevice(h->device));
  AM24_CUDA(cudaMemcpy2DAsync(B, sizeof(float) * (size_t)ldB, M.Bc, sizeof(float) * M.ldm,
                              sizeof(float) * M.m, M.n, cudaMemcpyDeviceToHost, h->stream));
  AM24_CUDA(cudaStreamSynchronize(h->stream));
  return AM24_OK;
}

am24_status am24_matrix_destroy(am24_handle h, am24_matrix mat) {
  if (!mat) return AM24_OK;
  if (h) {
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->stream);
  }
  delete mat;
  return AM24_OK;
}

// ============================================================== batches
am24_status am24_batch_create(am24_handle h, am24_matrix mat, const am24_settings *settings,
                              uint32_t batch_size, am24_batch *out) {
  if (!h || !mat || !out) return fail(AM24_ERR_INVALID_ARG, "NULL argument");
  *out = nullptr;
  AM24_TRY(validate_settings(settings));
  if (batch_size == 0 || batch_size > (1u << 20))
    return fail(AM24_ERR_INVALID_ARG, "batch_size must be in [1, 2^20]");
  if (is_constrained(settings->formulation) && settings->constraint > (uint32_t)mat->d.n)
    return fail(AM24_ERR_INVALID_ARG, "constraint exceeds n (run am24_check_input first)");
  if (mat->sparse)
    return fail(AM24_ERR_UNSUPPORTED, "sparse-resident matrices are solved by am24_solve_resident_f32 only");
  AM24_CUDA(cudaSetDevice(h->device));
  auto *b = new am24_batch_s();
  b->mem.stream = h->stream;  // used on this handle's stream only
  b->mem.ordered = true;
  b->mat = mat;
  b->s = *settings;
  const MatrixDev &M = mat->d;
  BatchDev &d = b->d;
  const int k = (int)batch_size;
  d.k = k;
  d.bn1 = pick_bn(k);
  d.bn2 = pick_bn(k);
  d.m_tiles1 = (M.m + BM - 1) / BM;
  d.n_tiles1 = (k + d.bn1 - 1) / d.bn1;
  d.m_tiles2 = (M.n + BM - 1) / BM;
  d.n_tiles2 = (k + d.bn2 - 1) / d.bn2;
  d.bk = BK_DEFAULT;
  if (const char *e = getenv("AM24_GEMM_BK")) d.bk = (atoi(e) == 16) ? 16 : 32;
  // V = B^T Z on CTA pairs when its N tile is 256 (AM24_GEMM_PAIR=0 turns it off),
  // with split FP16 operands (AM24_GEMM_FP16=0 turns that off), else with exact
  // BF16 operands for the L1-variance forms (AM24_GEMM_BF16=0 turns that off)
  // or TF32 hi/lo planes
  d.pair2 = d.bn2 == 256;
  if (const char *e = getenv("AM24_GEMM_PAIR")) d.pair2 = d.pair2 && atoi(e) != 0;
  d.fp16_2 = d.pair2;
  if (const char *e = getenv("AM24_GEMM_FP16")) d.fp16_2 = d.fp16_2 && atoi(e) != 0;
  // Z = B V on FP16 CTA pairs under the same switches, when its N tile is 256
  d.fp16_1 = d.fp16_2 && d.bn1 == 256;
  d.bf16_2 = d.pair2 && !d.fp16_2 && is_l1_variance(settings->formulation);
  if (const char *e = getenv("AM24_GEMM_BF16")) d.bf16_2 = d.bf16_2 && atoi(e) != 0;
  // MIXED runs its BF16 phase on CTA-pair tiles; narrower batches stay FP32
  d.mixed = settings->precision == AM24_PRECISION_MIXED && d.pair2;
  // the low-precision phase on single-pass FP16 operands (AM24_MIXED_BF16=1:
  // single-pass BF16, the FP16 planes off or not)
  d.mixed_fp16 = d.mixed && d.fp16_2;
  if (const char *e = getenv("AM24_MIXED_BF16")) d.mixed_fp16 = d.mixed_fp16 && atoi(e) == 0;
  d.k_stable = settings->stable_iterations;
  d.lead = settings->lead_iterations;
  d.need_stable = (uint32_t)std::max(1.0, std::ceil((double)settings->stable_share * k - 1e-9));
  d.need_stable = std::min(d.need_stable, (uint32_t)k);
  const bool need_bf16 = d.bf16_2 || (d.mixed && !d.mixed_fp16);
  // TF32 planes: Z = B V off the FP16 pairs; V = B^T Z with neither FP16 nor BF16 operands
  const bool tf32_1 = !d.fp16_1, tf32_2 = !d.fp16_2 && !d.bf16_2;
  const size_t zh_planes = is_l1_variance(settings->formulation) ? 1 : 2;
  // constrained forms: V = B^T Z's epilogue lists the selects' hinted
  // candidates (AM24_SELECT_LIST=0 leaves the gather to the select kernels)
  bool lists = is_constrained(settings->formulation);
  if (const char *e = getenv("AM24_SELECT_LIST")) lists = lists && atoi(e) != 0;
  const int bk2 = d.pair2 ? PAIR_BK_TF32 : d.bk;  // K box of the TF32 maps of V = B^T Z
  const int kb_total1 = (M.n + d.bk - 1) / d.bk;
  choose_splits(d.m_tiles1 * d.n_tiles1, kb_total1, num_sms(), &d.splits1, &d.kbps1);
  d.ws_len = ws_floats(d.splits1, d.m_tiles1, d.n_tiles1, d.bn1);
  if (d.fp16_1) {  // pair tiles of 256 rows, K blocks of 32, one unit per cluster (2 SMs)
    int kbps = 0;
    choose_splits(((d.m_tiles1 + 1) / 2) * d.n_tiles1, (M.n + PAIR_BK_BF16 - 1) / PAIR_BK_BF16,
                  std::max(1, num_sms() / 2), &d.splits1p, &kbps);
    d.ws_len = std::max(d.ws_len, ws_floats(d.splits1p, d.m_tiles1, d.n_tiles1, d.bn1));
  }
  const int parts = d.m_tiles2 * 4;
  d.log_capacity = std::max(settings->total_starts, k);
  am24_status st;
  auto &A = b->mem;
  const size_t kv = (size_t)k * M.ldn, kz = (size_t)k * M.ldm;
  if ((st = A.get(&d.Vx, kv)) ||
      (tf32_1 && ((st = A.get(&d.V_hi, kv)) || (st = A.get(&d.V_lo, kv)))) ||
      ((tf32_1 || tf32_2) && (st = ensure_tf32_planes(h, mat))) ||
      (st = A.get(&d.Vraw, kv)) ||
      (st = A.get(&d.Z_hi, kz)) || (st = A.get(&d.Z_lo, kz)) ||
      (st = A.get(&d.ws, d.ws_len)) ||
      (st = A.get(&d.fz, k)) || (st = A.get(&d.obj_part, (size_t)k * parts)) ||
      (st = A.get(&d.nnz_part, (size_t)k * parts)) || (st = A.get(&d.nnz, k)) ||
      (st = A.get(&d.val, k)) || (st = A.get(&d.err, k)) || (st = A.get(&d.max_err, 1)) ||
      (st = A.get(&d.iters, d.log_capacity)) || (st = A.get(&d.cards, d.log_capacity)) ||
      (st = A.get(&d.status, 1)) || (st = A.get(&d.vmask, (size_t)k * (M.ldn / 32))) ||
      (st = A.get(&d.max_nnz, 1)) || (st = A.get(&d.planes_nnz, 1)) ||
      (st = A.get(&d.sel_hint, k)) || (st = A.get(&d.ctl, (size_t)CTL_WORDS)) ||
      (lists && (st = A.get(&d.cmask, (size_t)k * (M.ldn / 32)))) ||
      (need_bf16 &&
       ((st = A.get(&d.Z_b, kz)) || (st = ensure_bf16_planes(h, mat, d.bf16_2 ? 3 : 1)))) ||
      (d.fp16_2 && ((st = A.get(&d.Z_h, zh_planes * kz)) || (st = A.get(&d.z_scale, k)) ||
                    (st = ensure_fp16_planes(h, mat)))) ||
      (d.fp16_1 && ((st = A.get(&d.V_h, 2 * kv)) || (st = A.get(&d.v_scale, k)) ||
                    (st = ensure_bt_fp16_planes(h, mat)))) ||
      (d.mixed && ((st = A.get(&d.vmask_prev, (size_t)k * (M.ldn / 32))) ||
                   (st = A.get(&d.stable, k)) || (st = A.get(&d.phase, 4))))) {
    delete b;
    return st;
  }
  cudaError_t e = cudaMemsetAsync(d.Vx, 0, sizeof(float) * kv, h->stream);
  if (!e && d.V_hi) e = cudaMemsetAsync(d.V_hi, 0, sizeof(float) * kv, h->stream);
  if (!e && d.V_lo) e = cudaMemsetAsync(d.V_lo, 0, sizeof(float) * kv, h->stream);
  if (!e) e = cudaMemsetAsync(d.Vraw, 0, sizeof(float) * kv, h->stream);
  if (!e) e = cudaMemsetAsync(d.Z_hi, 0, sizeof(float) * kz, h->stream);
  if (!e) e = cudaMemsetAsync(d.Z_lo, 0, sizeof(float) * kz, h->stream);
  if (!e) e = cudaMemsetAsync(d.val, 0, sizeof(float) * k, h->stream);
  if (!e) e = cudaMemsetAsync(d.err, 0, sizeof(float) * k, h->stream);
  if (!e) e = cudaMemsetAsync(d.fz, 0, sizeof(float) * k, h->stream);
  if (!e) e = cudaMemsetAsync(d.nnz, 0, sizeof(uint32_t) * k, h->stream);
  if (!e) e = cudaMemsetAsync(d.status, 0, sizeof(int), h->stream);
  if (!e) e = cudaMemsetAsync(d.vmask, 0, sizeof(uint32_t) * k * (M.ldn / 32), h->stream);
  if (!e) e = cudaMemsetAsync(d.max_nnz, 0xFF, sizeof(uint32_t), h->stream);
  if (!e) e = cudaMemsetAsync(d.planes_nnz, 0, sizeof(uint32_t), h->stream);
  if (!e) e = cudaMemsetAsync(d.sel_hint, 0, sizeof(float) * k, h->stream);
  if (!e) e = cudaMemsetAsync(d.ctl, 0, sizeof(uint32_t) * CTL_WORDS, h->stream);
  if (!e && d.cmask)
    e = cudaMemsetAsync(d.cmask, 0, sizeof(uint32_t) * k * (M.ldn / 32), h->stream);
  if (!e && d.Z_b) e = cudaMemsetAsync(d.Z_b, 0, sizeof(uint16_t) * kz, h->stream);
  if (!e && d.Z_h) e = cudaMemsetAsync(d.Z_h, 0, sizeof(uint16_t) * zh_planes * kz, h->stream);
  if (!e && d.z_scale) e = cudaMemsetAsync(d.z_scale, 0, sizeof(float) * k, h->stream);
  if (!e && d.V_h) e = cudaMemsetAsync(d.V_h, 0, sizeof(uint16_t) * 2 * kv, h->stream);
  if (!e && d.v_scale) e = cudaMemsetAsync(d.v_scale, 0, sizeof(float) * k, h->stream);
  d.row_scale = M.row_scale;
  d.bt_row_scale = M.bt_row_scale;
  if (!e && d.mixed)
    e = cudaMemsetAsync(d.vmask_prev, 0, sizeof(uint32_t) * k * (M.ldn / 32), h->stream);
  if (!e && d.mixed) e = reset_mixed(d, h->stream);
  if (!e) e = cudaMemsetAsync(d.iters, 0xFF, sizeof(int) * d.log_capacity, h->stream);
  if (!e) e = cudaMemsetAsync(d.cards, 0xFF, sizeof(int) * d.log_capacity, h->stream);
  if (!e) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) {
    delete b;
    return fail(AM24_ERR_CUDA, std::string("batch init: ") + cudaGetErrorString(e));
  }
  if ((tf32_1 && ((st = make_map(h, &b->tm.a1_hi, M.Bt_hi, M.n, M.m, M.ldn, BM, d.bk)) ||
                  (st = make_map(h, &b->tm.a1_lo, M.Bt_lo, M.n, M.m, M.ldn, BM, d.bk)) ||
                  (st = make_map(h, &b->tm.b1_hi, d.V_hi, M.n, k, M.ldn, d.bn1, d.bk)) ||
                  (st = make_map(h, &b->tm.b1_lo, d.V_lo, M.n, k, M.ldn, d.bn1, d.bk)))) ||
      (tf32_2 &&
       ((st = make_map(h, &b->tm.a2_hi, M.Bc_hi, M.m, M.n, M.ldm, BM, bk2)) ||
        (st = make_map(h, &b->tm.a2_lo, M.Bc_lo, M.m, M.n, M.ldm, BM, bk2)) ||
        (st = make_map(h, &b->tm.b2_hi, d.Z_hi, M.m, k, M.ldm, d.pair2 ? d.bn2 / 2 : d.bn2,
                       bk2)) ||
        (st = make_map(h, &b->tm.b2_lo, d.Z_lo, M.m, k, M.ldm, d.pair2 ? d.bn2 / 2 : d.bn2,
                       bk2))))) {
    delete b;
    return st;
  }
  if (need_bf16) {
    const size_t plane = (size_t)M.n * M.ldm;
    if ((st = make_map_bf16(h, &b->tm.a2_b0, M.Bc_b3, M.m, M.n, M.ldm, BM)) ||
        (d.bf16_2 &&
         ((st = make_map_bf16(h, &b->tm.a2_b1, M.Bc_b3 + plane, M.m, M.n, M.ldm, BM)) ||
          (st = make_map_bf16(h, &b->tm.a2_b2, M.Bc_b3 + 2 * plane, M.m, M.n, M.ldm, BM)))) ||
        (st = make_map_bf16(h, &b->tm.b2_b, d.Z_b, M.m, k, M.ldm, d.bn2 / 2))) {
      delete b;
      return st;
    }
  }
  if (d.fp16_2) {
    const size_t plane = (size_t)M.n * M.ldm;
    if ((st = make_map_bf16(h, &b->tm.a2_h0, M.Bc_h2, M.m, M.n, M.ldm, BM, true)) ||
        (st = make_map_bf16(h, &b->tm.a2_h1, M.Bc_h2 + plane, M.m, M.n, M.ldm, BM, true)) ||
        (st = make_map_bf16(h, &b->tm.b2_h0, d.Z_h, M.m, k, M.ldm, d.bn2 / 2, true)) ||
        (zh_planes == 2 &&
         (st = make_map_bf16(h, &b->tm.b2_h1, d.Z_h + kz, M.m, k, M.ldm, d.bn2 / 2, true)))) {
      delete b;
      return st;
    }
  }
  if (d.fp16_1) {
    const size_t plane = (size_t)M.m * M.ldn;
    if ((st = make_map_bf16(h, &b->tm.a1_h0, M.Bt_h2, M.n, M.m, M.ldn, BM, true)) ||
        (st = make_map_bf16(h, &b->tm.a1_h1, M.Bt_h2 + plane, M.n, M.m, M.ldn, BM, true)) ||
        (st = make_map_bf16(h, &b->tm.b1_h0, d.V_h, M.n, k, M.ldn, d.bn1 / 2, true)) ||
        (st = make_map_bf16(h, &b->tm.b1_h1, d.V_h + kv, M.n, k, M.ldn, d.bn1 / 2, true))) {
      delete b;
      return st;
    }
  }
  // a gather over V's non-zeros beats the dense product while they are few
  d.sparse_cap = (uint32_t)std::min(4096, M.n / 32);
  b->launches = (is_constrained(settings->formulation) ? 8 : 7) + (d.mixed ? 2 : 0);
  *out = b;
  return AM24_OK;
}

am24_status am24_batch_destroy(am24_handle h, am24_batch b) {
  if (!b) return AM24_OK;
  if (h) {
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->stream);
  }
  delete b;
  return AM24_OK;
}

am24_status am24_batch_load(am24_handle h, am24_batch b, const float *V, int32_t on_device) {
  if (!h || !b || !V) return fail(AM24_ERR_INVALID_ARG, "NULL argument");
  const MatrixDev &M = b->mat->d;
  const int k = b->d.k;
  if (on_device) {
    AM24_CUDA(cudaMemcpy2DAsync(b->d.Vraw, sizeof(float) * M.ldn, V, sizeof(float) * M.n,
                                sizeof(float) * M.n, k, cudaMemcpyDeviceToDevice, h->stream));
  } else {
    AM24_CUDA(cudaMemcpy2DAsync(b->d.Vraw, sizeof(float) * M.ldn, V, sizeof(float) * M.n,
                                sizeof(float) * M.n, k, cudaMemcpyHostToDevice, h->stream));
  }
  return load_from_vraw(h, b);
}

am24_status am24_batch_iterate(am24_handle h, am24_batch b, int32_t it0, int32_t iterations,
                               float *max_error) {
  if (!h || !b) return fail(AM24_ERR_INVALID_ARG, "NULL argument");
  for (int i = 0; i < iterations; i++) {
    const StepParams p = step_params(b->s, it0 + i, 0);
    AM24_CUDA(launch_am_step(b->mat->d, b->d, b->tm, p, h->stream, &b->launches));
  }
  if (max_error) {
    AM24_CUDA(cudaMemcpyAsync(max_error, b->d.max_err, sizeof(float), cudaMemcpyDeviceToHost,
                              h->stream));
    AM24_CUDA(cudaStreamSynchronize(h->stream));
    AM24_TRY(check_device_status(b));
  }
  return AM24_OK;
}

am24_status am24_batch_read(am24_handle h, am24_batch b, float *V, float *val, float *err,
                            uint32_t *nnz) {
  if (!h || !b) return fail(AM24_ERR_INVALID_ARG, "NULL argument");
  const MatrixDev &M = b->mat->d;
  const int k = b->d.k;
  if (V) {
    AM24_CUDA(launch_masked_copy(b->d.Vx, b->d.vmask, M.ldn, M.n, k, b->d.Vraw, M.ldn,
                                 h->stream));
    AM24_CUDA(cudaMemcpy2DAsync(V, sizeof(float) * M.n, b->d.Vraw, sizeof(float) * M.ldn,
                                sizeof(float) * M.n, k, cudaMemcpyDeviceToHost, h->stream));
  }
  if (val)
    AM24_CUDA(cudaMemcpyAsync(val, b->d.val, sizeof(float) * k, cudaMemcpyDeviceToHost, h->stream));
  if (err)
    AM24_CUDA(cudaMemcpyAsync(err, b->d.err, sizeof(float) * k, cudaMemcpyDeviceToHost, h->stream));
  if (nnz) {
    if (is_constrained(b->s.formulation)) {
      AM24_CUDA(cudaMemcpyAsync(nnz, b->d.nnz, sizeof(uint32_t) * k, cudaMemcpyDeviceToHost,
                                h->stream));
    } else {
      // penalized forms count non-zeros in the GEMM epilogue partials
      const int parts = b->d.m_tiles2 * 4;
      std::vector<float> np((size_t)k * parts);
      AM24_CUDA(cudaMemcpyAsync(np.data(), b->d.nnz_part, sizeof(float) * np.size(),
                                cudaMemcpyDeviceToHost, h->stream));
      AM24_CUDA(cudaStreamSynchronize(h->stream));
      for (int j = 0; j < k; j++) {
        double c = 0;
        for (int q = 0; q < parts; q++) c += np[(size_t)j * parts + q];
        nnz[j] = (uint32_t)c;
      }
    }
  }
  AM24_CUDA(cudaStreamSynchronize(h->stream));
  AM24_TRY(check_device_status(b));
  return AM24_OK;
}

am24_status am24_batch_step_timed(am24_handle h, am24_batch b, int32_t it, float *ms,
                                  int32_t *kinds, int32_t *count) {
  if (!h || !b || !ms || !kinds || !count) return fail(AM24_ERR_INVALID_ARG, "NULL argument");
  cudaEvent_t ev[17];
  int made = 0;
  am24_status st = AM24_OK;
  for (; made < 17; made++)
    if (cudaEventCreate(&ev[made]) != cudaSuccess) {
      st = fail(AM24_ERR_CUDA, "cudaEventCreate failed");
      break;
    }
  int nl = 0, kk[17] = {0};
  uint32_t gate = 0, phase = 1, planes = 0;
  if (st == AM24_OK &&
      cudaMemcpyAsync(&gate, b->d.max_nnz, sizeof gate, cudaMemcpyDeviceToHost, h->stream) ==
          cudaSuccess &&
      cudaMemcpyAsync(&planes, b->d.planes_nnz, sizeof planes, cudaMemcpyDeviceToHost,
                      h->stream) == cudaSuccess &&
      (!b->d.mixed || cudaMemcpyAsync(&phase, b->d.phase, sizeof phase, cudaMemcpyDeviceToHost,
                                      h->stream) == cudaSuccess) &&
      cudaStreamSynchronize(h->stream) == cudaSuccess) {
    const StepParams p = step_params(b->s, it, 0);
    cudaError_t e = launch_am_step(b->mat->d, b->d, b->tm, p, h->stream, &nl, ev, kk);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    for (int i = 0; e == cudaSuccess && i < nl; i++) e = cudaEventElapsedTime(&ms[i], ev[i], ev[i + 1]);
    if (e != cudaSuccess) st = fail(AM24_ERR_CUDA, std::string("timed step: ") + cudaGetErrorString(e));
  }
  for (int i = 0; i < made; i++) cudaEventDestroy(ev[i]);
  if (st != AM24_OK) return st;
  // mark the kernels that a gate turned into no-ops: the Z = B V path the
  // step does not take, and (MIXED) the V = B^T Z of the other phase
  const bool sparse = gate <= b->d.sparse_cap;
  const bool grouped = sparse && gate <= std::min(b->d.sparse_cap, GATHER_GROUP_MAX_NNZ);
  for (int i = 0; i < nl; i++) {
    bool skipped = sparse ? (kk[i] == AM24_KERNEL_GEMM_BV || kk[i] == AM24_KERNEL_Z_REDUCE ||
                             kk[i] == AM24_KERNEL_DENSIFY ||
                             kk[i] == (grouped ? AM24_KERNEL_GATHER_BV
                                               : AM24_KERNEL_GATHER_BV_GROUP))
                          : (kk[i] == AM24_KERNEL_GATHER_BV || kk[i] == AM24_KERNEL_GATHER_BV_GROUP ||
                             (kk[i] == AM24_KERNEL_DENSIFY && planes > b->d.sparse_cap));
    if (b->d.mixed)
      skipped = skipped || (phase == 0 ? kk[i] == AM24_KERNEL_GEMM_BTZ
                                       : kk[i] == AM24_KERNEL_GEMM_BTZ_LOW);
    kinds[i] = kk[i] | (skipped ? AM24_KERNEL_SKIPPED : 0);
  }
  *count = nl;
  return check_device_status(b);
}

void *am24_stream(am24_handle h) { return h ? static_cast<void *>(h->stream) : nullptr; }

am24_status am24_batch_phase(am24_handle h, am24_batch b, int32_t *refining) {
  if (!h || !b || !refining) return fail(AM24_ERR_INVALID_ARG, "NULL argument");
  uint32_t phase = 1;
  if (b->d.mixed) {
    AM24_CUDA(cudaMemcpyAsync(&phase, b->d.phase, sizeof phase, cudaMemcpyDeviceToHost,
                              h->stream));
    AM24_CUDA(cudaStreamSynchronize(h->stream));
  }
  *refining = phase != 0 ? 1 : 0;
  return AM24_OK;
}

am24_status am24_batch_launches_per_step(am24_handle h, am24_batch b, int32_t *launches) {
  if (!h || !b || !launches) return fail(AM24_ERR_INVALID_ARG, "NULL argument");
  *launches = b->launches;
  return AM24_OK;
}

// ============================================================== solver
am24_status am24_solve_resident_f32(am24_handle h, am24_matrix mat, float *x,
                                    am24_settings *settings, am24_statistics *stats,
                                    const float *start_points, float *fval_out) {
  const auto t_call = std::chrono::steady_clock::now();
  if (!h || !mat || !x || !settings) return fail(AM24_ERR_INVALID_ARG, "NULL argument");
  AM24_TRY(validate_settings(settings));
  if (settings->start_mode == AM24_START_INJECTED && !start_points)
    return fail(AM24_ERR_INVALID_ARG, "start_mode INJECTED needs start_points");
  AM24_CUDA(cudaSetDevice(h->device));
  const MatrixDev &M = mat->d;
  const unsigned n = (unsigned)M.n;
  AM24_TRY(am24_check_input(settings, n));
  if (mat->sparse) return solve_sparse(h, mat, x, *settings, stats, start_points, fval_out);
  am24_settings &s = *settings;
  const int bs = s.batch_size;
  Allocs local(h->stream);

  // The first batch's injected starts cross to the device on the copy stream
  // while the batch and the matrix layouts it needs are prepared on the main
  // stream; the main stream waits for them before its first load.
  float *pre = nullptr;
  cudaEvent_t pre_ready = nullptr, pre_done = nullptr;
  struct PreGuard {
    cudaEvent_t *a, *c;
    ~PreGuard() {
      if (*a) cudaEventDestroy(*a);
      if (*c) cudaEventDestroy(*c);
    }
  } preg{&pre_ready, &pre_done};
  if (s.start_mode == AM24_START_INJECTED && !s.use_otf) {
    AM24_TRY(local.get(&pre, (size_t)n * bs));
    AM24_CUDA(cudaEventCreateWithFlags(&pre_ready, cudaEventDisableTiming));
    AM24_CUDA(cudaEventCreateWithFlags(&pre_done, cudaEventDisableTiming));
    AM24_CUDA(cudaEventRecord(pre_ready, h->stream));  // `pre` is allocated from here on
    AM24_CUDA(cudaStreamWaitEvent(h->copy, pre_ready, 0));
    AM24_CUDA(cudaMemcpyAsync(pre, start_points, sizeof(float) * (size_t)n * bs,
                              cudaMemcpyHostToDevice, h->copy));
    AM24_CUDA(cudaEventRecord(pre_done, h->copy));
  }
  // the main stream never runs ahead of the copy's completion past this scope
  struct CopyJoin {
    am24_handle h;
    cudaEvent_t *done;
    ~CopyJoin() {
      if (*done) cudaStreamWaitEvent(h->stream, *done, 0);
    }
  } join{h, &pre_done};

  am24_batch b = nullptr;
  AM24_TRY(am24_batch_create(h, mat, &s, (uint32_t)bs, &b));
  struct BatchGuard {
    am24_handle h;
    am24_batch b;
    ~BatchGuard() { am24_batch_destroy(h, b); }
  } guard{h, b};

  // best loading so far, kept as hi/lo planes; starts as the caller's x, which
  // the reference returns normalised when no start ever improves on -1
  float *xb = nullptr, *x_dev = nullptr;
  double *ev_rows = nullptr;
  AM24_TRY(local.get(&xb, n));
  AM24_TRY(local.get(&x_dev, n));
  AM24_TRY(local.get(&ev_rows, ev_partial_len(M)));
  AM24_CUDA(cudaMemcpyAsync(xb, x, sizeof(float) * n, cudaMemcpyHostToDevice, h->stream));

  cudaEvent_t e0, e1;
  AM24_CUDA(cudaEventCreate(&e0));
  AM24_CUDA(cudaEventCreate(&e1));
  struct EvGuard {
    cudaEvent_t a, c;
    ~EvGuard() {
      cudaEventDestroy(a);
      cudaEventDestroy(c);
    }
  } evg{e0, e1};

  std::vector<float> staging, val(bs), err(bs);
  std::vector<int> slots(bs);
  std::vector<unsigned> gidx(bs);
  float best = -1.f;
  uint32_t total_it = 0;
  uint64_t start_its = 0;
  uint32_t low_its = 0;  // batch iterations in the BF16 phase (MIXED)
  double compute_s = 0.0;
  float last_max_err = 0.f;
  int degenerate = 0;
  const BatchDev &d = b->d;
  auto take_best = [&](int j) -> am24_status {
    AM24_CUDA(launch_masked_copy(d.Vx + (size_t)j * M.ldn, d.vmask + (size_t)j * (M.ldn / 32),
                                 M.ldn, (int)n, 1, xb, (int)n, h->stream));
    return AM24_OK;
  };

  if (!s.use_otf) {
    // ---------------------------------- batches (sparse_PCA_solver.h:171-232)
    for (unsigned batch = 0; batch < s.total_batches; batch++) {
      const unsigned shift = batch * (unsigned)bs;
      for (int j = 0; j < bs; j++) {
        gidx[j] = shift + j;
        slots[j] = j;
      }
      // the batch's starts, staged in Vraw by one copy (or generated there)
      if (s.start_mode == AM24_START_DEVICE_UNIFORM) {
        AM24_CUDA(launch_uniform_starts(d.Vraw, M.ldn, (int)n, bs, shift, h->stream));
      } else if (batch == 0 && pre) {  // already on the device
        AM24_CUDA(cudaStreamWaitEvent(h->stream, pre_done, 0));
        AM24_CUDA(cudaMemcpy2DAsync(d.Vraw, sizeof(float) * M.ldn, pre, sizeof(float) * n,
                                    sizeof(float) * n, bs, cudaMemcpyDeviceToDevice, h->stream));
      } else {
        const float *src = start_points + (size_t)shift * n;  // injected: read in place
        if (s.start_mode != AM24_START_INJECTED) {
          host_starts(s, n, start_points, gidx.data(), bs, staging);
          src = staging.data();
        }
        AM24_CUDA(cudaMemcpy2DAsync(d.Vraw, sizeof(float) * M.ldn, src, sizeof(float) * n,
                                    sizeof(float) * n, bs, cudaMemcpyHostToDevice, h->stream));
      }
      AM24_TRY(load_from_vraw(h, b));
      if (d.mixed) AM24_CUDA(reset_mixed(d, h->stream));
      AM24_CUDA(cudaEventRecord(e0, h->stream));
      BatchRun run;
      AM24_TRY(run_batch_steps(h, b, s, (int)shift, &run));
      AM24_CUDA(cudaEventRecord(e1, h->stream));
      total_it += (uint32_t)run.steps;
      low_its += run.low_steps;
      start_its += (uint64_t)run.steps * (uint64_t)bs;
      last_max_err = run.max_err;
      AM24_CUDA(cudaMemcpyAsync(val.data(), d.val, sizeof(float) * bs, cudaMemcpyDeviceToHost,
                                h->stream));
      AM24_CUDA(cudaStreamSynchronize(h->stream));
      float ms = 0.f;
      AM24_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      compute_s += ms * 1e-3;
      int sel = 0;
      float bv = val[0];
      if (s.store_all && stats && stats->values && shift < stats->per_start_capacity)
        stats->values[shift] = bv;
      for (int i = 1; i < bs; i++) {
        if (s.store_all && stats && stats->values && shift + i < stats->per_start_capacity)
          stats->values[shift + i] = val[i];
        if (val[i] > bv) {
          bv = val[i];
          sel = i;
        }
      }
      for (int i = 0; i < bs; i++) degenerate += std::isnan(val[i]) ? 1 : 0;
      if (best < bv) {
        best = bv;
        AM24_TRY(take_best(sel));
      }
    }
  } else {
    // ---------------------------------- on the fly (sparse_PCA_solver.h:83-168)
    s.store_all = 0;
    std::vector<unsigned> cur(bs, 0), order(bs);
    for (int j = 0; j < bs; j++) {
      order[j] = j;
      gidx[j] = j;
      slots[j] = j;
    }
    host_starts(s, n, start_points, gidx.data(), bs, staging);
    AM24_TRY(upload_columns(h, b, staging.data(), bs, slots.data()));
    AM24_CUDA(cudaMemsetAsync(d.val, 0, sizeof(float) * bs, h->stream));
    unsigned generated = (unsigned)bs;
    bool go = true;
    // MIXED: one BF16 phase for the whole run (starts refilled after the switch
    // run refinement steps only); the tolerance test applies to refinement steps
    if (d.mixed) AM24_CUDA(reset_mixed(d, h->stream));
    uint32_t phase = d.mixed ? mixed_first_phase(d.lead) : 1u;
    AM24_CUDA(cudaEventRecord(e0, h->stream));
    while (go) {
      total_it++;
      const bool refined = phase != 0;
      low_its += refined ? 0 : 1;
      const StepParams p = step_params(s, 0, 0);
      AM24_CUDA(launch_am_step(M, b->d, b->tm, p, h->stream, &b->launches));
      AM24_CUDA(cudaMemcpyAsync(err.data(), d.err, sizeof(float) * bs, cudaMemcpyDeviceToHost,
                                h->stream));
      AM24_CUDA(cudaMemcpyAsync(val.data(), d.val, sizeof(float) * bs, cudaMemcpyDeviceToHost,
                                h->stream));
      if (d.mixed)
        AM24_CUDA(cudaMemcpyAsync(&phase, d.phase, sizeof phase, cudaMemcpyDeviceToHost,
                                  h->stream));
      AM24_CUDA(cudaStreamSynchronize(h->stream));
      AM24_TRY(check_device_status(b));
      start_its += (uint64_t)bs;
      go = false;
      int nref = 0;
      for (int i = 0; i < bs; i++) {
        cur[i]++;
        // termination_criteria with it = cur > 0
        const bool conv = refined && (double)err[i] < s.tolerance;
        if (conv || cur[i] >= (unsigned)s.max_iter) {
          if (best < val[i]) {
            best = val[i];
            AM24_TRY(take_best(i));
          }
          if (generated < (unsigned)s.total_starts) {
            order[i] = generated++;
            cur[i] = 0;
            slots[nref] = i;
            gidx[nref] = order[i];
            nref++;
            go = true;
          }
        } else {
          go = true;
        }
      }
      if (nref > 0) {
        host_starts(s, n, start_points, gidx.data(), nref, staging);
        AM24_TRY(upload_columns(h, b, staging.data(), nref, slots.data()));
        for (int r = 0; r < nref; r++)
          AM24_CUDA(cudaMemsetAsync(d.val + slots[r], 0, sizeof(float), h->stream));
      }
    }
    AM24_CUDA(cudaEventRecord(e1, h->stream));
    AM24_CUDA(cudaStreamSynchronize(h->stream));
    float ms = 0.f;
    AM24_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    compute_s += ms * 1e-3;
    for (int i = 0; i < bs; i++) degenerate += std::isnan(val[i]) ? 1 : 0;
  }

  // x <- x / ||x|| and its FP64 explained variance ||B x||^2
  AM24_CUDA(launch_finalize_x(xb, (int)n, x_dev, h->stream));
  AM24_CUDA(launch_explained_variance(M, x_dev, ev_rows, h->ev_out, h->stream));
  double ev = 0.0;
  AM24_CUDA(cudaMemcpyAsync(x, x_dev, sizeof(float) * n, cudaMemcpyDeviceToHost, h->stream));
  AM24_CUDA(cudaMemcpyAsync(&ev, h->ev_out, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  AM24_CUDA(cudaStreamSynchronize(h->stream));

  if (stats) {
    stats->it = total_it;
    stats->fval = best;
    stats->error = last_max_err;
    stats->total_true_computation_time = compute_s;
    stats->n = n;
    stats->total_threads_used = 1;
    stats->explained_variance = ev;
    stats->start_iterations = start_its;
    stats->degenerate_starts = degenerate;
    stats->low_precision_iterations = low_its;
    if (s.store_all && stats->per_start_capacity > 0) {
      const int cap = std::min<int>((int)stats->per_start_capacity, d.log_capacity);
      if (stats->iters)
        AM24_CUDA(cudaMemcpy(stats->iters, d.iters, sizeof(int) * cap, cudaMemcpyDeviceToHost));
      if (stats->cardinalities)
        AM24_CUDA(
            cudaMemcpy(stats->cardinalities, d.cards, sizeof(int) * cap, cudaMemcpyDeviceToHost));
    }
    stats->total_elapsed_time =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t_call).count();
  }
  if (fval_out) *fval_out = best;
  return AM24_OK;
}

am24_status am24_solve_dense_f32(am24_handle h, const float *B, int32_t ldB, float *x, uint32_t m,
                                 uint32_t n, am24_settings *settings, am24_statistics *stats,
                                 const float *start_points, float *fval_out) {
  const auto t0 = std::chrono::steady_clock::now();
  am24_matrix mat = nullptr;
  AM24_TRY(create_matrix(h, B, ldB, m, n, 0, true, &mat));
  am24_status st = am24_solve_resident_f32(h, mat, x, settings, stats, start_points, fval_out);
  am24_matrix_destroy(h, mat);
  if (st == AM24_OK && stats)
    stats->total_elapsed_time =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return st;
}

am24_status am24_solve_device_f32(am24_handle h, const float *d_B, int32_t ldB, float *x,
                                  uint32_t m, uint32_t n, am24_settings *settings,
                                  am24_statistics *stats, const float *start_points,
                                  float *fval_out) {
  const auto t0 = std::chrono::steady_clock::now();
  am24_matrix mat = nullptr;
  AM24_TRY(create_matrix(h, d_B, ldB, m, n, 1, true, &mat));
  am24_status st = am24_solve_resident_f32(h, mat, x, settings, stats, start_points, fval_out);
  am24_matrix_destroy(h, mat);
  if (st == AM24_OK && stats)
    stats->total_elapsed_time =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return st;
}

}  // extern "C"

// ---- split-K workspace in a file-scope device array ------------------------
// am24_batch_iterate_static_ws runs the step of am24_batch_iterate with the
// split-K partial tiles of the dense Z = B V product in this array instead of
// the batch's own workspace.  Nothing in it has to start at zero: the GEMM of a
// step writes every slot that the step's reduction then reads.  Calls that
// overlap in time on one device (any handles, any threads) share the array
// and race.
static __device__ __align__(256) float am24_static_ws[AM24_STATIC_WS_BYTES / sizeof(float)];

namespace {

std::mutex g_static_ws_mu;
std::unordered_map<int, float *> g_static_ws_ptr;  // device -> address of am24_static_ws

// Address of am24_static_ws on `device`, looked up once per device with that
// device current.
am24_status static_ws_address(int device, float **out) {
  std::lock_guard<std::mutex> lock(g_static_ws_mu);
  auto it = g_static_ws_ptr.find(device);
  if (it != g_static_ws_ptr.end()) {
    *out = it->second;
    return AM24_OK;
  }
  AM24_CUDA(cudaSetDevice(device));
  float *ptr = nullptr;
  const cudaError_t e = cudaGetSymbolAddress((void **)&ptr, am24_static_ws);
  if (e != cudaSuccess || ptr == nullptr)
    return fail(AM24_ERR_CUDA, std::string("cudaGetSymbolAddress(am24_static_ws): ") +
                                   cudaGetErrorString(e));
  g_static_ws_ptr[device] = ptr;
  *out = ptr;
  return AM24_OK;
}

}  // namespace

extern "C" {

am24_status am24_batch_iterate_static_ws(am24_handle h, am24_batch b, int32_t it0,
                                         int32_t iterations, float *max_error) {
  if (!h || !b) return fail(AM24_ERR_INVALID_ARG, "NULL argument");
  const size_t need = b->d.ws_len * sizeof(float);
  if (need > AM24_STATIC_WS_BYTES)
    return fail(AM24_ERR_INVALID_ARG,
                "split-K workspace of " + std::to_string(need) +
                    " bytes exceeds the static workspace of " +
                    std::to_string((size_t)AM24_STATIC_WS_BYTES) +
                    " bytes; use am24_batch_iterate");
  float *ws = nullptr;
  AM24_TRY(static_ws_address(h->device, &ws));
  AM24_CUDA(cudaSetDevice(h->device));
  BatchDev d = b->d;
  d.ws = ws;
  for (int i = 0; i < iterations; i++) {
    const StepParams p = step_params(b->s, it0 + i, 0);
    AM24_CUDA(launch_am_step(b->mat->d, d, b->tm, p, h->stream, &b->launches));
  }
  if (max_error) {
    AM24_CUDA(cudaMemcpyAsync(max_error, d.max_err, sizeof(float), cudaMemcpyDeviceToHost,
                              h->stream));
    AM24_CUDA(cudaStreamSynchronize(h->stream));
    AM24_TRY(check_device_status(b));
  }
  return AM24_OK;
}

}  // extern "C"

// ---- FP64 host data --------------------------------------------------------
extern "C" {

am24_status am24_solve_dense_f64(am24_handle h, const double *B, int32_t ldB, double *x,
                                 uint32_t m, uint32_t n, am24_settings *settings,
                                 am24_statistics *stats, const double *start_points,
                                 double *fval_out) {
  if (!h || !B || !x || !settings) return fail(AM24_ERR_INVALID_ARG, "NULL argument");
  if (ldB < (int32_t)m) return fail(AM24_ERR_INVALID_ARG, "ldB must be >= m");
  std::vector<float> Bf((size_t)m * n), xf(n), sp;
  for (uint32_t c = 0; c < n; c++)
    for (uint32_t r = 0; r < m; r++) Bf[(size_t)c * m + r] = (float)B[(size_t)c * ldB + r];
  for (uint32_t i = 0; i < n; i++) xf[i] = (float)x[i];
  if (settings->start_mode == AM24_START_INJECTED && start_points) {
    am24_settings probe = *settings;
    AM24_TRY(am24_check_input(&probe, n));
    sp.resize((size_t)n * probe.total_starts);
    for (size_t i = 0; i < sp.size(); i++) sp[i] = (float)start_points[i];
  }
  float f = 0.f;
  AM24_TRY(am24_solve_dense_f32(h, Bf.data(), (int32_t)m, xf.data(), m, n, settings, stats,
                                sp.empty() ? nullptr : sp.data(), &f));
  if (stats) stats->input_rounded_to_f32 = 1;
  for (uint32_t i = 0; i < n; i++) x[i] = xf[i];
  if (fval_out) *fval_out = f;
  return AM24_OK;
}

}  // extern "C"
