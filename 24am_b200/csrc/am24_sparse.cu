// Sparse-resident matrices: the reference's sparse solver input
// (sparse_PCA_solver_CSC, c++/src/gpower/sparse_PCA_solver_for_CSC.h:111-117:
// CSC arrays, optional doMean / doRowMean centring) kept compressed on the
// device, and the batch driver that solves on it.  Device memory is O(nnz):
// CSC plus a CSR copy (8 bytes per non-zero each), the centring vectors, the
// segment lists of columns and rows longer than SP_LONG entries, and per batch
// the start-major and row-major planes of V and Z (4 (3 n + 2 m) bytes per
// start) plus the long entries' segment sums (4 bytes per segment and start).  The iteration is the dense path's (the
// reference's batch loop, c++/src/gpower/sparse_PCA_solver.h:171-232), so a
// sparse-resident solve gives the dense solve of the centred matrix up to FP32
// summation order; both products run as FP32 tile kernels on the compressed
// arrays (am24_sparse_kernels.cuh) and the selects and finalize are shared.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "am24.h"
#include "am24_internal.h"
#include "am24_host.h"

using namespace am24;
using namespace am24host;

namespace am24host {

am24_status validate_csc(const float *vals, const int32_t *row_ind, const int32_t *col_ptr,
                         uint32_t m, uint32_t n) {
  if (!col_ptr) return fail(AM24_ERR_INVALID_ARG, "NULL argument");
  if (m == 0 || n == 0) return fail(AM24_ERR_INVALID_ARG, "m and n must be positive");
  if (m > (1u << 30) || n > (1u << 30)) return fail(AM24_ERR_INVALID_ARG, "matrix too large");
  if (col_ptr[0] != 0) return fail(AM24_ERR_INVALID_ARG, "col_ptr[0] must be 0");
  for (uint32_t c = 0; c < n; c++)
    if (col_ptr[c + 1] < col_ptr[c])
      return fail(AM24_ERR_INVALID_ARG, "col_ptr must be non-decreasing");
  const size_t nnz = (size_t)col_ptr[n];
  if (nnz > 0 && (!vals || !row_ind)) return fail(AM24_ERR_INVALID_ARG, "NULL argument");
  for (size_t q = 0; q < nnz; q++)
    if (row_ind[q] < 0 || (uint32_t)row_ind[q] >= m)
      return fail(AM24_ERR_INVALID_ARG, "row index out of range at entry " + std::to_string(q));
  return AM24_OK;
}

// The segments of the outer entries longer than SP_LONG (host lists; see SparseLong).
struct LongLists {
  std::vector<int32_t> outer, first, e0, e1;
  void build(const int32_t *ptr, int outer_n) {
    for (int c = 0; c < outer_n; c++) {
      const int32_t a = ptr[c], z = ptr[c + 1];
      if (z - a <= SP_LONG) continue;
      outer.push_back(c);
      first.push_back((int32_t)e0.size());
      for (int32_t e = a; e < z; e += SP_SEG) {
        e0.push_back(e);
        e1.push_back(std::min(z, e + SP_SEG));
      }
    }
    first.push_back((int32_t)e0.size());
  }
};

}  // namespace am24host

extern "C" am24_status am24_matrix_create_csc_sparse_f32(am24_handle h, const float *vals,
                                                         const int32_t *row_ind,
                                                         const int32_t *col_ptr, uint32_t m,
                                                         uint32_t n, const float *means,
                                                         const float *row_means,
                                                         am24_matrix *out) {
  if (!out) return fail(AM24_ERR_INVALID_ARG, "NULL argument");
  *out = nullptr;
  // every index is checked on the host before any device write can use it
  AM24_TRY(validate_csc(vals, row_ind, col_ptr, m, n));
  if (!h) return fail(AM24_ERR_INVALID_ARG, "NULL handle");
  // canonical columns (rows strictly ascending): a column whose rows are not
  // is sorted by row (stably) and its duplicate entries added in entry order,
  // so that every column's rows are distinct on the device
  std::vector<int32_t> cp2, ri2;
  std::vector<float> v2;
  bool canonical = true;
  for (uint32_t c = 0; c < n && canonical; c++)
    for (int32_t e = col_ptr[c] + 1; e < col_ptr[c + 1]; e++)
      if (row_ind[e] <= row_ind[e - 1]) {
        canonical = false;
        break;
      }
  if (!canonical) {
    cp2.assign((size_t)n + 1, 0);
    ri2.reserve((size_t)col_ptr[n]);
    v2.reserve((size_t)col_ptr[n]);
    std::vector<int32_t> order;
    for (uint32_t c = 0; c < n; c++) {
      order.clear();
      for (int32_t e = col_ptr[c]; e < col_ptr[c + 1]; e++) order.push_back(e);
      std::stable_sort(order.begin(), order.end(),
                       [&](int32_t a, int32_t b2) { return row_ind[a] < row_ind[b2]; });
      for (size_t q = 0; q < order.size(); q++) {
        const int32_t e = order[q];
        if (q > 0 && row_ind[e] == ri2.back())
          v2.back() += vals[e];
        else {
          ri2.push_back(row_ind[e]);
          v2.push_back(vals[e]);
        }
      }
      cp2[c + 1] = (int32_t)ri2.size();
    }
    col_ptr = cp2.data();
    row_ind = ri2.data();
    vals = v2.data();
  }
  const size_t nnz = (size_t)col_ptr[n];
  // the CSR copy, built on the host by a counting pass: within each row the
  // columns come in ascending order, as the CSC arrays list them
  std::vector<int32_t> row_ptr((size_t)m + 1, 0), col_ind(nnz);
  std::vector<float> rvals(nnz);
  for (size_t e = 0; e < nnz; e++) row_ptr[(size_t)row_ind[e] + 1]++;
  for (uint32_t i = 0; i < m; i++) row_ptr[i + 1] += row_ptr[i];
  {
    std::vector<int32_t> fill(row_ptr.begin(), row_ptr.end() - 1);
    for (uint32_t c = 0; c < n; c++)
      for (int32_t e = col_ptr[c]; e < col_ptr[c + 1]; e++) {
        const int32_t at = fill[row_ind[e]]++;
        col_ind[at] = (int32_t)c;
        rvals[at] = vals[e];
      }
  }
  LongLists lc, lr;
  lc.build(col_ptr, (int)n);
  lr.build(row_ptr.data(), (int)m);
  AM24_CUDA(cudaSetDevice(h->device));
  auto *mat = new am24_matrix_s();
  mat->sparse = true;
  if (means) mat->means_host.assign(means, means + n);
  MatrixDev &M = mat->d;
  M.m = (int)m;
  M.n = (int)n;
  M.ldm = round_up((int)m, 32);
  M.ldn = round_up((int)n, 32);
  SparseDev &S = mat->sp;
  S.m = (int)m;
  S.n = (int)n;
  S.nnz = (int64_t)nnz;
  am24_status st;
  if ((st = mat->mem.get(&S.col_ptr, (size_t)n + 1)) || (st = mat->mem.get(&S.row_ind, nnz)) ||
      (st = mat->mem.get(&S.cvals, nnz)) || (st = mat->mem.get(&S.row_ptr, (size_t)m + 1)) ||
      (st = mat->mem.get(&S.col_ind, nnz)) || (st = mat->mem.get(&S.rvals, nnz)) ||
      (means && (st = mat->mem.get(&S.means, (size_t)n))) ||
      (row_means && (st = mat->mem.get(&S.row_means, (size_t)m)))) {
    delete mat;
    return st;
  }
  auto alloc_long = [&](const LongLists &l, SparseLong &L) -> am24_status {
    L.count = (int)l.outer.size();
    L.segs = (int)l.e0.size();
    if (L.count == 0) return AM24_OK;
    am24_status s2;
    if ((s2 = mat->mem.get(&L.outer, l.outer.size())) ||
        (s2 = mat->mem.get(&L.seg_first, l.first.size())) ||
        (s2 = mat->mem.get(&L.seg_e0, l.e0.size())) || (s2 = mat->mem.get(&L.seg_e1, l.e1.size())))
      return s2;
    return AM24_OK;
  };
  if ((st = alloc_long(lc, S.long_cols)) || (st = alloc_long(lr, S.long_rows))) {
    delete mat;
    return st;
  }
  cudaError_t e = cudaSuccess;
  auto up = [&](void *dst, const void *src, size_t bytes) {
    if (e == cudaSuccess && bytes)
      e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, h->stream);
  };
  up(S.col_ptr, col_ptr, sizeof(int32_t) * ((size_t)n + 1));
  up(S.row_ind, row_ind, sizeof(int32_t) * nnz);
  up(S.cvals, vals, sizeof(float) * nnz);
  up(S.row_ptr, row_ptr.data(), sizeof(int32_t) * ((size_t)m + 1));
  up(S.col_ind, col_ind.data(), sizeof(int32_t) * nnz);
  up(S.rvals, rvals.data(), sizeof(float) * nnz);
  if (means) up(S.means, means, sizeof(float) * n);
  if (row_means) up(S.row_means, row_means, sizeof(float) * m);
  for (auto [l, L] : {std::make_pair(&lc, &S.long_cols), std::make_pair(&lr, &S.long_rows)}) {
    if (L->count == 0) continue;
    up(L->outer, l->outer.data(), sizeof(int32_t) * l->outer.size());
    up(L->seg_first, l->first.data(), sizeof(int32_t) * l->first.size());
    up(L->seg_e0, l->e0.data(), sizeof(int32_t) * l->e0.size());
    up(L->seg_e1, l->e1.data(), sizeof(int32_t) * l->e1.size());
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);  // the host staging dies here
  if (e != cudaSuccess) {
    delete mat;
    return fail(e == cudaErrorMemoryAllocation ? AM24_ERR_OOM : AM24_ERR_CUDA,
                std::string("sparse matrix upload: ") + cudaGetErrorString(e));
  }
  *out = mat;
  return AM24_OK;
}

namespace am24host {

am24_status deflate_sparse(am24_handle h, am24_matrix mat, const float *x, int32_t on_device) {
  SparseDev &S = mat->sp;
  const int n = S.n, c = S.comps;
  if (c >= SP_DEFL_MAX)
    return fail(AM24_ERR_INVALID_ARG, "a sparse-resident matrix takes at most " +
                                          std::to_string(SP_DEFL_MAX) + " deflations");
  AM24_CUDA(cudaSetDevice(h->device));
  // work already queued on the handle's stream sees the old deflation
  AM24_CUDA(cudaStreamSynchronize(h->stream));
  std::vector<float> xh((size_t)n);
  AM24_CUDA(cudaMemcpy(xh.data(), x, sizeof(float) * n,
                       on_device ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost));
  if (!mat->defl_dev) {
    am24_status st;
    if ((st = mat->mem.get(&mat->defl_dev, (size_t)SP_DEFL_MAX * n)) ||
        (st = mat->mem.get(&mat->gram_dev, (size_t)SP_DEFL_MAX * SP_DEFL_MAX)) ||
        (st = mat->mem.get(&mat->defl_sum_dev, SP_DEFL_MAX)) ||
        (st = mat->mem.get(&mat->defl_mu_dev, SP_DEFL_MAX)))
      return st;
    mat->gram_host.assign((size_t)SP_DEFL_MAX * SP_DEFL_MAX, 0.0);
  }
  // x_c^T x_a for the earlier components and itself, 1^T x, means^T x (FP64)
  mat->defl_host.insert(mat->defl_host.end(), xh.begin(), xh.end());
  for (int a = 0; a <= c; a++) {
    const float *xa = mat->defl_host.data() + (size_t)a * n;
    double g = 0.0;
    for (int q = 0; q < n; q++) g += (double)xa[q] * (double)xh[q];
    mat->gram_host[(size_t)c * SP_DEFL_MAX + a] = g;
    mat->gram_host[(size_t)a * SP_DEFL_MAX + c] = g;
  }
  double sum = 0.0, mu = 0.0;
  for (int q = 0; q < n; q++) {
    sum += (double)xh[q];
    if (!mat->means_host.empty()) mu += (double)mat->means_host[q] * (double)xh[q];
  }
  AM24_CUDA(cudaMemcpy(mat->defl_dev + (size_t)c * n, xh.data(), sizeof(float) * n,
                       cudaMemcpyHostToDevice));
  AM24_CUDA(cudaMemcpy(mat->gram_dev, mat->gram_host.data(),
                       sizeof(double) * mat->gram_host.size(), cudaMemcpyHostToDevice));
  AM24_CUDA(cudaMemcpy(mat->defl_sum_dev + c, &sum, sizeof(double), cudaMemcpyHostToDevice));
  AM24_CUDA(cudaMemcpy(mat->defl_mu_dev + c, &mu, sizeof(double), cudaMemcpyHostToDevice));
  S.defl = mat->defl_dev;
  S.gram = mat->gram_dev;
  S.defl_sum = mat->defl_sum_dev;
  S.defl_mu = mat->defl_mu_dev;
  S.comps = c + 1;
  return AM24_OK;
}

// The reference's batch driver (denseDataSolver's batch mode,
// c++/src/gpower/sparse_PCA_solver.h:171-243) on a sparse-resident matrix:
// batches of batch_size starts (reference, injected or device starts), each
// iterated until the step the reference's loop ends on, the first best start
// over all batches, its loading normalised, and its explained variance in FP64.
am24_status solve_sparse(am24_handle h, am24_matrix mat, float *x, am24_settings &s,
                         am24_statistics *stats, const float *start_points, float *fval_out) {
  const auto t_call = std::chrono::steady_clock::now();
  if (s.use_otf)
    return fail(AM24_ERR_UNSUPPORTED, "on-the-fly mode is not supported on sparse-resident matrices");
  const SparseDev &S = mat->sp;
  const unsigned n = (unsigned)S.n;
  const int k = s.batch_size;
  SparseBatchDev b;
  b.k = k;
  b.kp = round_up(k, 32);
  b.ldn = mat->d.ldn;
  b.ldm = mat->d.ldm;
  b.log_capacity = std::max(s.total_starts, k);
  Allocs A(h->stream);
  float *xb = nullptr, *x_dev = nullptr;
  double *ev_scratch = nullptr;
  AM24_TRY(A.get(&b.Vx, (size_t)k * b.ldn));
  AM24_TRY(A.get(&b.vmask, (size_t)k * (b.ldn / 32)));
  AM24_TRY(A.get(&b.Vraw, (size_t)k * b.ldn));
  AM24_TRY(A.get(&b.Vt, (size_t)n * b.kp));
  AM24_TRY(A.get(&b.Zs, (size_t)k * b.ldm));
  AM24_TRY(A.get(&b.Zt, (size_t)S.m * b.kp));
  AM24_TRY(A.get(&b.fz, k));
  AM24_TRY(A.get(&b.val, k));
  AM24_TRY(A.get(&b.err, k));
  AM24_TRY(A.get(&b.max_err, 1));
  AM24_TRY(A.get(&b.sel_hint, k));
  AM24_TRY(A.get(&b.obj_part, k));
  AM24_TRY(A.get(&b.nnz_part, k));
  AM24_TRY(A.get(&b.nnz, k));
  AM24_TRY(A.get(&b.max_nnz, 1));
  AM24_TRY(A.get(&b.ctl, CTL_WORDS));
  AM24_TRY(A.get(&b.work, 1));
  AM24_TRY(A.get(&b.zgate, 1));
  AM24_TRY(A.get(&b.sum_v, k));
  AM24_TRY(A.get(&b.dot_mu, k));
  AM24_TRY(A.get(&b.zsum, k));
  AM24_TRY(A.get(&b.zdot, k));
  AM24_TRY(A.get(&b.status, 1));
  AM24_TRY(A.get(&b.iters, b.log_capacity));
  AM24_TRY(A.get(&b.cards, b.log_capacity));
  AM24_TRY(A.get(&xb, n));
  AM24_TRY(A.get(&x_dev, n));
  AM24_TRY(A.get(&ev_scratch, sparse_ev_scratch(S)));
  if (S.long_cols.segs) AM24_TRY(A.get(&b.part_cols, (size_t)S.long_cols.segs * b.kp));
  if (S.long_rows.segs) AM24_TRY(A.get(&b.part_rows, (size_t)S.long_rows.segs * b.kp));
  if (S.comps) AM24_TRY(A.get(&b.defl_a, (size_t)k * SP_DEFL_MAX));
  // every buffer starts defined: pool memory can hold an earlier call's state
  AM24_CUDA(cudaMemsetAsync(b.vmask, 0, sizeof(uint32_t) * (size_t)k * (b.ldn / 32), h->stream));
  AM24_CUDA(cudaMemsetAsync(b.Vx, 0, sizeof(float) * (size_t)k * b.ldn, h->stream));
  AM24_CUDA(cudaMemsetAsync(b.Vraw, 0, sizeof(float) * (size_t)k * b.ldn, h->stream));
  AM24_CUDA(cudaMemsetAsync(b.fz, 0, sizeof(float) * k, h->stream));
  AM24_CUDA(cudaMemsetAsync(b.obj_part, 0, sizeof(float) * k, h->stream));
  AM24_CUDA(cudaMemsetAsync(b.nnz_part, 0, sizeof(float) * k, h->stream));
  AM24_CUDA(cudaMemsetAsync(b.nnz, 0, sizeof(uint32_t) * k, h->stream));
  AM24_CUDA(cudaMemsetAsync(b.zsum, 0, sizeof(double) * k, h->stream));
  AM24_CUDA(cudaMemsetAsync(b.zdot, 0, sizeof(double) * k, h->stream));
  AM24_CUDA(cudaMemsetAsync(b.status, 0, sizeof(int), h->stream));
  AM24_CUDA(cudaMemsetAsync(b.iters, 0xFF, sizeof(int) * b.log_capacity, h->stream));
  AM24_CUDA(cudaMemsetAsync(b.cards, 0xFF, sizeof(int) * b.log_capacity, h->stream));
  // the best loading so far starts as the caller's x (returned normalised
  // when no start ever improves on -1, as the reference returns it)
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

  std::vector<float> staging, val(k);
  std::vector<unsigned> gidx(k);
  float best = -1.f;
  uint32_t total_it = 0;
  uint64_t start_its = 0;
  double compute_s = 0.0;
  float last_max_err = 0.f;
  int degenerate = 0;
  for (unsigned batch = 0; batch < s.total_batches; batch++) {
    const unsigned shift = batch * (unsigned)k;
    for (int j = 0; j < k; j++) gidx[j] = shift + j;
    // the batch's starts, staged in Vraw (or generated there), then split
    // into values and masks; ValueCoordinateHolder::reset
    if (s.start_mode == AM24_START_DEVICE_UNIFORM) {
      AM24_CUDA(launch_uniform_starts(b.Vraw, b.ldn, (int)n, k, shift, h->stream));
    } else {
      const float *src = start_points + (size_t)shift * n;
      if (s.start_mode != AM24_START_INJECTED) {
        host_starts(s, n, start_points, gidx.data(), k, staging);
        src = staging.data();
      }
      AM24_CUDA(cudaMemcpy2DAsync(b.Vraw, sizeof(float) * b.ldn, src, sizeof(float) * n,
                                  sizeof(float) * n, k, cudaMemcpyHostToDevice, h->stream));
    }
    AM24_CUDA(launch_load_columns(b.Vraw, b.ldn, (int)n, k, b.Vx, b.ldn, b.vmask, h->stream));
    AM24_CUDA(cudaMemsetAsync(b.sel_hint, 0, sizeof(float) * k, h->stream));
    AM24_CUDA(cudaMemsetAsync(b.val, 0, sizeof(float) * k, h->stream));
    AM24_CUDA(cudaMemsetAsync(b.err, 0, sizeof(float) * k, h->stream));
    AM24_CUDA(cudaMemsetAsync(b.ctl, 0, sizeof(uint32_t) * CTL_WORDS, h->stream));
    AM24_CUDA(cudaMemsetAsync(b.max_nnz, 0xFF, sizeof(uint32_t), h->stream));  // dense starts
    AM24_CUDA(cudaEventRecord(e0, h->stream));
    // the batch loop: finalize sets the stop word after the step the
    // reference's loop ends on; the host reads it after each step
    for (int it = 0; it < s.max_iter; it++) {
      StepParams p = step_params(s, it, (int)shift);
      p.stop_check = 1;
      AM24_CUDA(launch_sparse_step(S, b, p, h->stream));
      AM24_CUDA(cudaMemcpyAsync(&h->flags[0], b.ctl + CTL_STOP, sizeof(uint32_t),
                                cudaMemcpyDeviceToHost, h->stream));
      AM24_CUDA(cudaStreamSynchronize(h->stream));
      if (h->flags[0]) break;
    }
    AM24_CUDA(cudaEventRecord(e1, h->stream));
    uint32_t c[CTL_WORDS];
    int dev_status = 0;
    AM24_CUDA(cudaMemcpyAsync(c, b.ctl, sizeof c, cudaMemcpyDeviceToHost, h->stream));
    AM24_CUDA(cudaMemcpyAsync(&dev_status, b.status, sizeof(int), cudaMemcpyDeviceToHost,
                              h->stream));
    AM24_CUDA(cudaMemcpyAsync(val.data(), b.val, sizeof(float) * k, cudaMemcpyDeviceToHost,
                              h->stream));
    AM24_CUDA(cudaStreamSynchronize(h->stream));
    if (dev_status != 0) {
      char buf[96];
      snprintf(buf, sizeof buf, "device-side wait timed out (code 0x%x)", dev_status);
      return fail(AM24_ERR_DEVICE_TIMEOUT, buf);
    }
    float ms = 0.f;
    AM24_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    compute_s += ms * 1e-3;
    total_it += c[CTL_STEPS];
    start_its += (uint64_t)c[CTL_STEPS] * (uint64_t)k;
    memcpy(&last_max_err, &c[CTL_MAX_ERR], sizeof(float));
    // the first best start of the batch, then against the best so far
    // (sparse_PCA_solver.h:213-229)
    int sel = 0;
    float bv = val[0];
    for (int i = 0; i < k; i++) {
      if (s.store_all && stats && stats->values && shift + i < stats->per_start_capacity)
        stats->values[shift + i] = val[i];
      if (i > 0 && val[i] > bv) {
        bv = val[i];
        sel = i;
      }
      degenerate += std::isnan(val[i]) ? 1 : 0;
    }
    if (best < bv) {
      best = bv;
      AM24_CUDA(launch_masked_copy(b.Vx + (size_t)sel * b.ldn, b.vmask + (size_t)sel * (b.ldn / 32),
                                   b.ldn, (int)n, 1, xb, (int)n, h->stream));
    }
  }
  // x <- x / ||x|| and its FP64 explained variance ||(B - centring) P x||^2
  // (P the deflation, applied to x on the host in FP64: the last factor first)
  AM24_CUDA(launch_finalize_x(xb, (int)n, x_dev, h->stream));
  double ev = 0.0;
  AM24_CUDA(cudaMemcpyAsync(x, x_dev, sizeof(float) * n, cudaMemcpyDeviceToHost, h->stream));
  if (S.comps > 0) {
    AM24_CUDA(cudaStreamSynchronize(h->stream));
    std::vector<double> px(x, x + n);
    for (int c = S.comps - 1; c >= 0; c--) {
      const float *xc = mat->defl_host.data() + (size_t)c * n;
      double a = 0.0;
      for (unsigned q = 0; q < n; q++) a += (double)xc[q] * px[q];
      for (unsigned q = 0; q < n; q++) px[q] -= a * (double)xc[q];
    }
    std::vector<float> pxf(px.begin(), px.end());
    AM24_CUDA(cudaMemcpy(xb, pxf.data(), sizeof(float) * n, cudaMemcpyHostToDevice));
    AM24_CUDA(launch_sparse_ev(S, xb, ev_scratch, h->ev_out, h->stream));
  } else {
    AM24_CUDA(launch_sparse_ev(S, x_dev, ev_scratch, h->ev_out, h->stream));
  }
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
    stats->low_precision_iterations = 0;
    if (s.store_all && stats->per_start_capacity > 0) {
      const int cap = std::min<int>((int)stats->per_start_capacity, b.log_capacity);
      if (stats->iters)
        AM24_CUDA(cudaMemcpy(stats->iters, b.iters, sizeof(int) * cap, cudaMemcpyDeviceToHost));
      if (stats->cardinalities)
        AM24_CUDA(cudaMemcpy(stats->cardinalities, b.cards, sizeof(int) * cap,
                             cudaMemcpyDeviceToHost));
    }
    stats->total_elapsed_time =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t_call).count();
  }
  if (fval_out) *fval_out = best;
  return AM24_OK;
}

}  // namespace am24host
