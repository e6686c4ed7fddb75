/*
 * Drop-in for the reference's solver entry point
 *   template<F> F SPCASolver::MulticoreSolver::denseDataSolver(const F* B, const int ldB,
 *       F* x, const unsigned m, const unsigned n, OptimizationSettings*, OptimizationStatistics*)
 *   -- c++/src/gpower/sparse_PCA_solver.h:36-40
 * forwarding to the C ABI in am24.h (link with -lam24).  Same arguments, same
 * return value (the best objective), same rewriting of the settings
 * (chceckInputAndModifyIt and OTF's storeIterationsForAllPoints = false), same
 * statistics fields.  The solve runs on the GPU of settings->device; a
 * process-wide handle per device is created on first use.  The double
 * instantiation has no FP64 arithmetic: it rounds B and x to FP32 (2^-24
 * relative per entry), solves in FP32 (the library's arithmetic), returns x in
 * double and sets statistics->inputRoundedToFloat = 1.
 * On failure the return value is NaN and am24_last_error() says why.
 */
#ifndef AM24_SPARSE_PCA_SOLVER_H
#define AM24_SPARSE_PCA_SOLVER_H

#include <cmath>
#include <limits>
#include <mutex>
#include <vector>

#include "../am24.h"
#include "optimization_settings.h"
#include "optimization_statistics.h"

namespace SPCASolver {
namespace am24_detail {

inline am24_handle default_handle(int device) {
  static std::mutex mu;
  static std::vector<am24_handle> handles;
  std::lock_guard<std::mutex> lock(mu);
  if ((int)handles.size() <= device) handles.resize(device + 1, nullptr);
  if (!handles[device] && am24_create(&handles[device], device) != AM24_OK) return nullptr;
  return handles[device];
}

inline void to_c(const SolverStructures::OptimizationSettings &o, am24_settings *s) {
  am24_default_settings(s);
  s->formulation = (int32_t)o.formulation;
  s->constraint = o.constraintParameter;
  s->penalty = o.penaltyParameter;
  s->tolerance = o.tolerance;
  s->max_iter = o.maximumIterations;
  s->total_starts = o.totalStartingPoints;
  s->batch_size = o.batchSize;
  s->use_otf = o.useOTF ? 1 : 0;
  s->use_sort_hard = o.useSortForHardThresholding ? 1 : 0;
  s->store_all = o.storeIterationsForAllPoints ? 1 : 0;
  s->verbose = o.verbose ? 1 : 0;
  s->start_mode = o.startMode;
  s->l1_mode = o.l1Mode;
  s->timeout_ms = o.timeoutMs;
  s->precision = o.precision;
  s->stable_iterations = o.stableIterations;
  s->stable_share = o.stableShare;
  s->lead_iterations = o.leadIterations;
}

inline void from_c(const am24_settings &s, SolverStructures::OptimizationSettings *o) {
  o->constraintParameter = s.constraint;
  o->totalStartingPoints = s.total_starts;
  o->batchSize = s.batch_size;
  o->totalBatches = s.total_batches;
  o->storeIterationsForAllPoints = s.store_all != 0;
}

// One solve in FP32 through am24_solve_dense_f32 (host B), am24_solve_device_f32
// (device B) or, given a resident matrix, am24_solve_resident_f32 (B unused);
// fills the reference's statistics.
inline float solve_f32(const float *B, int ldB, float *x, unsigned m, unsigned n, bool on_device,
                       SolverStructures::OptimizationSettings *o,
                       SolverStructures::OptimizationStatistics *st,
                       am24_status *status = nullptr, const float *start_points = nullptr,
                       am24_matrix resident = nullptr) {
  const float nan = std::numeric_limits<float>::quiet_NaN();
  if (status) *status = AM24_ERR_CUDA;
  am24_handle h = default_handle(o->device);
  if (!h) return nan;
  am24_settings s;
  to_c(*o, &s);
  am24_settings probe = s;
  const am24_status pc = am24_check_input(&probe, n);
  if (status) *status = pc;
  if (pc != AM24_OK) return nan;
  const size_t cap = (size_t)probe.total_starts;
  st->values.assign(o->storeIterationsForAllPoints ? cap : 0, -1.0);
  st->iters.assign(o->storeIterationsForAllPoints ? cap : 0, -1);
  st->cardinalities.assign(o->storeIterationsForAllPoints ? cap : 0, -1);
  am24_statistics cs = {};
  if (o->storeIterationsForAllPoints && !o->useOTF) {
    cs.values = st->values.data();
    cs.iters = st->iters.data();
    cs.cardinalities = st->cardinalities.data();
    cs.per_start_capacity = (uint32_t)cap;
  }
  float f = nan;
  const am24_status rc =
      resident    ? am24_solve_resident_f32(h, resident, x, &s, &cs, start_points, &f)
      : on_device ? am24_solve_device_f32(h, B, ldB, x, m, n, &s, &cs, start_points, &f)
                  : am24_solve_dense_f32(h, B, ldB, x, m, n, &s, &cs, start_points, &f);
  from_c(s, o);
  if (status) *status = rc;
  if (rc != AM24_OK) return nan;
  st->it = cs.it;
  st->fval = cs.fval;
  st->error = cs.error;
  st->totalTrueComputationTime = cs.total_true_computation_time;
  st->n = n;
  st->totalThreadsUsed = cs.total_threads_used;
  st->explainedVariance = cs.explained_variance;
  st->startIterations = cs.start_iterations;
  st->degenerateStarts = cs.degenerate_starts;
  st->lowPrecisionIterations = cs.low_precision_iterations;
  st->inputRoundedToFloat = cs.input_rounded_to_f32;
  return f;
}

}  // namespace am24_detail

namespace MulticoreSolver {

template <typename F>
F denseDataSolver(const F *B, const int ldB, F *x, const unsigned int m, const unsigned int n,
                  SolverStructures::OptimizationSettings *optimizationSettings,
                  SolverStructures::OptimizationStatistics *optimizationStatistics);

template <>
inline float denseDataSolver<float>(const float *B, const int ldB, float *x, const unsigned int m,
                                    const unsigned int n,
                                    SolverStructures::OptimizationSettings *o,
                                    SolverStructures::OptimizationStatistics *st) {
  return am24_detail::solve_f32(B, ldB, x, m, n, false, o, st);
}

template <>
inline double denseDataSolver<double>(const double *B, const int ldB, double *x,
                                      const unsigned int m, const unsigned int n,
                                      SolverStructures::OptimizationSettings *o,
                                      SolverStructures::OptimizationStatistics *st) {
  std::vector<float> Bf((size_t)m * n), xf(n);
  for (unsigned c = 0; c < n; c++)
    for (unsigned r = 0; r < m; r++) Bf[(size_t)c * m + r] = (float)B[(size_t)c * ldB + r];
  for (unsigned i = 0; i < n; i++) xf[i] = (float)x[i];
  const float f = am24_detail::solve_f32(Bf.data(), (int)m, xf.data(), m, n, false, o, st);
  st->inputRoundedToFloat = 1;  // no FP64 arithmetic on this path
  for (unsigned i = 0; i < n; i++) x[i] = xf[i];
  return f;
}

}  // namespace MulticoreSolver
}  // namespace SPCASolver

#endif
