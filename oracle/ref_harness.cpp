/*
 * Harness around the reference's own AM solver (optml/24am), compiled from the
 * reference sources by oracle/Makefile into oracle/_ref/.  TEST INFRASTRUCTURE
 * ONLY: tests/ and bench.py's reference arm load it; the product never does.
 *
 * Three kinds of entry points, all extern "C" so Python can bind them:
 *   ref_dense_solver_*     the UNMODIFIED entry point
 *                          SPCASolver::MulticoreSolver::denseDataSolver<F>
 *                          (c++/src/gpower/sparse_PCA_solver.h:36-243), with the
 *                          reference's own rand_r starting points.
 *   ref_solver_injected_*  the same driver loop (batch c++/src/gpower/sparse_PCA_solver.h:171-232,
 *                          on-the-fly :83-168) restated here around the reference's
 *                          own per-iteration functions
 *                          perform_one_iteration_for_{constrained,penalized}_pca
 *                          (c++/src/gpower/gpower_commons.h:68-177), but with the
 *                          starting points supplied by the caller instead of
 *                          getSignleStartingPoint (which races under OpenMP:
 *                          c++/src/gpower/gpower_commons.h:27,39).
 *   ref_*_thresholding_*   the reference's thresholding operators
 *                          (c++/src/utils/thresh_functions.h:121-254).
 */
#include <cstring>
#include <vector>
#include <algorithm>

#include "c++/src/class/optimization_settings.h"
#include "c++/src/class/optimization_statistics.h"
#include "c++/src/gpower/sparse_PCA_solver.h"

extern "C" {

/* Flat mirror of the OptimizationSettings fields the AM path reads
 * (c++/src/class/optimization_settings.h:73-99). */
typedef struct {
  int formulation;        /* SPCA_Formulation enum value 0..7 */
  unsigned constraint;    /* constraintParameter (s) */
  double penalty;         /* penaltyParameter (gamma) */
  double tolerance;
  int max_iter;
  int total_starts;
  int batch_size;
  int use_otf;
  int use_sort_hard;      /* useSortForHardThresholding */
  int store_all;          /* storeIterationsForAllPoints */
  unsigned total_batches; /* output: set by chceckInputAndModifyIt */
} ref_settings;

typedef struct {
  unsigned it;
  double fval;
  double compute_time;
  int threads;
} ref_stats;

}  // extern "C"

namespace {

void to_ref(const ref_settings *s, SolverStructures::OptimizationSettings *o) {
  o->formulation = (SolverStructures::SPCA_Formulation)s->formulation;
  o->constraintParameter = s->constraint;
  o->penaltyParameter = s->penalty;
  o->tolerance = s->tolerance;
  o->maximumIterations = s->max_iter;
  o->totalStartingPoints = s->total_starts;
  o->batchSize = s->batch_size;
  o->useOTF = s->use_otf != 0;
  o->useSortForHardThresholding = s->use_sort_hard != 0;
  o->storeIterationsForAllPoints = s->store_all != 0;
  o->verbose = false;
}

void from_ref(const SolverStructures::OptimizationSettings *o, ref_settings *s) {
  s->constraint = o->constraintParameter;
  s->total_starts = o->totalStartingPoints;
  s->batch_size = o->batchSize;
  s->total_batches = o->totalBatches;
  s->store_all = o->storeIterationsForAllPoints ? 1 : 0;
}

template <typename F>
F run_dense_solver(const F *B, int ldB, F *x, unsigned m, unsigned n, ref_settings *s,
                   ref_stats *st, double *values, int *iters, int *cards) {
  SolverStructures::OptimizationSettings o;
  SolverStructures::OptimizationStatistics stats;
  to_ref(s, &o);
  F r = SPCASolver::MulticoreSolver::denseDataSolver<F>(B, ldB, x, m, n, &o, &stats);
  from_ref(&o, s);
  st->it = stats.it;
  st->fval = stats.fval;
  st->compute_time = stats.totalTrueComputationTime;
  st->threads = stats.totalThreadsUsed;
  if (o.storeIterationsForAllPoints) {
    for (size_t i = 0; i < stats.values.size(); i++) {
      if (values) values[i] = stats.values[i];
      if (iters) iters[i] = stats.iters[i];
      if (cards) cards[i] = stats.cardinalities[i];
    }
  }
  return r;
}

/* The driver of c++/src/gpower/sparse_PCA_solver.h:36-243 with injected starts.
 * V_all is n x total_starts column-major (after chceckInputAndModifyIt has
 * rounded total_starts up to whole batches).  Everything else -- iteration
 * functions, termination test, value holder, best-start pick -- is the
 * reference's own code. */
template <typename F>
F run_injected(const F *B, int ldB, F *x, unsigned m, unsigned n, ref_settings *s,
               ref_stats *st, const F *V_all, double *values, int *iters, int *cards) {
  SolverStructures::OptimizationSettings o;
  SolverStructures::OptimizationStatistics stats;
  to_ref(s, &o);
  o.chceckInputAndModifyIt(n);
  if (o.storeIterationsForAllPoints) {
    stats.iters.resize(o.totalStartingPoints, -1);
    stats.cardinalities.resize(o.totalStartingPoints, -1);
    stats.values.resize(o.totalStartingPoints, -1);
  }
  const unsigned bs = o.batchSize;
  std::vector<F> Z((size_t)m * bs, 0), V((size_t)n * bs, 0);
  std::vector<ValueCoordinateHolder<F>> vals(bs);
  for (auto &v : vals) { v.val = 0; v.prev_val = 0; v.tmp = 0; v.current_error = 0; }
  std::vector<std::vector<F>> buffer(bs);
  if (o.isConstrainedProblem())
    for (auto &b : buffer) b.resize(n);
  std::vector<F> max_errors(TOTAL_THREADS > 0 ? TOTAL_THREADS : 1);
  F best = -1;
  unsigned total_iterations = 0;
  double t0 = gettime();
  if (o.useOTF) {
    o.storeIterationsForAllPoints = false;
    for (unsigned j = 0; j < bs; j++)
      std::memcpy(&V[(size_t)j * n], &V_all[(size_t)j * n], sizeof(F) * n);
    unsigned generated = bs;
    bool do_iterate = true;
    std::vector<unsigned> cur_it(bs, 0), order(bs, 0);
    for (unsigned i = 0; i < bs; i++) order[i] = i;
    while (do_iterate) {
      total_iterations++;
      for (auto &e : max_errors) e = 0;
      if (o.isConstrainedProblem())
        perform_one_iteration_for_constrained_pca(V.data(), Z.data(), &o, &stats, bs, n, m, ldB,
                                                  B, max_errors.data(), vals.data(),
                                                  buffer.data(), 0, 0);
      else
        perform_one_iteration_for_penalized_pca(V.data(), Z.data(), &o, &stats, bs, n, m, ldB, B,
                                                max_errors.data(), vals.data(), 0, 0);
      do_iterate = false;
      for (unsigned i = 0; i < bs; i++) {
        cur_it[i]++;
        if (termination_criteria(vals[i].current_error, cur_it[i], &o) ||
            cur_it[i] >= (unsigned)o.maximumIterations) {
          if (best < vals[i].val) {
            best = vals[i].val;
            std::memcpy(x, &V[(size_t)n * i], sizeof(F) * n);
          }
          if (generated < (unsigned)o.totalStartingPoints) {
            vals[i].reset();
            order[i] = generated;
            generated++;
            cur_it[i] = 0;
            do_iterate = true;
          }
        } else {
          do_iterate = true;
        }
      }
      for (unsigned j = 0; j < bs; j++)
        if (cur_it[j] == 0)
          std::memcpy(&V[(size_t)j * n], &V_all[(size_t)order[j] * n], sizeof(F) * n);
    }
  } else {
    for (unsigned batch = 0; batch < o.totalBatches; batch++) {
      unsigned shift = batch * o.batchSize;
      std::memcpy(V.data(), &V_all[(size_t)shift * n], sizeof(F) * n * bs);
      for (unsigned j = 0; j < bs; j++) vals[j].reset();
      for (unsigned it = 0; it < (unsigned)o.maximumIterations; it++) {
        total_iterations++;
        for (auto &e : max_errors) e = 0;
        if (o.isConstrainedProblem())
          perform_one_iteration_for_constrained_pca(V.data(), Z.data(), &o, &stats, bs, n, m, ldB,
                                                    B, max_errors.data(), vals.data(),
                                                    buffer.data(), it, shift);
        else
          perform_one_iteration_for_penalized_pca(V.data(), Z.data(), &o, &stats, bs, n, m, ldB,
                                                  B, max_errors.data(), vals.data(), it, shift);
        F error = max_errors[cblas_vector_max_index((int)max_errors.size(), max_errors.data(), 1)];
        if (termination_criteria(error, it, &o)) break;
      }
      int sel = 0;
      F bv = vals[0].val;
      if (o.storeIterationsForAllPoints) stats.values[shift] = bv;
      for (unsigned i = 1; i < bs; i++) {
        if (o.storeIterationsForAllPoints) stats.values[i + shift] = vals[i].val;
        if (vals[i].val > bv) { bv = vals[i].val; sel = i; }
      }
      if (best < bv) {
        best = bv;
        std::memcpy(x, &V[(size_t)n * sel], sizeof(F) * n);
      }
    }
  }
  st->compute_time = gettime() - t0;
  st->it = total_iterations;
  F nx = cblas_l2_norm(n, x, 1);
  cblas_vector_scale(n, x, 1 / nx);
  st->fval = best;
  st->threads = 1;
  from_ref(&o, s);
  if (o.storeIterationsForAllPoints) {
    for (size_t i = 0; i < stats.values.size(); i++) {
      if (values) values[i] = stats.values[i];
      if (iters) iters[i] = stats.iters[i];
      if (cards) cards[i] = stats.cardinalities[i];
    }
  }
  return best;
}

template <typename F>
F run_soft(F *xv, unsigned len, unsigned s) {
  SolverStructures::OptimizationSettings o;
  std::vector<F> buf(len);
  return soft_thresholding(xv, len, s, buf, &o);
}

template <typename F>
F run_hard(F *xv, unsigned len, unsigned k, int use_sort) {
  SolverStructures::OptimizationSettings o;
  o.useSortForHardThresholding = use_sort != 0;
  std::vector<F> buf(len);
  return k_hard_thresholding(xv, len, k, buf, &o);
}

}  // namespace

extern "C" {

/* Sets TOTAL_THREADS and the thread-private my_thread_id
 * (c++/src/utils/openmp_helper.h:44-67) so per-thread error maxima do not race. */
void ref_init_threads(void) { init_random_seeds(); }
/* OpenMP team size for the reference's parallel regions; 1 makes its own
 * starting points reproducible (they share a global seed across threads). */
void ref_set_threads(int n) {
  omp_set_num_threads(n > 0 ? n : 1);
  init_random_seeds();
}
unsigned ref_total_threads(void) { return TOTAL_THREADS; }

float ref_dense_solver_f32(const float *B, int ldB, float *x, unsigned m, unsigned n,
                           ref_settings *s, ref_stats *st, double *values, int *iters,
                           int *cards) {
  return run_dense_solver<float>(B, ldB, x, m, n, s, st, values, iters, cards);
}
double ref_dense_solver_f64(const double *B, int ldB, double *x, unsigned m, unsigned n,
                            ref_settings *s, ref_stats *st, double *values, int *iters,
                            int *cards) {
  return run_dense_solver<double>(B, ldB, x, m, n, s, st, values, iters, cards);
}
float ref_solver_injected_f32(const float *B, int ldB, float *x, unsigned m, unsigned n,
                              ref_settings *s, ref_stats *st, const float *V_all, double *values,
                              int *iters, int *cards) {
  return run_injected<float>(B, ldB, x, m, n, s, st, V_all, values, iters, cards);
}
double ref_solver_injected_f64(const double *B, int ldB, double *x, unsigned m, unsigned n,
                               ref_settings *s, ref_stats *st, const double *V_all,
                               double *values, int *iters, int *cards) {
  return run_injected<double>(B, ldB, x, m, n, s, st, V_all, values, iters, cards);
}
float ref_soft_thresholding_f32(float *x, unsigned len, unsigned s) { return run_soft(x, len, s); }
double ref_soft_thresholding_f64(double *x, unsigned len, unsigned s) { return run_soft(x, len, s); }
float ref_k_hard_thresholding_f32(float *x, unsigned len, unsigned k, int use_sort) {
  return run_hard(x, len, k, use_sort);
}
double ref_k_hard_thresholding_f64(double *x, unsigned len, unsigned k, int use_sort) {
  return run_hard(x, len, k, use_sort);
}

}  // extern "C"
