/*
 * Drop-in for the reference's sparse-data entry point and its deflation
 * collection
 *   template<F> F SPCASolver::sparse_PCA_solver_CSC(F* B_CSC_Vals,
 *       int* B_CSC_Row_Id, int* B_CSC_Col_Ptr, F* x, int m, int n,
 *       OptimizationSettings*, OptimizationStatistics*, bool doMean, F* means,
 *       bool doRowMean, F* rowMeans, SparseDeflationCollection<F>&)
 *   -- c++/src/gpower/sparse_PCA_solver_for_CSC.h:111-117 (collection :55-106)
 * forwarding to am24_matrix_create_csc_f32, am24_matrix_deflate and
 * am24_solve_resident_f32 (link with -lam24).  Same arguments and return value
 * (the best objective), x normalised, the settings rewritten as the dense
 * entry point rewrites them.
 *
 * What differs, on purpose:
 * - B (with the means subtracted when doMean / doRowMean) is held on the GPU
 *   of settings->device either densely, solved by the dense tensor-core path,
 *   or (settings->sparseResident; by default when the dense FP32 form would
 *   exceed 8 GiB or the density is below 0.5 %) compressed, with the means
 *   applied implicitly (am24_matrix_create_csc_sparse_f32; no on-the-fly
 *   mode then);
 * - starting points follow settings->startMode (default: the reference's
 *   dense-solver generator, rand_r per global start index), where the
 *   reference's sparse driver draws its constrained starts from the
 *   process-wide rand() state;
 * - starts run in batches of settings->batchSize;
 * - each stored component x deflates B itself, B <- B (I - x x^T), the last
 *   one first.  For mutually orthogonal components that is the reference's
 *   projection of V before and after each product; for others the two sides'
 *   orders of projection differ, and this is the one that projects Z = B V's
 *   side as the reference does.
 * On failure the return value is NaN and am24_last_error() says why.
 */
#ifndef AM24_SPARSE_PCA_SOLVER_FOR_CSC_H
#define AM24_SPARSE_PCA_SOLVER_FOR_CSC_H

#include <limits>
#include <vector>

#include "sparse_PCA_solver.h"

namespace SPCASolver {

// One stored component: its non-zero positions and values.
template <typename F>
class SparseDeflation {
 public:
  std::vector<int> idx;
  std::vector<F> vals;
};

// The components found so far, with the reference's host-side operations on a
// block of n-vectors V (experiments columns): V <- (I - x x^T) V per component.
template <typename F>
class SparseDeflationCollection {
 public:
  std::vector<SparseDeflation<F> > list;
  std::vector<F> buffer;

  void deflateVByPV(F *V, int n, int experiments, SparseDeflation<F> &pv) {
    buffer.assign(experiments, F(0));
    for (int ex = 0; ex < experiments; ex++)
      for (size_t q = 0; q < pv.idx.size(); q++)
        buffer[ex] += V[pv.idx[q] + (size_t)n * ex] * pv.vals[q];
    for (int ex = 0; ex < experiments; ex++)
      for (size_t q = 0; q < pv.idx.size(); q++)
        V[pv.idx[q] + (size_t)n * ex] -= buffer[ex] * pv.vals[q];
  }

  void deflateV(F *V, int n, int experiments) {
    for (size_t p = 0; p < list.size(); p++) deflateVByPV(V, n, experiments, list[p]);
  }

  void addNewSparsePV(std::vector<F> &x) {
    SparseDeflation<F> pv;
    for (size_t i = 0; i < x.size(); i++)
      if (x[i] != 0) {
        pv.idx.push_back((int)i);
        pv.vals.push_back(x[i]);
      }
    list.push_back(pv);
  }
};

template <typename F>
F sparse_PCA_solver_CSC(F *B_CSC_Vals, int *B_CSC_Row_Id, int *B_CSC_Col_Ptr, F *x, int m, int n,
                        SolverStructures::OptimizationSettings *o,
                        SolverStructures::OptimizationStatistics *st, bool doMean, F *means,
                        bool doRowMean, F *rowMeans,
                        SparseDeflationCollection<F> &sparseDeflationCollection) {
  const F nan = std::numeric_limits<F>::quiet_NaN();
  if (m <= 0 || n <= 0 || !B_CSC_Col_Ptr || !x) return nan;
  am24_handle h = am24_detail::default_handle(o->device);
  if (!h) return nan;
  const size_t nnz = (size_t)B_CSC_Col_Ptr[n];
  std::vector<float> vals(B_CSC_Vals, B_CSC_Vals + nnz);
  std::vector<float> mu, rmu;
  if (doMean) mu.assign(means, means + n);
  if (doRowMean) rmu.assign(rowMeans, rowMeans + m);
  am24_matrix mat = nullptr;
  const double dense_bytes = 4.0 * (double)m * (double)n;
  const bool keep_sparse =
      o->sparseResident > 0 ||
      (o->sparseResident < 0 &&
       (dense_bytes > 8.0 * (1u << 30) || (double)nnz < 0.005 * (double)m * (double)n));
  if ((keep_sparse ? am24_matrix_create_csc_sparse_f32 : am24_matrix_create_csc_f32)(
          h, vals.data(), B_CSC_Row_Id, B_CSC_Col_Ptr, (uint32_t)m, (uint32_t)n,
          doMean ? mu.data() : nullptr, doRowMean ? rmu.data() : nullptr, &mat) != AM24_OK)
    return nan;
  std::vector<float> xf(n, 0.f);
  bool ok = true;
  const auto &list = sparseDeflationCollection.list;
  for (size_t p = list.size(); ok && p-- > 0;) {
    std::vector<float> pv(n, 0.f);
    for (size_t q = 0; q < list[p].idx.size(); q++) pv[list[p].idx[q]] = (float)list[p].vals[q];
    ok = am24_matrix_deflate(h, mat, pv.data(), 0) == AM24_OK;
  }
  for (int i = 0; i < n; i++) xf[i] = (float)x[i];
  const float f = ok ? am24_detail::solve_f32(nullptr, m, xf.data(), (unsigned)m, (unsigned)n,
                                              false, o, st, nullptr, nullptr, mat)
                     : std::numeric_limits<float>::quiet_NaN();
  am24_matrix_destroy(h, mat);
  for (int i = 0; i < n; i++) x[i] = (F)xf[i];
  return (F)f;
}

}  // namespace SPCASolver

#endif
