/*
 * Drop-in for the reference's GPU entry point
 *   template<F> int SPCASolver::GPUSolver::denseDataSolver(cublasHandle_t&, m, n,
 *       thrust::device_vector<F>& d_B, thrust::host_vector<F>& h_x, settings*, stats*,
 *       LD_M, LD_N) -- c++/src/gpugpower/gpu_sparse_PCA_solver.h:29-35
 * for the FP32 instantiation: d_B is read in place (leading dimension LD_M),
 * h_x receives the normalised loadings, the cuBLAS handle is not used.
 * Returns 0 on success (as the reference), 1 on failure.  Include from CUDA
 * translation units (needs thrust and cublas_v2.h).
 */
#ifndef AM24_GPU_SPARSE_PCA_SOLVER_H
#define AM24_GPU_SPARSE_PCA_SOLVER_H

#include <cublas_v2.h>
#include <thrust/device_vector.h>
#include <thrust/host_vector.h>

#include "sparse_PCA_solver.h"

namespace SPCASolver {
namespace GPUSolver {

template <typename F>
int denseDataSolver(cublasHandle_t &handle, const unsigned int m, const unsigned int n,
                    thrust::device_vector<F> &d_B, thrust::host_vector<F> &h_x,
                    SolverStructures::OptimizationSettings *optimizationSettings,
                    SolverStructures::OptimizationStatistics *optimizationStatistics,
                    const unsigned int LD_M, const unsigned int LD_N);

template <>
inline int denseDataSolver<float>(cublasHandle_t &, const unsigned int m, const unsigned int n,
                                  thrust::device_vector<float> &d_B,
                                  thrust::host_vector<float> &h_x,
                                  SolverStructures::OptimizationSettings *o,
                                  SolverStructures::OptimizationStatistics *st,
                                  const unsigned int LD_M, const unsigned int) {
  if (h_x.size() < n) h_x.resize(n, 0.f);
  am24_status rc = AM24_OK;
  am24_detail::solve_f32(thrust::raw_pointer_cast(d_B.data()), (int)LD_M, &h_x[0], m, n, true, o,
                         st, &rc);
  return rc == AM24_OK ? 0 : 1;
}

}  // namespace GPUSolver
}  // namespace SPCASolver
#endif
