/*
 * SolverStructures::OptimizationStatistics with the reference's members
 * (c++/src/class/optimization_statistics.h:27-46) plus this library's extras.
 * Times are in seconds (the reference's GPU solver reported milliseconds).
 */
#ifndef AM24_OPTIMIZATION_STATISTICS_H
#define AM24_OPTIMIZATION_STATISTICS_H
#include <vector>

namespace SolverStructures {
class OptimizationStatistics {
 public:
  unsigned int it;
  double fval;
  double error;
  double totalTrueComputationTime;
  double totalElapsedTime;
  unsigned int n;
  std::vector<double> values;
  std::vector<int> iters;
  std::vector<int> cardinalities;
  int totalThreadsUsed;
  // extras
  double explainedVariance;          // ||B x||^2 of the returned x, FP64
  unsigned long long startIterations;
  int degenerateStarts;
  unsigned lowPrecisionIterations;  // batch iterations with BF16 operands (precision 1)
  int inputRoundedToFloat;  // 1: the double data were rounded to float and solved in FP32
  OptimizationStatistics()
      : it(0), fval(0), error(0), totalTrueComputationTime(0), totalElapsedTime(0), n(0),
        totalThreadsUsed(1), explainedVariance(0), startIterations(0), degenerateStarts(0),
        lowPrecisionIterations(0), inputRoundedToFloat(0) {}
};
}  // namespace SolverStructures
#endif
