/*
 * SolverStructures::OptimizationSettings and SPCA_Formulation with the
 * reference's member names, types and defaults
 * (c++/src/class/optimization_settings.h:27-170), so code written against the
 * reference compiles unchanged.  Extra members (startMode, l1Mode, timeoutMs,
 * precision, stableIterations, stableShare, leadIterations, device, sparseResident) select this library's options and
 * default to reference behaviour.
 */
#ifndef AM24_OPTIMIZATION_SETTINGS_H
#define AM24_OPTIMIZATION_SETTINGS_H

namespace SolverStructures {

enum SPCA_Formulation {
  L0_constrained_L2_PCA = 0,
  L0_constrained_L1_PCA,
  L1_constrained_L2_PCA,
  L1_constrained_L1_PCA,
  L0_penalized_L2_PCA,
  L0_penalized_L1_PCA,
  L1_penalized_L2_PCA,
  L1_penalized_L1_PCA
};

template <typename T>
T &operator<<(T &stream, SPCA_Formulation &f) {
  static const char *names[] = {"L0_constrained_L2_PCA", "L0_constrained_L1_PCA",
                                "L1_constrained_L2_PCA", "L1_constrained_L1_PCA",
                                "L0_penalized_L2_PCA",   "L0_penalized_L1_PCA",
                                "L1_penalized_L2_PCA",   "L1_penalized_L1_PCA"};
  if ((int)f >= 0 && (int)f < 8) stream << names[(int)f];
  return stream;
}

class OptimizationSettings {
 public:
  int proccessNode;
  int distributedRowGridFile;
  double tolerance;
  bool verbose;
  bool useSortForHardThresholding;
  bool useKSelectionAlgorithmGPU;
  bool useDoublePrecision;
  double penaltyParameter;
  unsigned int constraintParameter;
  char *inputFilePath;
  char *outputFilePath;
  int gpu_sm_count;
  int gpu_max_threads;
  enum SPCA_Formulation formulation;
  bool getValuesForAllStartingPoints;
  bool storeIterationsForAllPoints;
  int maximumIterations;
  int totalStartingPoints;
  int batchSize;
  unsigned int totalBatches;
  bool useOTF;
  bool doColumnMean;
  bool doRowMean;
  bool L2RowNormalization;
  bool tfidf;
  // this library's options
  int startMode;       // 0: reference generator (rand_r per start index), 1: injected
  int l1Mode;          // 0: the reference's L1-ball scan, 1: exact projection
  unsigned timeoutMs;  // bound on any device-side wait
  int precision;       // 0: FP32-accurate products, 1: BF16 until supports settle, then FP32
  unsigned stableIterations;  // precision 1: iterations of unchanged supports before refining
  float stableShare;          // precision 1: share of the starts that must be that stable
  unsigned leadIterations;    // precision 1: FP32-accurate iterations before the single-pass phase
  int device;          // CUDA device of the default handle
  int sparseResident;  // sparse_PCA_solver_CSC: 1 keeps B compressed on the device, 0
                       // densifies it, -1 (default) keeps it compressed when its dense
                       // FP32 form would exceed 8 GiB or its density is below 0.5 %

  OptimizationSettings()
      : proccessNode(0), distributedRowGridFile(0), tolerance(0.01), verbose(false),
        useSortForHardThresholding(false), useKSelectionAlgorithmGPU(true),
        useDoublePrecision(false), penaltyParameter(0), constraintParameter(10),
        inputFilePath(0), outputFilePath(0), gpu_sm_count(0), gpu_max_threads(0),
        formulation(L0_constrained_L2_PCA), getValuesForAllStartingPoints(true),
        storeIterationsForAllPoints(false), maximumIterations(20), totalStartingPoints(64),
        batchSize(64), totalBatches(0), useOTF(false), doColumnMean(true), doRowMean(false),
        L2RowNormalization(true), tfidf(true), startMode(0), l1Mode(0), timeoutMs(5000),
        precision(0), stableIterations(5), stableShare(1.0f), leadIterations(0),
        device(0), sparseResident(-1) {}

  bool isConstrainedProblem() const { return (int)formulation <= 3; }
  bool isL1ConstrainedProblem() const {
    return !(formulation == L0_constrained_L1_PCA || formulation == L0_constrained_L2_PCA);
  }
  bool isL1PenalizedProblem() const {
    return !(formulation == L0_penalized_L1_PCA || formulation == L0_penalized_L2_PCA);
  }
  // s <= n; batch 0 means all starts; starts rounded up to whole batches.
  void chceckInputAndModifyIt(unsigned int n) {
    if (constraintParameter > n) constraintParameter = n;
    if (batchSize == 0) batchSize = totalStartingPoints;
    totalBatches = totalStartingPoints / batchSize;
    if (totalBatches * batchSize < (unsigned)totalStartingPoints) totalBatches++;
    totalStartingPoints = totalBatches * batchSize;
  }
};

}  // namespace SolverStructures
#endif
