// am24_console -- command-line drop-in for the reference's multicore and GPU
// consoles (c++/src/frontends/multicore_console.cpp:24-56,
// c++/src/frontends/gpu_console.cu:81-158): same getopt flags
// (c++/src/utils/option_console_parser.h:43-156), same CSV input
// (c++/src/utils/file_reader.h:80-86: rows of comma-separated values, read as
// the column-major m x n matrix B) and same output files <out>_x ("i,x_i" for
// every non-zero loading) and <out>_optimizationStatistics
// (c++/src/utils/file_reader.h:100-146).  The solve runs through the drop-in
// SPCASolver::MulticoreSolver::denseDataSolver of <am24/sparse_PCA_solver.h>.
//
//   am24_console -i data.csv -o result -f 1..8 [-s s] [-g gamma] [-m maxIter]
//                [-t tol] [-l starts] [-r batch] [-u 0|1] [-d x] [-v x] [-x rows]
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "am24/sparse_PCA_solver.h"

using SolverStructures::OptimizationSettings;
using SolverStructures::OptimizationStatistics;

namespace {

// console -f numbering (c++/src/utils/option_console_parser.h:105-138)
const SolverStructures::SPCA_Formulation kFlagToFormulation[9] = {
    SolverStructures::L0_constrained_L2_PCA, SolverStructures::L0_constrained_L1_PCA,
    SolverStructures::L0_constrained_L2_PCA, SolverStructures::L1_constrained_L1_PCA,
    SolverStructures::L1_constrained_L2_PCA, SolverStructures::L0_penalized_L1_PCA,
    SolverStructures::L0_penalized_L2_PCA,   SolverStructures::L1_penalized_L1_PCA,
    SolverStructures::L1_penalized_L2_PCA};

int parse_options(OptimizationSettings *s, int argc, char **argv) {
  bool in = false, out = false, form = false;
  int c;
  while ((c = getopt(argc, argv, "i:f:o:m:t:l:r:u:v:d:s:g:x:")) != -1) {
    switch (c) {
      case 'x': s->distributedRowGridFile = atoi(optarg); break;
      case 'l': s->totalStartingPoints = atoi(optarg); break;
      case 'r': s->batchSize = atoi(optarg); break;
      case 's': s->constraintParameter = atoi(optarg); break;
      case 'g': s->penaltyParameter = atof(optarg); break;
      case 'm': s->maximumIterations = atoi(optarg); break;
      case 'i': s->inputFilePath = optarg; in = true; break;
      case 'o': s->outputFilePath = optarg; out = true; break;
      case 'u': s->useOTF = atoi(optarg) != 0; break;
      case 't': s->tolerance = atof(optarg); break;
      case 'd': s->useDoublePrecision = true; break;
      case 'v': s->verbose = true; break;
      case 'f': {
        const int f = atoi(optarg);
        if (f >= 1 && f <= 8) {
          s->formulation = kFlagToFormulation[f];
          form = true;
        }
        break;
      }
      default: break;
    }
  }
  if (!in || !out || !form) {
    std::cout << "Usage: am24_console -i <csv> -o <out> -f <1..8> [-s s] [-g gamma] [-m maxIter]"
                 " [-t tol] [-l starts] [-r batch] [-u otf] [-d] [-v]" << std::endl;
    return 1;
  }
  if (s->batchSize > s->totalStartingPoints) s->totalStartingPoints = s->batchSize;
  return 0;
}

// Rows of comma-separated numbers -> column-major m x n.
template <typename F>
bool read_csv(const char *path, std::vector<F> &B, unsigned &m, unsigned &n) {
  std::ifstream f(path);
  if (!f) return false;
  std::vector<std::vector<double>> rows;
  std::string line;
  while (std::getline(f, line)) {
    if (line.empty()) continue;
    std::vector<double> row;
    std::stringstream ls(line);
    std::string cell;
    while (std::getline(ls, cell, ',')) row.push_back(atof(cell.c_str()));
    rows.push_back(row);
  }
  m = rows.size();
  n = m ? rows[0].size() : 0;
  B.assign((size_t)m * n, 0);
  for (unsigned r = 0; r < m; r++)
    for (unsigned c = 0; c < n && c < rows[r].size(); c++) B[(size_t)c * m + r] = (F)rows[r][c];
  return true;
}

std::string with_suffix(const char *base, const char *suffix) {
  return std::string(base) + "_" + suffix;
}

template <typename F>
void save_x(const OptimizationSettings &s, const std::vector<F> &x) {
  std::ofstream o(with_suffix(s.outputFilePath, "x").c_str());
  for (size_t i = 0; i < x.size(); i++)
    if (x[i] != 0) o << i << "," << std::setprecision(16) << x[i] << '\n';
}

void save_stats(OptimizationSettings &s, const OptimizationStatistics &st) {
  std::ofstream f(with_suffix(s.outputFilePath, "optimizationStatistics").c_str());
  f << "Solver options " << '\n';
  f << "Formulation: " << s.formulation << '\n';
  if (s.isConstrainedProblem())
    f << "Constraint parameter: " << s.constraintParameter << '\n';
  else
    f << "penaltyParameter parameter: " << s.penaltyParameter << '\n';
  f << "Max iterations per starting point: " << s.maximumIterations << '\n';
  f << "Starting points: " << s.totalStartingPoints << '\n';
  f << "Batch size: " << s.batchSize << '\n';
  f << "Batching strategy (OTF): " << s.useOTF << '\n';
  f << "Double precision: " << s.useDoublePrecision << '\n';
  f << "tolerance: " << s.tolerance << '\n';
  f << '\n' << "Timing " << '\n';
  f << "Total computational time: " << std::setprecision(16) << st.totalTrueComputationTime
    << " sec" << '\n';
  f << "Total elapsed time: " << std::setprecision(16) << st.totalElapsedTime << " sec" << '\n';
  f << '\n' << "Result " << '\n';
  f << "Objective value: " << std::setprecision(16) << st.fval << '\n';
  f << "Elapsed it (total): " << st.it << '\n';
  f << "Average it (per starting point): " << std::setprecision(16)
    << st.it * s.batchSize / (0.0 + s.totalStartingPoints) << '\n';
}

template <typename F>
int run(OptimizationSettings *s) {
  const char *dev = getenv("AM24_DEVICE");
  if (dev) s->device = atoi(dev);
  std::vector<F> B;
  unsigned m = 0, n = 0;
  if (!read_csv(s->inputFilePath, B, m, n) || m == 0 || n == 0) {
    std::cerr << "cannot read " << s->inputFilePath << std::endl;
    return 2;
  }
  OptimizationStatistics st;
  st.n = n;
  std::vector<F> x(n, 0);
  const F f = SPCASolver::MulticoreSolver::denseDataSolver<F>(B.data(), (int)m, x.data(), m, n, s,
                                                              &st);
  if (f != f && st.it == 0) {
    std::cerr << "solve failed: " << am24_last_error() << std::endl;
    return 3;
  }
  save_x(*s, x);
  save_stats(*s, st);
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  OptimizationSettings s;
  const int rc = parse_options(&s, argc, argv);
  if (rc > 0) return rc;
  return s.useDoublePrecision ? run<double>(&s) : run<float>(&s);
}
