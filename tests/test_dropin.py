"""The C++ drop-in boundary: the adapter headers compile against reference-style
callers, and the console reproduces the reference console's runs."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CONSOLE = os.path.join(ROOT, "24am_b200", "am24_console")
GOLDEN = os.path.join(ROOT, "tests", "golden", "reference_small_csv.npz")

CALLER = r'''
#include <am24/sparse_PCA_solver.h>
#include <vector>
using namespace SolverStructures;
// the shape of the reference's multicore console call (multicore_console.cpp:35)
template <typename F> F run(std::vector<F>& B, unsigned m, unsigned n, OptimizationSettings* s) {
  OptimizationStatistics* st = new OptimizationStatistics();
  std::vector<F> x(n, 0);
  F f = SPCASolver::MulticoreSolver::denseDataSolver(&B[0], m, &x[0], m, n, s, st);
  delete st;
  return f;
}
int main() {
  OptimizationSettings s; s.formulation = L1_penalized_L2_PCA;
  std::vector<float> Bf(6, 1.f); std::vector<double> Bd(6, 1.0);
  return (run(Bf, 2, 3, &s) == run(Bd, 2, 3, &s)) ? 0 : 0;
}
'''

GPU_CALLER = r'''
#include <am24/gpu_sparse_PCA_solver.h>
// the shape of the reference GPU console's call (gpu_console.cu:132)
int call(cublasHandle_t& h, thrust::device_vector<float>& d_B, thrust::host_vector<float>& x,
         SolverStructures::OptimizationSettings* s, SolverStructures::OptimizationStatistics* st) {
  return SPCASolver::GPUSolver::denseDataSolver(h, 2u, 3u, d_B, x, s, st, 32u, 32u);
}
'''


CSC_CALLER = r'''
#include <am24/sparse_PCA_solver_for_CSC.h>
#include <vector>
using namespace SolverStructures;
// the shape of the reference's sparse solver call, with its deflation collection
// (c++/src/gpower/sparse_PCA_solver_for_CSC.h:111-117)
template <typename F> F run(std::vector<F>& v, std::vector<int>& r, std::vector<int>& c, int m,
                            int n, OptimizationSettings* s) {
  OptimizationStatistics* st = new OptimizationStatistics();
  SPCASolver::SparseDeflationCollection<F> defl;
  std::vector<F> x(n, 0), means(n, 0), rowMeans(m, 0);
  F f = SPCASolver::sparse_PCA_solver_CSC(&v[0], &r[0], &c[0], &x[0], m, n, s, st, true,
                                          &means[0], false, &rowMeans[0], defl);
  defl.addNewSparsePV(x);
  std::vector<F> V(n * 2, 1);
  defl.deflateV(&V[0], n, 2);
  delete st;
  return f;
}
int main() {
  OptimizationSettings s;
  std::vector<float> vf(2, 1.f); std::vector<double> vd(2, 1.0);
  std::vector<int> r = {0, 1}, c = {0, 1, 2};
  return (run(vf, r, c, 2, 2, &s) == run(vd, r, c, 2, 2, &s)) ? 0 : 0;
}
'''


def test_csc_adapter_compiles_for_reference_callers(tmp_path):
    src = tmp_path / "csc_caller.cpp"
    src.write_text(CSC_CALLER)
    subprocess.run(["g++", "-std=c++14", "-Wall", "-Werror", f"-I{ROOT}/include", "-c", str(src),
                    "-o", str(tmp_path / "csc_caller.o")], check=True)


def test_adapter_compiles_for_reference_callers(tmp_path):
    src = tmp_path / "caller.cpp"
    src.write_text(CALLER)
    subprocess.run(["g++", "-std=c++14", "-Wall", "-Werror", f"-I{ROOT}/include", "-c", str(src),
                    "-o", str(tmp_path / "caller.o")], check=True)


def test_gpu_adapter_compiles_with_nvcc(tmp_path):
    src = tmp_path / "gcaller.cu"
    src.write_text(GPU_CALLER)
    subprocess.run(["nvcc", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
                    f"-I{ROOT}/include", "-c", str(src), "-o", str(tmp_path / "g.o")], check=True)


def test_console_usage_without_required_flags():
    r = subprocess.run([CONSOLE], capture_output=True, text=True)
    assert r.returncode == 1 and "Usage" in r.stdout


def _write_csv(path, B):
    with open(path, "w") as f:
        for row in B:
            f.write(",".join(repr(float(v)) for v in row) + "\n")


def _read_x(path, n):
    x = np.zeros(n)
    for line in open(path):
        i, v = line.strip().split(",")
        x[int(i)] = float(v)
    return x


def _read_fval(path):
    for line in open(path):
        if line.startswith("Objective value:"):
            return float(line.split(":")[1])
    raise AssertionError("no objective in " + path)


@pytest.mark.gpu
@pytest.mark.parametrize("name,flags", [
    ("small_f1_s3", ["-f", "1", "-s", "3"]),
    ("small_f1_s2_l1000_r64", ["-l", "1000", "-r", "64", "-f", "1", "-s", "2"]),
    ("small_f1_s2_l1000_r64_otf", ["-l", "1000", "-r", "64", "-u", "1", "-f", "1", "-s", "2"]),
])
def test_console_matches_reference_console_runs(name, flags):
    """The reference Makefile's console runs on datasets/small.csv
    (c++/multicore.mk:18-21), against outputs the reference itself produced."""
    z = np.load(GOLDEN)
    B = z["B"]
    with tempfile.TemporaryDirectory() as d:
        csv = os.path.join(d, "small.csv")
        _write_csv(csv, B)
        out = os.path.join(d, "res")
        subprocess.run([CONSOLE, "-i", csv, "-o", out, "-v", "true", "-d", "double"] + flags,
                       check=True, timeout=120)
        x = _read_x(out + "_x", B.shape[1])
        f = _read_fval(out + "_optimizationStatistics")
    assert abs(f - float(z[f"{name}.fval"])) <= 1e-5 * abs(float(z[f"{name}.fval"]))
    assert np.allclose(x, z[f"{name}.x"], atol=1e-5)


COLLECTION_PROGRAM = r'''
#include <am24/sparse_PCA_solver_for_CSC.h>
#include <cstdio>
#include <vector>
// V (n x 2) <- the collection's projections, then printed: the host-side part
// of the sparse solver's deflation collection, which needs no device
int main() {
  const int n = 5;
  SPCASolver::SparseDeflationCollection<double> defl;
  std::vector<double> x1 = {0.6, 0.0, 0.8, 0.0, 0.0}, x2 = {0.0, 1.0, 0.0, 0.0, 0.0};
  defl.addNewSparsePV(x1);
  defl.addNewSparsePV(x2);
  std::vector<double> V = {1, 2, 3, 4, 5, -1, 0.5, 2, 0, 1};
  defl.deflateV(&V[0], n, 2);
  for (double v : V) printf("%.17g\n", v);
  return (defl.list.size() == 2 && defl.list[0].idx.size() == 2) ? 0 : 1;
}
'''


def test_deflation_collection_projects_like_the_reference(tmp_path):
    """SparseDeflationCollection keeps each component's non-zeros and projects a
    block of vectors by each component in turn, V <- (I - x x^T) V."""
    src = tmp_path / "coll.cpp"
    src.write_text(COLLECTION_PROGRAM)
    exe = tmp_path / "coll"
    subprocess.run(["g++", "-std=c++14", "-Wall", "-Werror", f"-I{ROOT}/include", str(src),
                    "-o", str(exe), f"-L{ROOT}/24am_b200", "-lam24",
                    f"-Wl,-rpath,{ROOT}/24am_b200"], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    got = np.array([float(t) for t in out.split()]).reshape(2, 5).T
    V = np.array([[1, 2, 3, 4, 5], [-1, 0.5, 2, 0, 1]], float).T
    for x in (np.array([0.6, 0, 0.8, 0, 0]), np.array([0, 1.0, 0, 0, 0])):
        V = V - np.outer(x, x @ V)
    assert np.allclose(got, V, rtol=0, atol=1e-15)


GPU_PROGRAM = r'''
#include <am24/gpu_sparse_PCA_solver.h>
#include <cstdio>
#include <cstdlib>
#include <vector>
// the reference GPU console's call (c++/src/frontends/gpu_console.cu:76): B copied
// into a thrust::device_vector with its leading dimension padded to 128 bytes,
// then SPCASolver::GPUSolver::denseDataSolver
int main(int argc, char** argv) {
  FILE* f = fopen(argv[1], "rb");
  unsigned m = 0, n = 0;
  if (fread(&m, 4, 1, f) != 1 || fread(&n, 4, 1, f) != 1) return 2;
  std::vector<float> B((size_t)m * n);
  if (fread(B.data(), 4, B.size(), f) != B.size()) return 2;
  fclose(f);
  const unsigned LD_M = (m + 31) / 32 * 32, LD_N = (n + 31) / 32 * 32;
  thrust::host_vector<float> hB((size_t)LD_M * n, 0.f);
  for (unsigned c = 0; c < n; c++)
    for (unsigned r = 0; r < m; r++) hB[(size_t)c * LD_M + r] = B[(size_t)c * m + r];
  thrust::device_vector<float> dB = hB;
  thrust::host_vector<float> x(LD_N, 0.f);
  SolverStructures::OptimizationSettings s;
  s.formulation = (SolverStructures::SPCA_Formulation)atoi(argv[2]);
  s.constraintParameter = atoi(argv[3]);
  s.penaltyParameter = atof(argv[4]);
  s.tolerance = 1e-6;
  s.maximumIterations = 60;
  s.totalStartingPoints = 40;
  s.batchSize = 16;
  SolverStructures::OptimizationStatistics st;
  cublasHandle_t handle = nullptr;  // the adapter does not use cuBLAS
  const int rc = SPCASolver::GPUSolver::denseDataSolver(handle, m, n, dB, x, &s, &st, LD_M, LD_N);
  printf("%d %.9g %u %u\n", rc, st.fval, s.totalStartingPoints, s.totalBatches);
  for (unsigned i = 0; i < n; i++) printf("%.9g\n", x[i]);
  return rc;
}
'''


@pytest.mark.gpu
@pytest.mark.parametrize("formulation,s,gamma", [(0, 12, 0.0), (3, 12, 0.0), (6, 0, 0.15),
                                                 (5, 0, 60.0)])
def test_gpu_adapter_solves_like_the_oracle(tmp_path, po, formulation, s, gamma):
    """A program written against the reference's GPU entry point, linked to
    libam24.so, solves a device-resident B (the reference's own starting
    points, batch mode) to the oracle's best objective and loading."""
    src = tmp_path / "gprog.cu"
    src.write_text(GPU_PROGRAM)
    exe = tmp_path / "gprog"
    subprocess.run(["nvcc", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
                    f"-I{ROOT}/include", str(src), "-o", str(exe), f"-L{ROOT}/24am_b200",
                    "-lam24", f"-Xlinker=-rpath,{ROOT}/24am_b200"], check=True)
    m, n = 120, 700
    B = po.low_rank_data(m, n, 6, 20, seed=formulation, dtype=np.float32)
    data = tmp_path / "B.bin"
    with open(data, "wb") as f:
        np.array([m, n], np.uint32).tofile(f)
        np.asfortranarray(B).T.astype(np.float32).tofile(f)
    out = subprocess.run([str(exe), str(data), str(formulation), str(max(s, 1)), repr(gamma)],
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    lines = out.stdout.split("\n")
    rc, fval, total, batches = lines[0].split()
    x = np.array([float(t) for t in lines[1:1 + n]])
    assert int(rc) == 0 and int(total) == 48 and int(batches) == 3
    B64 = B.astype(np.float64)
    st = po.make_settings(formulation, constraint=max(s, 1), penalty=gamma, tolerance=1e-6,
                          max_iter=60, total_starts=40, batch_size=16)
    r = po.oracle_solve(B64, st, po.reference_starts(n, 48, formulation <= 3, max(s, 1),
                                                     dtype=np.float32).astype(np.float64))
    assert abs(float(fval) - r["fval"]) <= 1e-5 * abs(r["fval"])
    # a whole solve with the batch-global stop near FP32 resolution of the
    # objective: the returned loadings can sit a step apart (the per-start 1e-5
    # parity is in test_gpu_baseline_parity.py)
    ev = np.linalg.norm(B64 @ x) ** 2
    ev_o = np.linalg.norm(B64 @ r["x"]) ** 2
    assert abs(ev - ev_o) <= 1e-4 * ev_o
