"""Sparse (CSC) data matrices with the sparse solver's implicit centring
(am24_matrix_create_csc_f32): the densified, centred matrix on the device
against the same arithmetic on the host, solves against the oracle on that
matrix, and malformed arrays rejected before any device write."""
import importlib

import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu


def _am():
    return importlib.import_module("24am_b200")


def _sparse(m, n, seed, density=0.05):
    S = sp.random(m, n, density=density, format="csc", random_state=seed, dtype=np.float64)
    S.data = (S.data * 4.0 - 1.0).astype(np.float32)
    return S.astype(np.float32)


@pytest.mark.parametrize("center", ["none", "columns", "rows", "both"])
def test_csc_densified_with_centring(solver, center):
    am = _am()
    m, n = 200, 1500
    S = _sparse(m, n, 7)
    A = S.toarray().astype(np.float32)
    mu = A.mean(axis=0).astype(np.float32) if center in ("columns", "both") else None
    rmu = A.mean(axis=1).astype(np.float32) if center in ("rows", "both") else None
    M = am.Matrix.from_csc(solver, S, None, None, None, None, means=mu, row_means=rmu)
    D = M.read()
    M.close()
    ref = A.copy()
    if mu is not None:
        ref = ref - mu[None, :]
    if rmu is not None:
        ref = ref - rmu[:, None]
    assert np.array_equal(D, ref)


@pytest.mark.parametrize("formulation", [0, 3, 5, 6])
def test_csc_solve_matches_oracle(solver, po, formulation):
    """Column-centred sparse data (the text-corpus case) solved from the
    reference's own starting points, against the oracle on the dense matrix."""
    am = _am()
    m, n = 150, 1200
    S = _sparse(m, n, 11, density=0.08)
    A = S.toarray().astype(np.float32)
    mu = A.mean(axis=0).astype(np.float32)
    C = (A - mu[None, :]).astype(np.float32)
    g = {5: 0.5, 6: 0.05}.get(formulation, 0.0)
    kw = dict(formulation=formulation, constraintParameter=10, penaltyParameter=g,
              tolerance=1e-6, maximumIterations=60, totalStartingPoints=32, batchSize=32)
    M = am.Matrix.from_csc(solver, S, None, None, None, None, means=mu)
    x, f, stats = M.solve(am.OptimizationSettings(**kw))
    M.close()
    s = po.make_settings(formulation, constraint=10, penalty=g, tolerance=1e-6, max_iter=60,
                         total_starts=32, batch_size=32)
    r = po.oracle_solve(C.astype(np.float64), s,
                        po.reference_starts(n, 32, formulation <= 3, 10,
                                            dtype=np.float32).astype(np.float64))
    assert abs(f - r["fval"]) <= 1e-4 * abs(r["fval"])
    C64 = C.astype(np.float64)
    ev = float(np.linalg.norm(C64 @ x.astype(np.float64)) ** 2)
    ev_o = float(np.linalg.norm(C64 @ np.asarray(r["x"], np.float64)) ** 2)
    assert abs(ev - ev_o) <= 1e-4 * ev_o


def test_csc_rejects_malformed_arrays(solver):
    am = _am()
    vals = np.ones(3, np.float32)
    good_rows = np.array([0, 2, 1], np.int32)
    good_ptr = np.array([0, 2, 3], np.int32)
    M = am.Matrix.from_csc(solver, vals, good_rows, good_ptr, 3, 2)
    assert np.array_equal(M.read(), np.array([[1, 0], [0, 1], [1, 0]], np.float32))
    M.close()
    for rows, ptr in ((np.array([0, 3, 1], np.int32), good_ptr),      # row out of range
                      (np.array([0, -1, 1], np.int32), good_ptr),     # negative row
                      (good_rows, np.array([0, 3, 2], np.int32)),     # decreasing col_ptr
                      (good_rows, np.array([1, 2, 3], np.int32))):    # col_ptr[0] != 0
        with pytest.raises(am.Am24Error) as e:
            am.Matrix.from_csc(solver, vals, rows, ptr, 3, 2)
        assert e.value.status == 1  # AM24_ERR_INVALID_ARG


CSC_PROGRAM = r'''
#include <am24/sparse_PCA_solver_for_CSC.h>
#include <cstdio>
#include <vector>
// input: m n nnz, col_ptr, row_ind, vals, means (n), one component pv (n);
// output: the objectives and x of a solve, of a solve after adding pv to the
// deflation collection, and of a solve with B kept compressed on the device
static SolverStructures::OptimizationSettings settings() {
  SolverStructures::OptimizationSettings s;
  s.formulation = SolverStructures::L0_constrained_L2_PCA;
  s.constraintParameter = 10;
  s.tolerance = 1e-6;
  s.maximumIterations = 60;
  s.totalStartingPoints = 32;
  s.batchSize = 32;
  return s;
}
int main(int argc, char **argv) {
  FILE *f = fopen(argv[1], "rb");
  int m = 0, n = 0, nnz = 0;
  size_t got = fread(&m, 4, 1, f) + fread(&n, 4, 1, f) + fread(&nnz, 4, 1, f);
  std::vector<int> cp(n + 1), ri(nnz);
  std::vector<float> v(nnz), mu(n), pv(n), rmu(m, 0.f);
  got += fread(cp.data(), 4, n + 1, f) + fread(ri.data(), 4, nnz, f) + fread(v.data(), 4, nnz, f);
  got += fread(mu.data(), 4, n, f) + fread(pv.data(), 4, n, f);
  fclose(f);
  if (got != (size_t)(3 + n + 1 + 2 * nnz + 2 * n)) return 2;
  SPCASolver::SparseDeflationCollection<float> defl;
  std::vector<float> x0(n, 0.f), x1(n, 0.f);
  SolverStructures::OptimizationSettings s0 = settings(), s1 = settings();
  SolverStructures::OptimizationStatistics st0, st1;
  float f0 = SPCASolver::sparse_PCA_solver_CSC(v.data(), ri.data(), cp.data(), x0.data(), m, n,
                                               &s0, &st0, true, mu.data(), false, rmu.data(),
                                               defl);
  defl.addNewSparsePV(pv);
  float f1 = SPCASolver::sparse_PCA_solver_CSC(v.data(), ri.data(), cp.data(), x1.data(), m, n,
                                               &s1, &st1, true, mu.data(), false, rmu.data(),
                                               defl);
  SPCASolver::SparseDeflationCollection<float> none;
  std::vector<float> x2(n, 0.f);
  SolverStructures::OptimizationSettings s2 = settings();
  s2.sparseResident = 1;
  SolverStructures::OptimizationStatistics st2;
  float f2 = SPCASolver::sparse_PCA_solver_CSC(v.data(), ri.data(), cp.data(), x2.data(), m, n,
                                               &s2, &st2, true, mu.data(), false, rmu.data(),
                                               none);
  FILE *o = fopen(argv[2], "wb");
  fwrite(&f0, 4, 1, o);
  fwrite(&f1, 4, 1, o);
  fwrite(&f2, 4, 1, o);
  fwrite(x0.data(), 4, n, o);
  fwrite(x1.data(), 4, n, o);
  fwrite(x2.data(), 4, n, o);
  fclose(o);
  return (f0 == f0 && f1 == f1 && f2 == f2) ? 0 : 1;
}
'''


def test_csc_adapter_runs_like_the_python_mirror(solver, tmp_path):
    """A C++ caller of the reference's sparse_PCA_solver_CSC signature, linked to
    the library: a solve, one with a component in the deflation collection, and
    one with the matrix kept compressed (settings.sparseResident = 1), equal to
    the same three solves through the ABI (the mirror's Matrix.from_csc,
    deflate and solve)."""
    import os
    import subprocess
    am = _am()
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    m, n = 150, 1200
    S = _sparse(m, n, 21, density=0.08)
    S.sum_duplicates()
    A = S.toarray().astype(np.float32)
    mu = A.mean(axis=0).astype(np.float32)
    rng = np.random.default_rng(22)
    pv = np.zeros(n, np.float32)
    pick = rng.permutation(n)[:15]
    pv[pick] = rng.standard_normal(15).astype(np.float32)
    pv /= np.linalg.norm(pv)
    pv = pv.astype(np.float32)
    inp = tmp_path / "in.bin"
    with open(inp, "wb") as fh:
        np.array([m, n, S.nnz], np.int32).tofile(fh)
        S.indptr.astype(np.int32).tofile(fh)
        S.indices.astype(np.int32).tofile(fh)
        S.data.astype(np.float32).tofile(fh)
        mu.tofile(fh)
        pv.tofile(fh)
    src = tmp_path / "csc_run.cpp"
    src.write_text(CSC_PROGRAM)
    exe = tmp_path / "csc_run"
    lib = os.path.join(root, "24am_b200")
    subprocess.run(["g++", "-std=c++14", "-O1", f"-I{root}/include", str(src), f"-L{lib}",
                    "-lam24", f"-Wl,-rpath,{lib}", "-o", str(exe)], check=True)
    out = tmp_path / "out.bin"
    subprocess.run([str(exe), str(inp), str(out)], check=True)
    r = np.fromfile(out, np.float32)
    f0, f1, f2 = r[0], r[1], r[2]
    x0, x1, x2 = r[3:3 + n], r[3 + n:3 + 2 * n], r[3 + 2 * n:]
    kw = dict(formulation=0, constraintParameter=10, tolerance=1e-6, maximumIterations=60,
              totalStartingPoints=32, batchSize=32)
    M = am.Matrix.from_csc(solver, S, None, None, None, None, means=mu)
    y0, g0, _ = M.solve(am.OptimizationSettings(**kw))
    M.deflate(pv)
    y1, g1, _ = M.solve(am.OptimizationSettings(**kw))
    M.close()
    assert f0 == np.float32(g0) and np.array_equal(x0, y0)
    assert f1 == np.float32(g1) and np.array_equal(x1, y1)
    # settings.sparseResident = 1: the sparse-resident path of the mirror
    M = am.Matrix.from_csc(solver, S, None, None, None, None, means=mu, keep_sparse=True)
    y2, g2, _ = M.solve(am.OptimizationSettings(**kw))
    M.close()
    assert f2 == np.float32(g2) and np.array_equal(x2, y2)
