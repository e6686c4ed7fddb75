"""Deflation between components (am24_matrix_deflate): B <- B (I - x x^T) on
the device against the same update in FP64 on the host, several components
against the oracle's solves on host-deflated data, and batches made before a
deflation reading the deflated matrix afterwards."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _am():
    return importlib.import_module("24am_b200")


def _unit(n, seed, nnz=None):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(n)
    if nnz is not None:
        x[rng.permutation(n)[nnz:]] = 0.0
    return (x / np.linalg.norm(x)).astype(np.float32)


@pytest.mark.parametrize("nnz", [None, 20], ids=["dense_x", "sparse_x"])
def test_deflate_matches_fp64_update(solver, po, nnz):
    m, n = 300, 2000
    B = po.low_rank_data(m, n, 8, 30, seed=31, dtype=np.float32)
    x = _unit(n, 32, nnz)
    M = solver.matrix(B)
    M.deflate(x)
    D = M.read()
    M.close()
    B64, x64 = B.astype(np.float64), x.astype(np.float64)
    ref = B64 - np.outer(B64 @ x64, x64)
    # the device sums y = B x in another order, then rounds each entry once:
    # at most one FP32 step from the FP64 update rounded to FP32
    tol = np.spacing(np.abs(ref).astype(np.float32)).astype(np.float64) + 1e-12 * np.abs(B64).max()
    assert np.all(np.abs(D.astype(np.float64) - ref) <= tol)
    # a projection: the deflated B annihilates x up to FP32 rounding of its entries
    assert np.linalg.norm(D.astype(np.float64) @ x64) <= 1e-5 * np.linalg.norm(B64)


@pytest.mark.parametrize("formulation", [0, 7])
def test_components_match_oracle(solver, po, formulation):
    """Three components from the same injected starts, B deflated by each
    loading in between, against the oracle doing the same in FP64."""
    am = _am()
    m, n, k = 150, 900, 32
    B = po.low_rank_data(m, n, 6, 20, seed=41, dtype=np.float32)
    V = po.uniform_starts(n, k, seed=42, dtype=np.float32)
    g = {7: 3.0}.get(formulation, 0.0)
    st = am.OptimizationSettings(formulation=formulation, constraintParameter=12,
                                 penaltyParameter=g, tolerance=1e-6, maximumIterations=100,
                                 totalStartingPoints=k, batchSize=k,
                                 startMode=am.START_INJECTED)
    M = solver.matrix(B)
    X, f, _ = M.components(st, 3, start_points=V)
    M.close()
    s = po.make_settings(formulation, constraint=12, penalty=g, tolerance=1e-6, max_iter=100,
                         total_starts=k, batch_size=k)
    Bo = B.astype(np.float64)
    for i in range(3):
        r = po.oracle_solve(Bo, s, V.astype(np.float64))
        assert abs(f[i] - r["fval"]) <= 1e-4 * abs(r["fval"]), f"component {i}"
        x = np.asarray(r["x"], np.float64)
        ev, ev_o = (float(np.linalg.norm(Bo @ X[:, i].astype(np.float64)) ** 2),
                    float(np.linalg.norm(Bo @ x) ** 2))
        assert abs(ev - ev_o) <= 1e-4 * ev_o, f"component {i}"
        Bo = Bo - np.outer(Bo @ x, x)
    # every component's loading has unit norm
    assert np.all(np.abs(np.linalg.norm(X.astype(np.float64), axis=0) - 1.0) <= 1e-5)


@pytest.mark.parametrize("k", [96, 256], ids=["one_cta", "cta_pairs"])
@pytest.mark.parametrize("formulation", [0, 5])
def test_batches_made_before_a_deflation_read_the_new_matrix(solver, po, formulation, k):
    """Every layout the matrix holds (the FP16 planes on CTA pairs, the TF32
    planes on one-CTA tiles) is rebuilt in place: a batch made before the
    deflation steps exactly as one made on a fresh copy of the deflated data."""
    am = _am()
    m, n = 300, 3000
    B = po.low_rank_data(m, n, 8, 30, seed=51, dtype=np.float32)
    V = po.uniform_starts(n, k, seed=52, dtype=np.float32)
    st = am.OptimizationSettings(formulation=formulation, constraintParameter=16,
                                 penaltyParameter=0.02 if formulation == 5 else 0.0,
                                 tolerance=1e-6, maximumIterations=10, totalStartingPoints=k,
                                 batchSize=k)
    M = solver.matrix(B)
    b = M.batch(st, k)
    M.deflate(_unit(n, 53))
    b.load(V)
    b.iterate(0, 3)
    after = b.read()
    D = M.read()
    b.close()
    M.close()
    M2 = solver.matrix(D)
    b2 = M2.batch(st, k)
    b2.load(V)
    b2.iterate(0, 3)
    fresh = b2.read()
    b2.close()
    M2.close()
    for a, c in zip(after, fresh):
        assert np.array_equal(a, c, equal_nan=True)
