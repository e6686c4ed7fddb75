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
