"""am24_batch_iterate_static_ws (split-K partial sums of Z = B V in the
library's file-scope device array, no allocation) against am24_batch_iterate
on the same matrix, settings and starting points: two calls in a row."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STATIC_WS_BYTES = 16 << 20


def _gamma(B, formulation):
    Bd = B.astype(np.float64)
    c2 = np.linalg.norm(Bd, axis=0).max()
    c1 = np.abs(Bd).sum(0).max()
    # small penalties keep most loadings non-zero, so every step takes the
    # dense tensor-core Z = B V path that uses the split-K workspace
    return {0: 0.0, 4: (0.002 * c2) ** 2, 5: (0.002 * c1) ** 2, 6: 0.002 * c2}[formulation]


@pytest.mark.parametrize("k", [64, 256])
@pytest.mark.parametrize("formulation", [4, 5, 6, 0])
def test_static_ws_matches_iterate(solver, po, formulation, k):
    """k = 64 runs Z = B V on one-CTA tiles; k = 256 on CTA-pair tiles with
    split FP16 operands, whose split-K layout differs.  m = 300 samples make
    three 128-row blocks, so the second half of the last pair tile lies past
    the matrix and its partial tiles are skipped."""
    am = importlib.import_module("24am_b200")
    m, n = 300, 2048
    B = po.low_rank_data(m, n, 8, 30, seed=11, dtype=np.float32)
    V0 = po.uniform_starts(n, k, seed=5, dtype=np.float32)
    st = am.OptimizationSettings(formulation=formulation, constraintParameter=16,
                                 penaltyParameter=_gamma(B, formulation), tolerance=1e-6,
                                 maximumIterations=10, totalStartingPoints=k, batchSize=k)
    M = solver.matrix(B)
    ref, stat = M.batch(st, k), M.batch(st, k)
    ref.load(V0)
    stat.load(V0)
    for call in range(2):
        e_ref = ref.iterate(call, 1)
        e_stat = stat.iterate_static_ws(call, 1)
        Vr, valr, errr, nnzr = ref.read()
        Vs, vals, errs, nnzs = stat.read()
        # same kernels and operands; only the workspace address differs
        tol = 1e-6
        np.testing.assert_allclose(Vs, Vr, rtol=tol, atol=tol * np.abs(Vr).max())
        np.testing.assert_allclose(vals, valr, rtol=tol, atol=0)
        np.testing.assert_allclose(errs, errr, rtol=tol, atol=1e-12)
        np.testing.assert_array_equal(nnzs, nnzr)
        assert e_stat == pytest.approx(e_ref, rel=tol, abs=1e-12)
        if formulation >= 4:
            # more non-zeros than the sparse gather takes: the next step is dense too
            assert nnzr.max() > n // 32
    ref.close()
    stat.close()
    M.close()


def test_static_ws_rejects_large_workspace(solver, am):
    # 33 row tiles x 4 column tiles of 256 x 128 floats, one split: 17.3 MB
    m, n, k = 33 * 128, 256, 1024
    rng = np.random.default_rng(1)
    B = rng.standard_normal((m, n)).astype(np.float32)
    st = am.OptimizationSettings(formulation=0, constraintParameter=8, tolerance=1e-6,
                                 maximumIterations=5, totalStartingPoints=k, batchSize=k)
    M = solver.matrix(B)
    b = M.batch(st, k)
    with pytest.raises(am.Am24Error) as ex:
        b.iterate_static_ws(0, 1)
    assert ex.value.status == 1
    assert "exceeds the static workspace" in str(ex.value)
    b.close()
    M.close()
