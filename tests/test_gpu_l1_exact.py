"""AM24_L1_EXACT (the exact L1-ball projection, ||x||_1 / ||x||_2 = sqrt(s))
against the exact FP64 level on the same FP32 data and starting points: one
step from dense starts and three steps in a row (the later ones start their
search from the previous level), for the two L1-constraint formulations, on
one-CTA (k = 64) and CTA-pair (k = 256) tiles.  It replaces the reference's
first-break scan (c++/src/utils/thresh_functions.h:162-254), which often
misses the ratio; the exact mode always reaches it."""
import importlib

import numpy as np
import pytest

import fast_oracle as fo

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("k", [64, 256])
@pytest.mark.parametrize("s", [4, 30])
@pytest.mark.parametrize("formulation", [2, 3])
def test_l1_exact_matches_fp64_level(solver, po, formulation, s, k):
    am = importlib.import_module("24am_b200")
    m, n = 300, 4096
    B = po.low_rank_data(m, n, 8, 30, seed=31 + s, dtype=np.float32)
    B64 = B.astype(np.float64)
    V0 = po.uniform_starts(n, k, seed=32, dtype=np.float32)
    st = am.OptimizationSettings(formulation=formulation, constraintParameter=s, tolerance=1e-6,
                                 maximumIterations=10, totalStartingPoints=k, batchSize=k,
                                 l1Mode=am.L1_EXACT)
    M = solver.matrix(B)
    b = M.batch(st, k)
    b.load(V0)
    Vo, valo = V0.astype(np.float64), np.zeros(k)
    ill = np.zeros(k, bool)
    for it in range(3):
        b.iterate(it, 1)
        Vg, valg, _, nnz = b.read()
        r = fo.iteration(B64, Vo, formulation, s, 0.0, valo, l1_exact=True, keep_vraw=True)
        Vo, valo = r.V, r.val
        ill |= r.ill
        # x = (|v| - w)_+ / N: an error e|v| in v moves x by about e max|v| / N
        w = fo.exact_l1_levels(r.vraw, s)
        N = np.linalg.norm(np.maximum(np.abs(r.vraw) - w[None, :], 0.0), axis=0)
        scales = np.abs(r.vraw).max(axis=0) / N
        keep = np.flatnonzero(~ill)
        print(f"formulation {formulation}, s = {s}, k = {k}, step {it + 1}: {len(keep)} "
              f"columns compared, {k - len(keep)} set aside as ill-conditioned")
        assert len(keep) >= k // 2, f"{k - len(keep)} of {k} columns ill-conditioned"
        for j in keep:
            assert np.array_equal(Vg[:, j] != 0, Vo[:, j] != 0), f"step {it}: support of {j}"
            # the level sums every kept entry, so its FP32 error is that of a
            # sum over the support: a few times one entry's
            assert np.abs(Vg[:, j] - Vo[:, j]).max() <= 5e-5 * scales[j], \
                f"step {it}: column {j}"
            x = Vg[:, j].astype(np.float64)
            ratio = np.abs(x).sum() / np.linalg.norm(x)
            assert abs(ratio - np.sqrt(s)) <= 1e-5 * np.sqrt(s), (it, j, ratio)
        # the objective follows the loadings: held to the same 5e-5
        rel = np.abs(valg[keep] - valo[keep]) / np.abs(valo[keep])
        print(f"  objective max rel err {rel.max(initial=0):.2e}")
        assert rel.max(initial=0) <= 5e-5
    b.close()
    M.close()
