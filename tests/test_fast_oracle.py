"""The BLAS-backed FP64 iteration (oracle/fast_oracle.py) against the C
oracle's orc_iteration_f64, which is pinned bit for bit to the reference:
identical supports and values within FP64 rounding, every formulation, a few
steps from the same starts; and its exact L1-ball level against the definition."""
import numpy as np
import pytest

import fast_oracle as fo

GAMMA = {4: 0.3, 5: 60.0, 6: 0.15, 7: 3.0}


@pytest.mark.parametrize("formulation", range(8))
def test_fast_iteration_matches_c_oracle(po, formulation):
    m, n, k, s = 60, 300, 12, 9
    B = po.low_rank_data(m, n, 5, 20, seed=3 + formulation)
    V = po.uniform_starts(n, k, seed=4)
    g = GAMMA.get(formulation, 0.0)
    st = po.make_settings(formulation, constraint=s, penalty=g, tolerance=1e-6, max_iter=10,
                          total_starts=k, batch_size=k)
    Vc, valc = V.copy(), np.zeros(k)
    Vf, valf = V.copy(), np.zeros(k)
    for it in range(4):
        Vc, _, valc, errc, mec = po.oracle_iteration(B, Vc, st, valc, it=it)
        r = fo.iteration(B, Vf, formulation, s, g, valf)
        Vf, valf = r.V, r.val
        assert np.array_equal(Vc != 0, Vf != 0), f"support differs at step {it}"
        assert np.allclose(Vf, Vc, rtol=1e-12, atol=1e-13 * np.abs(Vc).max())
        assert np.allclose(valf, valc, rtol=1e-12)
        fin = ~np.isnan(errc)
        assert np.allclose(r.err[fin], errc[fin], rtol=1e-9, atol=1e-15)
        assert abs(r.max_err - mec) <= 1e-9 * max(abs(mec), 1e-300) or (it == 0)


@pytest.mark.parametrize("formulation", [0, 3, 4, 7])
def test_fast_batch_solve_matches_c_oracle(po, formulation):
    m, n, k, s = 50, 200, 8, 7
    B = po.low_rank_data(m, n, 4, 16, seed=9)
    V = po.uniform_starts(n, k, seed=10)
    g = GAMMA.get(formulation, 0.0)
    st = po.make_settings(formulation, constraint=s, penalty=g, tolerance=1e-6, max_iter=40,
                          total_starts=k, batch_size=k)
    r = po.oracle_solve(B, st, V)
    Vf, valf, steps, ill = fo.batch_solve(B, V, formulation, s, g, tol=1e-6, max_iter=40)
    assert steps == r["it"]
    best = int(np.nanargmax(valf))
    assert abs(valf[best] - r["fval"]) <= 1e-10 * abs(r["fval"])


@pytest.mark.parametrize("s", [2, 5, 30])
def test_exact_l1_level(s):
    rng = np.random.default_rng(s)
    v = rng.standard_normal(400)
    w = fo.exact_l1_level(v, s)
    x = np.maximum(np.abs(v) - w, 0)
    assert abs(x.sum() / np.linalg.norm(x) - np.sqrt(s)) <= 1e-9 * np.sqrt(s)


def test_exact_l1_levels_vectorised_matches_closed_form():
    rng = np.random.default_rng(7)
    V = rng.standard_normal((500, 6))
    for s in (2, 9, 40):
        w = fo.exact_l1_levels(V, s)
        for j in range(V.shape[1]):
            assert abs(w[j] - fo.exact_l1_level(V[:, j], s)) <= 1e-12 * np.abs(V[:, j]).max()
