"""The oracle against the reference solver compiled from its sources
(oracle/_ref/libref24_naive.so), live, on fresh random inputs.  Skipped where
that build is absent."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def ref(po):
    if not po.ref_available():
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    assert po.ref_set_threads(1) == 1  # the reference's own starts race otherwise
    return po


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("formulation", range(8))
def test_solver_bit_exact(ref, dtype, formulation):
    po = ref
    rng = np.random.default_rng(100 + formulation)
    m, n = int(rng.integers(5, 40)), int(rng.integers(10, 90))
    B = po.low_rank_data(m, n, 3, 8, seed=formulation, dtype=dtype)
    Bd = B.astype(np.float64)
    g = {4: 0.05 * (np.linalg.norm(Bd, axis=0) ** 2).max(), 5: 0.05 * np.abs(Bd).sum(0).max() ** 2,
         6: 0.1 * np.linalg.norm(Bd, axis=0).max(), 7: 0.1 * np.abs(Bd).sum(0).max()}.get(formulation, 0)
    for otf in (False, True):
        for inj in (False, True):
            s = po.make_settings(formulation, constraint=int(rng.integers(1, n)), penalty=g,
                                 tolerance=1e-4, max_iter=25, total_starts=int(rng.integers(3, 20)),
                                 batch_size=int(rng.integers(1, 8)), use_otf=otf, store_all=True)
            s2 = po.Settings.from_buffer_copy(s)
            s2.total_starts = s.total_starts
            V = po.uniform_starts(n, 64, seed=5, dtype=dtype) if inj else None
            a = po.oracle_solve(B, s, V)
            b = po.ref_solve(B, s2, V)
            assert np.array_equal(a["x"], b["x"], equal_nan=True)
            assert a["fval"] == b["fval"] or (np.isnan(a["fval"]) and np.isnan(b["fval"]))
            assert a["it"] == b["it"]
            assert np.array_equal(a["iters"], b["iters"]) and np.array_equal(a["cards"], b["cards"])
