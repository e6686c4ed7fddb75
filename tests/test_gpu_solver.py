"""Whole solves through the drop-in entry point (am24_solve_dense_f32) against
the oracle's restated denseDataSolver in FP64 on the same FP32 data."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _am():
    return importlib.import_module("24am_b200")


def explained_variance(B64, x):
    x = np.asarray(x, np.float64)
    return float(np.linalg.norm(B64 @ x) ** 2)


@pytest.mark.parametrize("formulation", range(8))
@pytest.mark.parametrize("otf", [False, True], ids=["batch", "otf"])
def test_solve_reference_starts(solver, po, formulation, otf):
    """Same seeded data, the reference's own starting points (rand_r seeded by
    the global start index, c++/src/gpower/gpower_commons.h:22-47)."""
    am = _am()
    m, n = 120, 700
    B = po.low_rank_data(m, n, 6, 20, seed=formulation, dtype=np.float32)
    B64 = B.astype(np.float64)
    g = {4: 0.3, 5: 60.0, 6: 0.15, 7: 3.0}.get(formulation, 0.0)
    kw = dict(formulation=formulation, constraintParameter=12, penaltyParameter=g,
              tolerance=1e-6, maximumIterations=60, totalStartingPoints=40, batchSize=16,
              useOTF=otf)
    st = am.OptimizationSettings(**kw)
    x, f, stats = solver.solve(B, st)
    s = po.make_settings(formulation, constraint=12, penalty=g, tolerance=1e-6, max_iter=60,
                         total_starts=40, batch_size=16, use_otf=otf)
    r = po.oracle_solve(B64, s, po.reference_starts(n, 48, formulation <= 3, 12,
                                                    dtype=np.float32).astype(np.float64))
    assert st.totalStartingPoints == 48 and st.totalBatches == 3
    assert abs(f - r["fval"]) <= 1e-4 * abs(r["fval"])
    ev_gpu, ev_orc = explained_variance(B64, x), explained_variance(B64, r["x"])
    assert abs(ev_gpu - ev_orc) <= 1e-4 * ev_orc
    assert abs(stats.explainedVariance - ev_gpu) <= 1e-6 * ev_gpu


@pytest.mark.parametrize("formulation", range(8))
def test_solve_injected_starts_store_all(solver, po, formulation):
    am = _am()
    m, n, k = 300, 2000, 64
    B = po.low_rank_data(m, n, 10, 40, seed=10 + formulation, dtype=np.float32)
    B64 = B.astype(np.float64)
    V = po.uniform_starts(n, k, seed=formulation, dtype=np.float32)
    g = {4: 0.3, 5: 300.0, 6: 0.2, 7: 8.0}.get(formulation, 0.0)
    st = am.OptimizationSettings(formulation=formulation, constraintParameter=16,
                                 penaltyParameter=g, tolerance=1e-6, maximumIterations=100,
                                 totalStartingPoints=k, batchSize=32, startMode=am.START_INJECTED,
                                 storeIterationsForAllPoints=True)
    x, f, stats = solver.solve(B, st, start_points=V)
    s = po.make_settings(formulation, constraint=16, penalty=g, tolerance=1e-6, max_iter=100,
                         total_starts=k, batch_size=32, store_all=True)
    r = po.oracle_solve(B64, s, V.astype(np.float64))
    assert abs(f - r["fval"]) <= 1e-4 * abs(r["fval"])
    assert abs(explained_variance(B64, x) - explained_variance(B64, r["x"])) <= \
        1e-4 * explained_variance(B64, r["x"])
    vals = np.array(stats.values)
    ok = np.abs(vals - r["values"]) <= 1e-4 * np.abs(r["values"]) + 1e-12
    assert ok.mean() >= 0.9
    # batch-global termination at tol = 1e-6 sits near FP32 resolution of the
    # objective, so the stopping iteration may move by a few steps
    assert abs(int(stats.it) - int(r["it"])) <= max(3, int(0.25 * r["it"]))


def test_power_method_known_answer(solver, po):
    """s = n for L2var_L0cons is the power method on B^T B: the loading must
    converge to the top right singular vector (explained variance = sigma_1^2)."""
    am = _am()
    B = po.low_rank_data(200, 500, 5, 500, seed=3, dtype=np.float32)
    B64 = B.astype(np.float64)
    st = am.OptimizationSettings(formulation=0, constraintParameter=500, tolerance=1e-9,
                                 maximumIterations=300, totalStartingPoints=8, batchSize=8)
    x, f, stats = solver.solve(B, st)
    sv = np.linalg.svd(B64, compute_uv=False)
    assert abs(stats.explainedVariance - sv[0] ** 2) <= 1e-4 * sv[0] ** 2
    assert abs(f - sv[0]) <= 1e-4 * sv[0]


def test_large_gamma_is_degenerate_like_reference(solver, po):
    """gamma above every |v| empties every support: the reference divides 0/0
    and returns NaN loadings; the library reports the NaN starts."""
    am = _am()
    B = po.low_rank_data(50, 200, 3, 20, seed=4, dtype=np.float32)
    st = am.OptimizationSettings(formulation=6, penaltyParameter=1e6, maximumIterations=5,
                                 totalStartingPoints=8, batchSize=8)
    x, f, stats = solver.solve(B, st)
    r = po.oracle_solve(B.astype(np.float64), po.make_settings(6, penalty=1e6, max_iter=5,
                                                                total_starts=8, batch_size=8))
    assert np.isnan(r["x"]).all() == np.isnan(x).all()


def test_device_wait_gives_up_and_handle_stays_usable(solver, po):
    """A wait that nothing satisfies ends after its limit with the timeout
    status (no trap, no hang); the same handle then solves normally."""
    import time
    am = _am()
    t0 = time.perf_counter()
    status = am.lib().am24_selftest_bounded_wait(solver.h, 20000)  # 20 ms
    elapsed = time.perf_counter() - t0
    assert status == 4, am.last_error()  # AM24_ERR_DEVICE_TIMEOUT
    assert "timed out" in am.last_error()
    assert 0.015 <= elapsed < 2.0
    B = po.low_rank_data(120, 700, 6, 20, seed=3, dtype=np.float32)
    st = am.OptimizationSettings(formulation=0, constraintParameter=12, tolerance=1e-6,
                                 maximumIterations=30, totalStartingPoints=32, batchSize=32)
    x, f, stats = solver.solve(B, st)
    assert np.isfinite(f) and stats.it > 0


@pytest.mark.parametrize("formulation", [0, 3, 4, 7])
@pytest.mark.parametrize("k", [64, 256])
def test_run_ahead_loop_stops_where_a_host_loop_stops(solver, po, formulation, k):
    """The solve's batch loop queues steps ahead of its convergence check (the
    check runs on the device and gates the steps queued past it); it must stop
    at the same step as a loop that checks the largest change after every step
    on the host, with the same best objective."""
    am = _am()
    m, n = 300, 2500
    B = po.low_rank_data(m, n, 8, 30, seed=21 + formulation, dtype=np.float32)
    V = po.uniform_starts(n, k, seed=22, dtype=np.float32)
    g = {4: 0.05, 5: 4.0, 6: 0.02, 7: 1.0}.get(formulation, 0.0)
    tol = 1e-5
    st = am.OptimizationSettings(formulation=formulation, constraintParameter=10,
                                 penaltyParameter=g, tolerance=tol, maximumIterations=80,
                                 totalStartingPoints=k, batchSize=k, startMode=am.START_INJECTED)
    M = solver.matrix(B)
    b = M.batch(st, k)
    b.load(V)
    steps = 0
    for it in range(80):
        me = b.iterate(it, 1)
        steps += 1
        if it > 0 and me < tol:
            break
    _, val, _, _ = b.read()
    b.close()
    x, f, stats = M.solve(st, start_points=V)
    M.close()
    assert int(stats.it) == steps
    assert int(stats.start_iterations) == steps * k
    assert f == np.nanmax(val)
