"""The serving layer (am24_server_*, am24_submit / am24_poll / am24_wait) and
the FP64 host entry point."""
import ctypes as C
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _am():
    return importlib.import_module("24am_b200")


def _req(am, f, k, s=16, g=0.0, max_iter=100, tol=1e-6, injected=True, precision=0):
    return am.OptimizationSettings(formulation=f, constraintParameter=s, penaltyParameter=g,
                                   tolerance=tol, maximumIterations=max_iter,
                                   totalStartingPoints=k, batchSize=k, precision=precision,
                                   startMode=am.START_INJECTED if injected
                                   else am.START_DEVICE_UNIFORM)


@pytest.mark.parametrize("precision", [0, 1], ids=["fp32", "mixed"])
def test_request_is_the_same_alone_and_in_the_mix(solver, po, precision):
    """Continuous batching: a request served alone and the same request served
    while seven others of other matrices, formulations and start counts run,
    arrive and leave, give the same x, objective, explained variance and
    iteration count, bit for bit."""
    am = _am()
    m, n, k = 300, 2000, 256
    B = po.low_rank_data(m, n, 8, 30, seed=41, dtype=np.float32)
    big = po.low_rank_data(1500, 20000, 8, 30, seed=42, dtype=np.float32)
    V = po.uniform_starts(n, k, seed=50, dtype=np.float32)
    st = _req(am, 0, k, precision=precision)
    srv = am.Server(0, 40 << 30)
    mid = srv.add_matrix(B)
    mbig = srv.add_matrix(big)
    xa, sa = srv.wait(srv.submit(mid, st, start_points=V))
    # long requests first, then the request, then more while it runs
    holds = [srv.submit(mbig, _req(am, f, 300 + 37 * f, s=16 + f, g=0.2, tol=0.0,
                                   max_iter=120, injected=False, precision=precision))
             for f in (0, 3, 4, 7)]
    t = srv.submit(mid, st, start_points=V)
    more = [srv.submit(mid, _req(am, f, 64 + 100 * f, g=0.3, injected=False))
            for f in (1, 2, 6)]
    xb, sb = srv.wait(t)
    for h in holds + more:
        srv.wait(h)
    assert np.array_equal(xa, xb)
    assert sa.fval == sb.fval and sa.it == sb.it
    assert sa.explained_variance == sb.explained_variance
    assert sa.start_iterations == sb.start_iterations == k * sa.it
    assert sb.total_elapsed_time >= sb.total_true_computation_time > 0
    srv.remove_matrix(mbig)
    srv.close()


def test_request_matches_a_one_call_solve(solver, po):
    """A served request of more than 128 starts runs the one-call solve's
    kernels: the same x, objective and iteration count bit for bit."""
    am = _am()
    m, n, k = 300, 2000, 300
    B = po.low_rank_data(m, n, 8, 30, seed=43, dtype=np.float32)
    V = po.uniform_starts(n, k, seed=51, dtype=np.float32)
    srv = am.Server(0, 40 << 30)
    mid = srv.add_matrix(B)
    for f, g in ((0, 0.0), (3, 0.0), (5, 240.0), (6, 0.15)):
        st = _req(am, f, k, s=12, g=g)
        x, s = srv.wait(srv.submit(mid, st, start_points=V))
        M = solver.matrix(B)
        xs, fs, ss = M.solve(_req(am, f, k, s=12, g=g), start_points=V)
        M.close()
        assert np.array_equal(x, xs), f
        assert s.fval == fs and s.it == ss.it and s.explained_variance == ss.explained_variance
    srv.close()


def test_requests_join_while_others_run(solver, po):
    """A short request submitted while a long one is on the device is admitted
    at the next step boundary and finishes first."""
    am = _am()
    B = po.low_rank_data(300, 2000, 8, 30, seed=44, dtype=np.float32)
    big = po.low_rank_data(2000, 40000, 8, 30, seed=45, dtype=np.float32)
    srv = am.Server(0, 40 << 30)
    mid, mbig = srv.add_matrix(B), srv.add_matrix(big)
    long_t = srv.submit(mbig, _req(am, 0, 1024, tol=0.0, max_iter=200, injected=False))
    import time
    time.sleep(0.05)
    short_t = srv.submit(mid, _req(am, 0, 64, injected=False))
    xs, ss = srv.wait(short_t)
    done, _, _ = srv.poll(long_t)
    assert not done  # the short request did not wait for the long one
    xl, sl = srv.wait(long_t)
    assert sl.it == 200 and ss.total_elapsed_time < sl.total_elapsed_time
    srv.close()


def test_admission_by_hbm_budget(po):
    am = _am()
    B = po.low_rank_data(300, 2000, 8, 30, seed=43, dtype=np.float32)
    srv = am.Server(0, 4 << 20)  # 4 MiB: less than the matrix's layouts (about 7.5 MB)
    with pytest.raises(am.Am24Error) as ex:
        srv.add_matrix(B)
    assert ex.value.status == 7
    srv.close()
    srv = am.Server(0, 64 << 20)  # the matrix fits, a large batch does not
    mid = srv.add_matrix(B)
    st = am.OptimizationSettings(formulation=0, constraintParameter=16, tolerance=1e-6,
                                 maximumIterations=10, totalStartingPoints=4096,
                                 batchSize=4096)
    with pytest.raises(am.Am24Error) as ex:
        srv.submit(mid, st)
    assert ex.value.status == 7
    small = am.OptimizationSettings(formulation=0, constraintParameter=16, tolerance=1e-6,
                                    maximumIterations=10, totalStartingPoints=32, batchSize=32)
    x, s = srv.wait(srv.submit(mid, small))
    assert s.it > 0 and np.isfinite(x).all()
    srv.close()


def test_f64_entry_matches_f32_on_float_data(solver, po):
    """FP64 host data rounds to FP32 and solves as the FP32 entry point does:
    on data that are FP32 values, x is the same bit for bit."""
    am = _am()
    m, n = 200, 1500
    B = po.low_rank_data(m, n, 6, 20, seed=44, dtype=np.float32)
    st32 = am.OptimizationSettings(formulation=2, constraintParameter=12, tolerance=1e-6,
                                   maximumIterations=50, totalStartingPoints=64, batchSize=32)
    x32, f32, _ = solver.solve(B, st32)
    B64 = np.asfortranarray(B.astype(np.float64))
    x64 = np.zeros(n, np.float64)
    s = am.OptimizationSettings(formulation=2, constraintParameter=12, tolerance=1e-6,
                                maximumIterations=50, totalStartingPoints=64,
                                batchSize=32).to_c()
    stc = am.am24_statistics()
    f = C.c_double()
    am.check(am.lib().am24_solve_dense_f64(solver.h, B64.ctypes.data_as(C.c_void_p), m,
                                           x64.ctypes.data_as(C.c_void_p), m, n, C.byref(s),
                                           C.byref(stc), None, C.byref(f)))
    assert np.array_equal(x64.astype(np.float32), x32)
    assert f.value == pytest.approx(f32, rel=0, abs=0)
    assert stc.input_rounded_to_f32 == 1


@pytest.mark.parametrize("formulation", [0, 6])
def test_f64_entry_on_double_data_reports_the_rounding(solver, po, formulation):
    """Genuine FP64 data (not FP32 values): the entry point says it rounded
    the input (input_rounded_to_f32 = 1), and its best objective and explained
    variance differ from the FP64 oracle's solve of the unrounded data by the
    rounding's effect, printed here: the objective to 1e-5 relative; the
    explained variance to 1e-4, since under a penalty the rounding of the data
    (2^-24 relative per entry) moves entries near gamma in or out of x."""
    am = _am()
    m, n, k = 200, 1500, 64
    B64 = po.low_rank_data(m, n, 6, 20, seed=46, dtype=np.float64)
    assert not np.array_equal(B64.astype(np.float32).astype(np.float64), B64)
    V = po.uniform_starts(n, k, seed=47, dtype=np.float64)
    g = 0.15 if formulation == 6 else 0.0
    s = am.OptimizationSettings(formulation=formulation, constraintParameter=12,
                                penaltyParameter=g, tolerance=1e-6, maximumIterations=80,
                                totalStartingPoints=k, batchSize=k,
                                startMode=am.START_INJECTED).to_c()
    x64 = np.zeros(n, np.float64)
    stc = am.am24_statistics()
    f = C.c_double()
    Vf = np.asfortranarray(V)
    am.check(am.lib().am24_solve_dense_f64(solver.h, B64.ctypes.data_as(C.c_void_p), m,
                                           x64.ctypes.data_as(C.c_void_p), m, n, C.byref(s),
                                           C.byref(stc), Vf.ctypes.data_as(C.c_void_p),
                                           C.byref(f)))
    assert stc.input_rounded_to_f32 == 1
    r = po.oracle_solve(B64, po.make_settings(formulation, constraint=12, penalty=g,
                                              tolerance=1e-6, max_iter=80, total_starts=k,
                                              batch_size=k), V)
    ev = float(np.linalg.norm(B64 @ x64) ** 2)
    ev_o = float(np.linalg.norm(B64 @ r["x"]) ** 2)
    e_f, e_ev = abs(f.value - r["fval"]) / abs(r["fval"]), abs(ev - ev_o) / ev_o
    print(f"FP64 data through the FP32 path, formulation {formulation}: objective rel err "
          f"{e_f:.2e}, explained variance rel err {e_ev:.2e} against the FP64 oracle")
    assert e_f <= 1e-5 and e_ev <= (1e-4 if formulation >= 4 else 1e-5)


def splitmix64(x):
    """The splitmix64 output mixer on uint64 arrays (wrapping arithmetic)."""
    x = (x + np.uint64(0x9E3779B97F4A7C15))
    x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def test_device_starts_follow_their_definition(solver, po):
    """AM24_START_DEVICE_UNIFORM: entry i of start c is U[-1, 1) from the top 24
    bits of splitmix64((c << 32) | i), then the column is normalised.  A solve
    from device starts and one from the same starts computed here agree."""
    am = _am()
    m, n, k = 200, 1500, 64
    B = po.low_rank_data(m, n, 6, 20, seed=45, dtype=np.float32)
    with np.errstate(over="ignore"):
        key = (np.arange(k, dtype=np.uint64)[None, :] << np.uint64(32)) | \
            np.arange(n, dtype=np.uint64)[:, None]
        z = splitmix64(key)
    U = (z >> np.uint64(40)).astype(np.float64) * (2.0 / 16777216.0) - 1.0
    V = (U / np.linalg.norm(U, axis=0)).astype(np.float32)
    common = dict(formulation=0, constraintParameter=12, tolerance=1e-6, maximumIterations=60,
                  totalStartingPoints=k, batchSize=k)
    xd, fd, sd = solver.solve(B, am.OptimizationSettings(startMode=am.START_DEVICE_UNIFORM,
                                                         **common))
    xi, fi, si = solver.solve(B, am.OptimizationSettings(startMode=am.START_INJECTED, **common),
                              start_points=V)
    assert abs(fd - fi) <= 1e-5 * abs(fi)
    assert abs(sd.explainedVariance - si.explainedVariance) <= 1e-5 * si.explainedVariance
