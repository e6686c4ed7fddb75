"""The MIXED precision mode: single-pass V = B^T Z (FP16 operands on the
scaled h0 / g0 planes, or BF16 with AM24_MIXED_BF16=1) while the supports
settle, then the FP32-accurate products.  One low-precision step against the
FP64 product within the single pass's rounding (and, for BF16, against the
product of the BF16-rounded operands), the phase switch, and whole solves
that reach the FP32 path's explained variance within 1e-4."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _am():
    return importlib.import_module("24am_b200")


def bf16_round(x):
    """Round FP32 values to the nearest BF16 (ties to even), as FP32."""
    b = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return r.astype(np.uint32).view(np.float32)


@pytest.mark.parametrize("formulation", [5, 4])
def test_bf16_step_matches_rounded_product(solver, po, formulation, monkeypatch):
    """With AM24_MIXED_BF16=1 the first phase runs single-pass BF16.  With
    gamma = 0 the L0 penalty keeps every non-zero v, so one such step returns
    V = b0(B)^T Z_b, b0 the BF16 rounding of B and Z_b that of Z (exact for the
    L1-variance sgn)."""
    monkeypatch.setenv("AM24_MIXED_BF16", "1")
    am = _am()
    m, n, k = 300, 2000, 256  # k > 128: CTA-pair tiles, where MIXED applies
    B = po.low_rank_data(m, n, 8, 30, seed=3, dtype=np.float32)
    V0 = po.uniform_starts(n, k, seed=4, dtype=np.float32)
    st = am.OptimizationSettings(formulation=formulation, penaltyParameter=0.0, tolerance=1e-6,
                                 maximumIterations=10, totalStartingPoints=k, batchSize=k,
                                 precision=am.PRECISION_MIXED)
    M = solver.matrix(B)
    b = M.batch(st, k)
    b.load(V0)
    b.iterate(0, 1)
    assert not b.refining()
    V1 = b.read()[0].astype(np.float64)
    Y = B.astype(np.float64) @ V0.astype(np.float64)
    if formulation == 5:
        Z = np.sign(Y)
        # a sign decided within FP32 rounding of zero is not a fair test
        ok = np.abs(Y).min(0) > 1e-4 * np.abs(Y).max(0)
    else:
        Z = bf16_round((Y / np.linalg.norm(Y, axis=0)).astype(np.float32)).astype(np.float64)
        ok = np.ones(k, bool)
    b0 = bf16_round(B).astype(np.float64)
    Vref = b0.T @ Z
    scale = np.abs(b0).T @ np.abs(Z)  # sum_i |b0_ij| |z_i| per entry
    err = np.abs(V1 - Vref)
    if formulation == 5:
        # exact products, FP32 accumulation over K = m
        assert np.all(err[:, ok] <= 5e-5 * scale[:, ok] + 1e-30), np.max(err / scale)
    else:
        # Z from the FP32 path (normalised as y * (1/||y||) in FP32, a few ulps
        # from the FP64 value here) can round to the other BF16 neighbour where
        # it sits that close to a BF16 rounding boundary; such a flip moves z_i
        # by at most 2^-7 |z_i| and touches one column.  Most columns meet the
        # tight bound, every column the bound plus two flips.
        tight = err <= 5e-5 * scale
        ab = np.abs(b0).T
        flips = 2.0 * 2.0 ** -7 * np.stack([(ab * np.abs(Z[:, c])).max(1) for c in range(k)], 1)
        assert np.mean(tight.all(0)) >= 0.95, np.max(err / scale)
        assert np.all(err <= 5e-5 * scale + flips)
    b.close()
    M.close()


@pytest.mark.parametrize("formulation", [5, 4])
def test_fp16_step_is_within_the_single_pass_bound(solver, po, formulation):
    """The default first phase: one FP16 MMA per product on the scaled h0 / g0
    planes (each operand rounded to 11 significant bits after a power-of-two
    scale per feature and per start).  With gamma = 0 one step returns V = B^T Z
    up to that rounding: each term within 2^-11 (the L1-variance forms, whose
    sgn(z) is exact) or 2 x 2^-11 of |b| |z|, plus FP32 accumulation; and the
    error is that of a single pass, far above the FP32-accurate products'."""
    am = _am()
    m, n, k = 300, 2000, 256
    B = po.low_rank_data(m, n, 8, 30, seed=3, dtype=np.float32)
    V0 = po.uniform_starts(n, k, seed=4, dtype=np.float32)
    st = am.OptimizationSettings(formulation=formulation, penaltyParameter=0.0, tolerance=1e-6,
                                 maximumIterations=10, totalStartingPoints=k, batchSize=k,
                                 precision=am.PRECISION_MIXED)
    M = solver.matrix(B)
    b = M.batch(st, k)
    b.load(V0)
    kinds = dict(b.step_timed(0))
    assert "gemm_BtZ_low" in kinds and "gemm_BtZ(skipped)" in kinds
    assert not b.refining()
    V1 = b.read()[0].astype(np.float64)
    B64 = B.astype(np.float64)
    Y = B64 @ V0.astype(np.float64)
    if formulation == 5:
        Z = np.sign(Y)
        ok = np.abs(Y).min(0) > 1e-4 * np.abs(Y).max(0)
        unit = 2.0 ** -11
    else:
        Z = Y / np.linalg.norm(Y, axis=0)
        ok = np.ones(k, bool)
        unit = 2.0 * 2.0 ** -11
    Vref = B64.T @ Z
    scale = np.abs(B64).T @ np.abs(Z)
    rel = np.abs(V1 - Vref)[:, ok] / scale[:, ok]
    assert rel.max() <= unit + 5e-5, rel.max()
    assert rel.max() > 1e-5  # a single pass, not the FP32-accurate split
    b.close()
    M.close()


def test_phase_switches_to_fp32_products(solver, po):
    """Step kernels before and after the switch: the BF16 V = B^T Z runs while
    the supports move, the FP32-accurate one after every start has kept its
    support for stableIterations steps."""
    am = _am()
    m, n, k = 300, 2000, 256
    B = po.low_rank_data(m, n, 8, 30, seed=5, dtype=np.float32)
    V0 = po.uniform_starts(n, k, seed=6, dtype=np.float32)
    st = am.OptimizationSettings(formulation=0, constraintParameter=16, tolerance=1e-6,
                                 maximumIterations=100, totalStartingPoints=k, batchSize=k,
                                 precision=am.PRECISION_MIXED, stableIterations=3)
    M = solver.matrix(B)
    b = M.batch(st, k)
    b.load(V0)
    first = dict(b.step_timed(0))
    assert "gemm_BtZ_low" in first and "gemm_BtZ(skipped)" in first and "support" in first
    switched_at = None
    for it in range(1, 60):
        b.iterate(it, 1)
        if b.refining():
            switched_at = it
            break
    assert switched_at is not None and switched_at >= 3
    after = dict(b.step_timed(switched_at + 1))
    assert "gemm_BtZ" in after and "gemm_BtZ_low(skipped)" in after
    b.close()
    M.close()


@pytest.mark.parametrize("formulation", [0, 7])
def test_mixed_solve_reaches_fp32_variance(solver, po, formulation):
    """Whole solves (batch mode) from the same injected starts: the MIXED run
    ends within 1e-4 of the FP32 run's best explained variance, after a BF16
    phase and refinement steps."""
    am = _am()
    m, n, k = 400, 3000, 256
    B = po.low_rank_data(m, n, 10, 40, seed=20 + formulation, dtype=np.float32)
    B64 = B.astype(np.float64)
    V = po.uniform_starts(n, k, seed=30 + formulation, dtype=np.float32)
    g = {7: 8.0}.get(formulation, 0.0)
    out = {}
    for prec in (am.PRECISION_FP32, am.PRECISION_MIXED):
        st = am.OptimizationSettings(formulation=formulation, constraintParameter=32,
                                     penaltyParameter=g, tolerance=1e-6, maximumIterations=200,
                                     totalStartingPoints=k, batchSize=k,
                                     startMode=am.START_INJECTED, precision=prec)
        x, f, stats = solver.solve(B, st, start_points=V)
        ev = float(np.linalg.norm(B64 @ np.asarray(x, np.float64)) ** 2)
        out[prec] = (ev, stats)
    ev32, s32 = out[am.PRECISION_FP32]
    evmx, smx = out[am.PRECISION_MIXED]
    assert s32.lowPrecisionIterations == 0
    assert 5 <= smx.lowPrecisionIterations < smx.it
    assert abs(evmx - ev32) <= 1e-4 * ev32


def test_lead_in_runs_fp32_products_first(solver, po):
    """leadIterations = 4: the first four steps run the FP32-accurate
    V = B^T Z (the batch reports refining), then the single-pass phase, which
    lasts at least stableIterations steps (no start counts as stable during the
    lead-in) before the switch back to the accurate products."""
    am = _am()
    m, n, k = 300, 2000, 256
    B = po.low_rank_data(m, n, 8, 30, seed=5, dtype=np.float32)
    V0 = po.uniform_starts(n, k, seed=6, dtype=np.float32)
    st = am.OptimizationSettings(formulation=0, constraintParameter=16, tolerance=1e-6,
                                 maximumIterations=100, totalStartingPoints=k, batchSize=k,
                                 precision=am.PRECISION_MIXED, stableIterations=3,
                                 leadIterations=4)
    M = solver.matrix(B)
    b = M.batch(st, k)
    b.load(V0)
    for it in range(4):
        kinds = dict(b.step_timed(it))
        assert "gemm_BtZ" in kinds and "gemm_BtZ_low(skipped)" in kinds, (it, kinds)
        # the last lead-in step hands over: the next step is single-pass
        assert b.refining() == (it < 3), it
    low = dict(b.step_timed(4))
    assert "gemm_BtZ_low" in low and "gemm_BtZ(skipped)" in low
    assert not b.refining()
    switched_at = None
    for it in range(5, 80):
        b.iterate(it, 1)
        if b.refining():
            switched_at = it
            break
    assert switched_at is not None and switched_at >= 4 + 3
    b.close()
    M.close()


@pytest.mark.parametrize("formulation", [0, 7])
def test_lead_in_solve_counts_and_group(solver, po, formulation):
    """Whole solves with a lead-in: the single-pass iterations exclude the
    lead-in, the result reaches the FP32 run's explained variance within 1e-4,
    and the same problem in a group gives the one-problem path's result bit for
    bit (same kernels, same phase rule)."""
    am = _am()
    m, n, k = 400, 3000, 256
    B = po.low_rank_data(m, n, 10, 40, seed=20 + formulation, dtype=np.float32)
    B64 = B.astype(np.float64)
    g = {7: 8.0}.get(formulation, 0.0)
    kw = dict(formulation=formulation, constraintParameter=32, penaltyParameter=g,
              tolerance=1e-6, maximumIterations=200, totalStartingPoints=k, batchSize=k,
              startMode=am.START_DEVICE_UNIFORM)
    M = solver.matrix(B)
    x32, _, s32 = M.solve(am.OptimizationSettings(**kw))
    mixed = am.OptimizationSettings(precision=am.PRECISION_MIXED, leadIterations=6, **kw)
    xmx, fmx, smx = M.solve(mixed)
    ev32 = float(np.linalg.norm(B64 @ np.asarray(x32, np.float64)) ** 2)
    evmx = float(np.linalg.norm(B64 @ np.asarray(xmx, np.float64)) ** 2)
    assert 1 <= smx.low_precision_iterations <= smx.it - 6
    assert abs(evmx - ev32) <= 1e-4 * ev32
    grp = am.Group(solver, capacity=2)
    pid = grp.add(M, am.OptimizationSettings(precision=am.PRECISION_MIXED, leadIterations=6, **kw))
    grp.run()
    xg, sg = grp.result(pid)
    assert sg.low_precision_iterations == smx.low_precision_iterations
    assert sg.it == smx.it
    assert np.array_equal(xg, xmx)
    grp.close()
    M.close()
