"""The MIXED precision mode: single-pass BF16 V = B^T Z while the supports
settle, then the FP32-accurate products.  One BF16 step against an FP64
product of the BF16-rounded operands, the phase switch, and whole solves that
reach the FP32 path's explained variance within 1e-4."""
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
def test_bf16_step_matches_rounded_product(solver, po, formulation):
    """With gamma = 0 the L0 penalty keeps every non-zero v, so one BF16-phase
    step returns V = b0(B)^T Z_b, b0 the BF16 rounding of B and Z_b that of Z
    (exact for the L1-variance sgn)."""
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
    assert "gemm_BtZ_bf16" in first and "gemm_BtZ(skipped)" in first and "support" in first
    switched_at = None
    for it in range(1, 60):
        b.iterate(it, 1)
        if b.refining():
            switched_at = it
            break
    assert switched_at is not None and switched_at >= 3
    after = dict(b.step_timed(switched_at + 1))
    assert "gemm_BtZ" in after and "gemm_BtZ_bf16(skipped)" in after
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
