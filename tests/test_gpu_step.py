"""One AM step on the GPU (am24_batch_iterate) against one oracle step in FP64
on the same FP32 data and starting points: every formulation, ragged shapes."""
import numpy as np
import pytest

import parity

pytestmark = pytest.mark.gpu

SHAPES = [(200, 300, 64), (257, 1000, 130), (33, 70, 1), (129, 4097, 257), (1000, 5000, 256)]


def gammas(B):
    Bd = B.astype(np.float64)
    c2 = np.linalg.norm(Bd, axis=0).max()
    c1 = np.abs(Bd).sum(0).max()
    # the scale of B^T sgn(B x) (L1 variance) and of B^T (B x / ||B x||) (L2)
    return {4: (0.02 * c2) ** 2, 5: (0.05 * c1) ** 2, 6: 0.05 * c2, 7: 0.05 * c1}


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("formulation", range(8))
def test_step_matches_oracle(solver, po, shape, formulation):
    m, n, k = shape
    check_step(solver, po, po.low_rank_data(m, n, 8, 30, seed=m + n, dtype=np.float32), k,
               formulation)


@pytest.mark.parametrize("formulation,spread", [(0, 6), (1, 6), (2, 0.5), (3, 0.5), (4, 6),
                                                (5, 6), (6, 6), (7, 6)])
def test_step_with_feature_scales_far_apart(solver, po, formulation, spread):
    """Features scaled from 10^-spread to 10^spread (and one all zero): the
    FP16 operands of V = B^T Z carry a power-of-two scale per feature, so every
    feature keeps its relative accuracy.  (The L1-ball forms 2 and 3 take a
    narrow spread: with a wide one the projection keeps only the largest
    feature, the tie case the parity check sets aside.)"""
    m, n, k = 300, 2000, 256
    B = po.low_rank_data(m, n, 8, 30, seed=11, dtype=np.float64)
    B *= 10.0 ** np.random.default_rng(12).uniform(-spread, spread, n)
    B[:, 7] = 0.0
    check_step(solver, po, B.astype(np.float32), k, formulation)


@pytest.mark.parametrize("scheme", ["tf32_bf16", "tf32", "one_cta", "select_gather"])
@pytest.mark.parametrize("shape", [(1000, 5000, 256), (129, 4097, 257)],
                         ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("formulation", range(8))
def test_step_matches_oracle_other_pair_schemes(solver, po, shape, formulation, scheme,
                                                monkeypatch):
    """The switches of a wide batch: the CTA-pair products without the FP16
    operands (3xTF32 for every formulation, or with exact BF16 operands for the
    L1-variance forms), every product on one-CTA tiles, and the selects doing
    their own hinted gather instead of reading V = B^T Z's candidate marks."""
    if scheme in ("tf32_bf16", "tf32"):
        monkeypatch.setenv("AM24_GEMM_FP16", "0")
    if scheme == "tf32":
        monkeypatch.setenv("AM24_GEMM_BF16", "0")
    if scheme == "one_cta":
        monkeypatch.setenv("AM24_GEMM_PAIR", "0")
    if scheme == "select_gather":
        monkeypatch.setenv("AM24_SELECT_LIST", "0")
    m, n, k = shape
    check_step(solver, po, po.low_rank_data(m, n, 8, 30, seed=m + n, dtype=np.float32), k,
               formulation)


def check_step(solver, po, B, k, formulation):
    m, n = B.shape
    B64 = B.astype(np.float64)
    V0 = po.uniform_starts(n, k, seed=n, dtype=np.float32)
    s = min(16, n)
    g = gammas(B).get(formulation, 0.0)
    import importlib
    am = importlib.import_module("24am_b200")
    st = am.OptimizationSettings(formulation=formulation, constraintParameter=s, penaltyParameter=g,
                                 tolerance=1e-6, maximumIterations=10, totalStartingPoints=k,
                                 batchSize=k)
    M = solver.matrix(B)
    b = M.batch(st, k)
    val_prev = np.linspace(1.0, 2.0, k).astype(np.float32)
    b.load(V0)
    b.iterate(0, 1)
    V1, val, err, nnz = b.read()
    os_ = po.make_settings(formulation, constraint=s, penalty=g, tolerance=1e-6, max_iter=10,
                           total_starts=k, batch_size=k)
    Vo, Zo, valo, erro, _ = po.oracle_iteration(B64, V0.astype(np.float64), os_, np.zeros(k))
    # the raw B^T z the oracle thresholded, for the conditioning checks
    Z = B64 @ V0.astype(np.float64)
    if formulation in (1, 3, 5, 7):
        Z = np.sign(Z)
    elif formulation >= 4:
        Z = Z / np.linalg.norm(Z, axis=0)
    Vraw = B64.T @ Z
    bad = 0
    for j in range(k):
        v = Vraw[:, j]
        if formulation in (0, 1):
            ill = parity.hard_ill_conditioned(v, s)
        elif formulation in (2, 3):
            # the reference scan's first step (t = 1) has a discriminant of exactly
            # zero in exact arithmetic, so stopping there is decided by the last
            # bit of the largest |v|; a 1-sparse result on either side is that case
            ill = (parity.soft_ill_conditioned(po, v, s) or
                   (nnz[j] == 1) != (np.count_nonzero(Vo[:, j]) == 1))
        else:
            ill = parity.penalty_ill_conditioned(v, g, formulation >= 6)
        if ill:
            bad += 1
            continue
        assert np.array_equal(V1[:, j] != 0, Vo[:, j] != 0), f"support differs in column {j}"
        # thresholds subtract from |v|; errors scale with |v| before the threshold,
        # relative to the normalisation the formulation applies
        if formulation <= 1:
            scale = np.abs(Vo[:, j]).max()
        elif formulation <= 3:
            scale = parity.soft_scale(po, v, s)
        else:
            scale = np.abs(v).max()
        assert np.abs(V1[:, j] - Vo[:, j]).max() <= 1e-5 * scale, f"column {j}"
        assert nnz[j] == np.count_nonzero(Vo[:, j])
        sc = parity.objective_scale(formulation, v, g)
        tol = 1e-5 * (sc if sc is not None else abs(valo[j]))
        assert abs(val[j] - valo[j]) <= tol + 1e-30, f"objective of column {j}"
    assert bad <= max(2, k // 10), f"{bad} ill-conditioned columns of {k}"
    b.close()
    M.close()


def test_step_is_deterministic(solver, po):
    import importlib
    am = importlib.import_module("24am_b200")
    B = po.low_rank_data(500, 3000, 8, 30, seed=1, dtype=np.float32)
    V0 = po.uniform_starts(3000, 200, seed=2, dtype=np.float32)
    M = solver.matrix(B)
    outs = []
    for f in (0, 3, 4, 7):
        st = am.OptimizationSettings(formulation=f, constraintParameter=16, penaltyParameter=0.5,
                                     totalStartingPoints=200, batchSize=200)
        for _ in range(2):
            b = M.batch(st, 200)
            b.load(V0)
            b.iterate(0, 3)
            outs.append(b.read())
            b.close()
        a, c = outs[-2], outs[-1]
        for x, y in zip(a, c):
            assert np.array_equal(x, y, equal_nan=True)


@pytest.mark.parametrize("k,marks", [(96, True), (98, True), (256, True), (256, False)],
                         ids=["k96", "k98", "k256", "k256-select-gather"])
@pytest.mark.parametrize("formulation", range(8))
def test_steps_through_sparse_gather_match_oracle(solver, po, formulation, k, marks,
                                                  monkeypatch):
    """Three steps: after the first, V is sparse and Z = B V runs as the gather
    kernel (every column at most min(4096, n/32) non-zeros); from the second the
    selects start from the previous level, reading the candidates V = B^T Z's
    epilogue marked (or, with marks off, gathering them themselves).  The
    loadings stay with the oracle's."""
    import importlib
    am = importlib.import_module("24am_b200")
    if not marks:
        monkeypatch.setenv("AM24_SELECT_LIST", "0")
    m, n = 300, 4096
    B = po.low_rank_data(m, n, 8, 30, seed=77, dtype=np.float32)
    B64 = B.astype(np.float64)
    V0 = po.uniform_starts(n, k, seed=78, dtype=np.float32)
    s = 12
    g = {4: 2.0, 5: 2000.0, 6: 1.0, 7: 40.0}.get(formulation, 0.0)
    st = am.OptimizationSettings(formulation=formulation, constraintParameter=s,
                                 penaltyParameter=g, tolerance=1e-6, maximumIterations=10,
                                 totalStartingPoints=k, batchSize=k)
    M = solver.matrix(B)
    b = M.batch(st, k)
    b.load(V0)
    os_ = po.make_settings(formulation, constraint=s, penalty=g, tolerance=1e-6, max_iter=10,
                           total_starts=k, batch_size=k)
    Vo, val_o = V0.astype(np.float64), np.zeros(k)
    kinds = []
    for it in range(3):
        kinds.append([name for name, _ in b.step_timed(it)])
        Vo, _, val_o, _, _ = po.oracle_iteration(B64, Vo, os_, val_o, it=it)
    V, val, err, nnz = b.read()
    assert "gemm_BV" in kinds[0] and "gather_BV(skipped)" in kinds[0]
    assert "gather_BV_group(skipped)" in kinds[0]
    if formulation <= 3 or np.count_nonzero(Vo, axis=0).max() <= n // 32:
        # four starts per block while no column has more than 1024 non-zeros
        assert ("gather_BV" in kinds[2]) != ("gather_BV_group" in kinds[2]), kinds[2]
    agree = []
    for j in range(k):
        same = np.array_equal(V[:, j] != 0, Vo[:, j] != 0)
        close = np.abs(V[:, j] - Vo[:, j]).max() <= 1e-4 * max(np.abs(Vo[:, j]).max(), 1e-30)
        agree.append(same and close and abs(val[j] - val_o[j]) <= 1e-4 * abs(val_o[j]) + 1e-20)
    assert sum(agree) >= 0.9 * k, f"{sum(agree)} of {k} starts agree after 3 steps"
    # a batch that is not a multiple of four ends in a partial group of the
    # grouped gather: its starts are held to the same bar as the others
    tail = agree[k - k % 4:] if k % 4 else []
    assert sum(tail) >= len(tail) - (1 if len(tail) > 1 else 0), tail
    b.close()
    M.close()


@pytest.mark.parametrize("k,fp16", [(96, True), (256, False), (256, True)])
@pytest.mark.parametrize("formulation", [4, 5, 6, 7])
def test_dense_penalized_steps(solver, po, formulation, k, fp16, monkeypatch):
    """Penalties small enough to keep V dense step after step.  On one-CTA
    tiles (k = 96), and on CTA pairs without FP16 operands, from the second step
    on Z = B V reads the TF32 planes the previous step's penalty epilogue wrote
    (densify returns at once); on CTA pairs with FP16 operands densify writes
    V's scaled FP16 planes every dense step.  The loadings stay with the
    oracle's."""
    import importlib
    am = importlib.import_module("24am_b200")
    if not fp16:
        monkeypatch.setenv("AM24_GEMM_FP16", "0")
    reuse = k <= 128 or not fp16
    m, n = 300, 2048
    B = po.low_rank_data(m, n, 8, 30, seed=91, dtype=np.float32)
    B64 = B.astype(np.float64)
    V0 = po.uniform_starts(n, k, seed=92, dtype=np.float32)
    g = {4: 1e-4, 5: 1e-2, 6: 1e-3, 7: 1e-2}[formulation]
    st = am.OptimizationSettings(formulation=formulation, penaltyParameter=g, tolerance=1e-6,
                                 maximumIterations=10, totalStartingPoints=k, batchSize=k)
    M = solver.matrix(B)
    b = M.batch(st, k)
    b.load(V0)
    os_ = po.make_settings(formulation, penalty=g, tolerance=1e-6, max_iter=10, total_starts=k,
                           batch_size=k)
    Vo, val_o = V0.astype(np.float64), np.zeros(k)
    kinds = []
    for it in range(4):
        kinds.append([name for name, _ in b.step_timed(it)])
        Vo, _, val_o, _, _ = po.oracle_iteration(B64, Vo, os_, val_o, it=it)
    V, val, err, nnz = b.read()
    assert np.count_nonzero(Vo, axis=0).max() > n // 32  # dense every step
    assert "densify" in kinds[0]
    for ks in kinds[1:]:
        assert ("densify(skipped)" if reuse else "densify") in ks and "gemm_BV" in ks, ks
    ok = 0
    for j in range(k):
        same = np.array_equal(V[:, j] != 0, Vo[:, j] != 0)
        close = np.abs(V[:, j] - Vo[:, j]).max() <= 1e-4 * max(np.abs(Vo[:, j]).max(), 1e-30)
        ok += same and close and abs(val[j] - val_o[j]) <= 1e-4 * abs(val_o[j]) + 1e-20
    assert ok >= 0.9 * k, f"{ok} of {k} starts agree after 4 steps"
    b.close()
    M.close()


@pytest.mark.parametrize("formulation", [0, 1])
def test_partial_gather_group_matches_a_full_one(solver, po, formulation):
    """The grouped sparse gather takes four starts per block; a batch of 98
    ends in a group of two.  Every start's sums run over its own non-zeros in
    index order whatever group it lands in, so the first 98 starts of a batch
    of 100 step bit for bit as the batch of 98 does (top-s keeps every column
    under the gather's bound, so both batches take the same path each step)."""
    import importlib
    am = importlib.import_module("24am_b200")
    m, n = 300, 4096
    B = po.low_rank_data(m, n, 8, 30, seed=61, dtype=np.float32)
    V = po.uniform_starts(n, 100, seed=62, dtype=np.float32)
    M = solver.matrix(B)
    outs = []
    for k in (98, 100):
        st = am.OptimizationSettings(formulation=formulation, constraintParameter=12,
                                     tolerance=1e-6, maximumIterations=10,
                                     totalStartingPoints=k, batchSize=k)
        b = M.batch(st, k)
        b.load(np.asfortranarray(V[:, :k]))
        kinds = [[name for name, _ in b.step_timed(it)] for it in range(3)]
        assert "gather_BV_group" in kinds[2], kinds[2]
        outs.append(b.read())
        b.close()
    M.close()
    (V98, val98, err98, nnz98), (V100, val100, err100, nnz100) = outs
    assert np.array_equal(V98, V100[:, :98])
    assert np.array_equal(val98, val100[:98])
    assert np.array_equal(err98, err100[:98], equal_nan=True)
    assert np.array_equal(nnz98, nnz100[:98])
