"""Parity at the benchmark configurations, per start, at 1e-5.

  * config 0's problem (n = 400 samples x p = 10304 features, r = 20, 64
    non-zeros per loading, seed 1; 64 starts; s = 16; tol 1e-6; maxIter 200),
    whole batch solves of all 8 formulations;
  * config 1's shape (2000 x 50000, r = 50, 256 non-zeros per loading; 1024
    starts), one step and three more of all 8 formulations with s in {16, 128}
    (constraints) and gamma = {0.1, 0.5} x the largest column norm and one that
    keeps 0.6 % of the entries (penalties), each step against the oracle's step
    from the same state.

The checker is the FP64 iteration of oracle/fast_oracle.py (BLAS products, the
C oracle's thresholds), on the same FP32 data and starting points.  Per start
the GPU must give the oracle's support (exact index set) and its objective and
explained variance ||B x||^2 within 1e-5 relative, wherever no step of the
start's trajectory made a decision that FP32 rounding of its inputs can flip
(fast_oracle's ill-conditioning flags).  The share of such starts is printed;
a lower bound on the starts compared guards against a check that sets
everything aside."""
import importlib

import numpy as np
import pytest

import fast_oracle as fo

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _am():
    return importlib.import_module("24am_b200")


def _ev(B64, V):
    """||B x||^2 per column of V, x = v / ||v|| (FP64)."""
    V = np.asarray(V, np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        X = V / np.linalg.norm(V, axis=0)[None, :]
    return np.linalg.norm(B64 @ X, axis=0) ** 2


def _gammas(am, B64, c):
    col2 = float(np.linalg.norm(B64, axis=0).max())
    col1 = float(np.abs(B64).sum(axis=0).max())
    return am.workloads.penalty_gammas(col2, col1, c)


def _objective_scales(formulation, Vr, gamma):
    """Per start, the size of the terms a penalized objective is formed from
    (its FP32 error is relative to that, not to the objective: every kept term
    has gamma subtracted from it): sum v^2 over the kept entries (L0 penalty),
    the 2-norm of the kept v (L1 penalty)."""
    if formulation in (4, 5):
        return np.where(Vr * Vr > gamma, Vr * Vr, 0.0).sum(axis=0)
    return np.sqrt(np.where(np.abs(Vr) > gamma, Vr * Vr, 0.0).sum(axis=0))


def _describe(j, Vg, Vo, vraw, gamma):
    """Where start j's supports differ: the rows, the GPU's and the oracle's
    values there and, with the oracle's v = B^T z, how close |v| (or v^2) lies
    to gamma relative to gamma."""
    rows = np.flatnonzero((Vg[:, j] != 0) != (Vo[:, j] != 0))[:5]
    out = [f"start {j}: rows {rows.tolist()} gpu {Vg[rows, j].tolist()} "
           f"oracle {Vo[rows, j].tolist()}"]
    if vraw is not None and gamma:
        v = vraw[rows, j]
        out.append(f"|v| {np.abs(v).tolist()} gamma {gamma} "
                   f"margin (|v|-gamma)/gamma {((np.abs(v) - gamma) / gamma).tolist()} "
                   f"(v^2-gamma)/gamma {((v * v - gamma) / gamma).tolist()}")
    return "; ".join(out)


def _compare(B64, Vg, valg, Vo, valo, ill, what, scale=None, vraw=None, gamma=0.0):
    """Per-start supports, objectives and explained variances.  Starts whose
    objective is NaN (an empty support earlier: the reference divides 0/0) must
    be NaN on both sides; starts with an empty support (objective 0) must be
    empty on both.  The objective's error is relative to `scale` where given
    (penalized forms), else to the objective.  Returns the number of starts
    compared."""
    k = Vo.shape[1]
    nan_o = np.isnan(valo)
    assert np.array_equal(np.isnan(valg), nan_o), f"{what}: NaN starts differ"
    keep = ~ill & ~nan_o
    sup_g, sup_o = Vg != 0, Vo != 0
    bad_sup = [j for j in np.flatnonzero(keep) if not np.array_equal(sup_g[:, j], sup_o[:, j])]
    assert not bad_sup, (f"{what}: support differs for starts {bad_sup[:10]}; " +
                         " | ".join(_describe(j, Vg, Vo, vraw, gamma) for j in bad_sup[:3]))
    empty = keep & (valo == 0)
    assert np.all(valg[empty] == 0), f"{what}: an empty support is not empty on the GPU"
    full = keep & (valo != 0)
    den = np.abs(valo[full]) if scale is None else scale[full]
    rel = np.abs(valg[full] - valo[full]) / den
    assert rel.max(initial=0.0) <= TOL, f"{what}: objective rel err {rel.max():.3g}"
    evg, evo = _ev(B64, Vg[:, full]), _ev(B64, Vo[:, full])
    rel_ev = np.abs(evg - evo) / evo
    assert rel_ev.max(initial=0.0) <= TOL, f"{what}: explained variance rel err {rel_ev.max():.3g}"
    print(f"{what}: {keep.sum()} of {k} starts compared ({full.sum()} non-empty, "
          f"{nan_o.sum()} NaN on both sides), {int(ill.sum())} set aside as "
          f"ill-conditioned; max rel err objective {rel.max(initial=0):.2e}, "
          f"explained variance {rel_ev.max(initial=0):.2e}")
    return int(keep.sum() + nan_o.sum())


# ------------------------------------------------------------------ config 0
@pytest.fixture(scope="module")
def config0():
    am = _am()
    B = am.workloads.low_rank_data(400, 10304, 20, 64, seed=1, dtype=np.float32)
    V = am.workloads.uniform_starts(10304, 64, seed=1001, dtype=np.float32)
    return B, V


@pytest.mark.parametrize("formulation", range(8))
def test_config0_whole_solves_per_start(solver, config0, formulation):
    """Batch solves to tol 1e-6 (maxIter 200): the GPU's batch loop stops within
    a step or two of the oracle's (the change test sits near FP32 resolution of
    the objective); run to the oracle's step count, every start that stayed
    well-conditioned has the oracle's support and objective, and explained
    variance within 1e-5; so does the best start."""
    am = _am()
    B, V = config0
    B64 = B.astype(np.float64)
    k, s, tol, max_iter = V.shape[1], 16, 1e-6, 200
    g = _gammas(am, B64, 0.1).get(formulation, 0.0)
    Vo, valo, steps_o, ill = fo.batch_solve(B64, V.astype(np.float64), formulation, s, g,
                                            tol=tol, max_iter=max_iter)
    st = am.OptimizationSettings(formulation=formulation, constraintParameter=s,
                                 penaltyParameter=g, tolerance=tol, maximumIterations=max_iter,
                                 totalStartingPoints=k, batchSize=k)
    M = solver.matrix(B)
    b = M.batch(st, k)
    b.load(V)
    steps_g = max_iter
    for it in range(max_iter):
        me = b.iterate(it, 1)
        if it > 0 and me < tol:
            steps_g = it + 1
            break
    print(f"config 0, formulation {formulation}: the batch loop stops after {steps_g} steps "
          f"(oracle {steps_o})")
    if formulation not in (2, 3):
        # the reference's L1-ball scan can leave a start cycling between two
        # stopping ranks near a tie, and which side FP32 rounding takes decides
        # whether the batch-global change ever falls below tol: the stopping
        # step is compared for the other forms only
        assert abs(steps_g - steps_o) <= max(2, steps_o // 20), (steps_g, steps_o)
    if steps_g != steps_o:  # compare at the oracle's step
        b.load(V)
        b.iterate(0, steps_o)
    Vg, valg, _, _ = b.read()
    b.close()
    M.close()
    compared = _compare(B64, Vg, valg.astype(np.float64), Vo, valo, ill,
                        f"config 0, formulation {formulation}, {steps_o} steps")
    # over a whole solve the L1-ball forms meet the scan's knife-edges (a
    # level within rounding of an entry, a stop at the first rank) often
    assert compared >= (k // 4 if formulation in (2, 3) else k // 2)
    # the best start among those compared (the reference's choice: largest
    # objective, first on ties; starts in one optimum tie up to rounding, so
    # the two sides may name different ones): explained variance within 1e-5.  (The best of all starts may be one whose cycle
    # between two supports near a tie FP32 rounding decides; it is printed.)
    keep = ~ill & np.isfinite(valo) & np.isfinite(valg)
    if np.any(keep & (valo > 0)):
        idx = np.flatnonzero(keep)
        jo = int(idx[np.argmax(valo[idx])])
        jg = int(idx[np.argmax(valg[idx])])
        ev_o = _ev(B64, Vo[:, [jo]])[0]
        ev_g = _ev(B64, Vg[:, [jg]])[0]
        assert abs(ev_g - ev_o) <= TOL * ev_o, (ev_g, ev_o)
    if np.nanmax(valo, initial=0.0) > 0:
        ev_all_o = _ev(B64, Vo[:, [int(np.nanargmax(valo))]])[0]
        ev_all_g = _ev(B64, Vg[:, [int(np.nanargmax(valg))]])[0]
        print(f"config 0, formulation {formulation}: best of all starts, explained variance "
              f"GPU {ev_all_g:.9g}, oracle {ev_all_o:.9g}")


# ------------------------------------------------------------------ config 1
@pytest.fixture(scope="module")
def config1():
    am = _am()
    B = am.workloads.low_rank_data(2000, 50000, 50, 256, seed=1, dtype=np.float32)
    V = am.workloads.uniform_starts(50000, 1024, seed=1001, dtype=np.float32)
    return B, B.astype(np.float64), V


CASES = ([(f, p) for f in range(4) for p in (16, 128)]
         + [(f, p) for f in range(4, 8) for p in (0.1, 0.5, "q")])


def _quantile_gamma(B64, V, formulation, share=0.006):
    """A gamma that keeps about `share` of the entries of the first step's
    v = B^T z over all starts (the column-norm multiples leave the L0-penalty
    forms with empty supports at this shape, so these cases exercise the kept
    entries)."""
    r = fo.iteration(B64, V, formulation, 0, 0.0, check=False, keep_vraw=True)
    t = r.vraw * r.vraw if formulation in (4, 5) else np.abs(r.vraw)
    return float(np.quantile(t, 1.0 - share))


@pytest.mark.parametrize("formulation,param", CASES, ids=[f"f{f}-{p}" for f, p in CASES])
def test_config1_shape_steps_per_start(solver, config1, formulation, param):
    """One step from the dense starts (tensor-core Z = B V, split-FP16 pair
    GEMMs at K = 2000 and K = 50000), then three more (sparse gather, hinted
    selects from the second on), all 1024 columns.  Each GPU step is checked
    against the FP64 oracle's step from the same state: the starting points for
    step 1, the GPU's own loadings after step t for step t + 1.  (Along a whole
    trajectory the thresholds amplify rounding: x = |v| - gamma or |v| - w has
    few correct digits for |v| near the level, and the next step's signs or
    supports can turn on them; stepping both sides from the same x checks every
    step's kernels without that amplification.)

    Penalties: gamma = 0.1 and 0.5 x the largest column norm (the benchmark's
    choice) and "q", a gamma that keeps about 0.6% of the entries.  The L1-ball
    forms: the reference's scan at its first rank solves a quadratic whose
    discriminant is exactly zero, so whether it stops there (a support of one
    entry) is decided by the last bits of the largest |v|; a start that stopped
    there on the GPU's side is set aside with the oracle's ill-conditioned
    starts (which include its own first-rank stops)."""
    am = _am()
    B, B64, V = config1
    k = V.shape[1]
    s = param if formulation <= 3 else 0
    if formulation <= 3:
        g = 0.0
    elif param == "q":
        g = _quantile_gamma(B64, V.astype(np.float64), formulation)
    else:
        g = _gammas(am, B64, param)[formulation]
    st = am.OptimizationSettings(formulation=formulation, constraintParameter=max(s, 1),
                                 penaltyParameter=g, tolerance=1e-6, maximumIterations=200,
                                 totalStartingPoints=k, batchSize=k)
    M = solver.matrix(B)
    b = M.batch(st, k)
    b.load(V)
    prev_V, prev_val = V.astype(np.float64), np.zeros(k)
    counts = []
    for it in range(4):
        b.iterate(it, 1)
        Vg, valg, _, nnz = b.read()
        r = fo.iteration(B64, prev_V, formulation, s, g, prev_val, keep_vraw=True)
        ill = r.ill.copy()
        if formulation in (2, 3):
            ill |= np.count_nonzero(Vg, axis=0) == 1  # the GPU's first-rank stops
        scale = _objective_scales(formulation, r.vraw, g) if formulation >= 4 else None
        counts.append(_compare(B64, Vg, valg.astype(np.float64), r.V, r.val, ill,
                               f"config 1 shape, formulation {formulation} ({param}), "
                               f"step {it + 1}", scale, r.vraw, g))
        prev_V, prev_val = Vg.astype(np.float64), valg.astype(np.float64)
    b.close()
    M.close()
    # every start that is compared must match, and enough must be comparable:
    # half, or a fifth for the L1-ball forms, whose scan meets a knife-edge
    # (its first-rank stop, a level within rounding of an entry) on many
    # starts once the supports are small
    assert min(counts) >= (k // 5 if formulation in (2, 3) else k // 2), counts
