"""Comparison rules between the CUDA path (FP32 data, FP32-accurate products)
and the oracle run in FP64 on the same data.

A discrete decision (which entries survive a threshold) can only be required
to match where the oracle's decision is stable under FP32 rounding of its
inputs; the helpers below find the unstable ("ill-conditioned") columns.
"""
import numpy as np

# FP32 products over K terms carry ~1e-6 relative error; decisions closer than
# this to a tie are not asked to match.
MARGIN = 1e-5


def hard_ill_conditioned(v, s):
    """L0 constraint: the s-th and (s+1)-th largest |v| within MARGIN."""
    a = np.sort(np.abs(v))[::-1]
    if s >= len(a):
        return False
    return (a[s - 1] - a[s]) <= MARGIN * a[s - 1]


def penalty_ill_conditioned(v, gamma, l1):
    """Penalties: some entry within MARGIN of the threshold."""
    t = np.abs(v) if l1 else v * v
    return bool(np.any(np.abs(t - gamma) <= MARGIN * max(gamma, 1e-300)))


def soft_ill_conditioned(po, v, s, trials=4, seed=0):
    """L1 constraint: the oracle's scan stops at a different rank, or gives a
    different level, once v is perturbed at FP32 rounding size."""
    w0, b0 = po.oracle_soft_level(np.asarray(v, np.float64), s)
    rng = np.random.default_rng(seed)
    vv = [np.asarray(v, np.float32).astype(np.float64)]
    scale = np.abs(v).max()
    for _ in range(trials):
        vv.append(v + MARGIN * scale * rng.standard_normal(v.shape) / np.sqrt(len(v)))
    for u in vv:
        w, b = po.oracle_soft_level(u, s)
        if b != b0 or abs(w - w0) > 1e-4 * max(abs(w0), 1e-300):
            return True
    # an entry within rounding of the level may land on either side of it
    return bool(np.min(np.abs(np.abs(v) - w0)) <= MARGIN * scale)


def soft_scale(po, v, s):
    """x = (|v| - w)_+ / N: an error e|v| in v moves x by about e|v|/N."""
    w, _ = po.oracle_soft_level(np.asarray(v, np.float64), s)
    N = np.linalg.norm(np.maximum(np.abs(v) - w, 0.0))
    return float(np.abs(v).max() / max(N, 1e-300))


def objective_scale(formulation, v_raw, gamma):
    """Size of the terms the objective is formed from, for an absolute tolerance:
    the penalized objectives subtract gamma from each surviving term, so their
    relative error grows as the terms approach gamma."""
    if formulation in (4, 5):
        keep = v_raw * v_raw > gamma
        return float(np.sum(v_raw[keep] ** 2)) + 1e-300
    if formulation in (6, 7):
        keep = np.abs(v_raw) > gamma
        return float(np.sqrt(np.sum(v_raw[keep] ** 2))) + 1e-300
    return None
