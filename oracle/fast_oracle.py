"""ORACLE -- test infrastructure, not product code.

A batch AM iteration in FP64 with the two products on numpy's BLAS, for the
parity tests at the benchmark shapes (400 x 10304 whole solves, 2000 x 50000
steps over 1024 starts), where the sequential loops of oracle/am_oracle.c
(orc_iteration_f64) would take hours.  It restates the same iteration
(perform_one_iteration_for_{constrained,penalized}_pca,
c++/src/gpower/gpower_commons.h:68-177; the ValueCoordinateHolder bookkeeping
of c++/src/utils/various.h:19-42; the relative change of
c++/src/utils/termination_criteria.h:30-36):

  * Z = B V and V = B^T Z in FP64 on BLAS (the C oracle sums each product
    sequentially; the two differ by FP64 rounding, ~1e-16 relative);
  * the thresholds of the constrained forms are the C oracle's own functions
    (orc_hard_level_set_f64 -- the reference's ordered-set level with its
    de-duplication -- and orc_soft_level_f64, the reference's L1-ball scan),
    called per column on a thread pool;
  * the penalties (c++/src/gpower/sparse_PCA_thresholding.h:26-102) in numpy:
    x = sgn(v)(|v| - gamma)_+ with f = sqrt(sum (|v| - gamma)_+^2), and
    x = v [v^2 > gamma] with f = sum (v^2 - gamma)_+.

Besides the iterate it reports, per start, whether any of the step's discrete
decisions is ill-conditioned under FP32 rounding of its inputs: a sign of
B v within rounding of zero (L1 variance), the s-th and (s+1)-th |v| within
MARGIN (L0 constraint), an entry within MARGIN of gamma (penalties), or an
L1-ball scan whose stopping rank or level moves under FP32-size perturbations
(or stops at its first rank, where the discriminant is exactly zero).  A test
asks for identical supports only where no step of the start's trajectory was
ill-conditioned.

tests/test_fast_oracle.py pins this module to orc_iteration_f64 on small
shapes (identical supports, values within 1e-12).
"""
import ctypes as C
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np

import pyoracle

MARGIN = 1e-5  # relative closeness to a tie that FP32 products may resolve either way

_POOL = None


def _pool():
    global _POOL
    if _POOL is None:
        _POOL = ThreadPoolExecutor(max_workers=max(1, min(32, os.cpu_count() or 1)))
    return _POOL


def _fn(name):
    f = getattr(pyoracle.oracle_lib(), name)
    f.restype = C.c_double
    return f


def _col_map(fn, cols, chunk=16):
    """fn(j) for every j in cols, on the thread pool (the C calls release the GIL)."""
    cols = list(cols)
    if len(cols) <= chunk:
        return [fn(j) for j in cols]
    parts = [cols[i:i + chunk] for i in range(0, len(cols), chunk)]
    out = []
    for r in _pool().map(lambda p: [fn(j) for j in p], parts):
        out.extend(r)
    return out


def hard_levels(Vr, s):
    """orc_hard_level_set_f64 of every column of Vr (n x k, FP64)."""
    n, k = Vr.shape
    f = _fn("orc_hard_level_set_f64")

    def one(j):
        col = np.ascontiguousarray(Vr[:, j])
        buf = np.zeros(s + 2, np.float64)
        return f(col.ctypes.data_as(C.c_void_p), C.c_uint(n), C.c_uint(s),
                 buf.ctypes.data_as(C.c_void_p))
    return np.array(_col_map(one, range(k)))


def soft_levels(Vr, s, cols=None):
    """(w, brk) of orc_soft_level_f64 for the columns of Vr (n x k, FP64)."""
    n, k = Vr.shape
    f = _fn("orc_soft_level_f64")

    def one(j):
        col = np.ascontiguousarray(Vr[:, j])
        buf = np.zeros(n + 2, np.float64)
        brk = C.c_uint(0)
        w = f(col.ctypes.data_as(C.c_void_p), C.c_uint(n), C.c_uint(s),
              buf.ctypes.data_as(C.c_void_p), C.byref(brk))
        return w, brk.value
    r = _col_map(one, range(k) if cols is None else cols)
    return np.array([a for a, _ in r]), np.array([b for _, b in r], np.int64)


# Per-entry size of the noise the L1-ball check perturbs v with, relative to
# the column's largest |v|: a few times the error of an FP32-accurate product
# entry (about 1e-7 of that scale), the same for every column length.
SOFT_NOISE = 3e-7


def _soft_ill(Vr, s, w0, b0, trials=3, seed=0):
    """L1 ball: the scan's rank or level moves under noise of the size of the
    products' FP32 error, an entry lies within rounding of the level, or the
    scan stops at its first rank."""
    n, k = Vr.shape
    scale = np.abs(Vr).max(axis=0)
    ill = (b0 == 0)
    ill |= np.min(np.abs(np.abs(Vr) - w0[None, :]), axis=0) <= MARGIN * scale
    rng = np.random.default_rng(seed)
    for _ in range(trials):
        P = Vr + (SOFT_NOISE * scale)[None, :] * rng.standard_normal(Vr.shape)
        w, b = soft_levels(P, s)
        ill |= (b != b0) | (np.abs(w - w0) > 1e-4 * np.maximum(np.abs(w0), 1e-300))
    return ill


def _hard_ill(Vr, s, lev):
    """L0 constraint: the s-th and (s+1)-th largest |v| within MARGIN."""
    n = Vr.shape[0]
    if s >= n:
        return np.zeros(Vr.shape[1], bool)
    nxt = hard_levels(Vr, s + 1)
    return (lev - nxt) <= MARGIN * lev


def _penalty_ill(Vr, gamma, l1):
    t = np.abs(Vr) if l1 else Vr * Vr
    return np.any(np.abs(t - gamma) <= MARGIN * max(gamma, 1e-300), axis=0)


class Step:
    """Result of one batch iteration."""

    def __init__(self, V, val, err, max_err, ill, vraw):
        self.V, self.val, self.err, self.max_err, self.ill, self.vraw = (
            V, val, err, max_err, ill, vraw)


def exact_l1_levels(Vr, s, iters=80):
    """exact_l1_level of every column of Vr, by bisection on w in FP64: the
    ratio ||(|v| - w)_+||_1 / ||(|v| - w)_+||_2 falls from ||v||_1 / ||v||_2
    at w = 0 to 1 as w reaches max |v|, so the level is its unique crossing
    of sqrt(s) (0 where the ratio is already at most sqrt(s))."""
    A = np.abs(np.asarray(Vr, np.float64))
    k = A.shape[1]
    target = np.sqrt(float(s))

    def ratio(w):
        X = np.maximum(A - w[None, :], 0.0)
        with np.errstate(divide="ignore", invalid="ignore"):
            return X.sum(axis=0) / np.sqrt((X * X).sum(axis=0))
    lo = np.zeros(k)
    hi = A.max(axis=0)
    done = ratio(lo) <= target
    for _ in range(iters):
        mid = 0.5 * (lo + hi)
        r = ratio(mid)
        above = r > target  # r decreases with w: the level lies above mid
        lo = np.where(above, mid, lo)
        hi = np.where(above, hi, mid)
    return np.where(done, 0.0, 0.5 * (lo + hi))


def iteration(B, V, formulation, s=0, gamma=0.0, val=None, check=True, keep_vraw=False,
              l1_exact=False):
    """One batch AM iteration in FP64 (orc_iteration_f64's semantics).

    B: m x n FP64, V: n x k FP64 (the current loadings), val: the previous
    objective per start (zeros before the first step).  Returns a Step with
    the new V, val, err, the NaN-ignoring batch maximum of err and, when
    `check`, the per-start ill-conditioning flags of this step.  With
    `l1_exact` the L1-constraint forms project exactly onto
    ||x||_1 / ||x||_2 = sqrt(s) (exact_l1_levels) instead of the reference's
    scan."""
    form = int(formulation)
    m, n = B.shape
    k = V.shape[1]
    val = np.zeros(k) if val is None else np.asarray(val, np.float64)
    l1var = form in (1, 3, 5, 7)
    Y = B @ V
    ill = np.zeros(k, bool)
    if check and l1var:
        # a sign within rounding of zero: |y_i| within MARGIN of the 2-norm of
        # the terms b_ij v_j it sums (the scale of a blocked FP32 sum's error)
        # (a column of zeros gives y = 0 and sign 0 on both sides: not a tie)
        bound = np.sqrt((B * B) @ (V * V))
        ill |= np.any((np.abs(Y) <= MARGIN * bound) & (bound > 0), axis=0)
    with np.errstate(divide="ignore", invalid="ignore"):
        if form <= 3:
            if l1var:
                f = np.abs(Y).sum(axis=0)
                Z = np.sign(Y)
            else:
                f = np.linalg.norm(Y, axis=0)
                Z = Y
            Vr = B.T @ Z
            if form <= 1:
                lev = hard_levels(Vr, s)
                X = np.where(np.abs(Vr) < lev[None, :], 0.0, Vr)
                if check:
                    ill |= _hard_ill(Vr, s, lev)
            elif l1_exact:
                w = exact_l1_levels(Vr, s)
                d = np.abs(Vr) - w[None, :]
                X = np.where(d > 0, d * np.sign(Vr), 0.0)
                if check:  # an entry within rounding of the level
                    scale = np.abs(Vr).max(axis=0)
                    ill |= np.min(np.abs(d), axis=0) <= MARGIN * scale
            else:
                w, brk = soft_levels(Vr, s)
                d = np.abs(Vr) - w[None, :]
                X = np.where(d > 0, d * np.sign(Vr), 0.0)
                if check:
                    ill |= _soft_ill(Vr, s, w, brk)
            nx = np.sqrt((X * X).sum(axis=0))
            Vn = X * (1.0 / nx)[None, :]
        else:
            Z = np.sign(Y) if l1var else Y / np.linalg.norm(Y, axis=0)[None, :]
            Vr = B.T @ Z
            if form >= 6:
                d = np.abs(Vr) - gamma
                keep = d > 0
                Vn = np.where(keep, d * np.sign(Vr), 0.0)
                f = np.sqrt(np.where(keep, d * d, 0.0).sum(axis=0))
            else:
                d = Vr * Vr - gamma
                keep = d > 0
                Vn = np.where(keep, Vr, 0.0)
                f = np.where(keep, d, 0.0).sum(axis=0)
            if check:
                ill |= _penalty_ill(Vr, gamma, form >= 6)
        err = np.abs(f - val) / val
    finite = err[~np.isnan(err)]
    max_err = float(max(0.0, finite.max())) if finite.size else 0.0
    return Step(Vn, f, err, max_err, ill, Vr if keep_vraw else None)


def batch_solve(B, V0, formulation, s=0, gamma=0.0, tol=1e-6, max_iter=200):
    """The reference's batch loop (c++/src/gpower/sparse_PCA_solver.h:192-212)
    over one batch: steps it = 0, 1, ... until it > 0 and the batch's largest
    change is below tol, or max_iter steps.  Returns (V, val, steps, ill), ill
    being whether any step of a start was ill-conditioned."""
    V = np.asarray(V0, np.float64)
    val = np.zeros(V.shape[1])
    ill = np.zeros(V.shape[1], bool)
    steps = 0
    for it in range(max_iter):
        r = iteration(B, V, formulation, s, gamma, val)
        V, val = r.V, r.val
        ill |= r.ill
        steps += 1
        if it > 0 and r.max_err < tol:
            break
    return V, val, steps, ill


def exact_l1_level(v, s):
    """The exact L1-ball level: w >= 0 with ||x||_1 / ||x||_2 = sqrt(s) for
    x = (|v| - w)_+, from the sorted magnitudes (on each interval between
    consecutive |v| the ratio's square is a ratio of quadratics in w, so the
    root is that of a quadratic; the ratio decreases as w grows).  Returns 0
    when ||v||_1 / ||v||_2 <= sqrt(s) already."""
    a = np.sort(np.abs(np.asarray(v, np.float64)))[::-1]
    a = a[a > 0]
    if a.size == 0:
        return 0.0
    target = float(s)
    c1 = np.cumsum(a)
    c2 = np.cumsum(a * a)
    if c1[-1] ** 2 <= target * c2[-1]:
        return 0.0
    # with t entries kept: (S1 - t w)^2 = s (S2 - 2 w S1 + t w^2)
    for t in range(1, a.size + 1):
        S1, S2 = c1[t - 1], c2[t - 1]
        lo = a[t] if t < a.size else 0.0
        hi = a[t - 1]
        A = t * t - target * t
        Bq = -2 * t * S1 + 2 * target * S1
        Cq = S1 * S1 - target * S2
        if abs(A) < 1e-300:
            roots = [-Cq / Bq] if Bq != 0 else []
        else:
            disc = max(Bq * Bq - 4 * A * Cq, 0.0)
            r = np.sqrt(disc)
            roots = [(-Bq - r) / (2 * A), (-Bq + r) / (2 * A)]
        for w in sorted(roots):
            if lo - 1e-15 * hi <= w < hi and (S1 - t * w) > 0:
                x = np.maximum(a - w, 0.0)
                if abs(x.sum() / np.linalg.norm(x) - np.sqrt(target)) <= 1e-9 * np.sqrt(target):
                    return float(w)
    raise ArithmeticError("no L1-ball level found")
