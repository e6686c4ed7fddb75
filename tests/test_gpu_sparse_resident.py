"""Sparse-resident matrices (am24_matrix_create_csc_sparse_f32): CSC data kept
compressed on the device, the centring applied implicitly, solved by the
dense path's iteration with both products on the compressed arrays.  Whole
solves against the oracle on the densified, centred matrix; against the
densified path; a matrix whose dense form would not fit in device memory; and
the entry points that do not take such a matrix."""
import importlib

import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu

FORMS = range(8)


def _am():
    return importlib.import_module("24am_b200")


def _sparse(m, n, seed, density):
    S = sp.random(m, n, density=density, format="csc", random_state=seed, dtype=np.float64)
    S.data = S.data * 4.0 - 1.0
    return S.astype(np.float32)


def _planted(m, n, seed, density, width=30, scale=40.0):
    """Sparse noise plus one planted sparse component (a rank-one block on
    `width` features), so that the best start of a whole solve lands on it
    whatever the first steps' near-ties decide."""
    rng = np.random.default_rng(seed)
    A = _sparse(m, n, seed, density).toarray()
    idx = rng.choice(n, width, replace=False)
    u = rng.standard_normal(m)
    w = rng.standard_normal(width)
    A[:, idx] += (scale * np.outer(u / np.linalg.norm(u), w / np.linalg.norm(w))).astype(np.float32)
    return sp.csc_matrix(A)


def _centring(A, center):
    mu = A.mean(axis=0).astype(np.float32) if center in ("columns", "both") else None
    rmu = A.mean(axis=1).astype(np.float32) if center in ("rows", "both") else None
    C = A.astype(np.float64)
    if mu is not None:
        C = C - mu[None, :].astype(np.float64)
    if rmu is not None:
        C = C - rmu[:, None].astype(np.float64)
    return mu, rmu, C


def _gamma(C, formulation, c=0.3):
    """A penalty that keeps a handful of loadings: a share of the largest |v|
    of V = C^T z at the top left singular vector z (L2 variance) or a share of
    the largest column 1-norm (L1 variance); the L0 penalties compare v^2 with
    gamma."""
    if formulation in (4, 6):
        u = np.linalg.svd(C, full_matrices=False)[0][:, 0]
        g = c * np.abs(C.T @ u).max()
        return g * g if formulation == 4 else g
    c1 = np.abs(C).sum(axis=0).max()
    return {5: (c * c1) ** 2, 7: c * c1}.get(formulation, 0.0)


@pytest.mark.parametrize("center", ["none", "columns", "rows", "both"])
@pytest.mark.parametrize("formulation", FORMS)
def test_sparse_resident_solve_matches_oracle(solver, po, formulation, center):
    """Reference starting points, 48 starts in two batches, on sparse noise
    with a planted sparse component; the oracle runs in FP64 on the densified,
    centred matrix from the same starts.  Best objective and FP64 explained
    variance within 1e-4.  The L1-ball form with L2 variance runs 8 steps: the
    reference's scan decides its first step on the last bit of max |v| (a
    discriminant of exactly zero), and on noise its later steps can cycle
    between supports, so longer runs compare rounding, not the kernels."""
    am = _am()
    m, n, k = 160, 1400, 48
    S = _planted(m, n, 11 + formulation, density=0.06)
    A = S.toarray()
    mu, rmu, C = _centring(A, center)
    g = _gamma(C, formulation)
    max_iter = 8 if formulation == 2 else 60
    kw = dict(formulation=formulation, constraintParameter=10, penaltyParameter=g,
              tolerance=1e-6, maximumIterations=max_iter, totalStartingPoints=k,
              batchSize=k // 2)
    M = am.Matrix.from_csc(solver, S, None, None, None, None, means=mu, row_means=rmu,
                           keep_sparse=True)
    x, f, stats = M.solve(am.OptimizationSettings(**kw))
    M.close()
    s = po.make_settings(formulation, constraint=10, penalty=g, tolerance=1e-6,
                         max_iter=max_iter, total_starts=k, batch_size=k // 2)
    starts = po.reference_starts(n, k, formulation <= 3, 10, dtype=np.float32)
    r = po.oracle_solve(C, s, starts.astype(np.float64))
    assert abs(f - r["fval"]) <= 1e-4 * abs(r["fval"]), (f, r["fval"])
    ev = float(np.linalg.norm(C @ x.astype(np.float64)) ** 2)
    ev_o = float(np.linalg.norm(C @ np.asarray(r["x"], np.float64)) ** 2)
    assert abs(ev - ev_o) <= 1e-4 * ev_o, (ev, ev_o)
    # the reported variance is the FP64 one of the returned x
    assert abs(stats.explained_variance - ev) <= 1e-9 * ev
    assert stats.low_precision_iterations == 0


@pytest.mark.parametrize("formulation", FORMS)
def test_sparse_resident_matches_densified_path(solver, formulation):
    """The same column-centred CSC input through both entry points, device
    starts: the same iteration with other products (split-FP16 tensor-core
    tiles against FP32 sums over the non-zeros), so the best explained variance
    agrees within 1e-4 and the step counts within three."""
    am = _am()
    m, n, k = 300, 2500, 256
    S = _sparse(m, n, 40 + formulation, density=0.04)
    A = S.toarray()
    mu, _, C = _centring(A, "columns")
    g = _gamma(C, formulation)
    kw = dict(formulation=formulation, constraintParameter=12, penaltyParameter=g,
              tolerance=1e-6, maximumIterations=80, totalStartingPoints=k, batchSize=k,
              startMode=am.START_DEVICE_UNIFORM)
    out = {}
    for keep in (False, True):
        M = am.Matrix.from_csc(solver, S, None, None, None, None, means=mu, keep_sparse=keep)
        x, f, stats = M.solve(am.OptimizationSettings(**kw))
        M.close()
        out[keep] = (x, f, stats)
    (_, fd, sd), (_, fs, ss) = out[False], out[True]
    assert abs(ss.explained_variance - sd.explained_variance) <= 1e-4 * sd.explained_variance
    assert abs(fs - fd) <= 1e-4 * abs(fd)
    assert abs(ss.it - sd.it) <= 3, (ss.it, sd.it)


def _with_long_entries(m, n, seed):
    """1 % noise plus four columns with 90 % of the rows filled and two rows
    with 60 % of the columns filled: both products then have outer entries
    longer than the 1024 entries one warp sums alone (SP_LONG)."""
    rng = np.random.default_rng(seed)
    A = _sparse(m, n, seed, density=0.01).toarray()
    for c in rng.choice(n, 4, replace=False):
        rows = rng.random(m) < 0.9
        A[rows, c] = rng.standard_normal(int(rows.sum())).astype(np.float32) + 1.0
    for r in rng.choice(m, 2, replace=False):
        cols = rng.random(n) < 0.6
        A[r, cols] = rng.standard_normal(int(cols.sum())).astype(np.float32)
    return sp.csc_matrix(A)


@pytest.mark.parametrize("formulation", [0, 1, 4, 6])
def test_sparse_resident_long_columns_and_rows(solver, po, formulation):
    """Columns and rows longer than SP_LONG entries (summed in segments, then
    combined): whole solves against the densified path (device starts, 256
    starts), and for the top-s form against the oracle (reference starts, 16
    starts, 10 steps).  The L1-ball forms are left out here: their reference
    scan cycles on such data, so two roundings of the same solve end on
    different supports (the other tests hold them to the oracle)."""
    am = _am()
    m, n = 3000, 2000
    S = _with_long_entries(m, n, 70 + formulation)
    assert np.diff(S.indptr).max() > 1024 and np.diff(S.tocsr().indptr).max() > 1024
    A = S.toarray()
    mu, _, C = _centring(A, "columns")
    g = _gamma(C, formulation, c=0.1)  # the long columns dominate the singular vector
    kw = dict(formulation=formulation, constraintParameter=12, penaltyParameter=g,
              tolerance=1e-6, maximumIterations=80, totalStartingPoints=256, batchSize=256,
              startMode=am.START_DEVICE_UNIFORM)
    out = {}
    for keep in (False, True):
        M = am.Matrix.from_csc(solver, S, None, None, None, None, means=mu, keep_sparse=keep)
        _, f, stats = M.solve(am.OptimizationSettings(**kw))
        M.close()
        out[keep] = (f, stats)
    (fd, sd), (fs, ss) = out[False], out[True]
    assert abs(ss.explained_variance - sd.explained_variance) <= 1e-4 * sd.explained_variance
    assert abs(fs - fd) <= 1e-4 * abs(fd)
    if formulation == 0:
        k = 16
        kw = dict(formulation=0, constraintParameter=12, tolerance=1e-6, maximumIterations=10,
                  totalStartingPoints=k, batchSize=k)
        M = am.Matrix.from_csc(solver, S, None, None, None, None, means=mu, keep_sparse=True)
        x, f, _ = M.solve(am.OptimizationSettings(**kw))
        M.close()
        s = po.make_settings(0, constraint=12, tolerance=1e-6, max_iter=10, total_starts=k,
                             batch_size=k)
        starts = po.reference_starts(n, k, True, 12, dtype=np.float32)
        r = po.oracle_solve(C, s, starts.astype(np.float64))
        assert abs(f - r["fval"]) <= 1e-5 * abs(r["fval"]), (f, r["fval"])


def test_sparse_resident_beyond_dense_memory(solver):
    """400000 x 200000 at 2.5e-5 density (2 M non-zeros): its dense FP32 form
    alone (320 GB) would not fit in device memory.  A few iterations of the
    top-s form from device starts; the reported FP64 explained variance is that
    of the returned x, recomputed on the host from the CSC arrays."""
    am = _am()
    m, n, k = 400_000, 200_000, 64
    rng = np.random.default_rng(3)
    nnz = 2_000_000
    rows = rng.integers(0, m, nnz)
    cols = rng.integers(0, n, nnz)
    S = sp.csc_matrix((rng.standard_normal(nnz).astype(np.float32), (rows, cols)),
                      shape=(m, n), dtype=np.float32)
    S.sum_duplicates()
    mu = np.asarray(S.mean(axis=0), np.float32).ravel()
    kw = dict(formulation=0, constraintParameter=20, tolerance=1e-6, maximumIterations=8,
              totalStartingPoints=k, batchSize=k, startMode=am.START_DEVICE_UNIFORM)
    M = am.Matrix.from_csc(solver, S, None, None, None, None, means=mu, keep_sparse=True)
    x, f, stats = M.solve(am.OptimizationSettings(**kw))
    M.close()
    x64 = x.astype(np.float64)
    assert np.count_nonzero(x) == 20 and abs(np.linalg.norm(x64) - 1.0) < 1e-6
    y = S.astype(np.float64) @ x64 - float(mu.astype(np.float64) @ x64)
    ev = float(y @ y)
    assert abs(stats.explained_variance - ev) <= 1e-9 * ev
    assert f > 0 and stats.it == 8


def test_sparse_resident_rejections(solver):
    """Batches, groups and reads take dense matrices only; the on-the-fly mode
    is not offered on a sparse-resident one."""
    am = _am()
    S = _sparse(64, 300, 5, density=0.1)
    M = am.Matrix.from_csc(solver, S, None, None, None, None, keep_sparse=True)
    st = am.OptimizationSettings(formulation=0, constraintParameter=5, totalStartingPoints=32,
                                 batchSize=32)
    for call in (lambda: M.batch(st, 32), lambda: M.read(),
                 lambda: M.solve(am.OptimizationSettings(formulation=0, constraintParameter=5,
                                                         useOTF=True, totalStartingPoints=32,
                                                         batchSize=8))):
        with pytest.raises(am.Am24Error) as ex:
            call()
        assert ex.value.status == 5  # AM24_ERR_UNSUPPORTED
    grp = am.Group(solver, capacity=1)
    with pytest.raises(am.Am24Error):
        grp.add(M, st)
    grp.close()
    M.close()


def test_sparse_resident_unsorted_and_duplicate_entries(solver):
    """CSC columns with unsorted rows and repeated (row, column) entries are
    sorted and summed on the host: the solve equals the one on the canonical
    arrays bit for bit (values are small integers, so every sum is exact)."""
    am = _am()
    m, n = 120, 700
    rng = np.random.default_rng(9)
    A = _planted(m, n, 19, density=0.08).toarray()
    A = np.round(A * 4.0).astype(np.float32)
    S = sp.csc_matrix(A)
    S.sort_indices()
    # split every entry in two halves at random positions of its column, shuffled
    ptr, rows, vals = [0], [], []
    for c in range(n):
        r = S.indices[S.indptr[c]:S.indptr[c + 1]]
        v = S.data[S.indptr[c]:S.indptr[c + 1]]
        half = np.floor(v / 2.0).astype(np.float32)
        rr = np.concatenate([r, r])
        vv = np.concatenate([half, (v - half).astype(np.float32)])
        perm = rng.permutation(rr.size)
        rows.extend(rr[perm])
        vals.extend(vv[perm])
        ptr.append(len(rows))
    mu = np.asarray(A.mean(axis=0), np.float32)
    kw = dict(formulation=0, constraintParameter=10, tolerance=1e-6, maximumIterations=40,
              totalStartingPoints=64, batchSize=64)
    M1 = am.Matrix.from_csc(solver, S, None, None, None, None, means=mu, keep_sparse=True)
    x1, f1, _ = M1.solve(am.OptimizationSettings(**kw))
    M1.close()
    M2 = am.Matrix.from_csc(solver, np.array(vals, np.float32), np.array(rows, np.int32),
                            np.array(ptr, np.int32), m, n, means=mu, keep_sparse=True)
    x2, f2, _ = M2.solve(am.OptimizationSettings(**kw))
    M2.close()
    assert f1 == f2 and np.array_equal(x1, x2)


@pytest.mark.parametrize("formulation", [0, 3, 6])
def test_sparse_resident_deflation_matches_densified(solver, formulation):
    """Three components, the reference's multi-component loop: after each
    solve both matrices are deflated by the same loading (the densified
    path's), B <- B (I - x x^T).  The densified matrix is rewritten; the
    sparse-resident one projects the loadings instead.  Each solve's best
    explained variance (of the deflated matrix) agrees within 1e-4."""
    am = _am()
    m, n, k = 300, 2500, 256
    S = _planted(m, n, 90 + formulation, density=0.04)
    A = S.toarray()
    mu, _, C = _centring(A, "columns")
    Md = am.Matrix.from_csc(solver, S, None, None, None, None, means=mu)
    Ms = am.Matrix.from_csc(solver, S, None, None, None, None, means=mu, keep_sparse=True)
    for comp in range(3):
        # the penalty from the deflated matrix, so that each solve keeps loadings
        kw = dict(formulation=formulation, constraintParameter=12,
                  penaltyParameter=_gamma(C, formulation), tolerance=1e-6,
                  maximumIterations=80, totalStartingPoints=k, batchSize=k,
                  startMode=am.START_DEVICE_UNIFORM)
        xd, fd, sd = Md.solve(am.OptimizationSettings(**kw))
        xs, fs, ss = Ms.solve(am.OptimizationSettings(**kw))
        assert abs(ss.explained_variance - sd.explained_variance) <= \
            1e-4 * sd.explained_variance, (comp, ss.explained_variance, sd.explained_variance)
        assert abs(fs - fd) <= 1e-4 * abs(fd), (comp, fs, fd)
        Md.deflate(xd)
        Ms.deflate(xd)
        x64 = xd.astype(np.float64)
        C = C - np.outer(C @ x64, x64)
    Md.close()
    Ms.close()
