"""The oracle against fixtures produced by the reference itself
(tests/golden/make_golden.py): bit-identical outputs required."""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and np.array_equal(a, b, equal_nan=True)


def _solver_cases():
    z = np.load(os.path.join(GOLDEN, "reference_solver.npz"))
    names = sorted({k.rsplit(".", 1)[0] for k in z.files if k.count(".") == 1 and
                    not k.startswith(("B.", "V."))})
    return z, names


Z, NAMES = _solver_cases()


@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_reference_solver(po, name):
    """denseDataSolver (c++/src/gpower/sparse_PCA_solver.h:36-243), all 8
    formulations, batch / on-the-fly, reference / injected starts, f32 / f64."""
    tag = name.split("_")[0]
    B = Z[f"B.{tag}"]
    st = Z[f"{name}.settings"]
    s = po.make_settings(int(st[0]), constraint=int(st[1]), penalty=float(st[2]),
                         tolerance=float(st[3]), max_iter=int(st[4]), total_starts=int(st[5]),
                         batch_size=int(st[6]), use_otf=bool(st[7]), store_all=True)
    V = Z[f"V.{tag}"] if name.endswith("_inj") else None
    r = po.oracle_solve(B, s, V)
    assert _same(r["x"], Z[f"{name}.x"])
    assert _same(r["fval"], Z[f"{name}.fval"])
    assert int(r["it"]) == int(Z[f"{name}.it"])
    assert int(r["settings"].total_starts) == int(Z[f"{name}.total_starts"])
    if not s.use_otf:
        assert _same(r["values"], Z[f"{name}.values"])
        assert _same(r["iters"], Z[f"{name}.iters"])
        assert _same(r["cards"], Z[f"{name}.cards"])


def test_oracle_matches_reference_small_csv(po):
    """The reference's datasets/small.csv with its Makefile console runs
    (c++/multicore.mk:18-21: -f 1 -s 3 -d; -l 1000 -r 64 -f 1 -s 2 -d; -u 1)."""
    z = np.load(os.path.join(GOLDEN, "reference_small_csv.npz"))
    B = z["B"]
    assert B.shape == (2, 3)
    runs = {"small_f1_s3": dict(constraint=3),
            "small_f1_s2_l1000_r64": dict(constraint=2, total_starts=1000, batch_size=64),
            "small_f1_s2_l1000_r64_otf": dict(constraint=2, total_starts=1000, batch_size=64,
                                              use_otf=True)}
    for name, kw in runs.items():
        r = po.oracle_solve(B, po.make_settings(1, **kw))
        assert _same(r["x"], z[f"{name}.x"]), name
        assert _same(r["fval"], z[f"{name}.fval"]), name
        assert int(r["it"]) == int(z[f"{name}.it"]), name


def test_oracle_matches_reference_thresholds(po):
    """k_hard_thresholding (set and sort level) and soft_thresholding
    (c++/src/utils/thresh_functions.h:92-254), vectors with duplicates included."""
    z = np.load(os.path.join(GOLDEN, "reference_thresholds.npz"))
    keys = sorted({k.rsplit(".", 1)[0] for k in z.files})
    assert len(keys) >= 100
    for key in keys:
        x = z[f"{key}.x"]
        k, s = (int(v) for v in z[f"{key}.ks"])
        h, nh = po.oracle_hard_threshold(x, k, use_sort=True)
        assert _same(h, z[f"{key}.hard_sort"]) and nh == float(z[f"{key}.hard_sort_norm"]), key
        h, nh = po.oracle_hard_threshold(x, k, use_sort=False)
        assert _same(h, z[f"{key}.hard_set"]) and nh == float(z[f"{key}.hard_set_norm"]), key
        so, ns = po.oracle_soft_threshold(x, s)
        assert _same(so, z[f"{key}.soft"]), key
        assert _same(ns, z[f"{key}.soft_norm"]), key
