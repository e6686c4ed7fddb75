"""Generates tests/golden/*.npz by running the REFERENCE solver itself.

The reference (optml/24am) is compiled from its own sources by oracle/Makefile
(`make -C oracle ref`) into oracle/_ref/libref24_naive.so: its unmodified
SPCASolver::MulticoreSolver::denseDataSolver (c++/src/gpower/sparse_PCA_solver.h:36-243)
and its thresholding operators (c++/src/utils/thresh_functions.h:121-254), linked
against a deterministic CBLAS.  This script feeds it seeded inputs and stores
inputs and outputs; tests/test_golden.py replays the inputs through the oracle
and requires bit-identical outputs.  Needs the reference sources, so it runs
only where they are mounted:

    OMP_NUM_THREADS=1 python tests/golden/make_golden.py <reference source tree>
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import pyoracle as po  # noqa: E402


def read_csv(path):
    """The reference's CSV reader (c++/src/utils/file_reader.h:80-86) yields
    an m x n column-major matrix; numpy's loadtxt gives the same values."""
    return np.asfortranarray(np.loadtxt(path, delimiter=",", ndmin=2))


def solver_cases():
    """(name, B, settings, V_all or None)."""
    cases = []
    for dt in (np.float64, np.float32):
        tag = "f64" if dt == np.float64 else "f32"
        B = po.low_rank_data(40, 120, 4, 12, seed=7, dtype=dt)
        colmax = float(np.linalg.norm(B.astype(np.float64), axis=0).max())
        l1max = float(np.abs(B.astype(np.float64)).sum(axis=0).max())
        V_all = po.uniform_starts(120, 32, seed=1007, dtype=dt)
        for f in range(8):
            gamma = {4: 0.1 * colmax ** 2, 5: 0.1 * l1max ** 2, 6: 0.1 * colmax,
                     7: 0.1 * l1max}.get(f, 0.0)
            for otf in (False, True):
                for inj in (False, True):
                    s = po.make_settings(f, constraint=6, penalty=gamma, tolerance=1e-5,
                                         max_iter=40, total_starts=24, batch_size=8,
                                         use_otf=otf, store_all=True)
                    name = f"{tag}_f{f}_{'otf' if otf else 'batch'}_{'inj' if inj else 'ref'}"
                    cases.append((name, B, s, V_all if inj else None))
    return cases


def main(reference):
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    po.build(reference)
    po.ref_set_threads(1)
    out = {}
    for name, B, s, V in solver_cases():
        tag = name.split("_")[0]
        out[f"B.{tag}"] = B
        if V is not None:
            out[f"V.{tag}"] = V
        r = po.ref_solve(B, s, V)
        case = dict(
            settings=np.array([s.formulation, s.constraint, s.penalty, s.tolerance, s.max_iter,
                               24, 8, s.use_otf, 0, 1], np.float64),
            x=r["x"], fval=np.array(r["fval"]), it=np.array(r["it"]),
            values=r["values"], iters=r["iters"], cards=r["cards"],
            total_starts=np.array(r["settings"].total_starts),
        )
        out.update({f"{name}.{k}": v for k, v in case.items()})
    np.savez_compressed(os.path.join(HERE, "reference_solver.npz"), **out)

    # the reference's own 2 x 3 fixture and the console runs of its Makefile
    # (c++/multicore.mk:18-21): -f 1 -s 3; -l 1000 -r 64 -f 1 -s 2; and with -u 1
    small = read_csv(os.path.join(reference, "c++", "datasets", "small.csv"))
    runs = {"small_f1_s3": dict(constraint=3),
            "small_f1_s2_l1000_r64": dict(constraint=2, total_starts=1000, batch_size=64),
            "small_f1_s2_l1000_r64_otf": dict(constraint=2, total_starts=1000, batch_size=64,
                                              use_otf=True)}
    sm = {"B": small}
    for name, kw in runs.items():
        s = po.make_settings(1, **kw)
        r = po.ref_solve(small, s)
        sm[f"{name}.x"] = r["x"]
        sm[f"{name}.fval"] = np.array(r["fval"])
        sm[f"{name}.it"] = np.array(r["it"])
    np.savez_compressed(os.path.join(HERE, "reference_small_csv.npz"), **sm)

    # thresholding operators on vectors with and without exact duplicates
    rng = np.random.default_rng(11)
    th = {}
    for t in range(60):
        L = int(rng.integers(2, 200))
        x = rng.standard_normal(L)
        if t % 3 == 0:
            x = np.round(x * 4) / 4
        for dt, tag in ((np.float64, "f64"), (np.float32, "f32")):
            xv = x.astype(dt)
            k = int(rng.integers(1, L + 1))
            s = int(rng.integers(1, L + 1))
            hs, ns = po.ref_hard_threshold(xv, k, use_sort=True)
            hm, nm = po.ref_hard_threshold(xv, k, use_sort=False)
            so, no = po.ref_soft_threshold(xv, s)
            th[f"{t}.{tag}.x"] = xv
            th[f"{t}.{tag}.ks"] = np.array([k, s])
            th[f"{t}.{tag}.hard_sort"] = hs
            th[f"{t}.{tag}.hard_sort_norm"] = np.array(ns)
            th[f"{t}.{tag}.hard_set"] = hm
            th[f"{t}.{tag}.hard_set_norm"] = np.array(nm)
            th[f"{t}.{tag}.soft"] = so
            th[f"{t}.{tag}.soft_norm"] = np.array(no)
    np.savez_compressed(os.path.join(HERE, "reference_thresholds.npz"), **th)
    print("wrote", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <reference source tree>")
    main(sys.argv[1])
