"""Grouped solves (am24_group_*): many problems of uneven shape stepped by one
captured graph of grouped launches.

  * Bit for bit against the one-problem batch path wherever both run the same
    kernels (more than 128 starts: CTA-pair tiles with split FP16 operands on
    both paths), step by step and to convergence, FP32 and MIXED, in a group
    of problems of different shapes, formulations and start counts.
  * Against the FP64 oracle per start for the narrow problems (64 and 128
    starts), which the grouped path runs on CTA pairs where the one-problem
    path runs one-CTA 3xTF32 tiles.
  * The same result alone and among other problems, bit for bit.
  * Each problem stops after the step its own batch loop stops on."""
import importlib

import numpy as np
import pytest

import fast_oracle as fo

pytestmark = pytest.mark.gpu


def _am():
    return importlib.import_module("24am_b200")


GAMMA = {4: 0.3, 5: 60.0, 6: 0.15, 7: 3.0}

# (m, n, k, formulation, s): shapes that give one, two and odd numbers of
# row tiles and every N tile
PROBLEMS = [(300, 2048, 256, 0, 12), (129, 4097, 257, 1, 16), (500, 1000, 384, 2, 9),
            (257, 3000, 300, 3, 20), (200, 1500, 256, 4, 0), (400, 2500, 512, 5, 0),
            (150, 900, 260, 6, 0), (333, 2222, 256, 7, 0)]


def _setup(am, po, spec, seed, precision=0, tol=1e-6, max_iter=60):
    m, n, k, f, s = spec
    B = po.low_rank_data(m, n, 6, 24, seed=seed, dtype=np.float32)
    V = po.uniform_starts(n, k, seed=seed + 1, dtype=np.float32)
    g = GAMMA.get(f, 0.0) * (4.0 if f == 5 else 1.0)
    st = am.OptimizationSettings(formulation=f, constraintParameter=max(s, 1), penaltyParameter=g,
                                 tolerance=tol, maximumIterations=max_iter,
                                 totalStartingPoints=k, batchSize=k, startMode=am.START_INJECTED,
                                 precision=precision)
    return B, V, st


@pytest.mark.parametrize("precision", [0, 1], ids=["fp32", "mixed"])
def test_group_matches_batch_bit_for_bit(solver, po, precision):
    am = _am()
    mats, specs = [], []
    grp = am.Group(solver, capacity=16)
    for i, spec in enumerate(PROBLEMS):
        B, V, st = _setup(am, po, spec, 100 + i, precision)
        M = solver.matrix(B)
        pid = grp.add(M, st, start_points=V)
        mats.append(M)
        specs.append((pid, M, V, st))
    # three steps, then on to convergence
    grp.run(max_steps=3)
    outs3 = {pid: grp.read(pid) for pid, *_ in specs}
    grp.run()
    for pid, M, V, st in specs:
        b = M.batch(st, V.shape[1])
        b.load(V)
        b.iterate(0, 3)
        ref3 = b.read()
        for a, c in zip(outs3[pid], ref3):
            assert np.array_equal(a, c, equal_nan=True), f"problem {pid} after 3 steps"
        x, f, stats = M.solve(st, start_points=V)
        xg, sg = grp.result(pid)
        stopped, steps = grp.state(pid)
        assert stopped and steps == stats.it, (pid, steps, stats.it)
        assert np.array_equal(xg, x), f"problem {pid}: x"
        assert sg.fval == f and sg.explained_variance == stats.explained_variance
        assert sg.low_precision_iterations == stats.low_precision_iterations
        b.close()
    grp.close()
    for M in mats:
        M.close()


@pytest.mark.parametrize("k", [64, 128, 96])
@pytest.mark.parametrize("formulation", [0, 3, 4, 7])
def test_narrow_problems_match_the_oracle(solver, po, formulation, k):
    """64 / 96 / 128 starts: N tiles of 64 and 128 on CTA pairs, three steps
    against the FP64 oracle per start (supports, loadings, objectives)."""
    am = _am()
    m, n, s = 300, 3000, 12
    B = po.low_rank_data(m, n, 8, 30, seed=7 + k, dtype=np.float32)
    B64 = B.astype(np.float64)
    V = po.uniform_starts(n, k, seed=8, dtype=np.float32)
    g = GAMMA.get(formulation, 0.0)
    st = am.OptimizationSettings(formulation=formulation, constraintParameter=s,
                                 penaltyParameter=g, tolerance=1e-6, maximumIterations=20,
                                 totalStartingPoints=k, batchSize=k, startMode=am.START_INJECTED)
    M = solver.matrix(B)
    grp = am.Group(solver, capacity=4)
    pid = grp.add(M, st, start_points=V)
    Vo, valo = V.astype(np.float64), np.zeros(k)
    ill = np.zeros(k, bool)
    for it in range(3):
        grp.run(max_steps=1)
        r = fo.iteration(B64, Vo, formulation, s, g, valo)
        Vo, valo = r.V, r.val
        ill |= r.ill
    Vg, valg, _, _ = grp.read(pid)
    keep = np.flatnonzero(~ill)
    assert len(keep) >= k // 2, f"{k - len(keep)} of {k} starts ill-conditioned"
    for j in keep:
        assert np.array_equal(Vg[:, j] != 0, Vo[:, j] != 0), f"support of start {j}"
        assert np.abs(Vg[:, j] - Vo[:, j]).max() <= 1e-5 * np.abs(Vo[:, j]).max() * 10
    assert np.allclose(valg[keep], valo[keep], rtol=1e-5)
    grp.close()
    M.close()


def test_alone_and_among_others_bit_for_bit(solver, po):
    """A problem's loadings, objectives and stopping step are the same solved
    alone and solved with seven others of other shapes and formulations."""
    am = _am()
    B, V, st = _setup(am, po, (300, 2048, 200, 2, 10), 55)
    M = solver.matrix(B)
    alone = am.Group(solver, capacity=2)
    pa = alone.add(M, st, start_points=V)
    alone.run()
    ra = alone.read(pa), alone.result(pa)[0], alone.state(pa)
    alone.close()
    mix = am.Group(solver, capacity=16)
    others = []
    for i, spec in enumerate(PROBLEMS[:4] + PROBLEMS[5:]):
        Bo, Vo, so = _setup(am, po, spec, 300 + i)
        Mo = solver.matrix(Bo)
        others.append(Mo)
        mix.add(Mo, so, start_points=Vo)
    pm = mix.add(M, st, start_points=V)
    mix.run()
    rm = mix.read(pm), mix.result(pm)[0], mix.state(pm)
    for a, c in zip(ra[0], rm[0]):
        assert np.array_equal(a, c, equal_nan=True)
    assert np.array_equal(ra[1], rm[1])
    assert ra[2] == rm[2]
    mix.close()
    for Mo in others:
        Mo.close()
    M.close()


def test_slots_are_reused_and_results_stay_put(solver, po):
    """Problems removed after their run free their slots; a problem added to a
    freed slot solves like a fresh one, and a problem that has stopped is not
    stepped again by later runs."""
    am = _am()
    B, V, st = _setup(am, po, (200, 1500, 256, 0, 12), 71)
    M = solver.matrix(B)
    grp = am.Group(solver, capacity=2)
    p0 = grp.add(M, st, start_points=V)
    p1 = grp.add(M, st, start_points=V)
    grp.run()
    r0 = grp.read(p0)
    grp.remove(p1)
    p2 = grp.add(M, st, start_points=V)
    grp.run()
    for a, c, d in zip(r0, grp.read(p0), grp.read(p2)):
        assert np.array_equal(a, c, equal_nan=True)
        assert np.array_equal(a, d, equal_nan=True)
    with pytest.raises(am.Am24Error):
        grp.add(M, st, start_points=V)  # full
    grp.close()
    M.close()


def test_autotuned_tiles_solve_like_the_cost_model(solver, po, tmp_path):
    """Problems added with autotuning on take the tiles the tuner timed (kept
    per bucket: a second problem of the bucket reuses them); the solves reach
    the same explained variance as with the cost model's tiles, and the table
    saved and loaded back gives the same tiles without timing again."""
    am = _am()
    am.autotune_clear()
    specs = [(300, 2048, 200, 0, 12), (300, 2048, 200, 0, 12), (129, 4097, 300, 5, 0)]
    runs = []
    for tuned in (False, True):
        grp = am.Group(solver, capacity=8)
        grp.set_autotune(tuned)
        mats, ids = [], []
        for i, spec in enumerate(specs):
            B, V, st = _setup(am, po, spec, 400 + (i % 2 if i < 2 else i))
            M = solver.matrix(B)
            mats.append(M)
            ids.append(grp.add(M, st, start_points=V))
        grp.run()
        runs.append([grp.result(p) for p in ids])
        grp.close()
        for M in mats:
            M.close()
    for (x0, s0), (x1, s1) in zip(*runs):
        assert abs(s1.explained_variance - s0.explained_variance) <= 1e-5 * s0.explained_variance
        assert abs(int(s1.it) - int(s0.it)) <= 2
    path = str(tmp_path / "tune.txt")
    am.autotune_save(path)
    lines = [l for l in open(path) if not l.startswith("#")]
    assert len(lines) == 2  # two buckets
    am.autotune_clear()
    am.autotune_load(path)
    am.autotune_save(path + ".2")
    assert open(path).read() == open(path + ".2").read()


def test_admission_in_chunks_matches_solo_runs(solver, po):
    """The serving pattern: problems join a group while others are mid-solve,
    the group runs four steps at a time, stopped problems are read and removed
    and their slots refilled.  Every problem ends bit for bit as it does
    solved alone in a group of its own."""
    am = _am()
    specs = [(300, 2048, 256, 0, 12), (129, 4097, 257, 1, 16), (500, 1000, 384, 2, 9),
             (257, 3000, 300, 3, 20), (200, 1500, 256, 4, 0), (400, 2500, 512, 5, 0),
             (150, 900, 260, 6, 0), (333, 2222, 256, 7, 0), (300, 2048, 200, 0, 30),
             (200, 1500, 300, 6, 0), (129, 4097, 256, 3, 8), (400, 2500, 256, 1, 40)]
    probs = []
    for i, spec in enumerate(specs):
        B, V, st = _setup(am, po, spec, 500 + i, max_iter=40)
        probs.append((solver.matrix(B), V, st))
    solo = []
    for M, V, st in probs:
        g1 = am.Group(solver, capacity=1)
        p = g1.add(M, st, start_points=V)
        g1.run()
        solo.append((g1.read(p), g1.result(p)[0], g1.state(p)))
        g1.close()
    grp = am.Group(solver, capacity=4)
    queue = list(range(len(probs)))
    running, done = {}, {}
    chunks = 0
    while queue or running:
        while queue and len(running) < 4:
            i = queue.pop(0)
            M, V, st = probs[i]
            running[grp.add(M, st, start_points=V)] = i
        grp.run(max_steps=4)
        chunks += 1
        assert chunks < 200
        for pid in list(running):
            stopped, _ = grp.state(pid)
            if stopped:
                i = running.pop(pid)
                done[i] = (grp.read(pid), grp.result(pid)[0], grp.state(pid))
                grp.remove(pid)
    grp.close()
    for i, (ref, got) in enumerate(zip(solo, (done[i] for i in range(len(probs))))):
        for a, c in zip(ref[0], got[0]):
            assert np.array_equal(a, c, equal_nan=True), f"problem {i}"
        assert np.array_equal(ref[1], got[1]), f"problem {i}: x"
        assert ref[2] == got[2], (i, ref[2], got[2])
    for M, _, _ in probs:
        M.close()
