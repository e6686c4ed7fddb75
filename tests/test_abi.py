"""The C ABI without a GPU: the library loads, exports every entry point of
include/am24.h, mirrors the reference's settings logic, and reports errors."""
import ctypes as C

import numpy as np
import pytest


def test_exports_every_declared_symbol(am):
    L = am.lib()
    syms = am.header_symbols()
    assert len(syms) >= 19
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing
    assert L.am24_abi_version() == 1


def test_default_settings_are_reference_defaults(am):
    """OptimizationSettings() (c++/src/class/optimization_settings.h:101-123)."""
    s = am.am24_settings()
    am.lib().am24_default_settings(C.byref(s))
    assert (s.tolerance, s.constraint, s.penalty, s.total_starts, s.batch_size) == (0.01, 10, 0.0, 64, 64)
    assert (s.max_iter, s.use_otf, s.use_sort_hard, s.store_all) == (20, 0, 0, 0)
    assert s.start_mode == am.START_REFERENCE and s.l1_mode == am.L1_REFERENCE_SCAN


def test_mixed_settings_defaults_and_mirror(am):
    """The library's MIXED options: the single-pass phase from the first
    iteration unless a lead-in is asked for, and the Python mirror's fields
    reaching the C struct (leadIterations in the former reserved words: the
    struct's size and the offsets of the fields after it are unchanged)."""
    s = am.am24_settings()
    am.lib().am24_default_settings(C.byref(s))
    assert (s.precision, s.stable_iterations, s.stable_share, s.lead_iterations) == (0, 5, 1.0, 0)
    c = am.OptimizationSettings(precision=am.PRECISION_MIXED, stableIterations=3,
                                stableShare=0.5, leadIterations=20).to_c()
    assert (c.precision, c.stable_iterations, c.stable_share, c.lead_iterations) == (1, 3, 0.5, 20)
    assert am.am24_settings.lead_iterations.offset == am.am24_settings.stable_share.offset + 4
    assert am.am24_settings.reserved.offset == am.am24_settings.lead_iterations.offset + 4


def test_check_input_matches_reference(am, po):
    """chceckInputAndModifyIt (c++/src/class/optimization_settings.h:156-168)
    against the oracle's restatement, over random settings."""
    rng = np.random.default_rng(3)
    for _ in range(300):
        n = int(rng.integers(1, 500))
        total = int(rng.integers(1, 300))
        bs = int(rng.integers(0, 70))
        s_par = int(rng.integers(1, 1000))
        a = am.am24_settings()
        am.lib().am24_default_settings(C.byref(a))
        a.total_starts, a.batch_size, a.constraint = total, bs, s_par
        st = am.lib().am24_check_input(C.byref(a), n)
        b = po.make_settings(0, constraint=s_par, total_starts=total, batch_size=bs)
        po.oracle_lib().orc_check_input(C.byref(b), C.c_uint(n))
        assert st == 0
        assert (a.total_starts, a.batch_size, a.constraint, a.total_batches) == \
               (b.total_starts, b.batch_size, b.constraint, b.total_batches)


def test_python_mirror_settings(am):
    s = am.OptimizationSettings(totalStartingPoints=100, batchSize=64, constraintParameter=500)
    s.chceckInputAndModifyIt(300)
    assert (s.totalStartingPoints, s.totalBatches, s.constraintParameter) == (128, 2, 300)
    assert am.OptimizationSettings(formulation=am.L1_penalized_L2_PCA).isL1PenalizedProblem()
    assert not am.OptimizationSettings(formulation=am.L0_penalized_L2_PCA).isConstrainedProblem()


def test_errors_are_reported(am):
    L = am.lib()
    assert L.am24_check_input(None, 10) == 1
    assert "NULL" in am.last_error()
    x = np.zeros(3, np.float32)
    s = am.am24_settings()
    L.am24_default_settings(C.byref(s))
    assert L.am24_solve_dense_f32(None, None, 1, x.ctypes.data_as(C.c_void_p), 1, 3, C.byref(s),
                                  None, None, None) == 1
    assert L.am24_status_string(4).decode() == "device-side wait timed out"


def test_no_gpu_fails_loudly(am):
    """Without a usable sm_100 device the library refuses; there is no CPU path."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(am.Am24Error):
        am.Solver(0)


def test_struct_layouts_match_the_header(am, tmp_path):
    """The ctypes mirrors of am24_settings / am24_statistics have the C layout
    (offsets of every field, and the size), compiled from include/am24.h."""
    import ctypes as C
    import os
    import subprocess
    structs = {"am24_settings": am.am24_settings, "am24_statistics": am.am24_statistics}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "am24.h"', 'int main(void) {']
    for cname, py in structs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    subprocess.run(["gcc", "-I", inc, "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    for line in out.splitlines():
        cname, field, value = line.split()
        py = structs[cname]
        got = C.sizeof(py) if field == "size" else getattr(py, field).offset
        assert got == int(value), (cname, field, got, value)


@pytest.mark.parametrize("rows,ptr,msg", [
    ([0, 3, 1], [0, 2, 3], "row index out of range at entry 1"),
    ([0, -1, 1], [0, 2, 3], "row index out of range at entry 1"),
    ([0, 2, 1], [0, 3, 2], "non-decreasing"),
    ([0, 2, 1], [1, 2, 3], "col_ptr[0]"),
    ([0, 2, 1], [0, 2, 3], "NULL handle"),  # well formed: only the handle is missing
])
@pytest.mark.parametrize("entry", ["am24_matrix_create_csc_f32",
                                   "am24_matrix_create_csc_sparse_f32"])
def test_csc_arrays_checked_on_the_host(am, rows, ptr, msg, entry):
    """Both CSC entry points (densified and sparse-resident) check the CSC
    arrays on the host before they need a handle or a device: malformed arrays
    never reach a kernel."""
    L = am.lib()
    vals = np.ones(3, np.float32)
    r = np.array(rows, np.int32)
    p = np.array(ptr, np.int32)
    out = C.c_void_p()
    st = getattr(L, entry)(None, vals.ctypes.data_as(C.c_void_p),
                           r.ctypes.data_as(C.c_void_p), p.ctypes.data_as(C.c_void_p),
                           3, 2, None, None, C.byref(out))
    assert st == 1 and msg in am.last_error()


def test_autotune_table_round_trip(am, tmp_path):
    """The autotuner's table: a file loaded, saved back the same, a malformed
    entry rejected (no device needed)."""
    src = tmp_path / "t.txt"
    src.write_text("# header\n0 16 26 18 256 6\n1 14 24 16 128 0\n")
    am.autotune_clear()
    am.autotune_load(str(src))
    out = tmp_path / "o.txt"
    am.autotune_save(str(out))
    body = [l for l in out.read_text().splitlines() if not l.startswith("#")]
    assert body == ["0 16 26 18 256 6", "1 14 24 16 128 0"]
    bad = tmp_path / "bad.txt"
    bad.write_text("0 16 26 18 96 1\n")
    with pytest.raises(am.Am24Error):
        am.autotune_load(str(bad))
    am.autotune_clear()
