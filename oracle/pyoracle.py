"""ORACLE bindings -- test infrastructure, not product code.

ctypes wrappers around
  * oracle/liboracle.so            the C restatement of the reference AM core
                                   (oracle/am_oracle.c), and
  * oracle/_ref/libref24_*.so      the reference's own solver compiled from its
                                   sources (oracle/Makefile, oracle/ref_harness.cpp).

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs import this module.
Matrices follow the reference layout: B is m x n column-major (m samples,
n features, ldB = m); starting points are n x k column-major.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FORMULATIONS = [
    "L0_constrained_L2_PCA", "L0_constrained_L1_PCA", "L1_constrained_L2_PCA",
    "L1_constrained_L1_PCA", "L0_penalized_L2_PCA", "L0_penalized_L1_PCA",
    "L1_penalized_L2_PCA", "L1_penalized_L1_PCA",
]


class Settings(C.Structure):
    """Layout shared by orc_settings (am_oracle.h) and ref_settings (ref_harness.cpp)."""
    _fields_ = [
        ("formulation", C.c_int), ("constraint", C.c_uint), ("penalty", C.c_double),
        ("tolerance", C.c_double), ("max_iter", C.c_int), ("total_starts", C.c_int),
        ("batch_size", C.c_int), ("use_otf", C.c_int), ("use_sort_hard", C.c_int),
        ("store_all", C.c_int), ("total_batches", C.c_uint),
    ]


class Stats(C.Structure):
    _fields_ = [("it", C.c_uint), ("fval", C.c_double), ("compute_time", C.c_double),
                ("threads", C.c_int)]


def make_settings(formulation, constraint=10, penalty=0.0, tolerance=0.01, max_iter=20,
                  total_starts=64, batch_size=64, use_otf=False, use_sort_hard=False,
                  store_all=False):
    """Defaults are the reference's OptimizationSettings() defaults
    (c++/src/class/optimization_settings.h:101-123)."""
    return Settings(int(formulation), int(constraint), float(penalty), float(tolerance),
                    int(max_iter), int(total_starts), int(batch_size), int(bool(use_otf)),
                    int(bool(use_sort_hard)), int(bool(store_all)), 0)


def build(reference=None):
    """Compile liboracle.so (always) and, given the reference's source tree
    (`reference`, else the AM24_REFERENCE environment variable), the reference
    build in _ref/ against naive loops and against the OpenBLAS found beside
    the Python packages."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    reference = reference or os.environ.get("AM24_REFERENCE")
    if reference and os.path.isdir(reference):
        lib = _openblas_lib()
        if lib is None:
            raise FileNotFoundError("no libopenblas*.so found for the reference build")
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REFERENCE={reference}",
                        f"OPENBLAS_LIB={lib}"], check=True)


_LIBS = {}


def _load(path):
    if path not in _LIBS:
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (run `make -C {HERE}` / `make ref`)")
        _LIBS[path] = C.CDLL(path)
    return _LIBS[path]


def oracle_lib():
    return _load(os.path.join(HERE, "liboracle.so"))


def _openblas_dir():
    import site
    for d in site.getsitepackages() + [site.getusersitepackages()]:
        cand = os.path.join(d, "opencv_python_headless.libs")
        if os.path.isdir(cand):
            return cand
    return None


def _openblas_lib():
    d = _openblas_dir()
    if not d:
        return None
    for f in sorted(os.listdir(d)):
        if f.startswith("libopenblas") and f.endswith(".so"):
            return os.path.join(d, f)
    return None


def ref_lib(blas="naive"):
    if blas == "openblas" and "openblas-deps" not in _LIBS:
        # OpenBLAS's own runtime dependencies sit beside it; load them first so
        # the dynamic loader finds them by soname.
        d = _openblas_dir()
        if d:
            for prefix in ("libquadmath", "libgfortran"):
                for f in sorted(os.listdir(d)):
                    if f.startswith(prefix):
                        C.CDLL(os.path.join(d, f), mode=C.RTLD_GLOBAL)
        _LIBS["openblas-deps"] = True
    return _load(os.path.join(HERE, "_ref", f"libref24_{blas}.so"))


def ref_available(blas="naive"):
    return os.path.exists(os.path.join(HERE, "_ref", f"libref24_{blas}.so"))


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _dt(dtype):
    return "f32" if np.dtype(dtype) == np.float32 else "f64"


def _solve(lib, fn, B, settings, V_all=None, x0=None):
    dtype = B.dtype
    m, n = B.shape
    Bf = np.asfortranarray(B)
    x = np.zeros(n, dtype) if x0 is None else np.array(x0, dtype)
    s = Settings.from_buffer_copy(settings)
    st = Stats()
    total = max(s.total_starts, s.batch_size) + s.batch_size
    values = np.full(total, -1.0)
    iters = np.full(total, -1, np.int32)
    cards = np.full(total, -1, np.int32)
    f = getattr(lib, fn)
    f.restype = C.c_float if dtype == np.float32 else C.c_double
    args = [_ptr(Bf), C.c_int(m), _ptr(x), C.c_uint(m), C.c_uint(n), C.byref(s), C.byref(st)]
    if V_all is not None:
        args.append(_ptr(np.asfortranarray(V_all, dtype)))
    args += [_ptr(values), _ptr(iters), _ptr(cards)]
    ret = f(*args)
    k = s.total_starts
    return dict(fval=float(ret), x=x, it=st.it, settings=s, values=values[:k],
                iters=iters[:k], cards=cards[:k], compute_time=st.compute_time,
                threads=st.threads)


def oracle_solve(B, settings, V_all=None):
    """orc_dense_solver_*: the restated denseDataSolver (reference starts when V_all is None)."""
    lib = oracle_lib()
    dtype = B.dtype
    m, n = B.shape
    Bf = np.asfortranarray(B)
    x = np.zeros(n, dtype)
    s = Settings.from_buffer_copy(settings)
    st = Stats()
    total = max(s.total_starts, s.batch_size) + s.batch_size
    values = np.full(total, -1.0)
    iters = np.full(total, -1, np.int32)
    cards = np.full(total, -1, np.int32)
    f = getattr(lib, f"orc_dense_solver_{_dt(dtype)}")
    f.restype = C.c_float if dtype == np.float32 else C.c_double
    Va = None if V_all is None else np.asfortranarray(V_all, dtype)
    ret = f(_ptr(Bf), C.c_int(m), _ptr(x), C.c_uint(m), C.c_uint(n), C.byref(s), C.byref(st),
            _ptr(Va), _ptr(values), _ptr(iters), _ptr(cards))
    k = s.total_starts
    return dict(fval=float(ret), x=x, it=st.it, settings=s, values=values[:k],
                iters=iters[:k], cards=cards[:k])


def ref_solve(B, settings, V_all=None, blas="naive"):
    """The reference's solver: unmodified denseDataSolver when V_all is None,
    else its driver loop around its own iteration functions with injected starts."""
    lib = ref_lib(blas)
    fn = ("ref_dense_solver_" if V_all is None else "ref_solver_injected_") + _dt(B.dtype)
    return _solve(lib, fn, B, settings, V_all)


def ref_set_threads(n, blas="naive"):
    """OpenMP threads of the reference build (1 = reproducible reference starts)."""
    lib = ref_lib(blas)
    lib.ref_set_threads(C.c_int(int(n)))
    lib.ref_total_threads.restype = C.c_uint
    return lib.ref_total_threads()


def ref_init_threads(blas="naive"):
    lib = ref_lib(blas)
    lib.ref_init_threads()
    lib.ref_total_threads.restype = C.c_uint
    return lib.ref_total_threads()


def oracle_iteration(B, V, settings, val, tmpv=None, it=1):
    """One batch AM iteration (orc_iteration_*). Returns (V', Z, val', err, max_err)."""
    lib = oracle_lib()
    dtype = B.dtype
    m, n = B.shape
    bs = V.shape[1]
    Bf = np.asfortranarray(B)
    V = np.array(V, dtype, order="F")
    Z = np.zeros((m, bs), dtype, order="F")
    val = np.array(val, dtype)
    tmpv = np.zeros(bs, dtype) if tmpv is None else np.array(tmpv, dtype)
    err = np.zeros(bs, dtype)
    buf = np.zeros(n + 2, dtype)
    iters = np.full(bs, -1, np.int32)
    cards = np.full(bs, -1, np.int32)
    f = getattr(lib, f"orc_iteration_{_dt(dtype)}")
    f.restype = C.c_float if dtype == np.float32 else C.c_double
    s = Settings.from_buffer_copy(settings)
    me = f(_ptr(Bf), C.c_int(m), C.c_uint(m), C.c_uint(n), C.c_uint(bs), _ptr(V), _ptr(Z),
           C.byref(s), _ptr(val), _ptr(tmpv), _ptr(err), C.c_int(it), C.c_uint(0),
           _ptr(iters), _ptr(cards), _ptr(buf))
    return V, Z, val, err, float(me)


def reference_starts(n, k, constrained, s, dtype=np.float64, first=0):
    """The reference's own starting points for global indices first..first+k-1
    (orc_reference_start_*), n x k column-major."""
    lib = oracle_lib()
    V = np.zeros((n, k), dtype, order="F")
    f = getattr(lib, f"orc_reference_start_{_dt(dtype)}")
    for j in range(k):
        col = V[:, j]
        f(_ptr(col), C.c_uint(n), C.c_int(int(constrained)), C.c_uint(s), C.c_uint(first + j))
    return V


def _thr(lib, name, x, *args):
    x = np.array(x, order="C")
    f = getattr(lib, f"{name}_{_dt(x.dtype)}")
    f.restype = C.c_float if x.dtype == np.float32 else C.c_double
    r = f(_ptr(x), C.c_uint(x.size), *args)
    return x, float(r)


def oracle_soft_threshold(x, s):
    buf = np.zeros(np.size(x) + 2, np.asarray(x).dtype)
    x = np.array(x, order="C")
    f = getattr(oracle_lib(), f"orc_soft_threshold_{_dt(x.dtype)}")
    f.restype = C.c_float if x.dtype == np.float32 else C.c_double
    r = f(_ptr(x), C.c_uint(x.size), C.c_uint(s), _ptr(buf))
    return x, float(r)


def oracle_soft_level(x, s):
    x = np.array(x, order="C")
    buf = np.zeros(x.size + 2, x.dtype)
    brk = C.c_uint(0)
    f = getattr(oracle_lib(), f"orc_soft_level_{_dt(x.dtype)}")
    f.restype = C.c_float if x.dtype == np.float32 else C.c_double
    w = f(_ptr(x), C.c_uint(x.size), C.c_uint(s), _ptr(buf), C.byref(brk))
    return float(w), int(brk.value)


def oracle_hard_threshold(x, k, use_sort=False):
    x = np.array(x, order="C")
    buf = np.zeros(x.size + 2, x.dtype)
    f = getattr(oracle_lib(), f"orc_hard_threshold_{_dt(x.dtype)}")
    f.restype = C.c_float if x.dtype == np.float32 else C.c_double
    r = f(_ptr(x), C.c_uint(x.size), C.c_uint(k), C.c_int(int(use_sort)), _ptr(buf))
    return x, float(r)


def ref_soft_threshold(x, s, blas="naive"):
    return _thr(ref_lib(blas), "ref_soft_thresholding", x, C.c_uint(s))


def ref_hard_threshold(x, k, use_sort=False, blas="naive"):
    return _thr(ref_lib(blas), "ref_k_hard_thresholding", x, C.c_uint(k), C.c_int(int(use_sort)))


def _workloads():
    import importlib.util
    path = os.path.join(os.path.dirname(HERE), "24am_b200", "workloads.py")
    spec = importlib.util.spec_from_file_location("am24_workloads", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def low_rank_data(n, p, r, nnz_v, seed, noise=0.1, dtype=np.float64):
    """The benchmark workloads' low-rank-plus-noise generator (24am_b200/workloads.py)."""
    return _workloads().low_rank_data(n, p, r, nnz_v, seed, noise, dtype)


def uniform_starts(p, k, seed, dtype=np.float64):
    """Starting points i.i.d. U[-1, 1], each column normalised (24am_b200/workloads.py)."""
    return _workloads().uniform_starts(p, k, seed, dtype)
