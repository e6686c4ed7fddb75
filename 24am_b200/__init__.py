"""Python mirror of the AM sparse-PCA solver interface, over the C ABI of libam24.so.

The reference (optml/24am) exposes
    SPCASolver::MulticoreSolver::denseDataSolver<F>(B, ldB, x, m, n, settings, stats)
      -- c++/src/gpower/sparse_PCA_solver.h:36-40
with SolverStructures::OptimizationSettings / OptimizationStatistics
(c++/src/class/optimization_settings.h:71-170, optimization_statistics.h:27-46).
This module mirrors those names (``OptimizationSettings``, ``OptimizationStatistics``,
``denseDataSolver``) so tests read like the reference's own, and forwards to
include/am24.h.  All compute runs in libam24.so on an sm_100 GPU; there is no
CPU fallback: without the built library or a B200-class GPU the calls raise.

The package directory name starts with a digit, so import it with
``importlib.import_module("24am_b200")``.
"""
import ctypes as C
import os
import weakref

import numpy as np

from . import workloads  # noqa: F401  (seeded synthetic inputs)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libam24.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

# SPCA_Formulation (c++/src/class/optimization_settings.h:27-37)
L0_constrained_L2_PCA = 0
L0_constrained_L1_PCA = 1
L1_constrained_L2_PCA = 2
L1_constrained_L1_PCA = 3
L0_penalized_L2_PCA = 4
L0_penalized_L1_PCA = 5
L1_penalized_L2_PCA = 6
L1_penalized_L1_PCA = 7
FORMULATIONS = {
    "L2var_L0cons": 0, "L1var_L0cons": 1, "L2var_L1cons": 2, "L1var_L1cons": 3,
    "L2var_L0pen": 4, "L1var_L0pen": 5, "L2var_L1pen": 6, "L1var_L1pen": 7,
}

START_REFERENCE, START_INJECTED, START_DEVICE_UNIFORM = 0, 1, 2
L1_REFERENCE_SCAN, L1_EXACT = 0, 1
PRECISION_FP32, PRECISION_MIXED = 0, 1

STATUS = {0: "AM24_OK", 1: "AM24_ERR_INVALID_ARG", 2: "AM24_ERR_OOM", 3: "AM24_ERR_CUDA",
          4: "AM24_ERR_DEVICE_TIMEOUT", 5: "AM24_ERR_UNSUPPORTED", 6: "AM24_ERR_DEGENERATE",
          7: "AM24_ERR_ADMISSION_REJECTED"}


class Am24Error(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class am24_settings(C.Structure):
    _fields_ = [
        ("formulation", C.c_int32), ("constraint", C.c_uint32), ("penalty", C.c_double),
        ("tolerance", C.c_double), ("max_iter", C.c_int32), ("total_starts", C.c_int32),
        ("batch_size", C.c_int32), ("use_otf", C.c_int32), ("use_sort_hard", C.c_int32),
        ("store_all", C.c_int32), ("total_batches", C.c_uint32), ("verbose", C.c_int32),
        ("start_mode", C.c_int32), ("l1_mode", C.c_int32), ("timeout_ms", C.c_uint32),
        ("precision", C.c_int32), ("stable_iterations", C.c_uint32), ("stable_share", C.c_float),
        ("lead_iterations", C.c_uint32), ("reserved", C.c_uint32 * 3),
    ]


class am24_statistics(C.Structure):
    _fields_ = [
        ("it", C.c_uint32), ("fval", C.c_double), ("error", C.c_double),
        ("total_true_computation_time", C.c_double), ("total_elapsed_time", C.c_double),
        ("n", C.c_uint32), ("total_threads_used", C.c_int32),
        ("values", C.POINTER(C.c_double)), ("iters", C.POINTER(C.c_int32)),
        ("cardinalities", C.POINTER(C.c_int32)), ("per_start_capacity", C.c_uint32),
        ("explained_variance", C.c_double), ("start_iterations", C.c_uint64),
        ("degenerate_starts", C.c_int32), ("low_precision_iterations", C.c_uint32),
        ("input_rounded_to_f32", C.c_int32), ("reserved", C.c_uint32 * 5),
    ]


# every entry point of include/am24.h with its ctypes signature
_VP = C.c_void_p
_SIGS = {
    "am24_abi_version": (C.c_uint32, []),
    "am24_last_error": (C.c_char_p, []),
    "am24_status_string": (C.c_char_p, [C.c_int]),
    "am24_default_settings": (None, [C.POINTER(am24_settings)]),
    "am24_check_input": (C.c_int, [C.POINTER(am24_settings), C.c_uint32]),
    "am24_create": (C.c_int, [C.POINTER(_VP), C.c_int]),
    "am24_destroy": (C.c_int, [_VP]),
    "am24_solve_dense_f32": (C.c_int, [_VP, _VP, C.c_int32, _VP, C.c_uint32, C.c_uint32,
                                       C.POINTER(am24_settings), C.POINTER(am24_statistics), _VP,
                                       C.POINTER(C.c_float)]),
    "am24_solve_device_f32": (C.c_int, [_VP, _VP, C.c_int32, _VP, C.c_uint32, C.c_uint32,
                                        C.POINTER(am24_settings), C.POINTER(am24_statistics), _VP,
                                        C.POINTER(C.c_float)]),
    "am24_matrix_create_f32": (C.c_int, [_VP, _VP, C.c_int32, C.c_uint32, C.c_uint32, C.c_int32,
                                         C.POINTER(_VP)]),
    "am24_matrix_destroy": (C.c_int, [_VP, _VP]),
    "am24_matrix_deflate": (C.c_int, [_VP, _VP, _VP, C.c_int32]),
    "am24_matrix_create_csc_f32": (C.c_int, [_VP, _VP, _VP, _VP, C.c_uint32, C.c_uint32, _VP,
                                             _VP, _VP]),
    "am24_matrix_create_csc_sparse_f32": (C.c_int, [_VP, _VP, _VP, _VP, C.c_uint32, C.c_uint32,
                                                    _VP, _VP, _VP]),
    "am24_matrix_read_f32": (C.c_int, [_VP, _VP, _VP, C.c_int32]),
    "am24_solve_resident_f32": (C.c_int, [_VP, _VP, _VP, C.POINTER(am24_settings),
                                          C.POINTER(am24_statistics), _VP, C.POINTER(C.c_float)]),
    "am24_batch_create": (C.c_int, [_VP, _VP, C.POINTER(am24_settings), C.c_uint32,
                                    C.POINTER(_VP)]),
    "am24_batch_destroy": (C.c_int, [_VP, _VP]),
    "am24_batch_load": (C.c_int, [_VP, _VP, _VP, C.c_int32]),
    "am24_batch_iterate": (C.c_int, [_VP, _VP, C.c_int32, C.c_int32, C.POINTER(C.c_float)]),
    "am24_batch_iterate_static_ws": (C.c_int, [_VP, _VP, C.c_int32, C.c_int32,
                                               C.POINTER(C.c_float)]),
    "am24_batch_read": (C.c_int, [_VP, _VP, _VP, _VP, _VP, _VP]),
    "am24_batch_launches_per_step": (C.c_int, [_VP, _VP, C.POINTER(C.c_int32)]),
    "am24_batch_phase": (C.c_int, [_VP, _VP, C.POINTER(C.c_int32)]),
    "am24_solve_dense_f64": (C.c_int, [_VP, _VP, C.c_int32, _VP, C.c_uint32, C.c_uint32,
                                       C.POINTER(am24_settings), C.POINTER(am24_statistics), _VP,
                                       C.POINTER(C.c_double)]),
    "am24_server_create": (C.c_int, [C.c_int, C.c_uint64, C.POINTER(_VP)]),
    "am24_server_destroy": (C.c_int, [_VP]),
    "am24_server_add_matrix_f32": (C.c_int, [_VP, _VP, C.c_int32, C.c_uint32, C.c_uint32,
                                             C.c_int32, C.POINTER(C.c_uint32)]),
    "am24_server_remove_matrix": (C.c_int, [_VP, C.c_uint32]),
    "am24_submit": (C.c_int, [_VP, C.c_uint32, C.POINTER(am24_settings), _VP,
                              C.POINTER(C.c_uint64)]),
    "am24_poll": (C.c_int, [_VP, C.c_uint64, _VP, C.POINTER(am24_statistics),
                            C.POINTER(C.c_int32)]),
    "am24_wait": (C.c_int, [_VP, C.c_uint64, _VP, C.POINTER(am24_statistics)]),
    "am24_sync": (C.c_int, [_VP]),
    "am24_selftest_bounded_wait": (C.c_int, [_VP, C.c_uint32]),
    "am24_stream": (C.c_void_p, [_VP]),
    "am24_batch_step_timed": (C.c_int, [_VP, _VP, C.c_int32, C.POINTER(C.c_float),
                                        C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "am24_group_create": (C.c_int, [_VP, C.c_uint32, C.POINTER(_VP)]),
    "am24_group_destroy": (C.c_int, [_VP]),
    "am24_group_add": (C.c_int, [_VP, _VP, C.POINTER(am24_settings), _VP,
                                 C.POINTER(C.c_uint32)]),
    "am24_group_run": (C.c_int, [_VP, C.c_uint32, C.POINTER(C.c_float)]),
    "am24_group_state": (C.c_int, [_VP, C.c_uint32, C.POINTER(C.c_int32),
                                   C.POINTER(C.c_uint32)]),
    "am24_group_result": (C.c_int, [_VP, C.c_uint32, _VP, C.POINTER(am24_statistics)]),
    "am24_group_read": (C.c_int, [_VP, C.c_uint32, _VP, _VP, _VP, _VP]),
    "am24_group_remove": (C.c_int, [_VP, C.c_uint32]),
    "am24_group_set_autotune": (C.c_int, [_VP, C.c_int32]),
    "am24_autotune_save": (C.c_int, [C.c_char_p]),
    "am24_autotune_load": (C.c_int, [C.c_char_p]),
    "am24_autotune_clear": (C.c_int, []),
}
KERNEL_KINDS = ["gemm_BV", "z_reduce", "gemm_BtZ", "select", "finalize", "gather_BV", "densify",
                "gemm_BtZ_low", "support", "gather_BV_group"]

_lib = None


def lib():
    """The loaded libam24.so.  Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise Am24Error(5, f"{LIB_PATH} is not built; run __graft_entry__.build()")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def last_error():
    return lib().am24_last_error().decode()


def check(status):
    if status != 0:
        raise Am24Error(status, last_error())


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class OptimizationSettings:
    """Mirror of SolverStructures::OptimizationSettings (reference field names
    and defaults, c++/src/class/optimization_settings.h:71-123), plus the
    extensions startMode / l1Mode / timeoutMs / precision / stableIterations /
    stableShare / leadIterations of this library."""

    def __init__(self, **kw):
        self.formulation = L0_constrained_L2_PCA
        self.constraintParameter = 10
        self.penaltyParameter = 0.0
        self.tolerance = 0.01
        self.maximumIterations = 20
        self.totalStartingPoints = 64
        self.batchSize = 64
        self.useOTF = False
        self.useSortForHardThresholding = False
        self.storeIterationsForAllPoints = False
        self.totalBatches = 0
        self.verbose = False
        self.startMode = START_REFERENCE
        self.l1Mode = L1_REFERENCE_SCAN
        self.timeoutMs = 5000
        self.precision = PRECISION_FP32
        self.stableIterations = 5
        self.stableShare = 1.0
        self.leadIterations = 0
        for k, v in kw.items():
            if not hasattr(self, k):
                raise AttributeError(f"OptimizationSettings has no field {k}")
            setattr(self, k, v)

    # predicates of c++/src/class/optimization_settings.h:125-153
    def isConstrainedProblem(self):
        return self.formulation <= 3

    def isL1ConstrainedProblem(self):
        return self.formulation not in (0, 1)

    def isL1PenalizedProblem(self):
        return self.formulation not in (4, 5)

    def chceckInputAndModifyIt(self, n):
        s = self.to_c()
        check(lib().am24_check_input(C.byref(s), n))
        self.from_c(s)

    def to_c(self):
        s = am24_settings()
        lib().am24_default_settings(C.byref(s))
        s.formulation = int(self.formulation)
        s.constraint = int(self.constraintParameter)
        s.penalty = float(self.penaltyParameter)
        s.tolerance = float(self.tolerance)
        s.max_iter = int(self.maximumIterations)
        s.total_starts = int(self.totalStartingPoints)
        s.batch_size = int(self.batchSize)
        s.use_otf = int(bool(self.useOTF))
        s.use_sort_hard = int(bool(self.useSortForHardThresholding))
        s.store_all = int(bool(self.storeIterationsForAllPoints))
        s.verbose = int(bool(self.verbose))
        s.start_mode = int(self.startMode)
        s.l1_mode = int(self.l1Mode)
        s.timeout_ms = int(self.timeoutMs)
        s.precision = int(self.precision)
        s.stable_iterations = int(self.stableIterations)
        s.stable_share = float(self.stableShare)
        s.lead_iterations = int(self.leadIterations)
        return s

    def from_c(self, s):
        """The fields a solve rewrites, as the reference rewrites them."""
        self.constraintParameter = s.constraint
        self.totalStartingPoints = s.total_starts
        self.batchSize = s.batch_size
        self.totalBatches = s.total_batches
        self.storeIterationsForAllPoints = bool(s.store_all)


class OptimizationStatistics:
    """Mirror of SolverStructures::OptimizationStatistics
    (c++/src/class/optimization_statistics.h:27-46) plus this library's extras."""

    def __init__(self):
        self.it = 0
        self.fval = 0.0
        self.error = 0.0
        self.totalTrueComputationTime = 0.0
        self.totalElapsedTime = 0.0
        self.n = 0
        self.values = []
        self.iters = []
        self.cardinalities = []
        self.totalThreadsUsed = 1
        self.explainedVariance = 0.0
        self.startIterations = 0
        self.degenerateStarts = 0
        self.lowPrecisionIterations = 0
        self.inputRoundedToF32 = False


class Solver:
    """One device handle (am24_create / am24_destroy).  Closing it closes the
    matrices (and their batches) still open on it first: the C API wants every
    batch and matrix destroyed before their handle."""

    def __init__(self, device=0):
        h = C.c_void_p()
        check(lib().am24_create(C.byref(h), int(device)))
        self.h = h
        self._matrices = weakref.WeakSet()
        self._groups = weakref.WeakSet()

    def close(self):
        if self.h:
            for g in list(self._groups):  # their problems read the matrices
                g.close()
            for m in list(self._matrices):
                m.close()
            lib().am24_destroy(self.h)
            self.h = None

    def stream(self):
        """The handle's cudaStream_t as an integer."""
        return lib().am24_stream(self.h)

    def sync(self):
        check(lib().am24_sync(self.h))

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def denseDataSolver(self, B, ldB, x, m, n, settings, stats, start_points=None):
        """SPCASolver::MulticoreSolver::denseDataSolver<float>: B (m x n column-major,
        float32), x (n, float32) written in place.  Returns the best objective."""
        B = np.asarray(B)
        if B.dtype != np.float32 or x.dtype != np.float32:
            raise TypeError("the FP32 path takes float32 B and x")
        s = settings.to_c()
        st = am24_statistics()
        cap = max(int(settings.totalStartingPoints), int(settings.batchSize)) * 2 + 8
        values = np.full(cap, -1.0)
        iters = np.full(cap, -1, np.int32)
        cards = np.full(cap, -1, np.int32)
        if settings.storeIterationsForAllPoints:
            st.values = values.ctypes.data_as(C.POINTER(C.c_double))
            st.iters = iters.ctypes.data_as(C.POINTER(C.c_int32))
            st.cardinalities = cards.ctypes.data_as(C.POINTER(C.c_int32))
            st.per_start_capacity = cap
        sp = None if start_points is None else np.asfortranarray(start_points, np.float32)
        fv = C.c_float()
        Bp = B if B.flags.f_contiguous or B.ndim == 1 else np.asfortranarray(B)
        check(lib().am24_solve_dense_f32(self.h, _ptr(Bp), int(ldB), _ptr(x), int(m), int(n),
                                         C.byref(s), C.byref(st), _ptr(sp), C.byref(fv)))
        settings.from_c(s)
        stats.it = st.it
        stats.fval = st.fval
        stats.error = st.error
        stats.totalTrueComputationTime = st.total_true_computation_time
        stats.totalElapsedTime = st.total_elapsed_time
        stats.n = st.n
        stats.totalThreadsUsed = st.total_threads_used
        stats.explainedVariance = st.explained_variance
        stats.startIterations = st.start_iterations
        stats.degenerateStarts = st.degenerate_starts
        stats.lowPrecisionIterations = st.low_precision_iterations
        stats.inputRoundedToF32 = bool(st.input_rounded_to_f32)
        if settings.storeIterationsForAllPoints:
            k = settings.totalStartingPoints
            stats.values = values[:k].tolist()
            stats.iters = iters[:k].tolist()
            stats.cardinalities = cards[:k].tolist()
        return fv.value

    def solve(self, B, settings, start_points=None):
        """Convenience: B (m x n) -> (x, fval, stats)."""
        B = np.asfortranarray(B, np.float32)
        m, n = B.shape
        x = np.zeros(n, np.float32)
        stats = OptimizationStatistics()
        f = self.denseDataSolver(B, m, x, m, n, settings, stats, start_points)
        return x, f, stats

    # ---- resident matrices and batch stepping
    def matrix(self, B):
        return Matrix(self, B)


class Matrix:
    """A resident data matrix (am24_matrix_create_f32)."""

    def __init__(self, solver, B, on_device_ptr=None, m=None, n=None, ldB=None):
        self.solver = solver
        mh = C.c_void_p()
        if on_device_ptr is None:
            B = np.asfortranarray(B, np.float32)
            m, n = B.shape
            check(lib().am24_matrix_create_f32(solver.h, _ptr(B), m, m, n, 0, C.byref(mh)))
        else:
            check(lib().am24_matrix_create_f32(solver.h, C.c_void_p(on_device_ptr), ldB or m, m,
                                               n, 1, C.byref(mh)))
        self.m, self.n = m, n
        self.mh = mh
        self._batches = weakref.WeakSet()
        solver._matrices.add(self)

    @classmethod
    def from_csc(cls, solver, vals, row_ind, col_ptr, m, n, means=None, row_means=None,
                 keep_sparse=False):
        """A resident matrix from compressed sparse columns, with the sparse
        solver's optional implicit centring: the matrix solved is
        B - 1 means^T - row_means 1^T.  Densified on the device
        (am24_matrix_create_csc_f32), or with keep_sparse=True kept compressed
        (am24_matrix_create_csc_sparse_f32: O(nnz) memory, solves only).  Also
        takes a scipy.sparse matrix as `vals` (then row_ind / col_ptr / m / n may
        be None)."""
        if hasattr(vals, "tocsc"):
            S = vals.tocsc(copy=True)
            S.sum_duplicates()  # canonical: one entry per (row, column), rows sorted
            m, n = S.shape
            vals, row_ind, col_ptr = S.data, S.indices, S.indptr
        vals = np.ascontiguousarray(vals, np.float32)
        row_ind = np.ascontiguousarray(row_ind, np.int32)
        col_ptr = np.ascontiguousarray(col_ptr, np.int32)
        mu = None if means is None else np.ascontiguousarray(means, np.float32)
        rmu = None if row_means is None else np.ascontiguousarray(row_means, np.float32)
        self = cls.__new__(cls)
        self.solver = solver
        mh = C.c_void_p()
        create = (lib().am24_matrix_create_csc_sparse_f32 if keep_sparse
                  else lib().am24_matrix_create_csc_f32)
        check(create(solver.h, _ptr(vals), _ptr(row_ind), _ptr(col_ptr), int(m), int(n),
                     _ptr(mu), _ptr(rmu), C.byref(mh)))
        self.m, self.n = int(m), int(n)
        self.mh = mh
        self._batches = weakref.WeakSet()
        solver._matrices.add(self)
        return self

    def close(self):
        """Destroys the matrix, after any batch still open on it and any group
        problem on it."""
        if self.mh:
            for b in list(self._batches):
                b.close()
            for g in list(getattr(self.solver, "_groups", ())):
                if not g.gh:
                    continue
                for pid, (mat, _) in list(g.problems.items()):
                    if mat is self:
                        g.remove(pid)
            lib().am24_matrix_destroy(self.solver.h, self.mh)
            self.mh = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve(self, settings, start_points=None, x0=None):
        x = np.zeros(self.n, np.float32) if x0 is None else np.array(x0, np.float32)
        s = settings.to_c()
        st = am24_statistics()
        sp = None if start_points is None else np.asfortranarray(start_points, np.float32)
        fv = C.c_float()
        check(lib().am24_solve_resident_f32(self.solver.h, self.mh, _ptr(x), C.byref(s),
                                            C.byref(st), _ptr(sp), C.byref(fv)))
        settings.from_c(s)
        return x, fv.value, st

    def batch(self, settings, batch_size):
        return Batch(self, settings, batch_size)

    def deflate(self, x):
        """B <- B (I - x x^T) on the device (am24_matrix_deflate): the update the
        reference's multi-component driver applies between solves."""
        x = np.ascontiguousarray(x, np.float32)
        assert x.shape == (self.n,)
        check(lib().am24_matrix_deflate(self.solver.h, self.mh, _ptr(x), 0))

    def read(self):
        """The current B (m x n, column-major float32)."""
        B = np.zeros((self.m, self.n), np.float32, order="F")
        check(lib().am24_matrix_read_f32(self.solver.h, self.mh, _ptr(B), self.m))
        return B

    def components(self, settings, count, start_points=None):
        """`count` sparse components one after another, deflating B by each
        (c++/matlab/run_example.m:29-34).  Returns X (n x count), the objectives
        and the statistics of each solve.  B is left deflated by all of them."""
        X = np.zeros((self.n, count), np.float32, order="F")
        fvals, stats = [], []
        for i in range(count):
            x, f, st = self.solve(settings, start_points=start_points)
            X[:, i] = x
            fvals.append(f)
            stats.append(st)
            if i + 1 < count:
                self.deflate(x)
        return X, fvals, stats


class Batch:
    """A batch of starting points stepped one AM iteration at a time."""

    def __init__(self, matrix, settings, batch_size):
        self.matrix = matrix
        self.k = int(batch_size)
        s = settings.to_c()
        check(lib().am24_check_input(C.byref(s), matrix.n))
        bh = C.c_void_p()
        check(lib().am24_batch_create(matrix.solver.h, matrix.mh, C.byref(s), self.k,
                                      C.byref(bh)))
        self.bh = bh
        matrix._batches.add(self)

    def close(self):
        if self.bh:
            lib().am24_batch_destroy(self.matrix.solver.h, self.bh)
            self.bh = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load(self, V=None, device_ptr=None):
        if device_ptr is not None:
            check(lib().am24_batch_load(self.matrix.solver.h, self.bh, C.c_void_p(device_ptr), 1))
        else:
            V = np.asfortranarray(V, np.float32)
            assert V.shape == (self.matrix.n, self.k)
            check(lib().am24_batch_load(self.matrix.solver.h, self.bh, _ptr(V), 0))

    def iterate(self, it0=0, iterations=1, sync=True):
        me = C.c_float()
        check(lib().am24_batch_iterate(self.matrix.solver.h, self.bh, int(it0), int(iterations),
                                       C.byref(me) if sync else None))
        return me.value if sync else None

    def iterate_static_ws(self, it0=0, iterations=1, sync=True):
        """iterate() with the split-K workspace in the library's static device
        array (am24_batch_iterate_static_ws)."""
        me = C.c_float()
        check(lib().am24_batch_iterate_static_ws(self.matrix.solver.h, self.bh, int(it0),
                                                 int(iterations),
                                                 C.byref(me) if sync else None))
        return me.value if sync else None

    def read(self):
        n, k = self.matrix.n, self.k
        V = np.zeros((n, k), np.float32, order="F")
        val = np.zeros(k, np.float32)
        err = np.zeros(k, np.float32)
        nnz = np.zeros(k, np.uint32)
        check(lib().am24_batch_read(self.matrix.solver.h, self.bh, _ptr(V), _ptr(val), _ptr(err),
                                    _ptr(nnz)))
        return V, val, err, nnz

    def step_timed(self, it=0):
        """One step with per-kernel CUDA-event durations: [(kind, ms), ...]."""
        ms = (C.c_float * 16)()
        kinds = (C.c_int32 * 16)()
        cnt = C.c_int32()
        check(lib().am24_batch_step_timed(self.matrix.solver.h, self.bh, int(it), ms, kinds,
                                          C.byref(cnt)))
        out = []
        for i in range(cnt.value):
            k = kinds[i]
            name = KERNEL_KINDS[k & 0xFF] + ("(skipped)" if k & 0x100 else "")
            out.append((name, ms[i]))
        return out

    def refining(self):
        """False while a MIXED batch steps with BF16 operands, True after it
        switched to the FP32-accurate products (and always for FP32 batches)."""
        v = C.c_int32()
        check(lib().am24_batch_phase(self.matrix.solver.h, self.bh, C.byref(v)))
        return bool(v.value)

    def launches_per_step(self):
        v = C.c_int32()
        check(lib().am24_batch_launches_per_step(self.matrix.solver.h, self.bh, C.byref(v)))
        return v.value


class Group:
    """Many independent problems solved together (am24_group_*): every step of
    every problem runs in one set of grouped launches inside one captured CUDA
    graph that loops on the device until all have stopped."""

    def __init__(self, solver, capacity=256):
        self.solver = solver
        gh = C.c_void_p()
        check(lib().am24_group_create(solver.h, int(capacity), C.byref(gh)))
        self.gh = gh
        self.problems = {}  # id -> (matrix, k)
        solver._groups.add(self)

    def close(self):
        if self.gh:
            lib().am24_group_destroy(self.gh)
            self.gh = None
            self.problems = {}
            self.solver._groups.discard(self)

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, matrix, settings, start_points=None):
        """One problem: all of settings.totalStartingPoints starts as one batch."""
        s = settings.to_c()
        sp = None if start_points is None else np.asfortranarray(start_points, np.float32)
        pid = C.c_uint32()
        check(lib().am24_group_add(self.gh, matrix.mh, C.byref(s), _ptr(sp), C.byref(pid)))
        chk = settings.to_c()
        check(lib().am24_check_input(C.byref(chk), matrix.n))
        self.problems[pid.value] = (matrix, int(chk.total_starts))
        return pid.value

    def run(self, max_steps=0):
        """Runs until every problem has stopped (or max_steps steps); returns the
        launch's device time in ms."""
        ms = C.c_float()
        check(lib().am24_group_run(self.gh, int(max_steps), C.byref(ms)))
        return ms.value

    def state(self, pid):
        stopped, steps = C.c_int32(), C.c_uint32()
        check(lib().am24_group_state(self.gh, int(pid), C.byref(stopped), C.byref(steps)))
        return bool(stopped.value), steps.value

    def result(self, pid):
        matrix, _ = self.problems[pid]
        x = np.zeros(matrix.n, np.float32)
        st = am24_statistics()
        check(lib().am24_group_result(self.gh, int(pid), _ptr(x), C.byref(st)))
        return x, st

    def read(self, pid):
        matrix, k = self.problems[pid]
        V = np.zeros((matrix.n, k), np.float32, order="F")
        val = np.zeros(k, np.float32)
        err = np.zeros(k, np.float32)
        nnz = np.zeros(k, np.uint32)
        check(lib().am24_group_read(self.gh, int(pid), _ptr(V), _ptr(val), _ptr(err), _ptr(nnz)))
        return V, val, err, nnz

    def remove(self, pid):
        check(lib().am24_group_remove(self.gh, int(pid)))
        self.problems.pop(pid, None)

    def set_autotune(self, on=True):
        """Tiles of problems added from now on chosen by timing (am24_group_set_autotune)."""
        check(lib().am24_group_set_autotune(self.gh, 1 if on else 0))


def autotune_save(path):
    check(lib().am24_autotune_save(os.fsencode(path)))


def autotune_load(path):
    check(lib().am24_autotune_load(os.fsencode(path)))


def autotune_clear():
    check(lib().am24_autotune_clear())


class Server:
    """A serving loop (am24_server_*): resident matrices under an HBM budget,
    queued solves batched on arrival by a worker thread."""

    def __init__(self, device=0, hbm_budget_bytes=150 << 30):
        sh = C.c_void_p()
        check(lib().am24_server_create(int(device), int(hbm_budget_bytes), C.byref(sh)))
        self.sh = sh
        self.shapes = {}

    def close(self):
        if self.sh:
            lib().am24_server_destroy(self.sh)
            self.sh = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_matrix(self, B=None, on_device_ptr=None, m=None, n=None, ldB=None):
        mid = C.c_uint32()
        if on_device_ptr is None:
            B = np.asfortranarray(B, np.float32)
            m, n = B.shape
            check(lib().am24_server_add_matrix_f32(self.sh, _ptr(B), m, m, n, 0, C.byref(mid)))
        else:
            check(lib().am24_server_add_matrix_f32(self.sh, C.c_void_p(on_device_ptr), ldB or m,
                                                   m, n, 1, C.byref(mid)))
        self.shapes[mid.value] = (m, n)
        return mid.value

    def remove_matrix(self, matrix_id):
        check(lib().am24_server_remove_matrix(self.sh, int(matrix_id)))
        self.shapes.pop(matrix_id, None)

    def submit(self, matrix_id, settings, start_points=None):
        s = settings.to_c()
        sp = None if start_points is None else np.asfortranarray(start_points, np.float32)
        t = C.c_uint64()
        check(lib().am24_submit(self.sh, int(matrix_id), C.byref(s), _ptr(sp), C.byref(t)))
        return (t.value, matrix_id)

    def poll(self, ticket):
        """(done, x, stats); x and stats are None while the request runs."""
        t, mid = ticket
        x = np.zeros(self.shapes[mid][1], np.float32)
        st = am24_statistics()
        done = C.c_int32()
        check(lib().am24_poll(self.sh, t, _ptr(x), C.byref(st), C.byref(done)))
        return (True, x, st) if done.value else (False, None, None)

    def wait(self, ticket):
        t, mid = ticket
        x = np.zeros(self.shapes[mid][1], np.float32)
        st = am24_statistics()
        check(lib().am24_wait(self.sh, t, _ptr(x), C.byref(st)))
        return x, st


def header_symbols():
    """Entry points declared in include/am24.h."""
    import re
    src = open(os.path.join(INCLUDE, "am24.h")).read()
    return sorted(set(re.findall(r"^\s*(?:[a-z_0-9]+\s*\*?\s+)+\*?(am24_[a-z_0-9]+)\s*\(",
                                 src, re.M)))
