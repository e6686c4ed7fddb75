/*
 * am24.h -- C ABI of the B200-native alternating-maximization (AM) sparse-PCA
 * core.  Plain C types only (no CUDA or torch types), so any FFI can bind it.
 *
 * The library replaces the reference's (optml/24am) dense AM solver:
 *   SPCASolver::MulticoreSolver::denseDataSolver<F>(const F* B, int ldB, F* x,
 *       unsigned m, unsigned n, OptimizationSettings*, OptimizationStatistics*)
 *       -- c++/src/gpower/sparse_PCA_solver.h:36-40
 *   SPCASolver::GPUSolver::denseDataSolver<F>(cublasHandle_t&, m, n,
 *       thrust::device_vector<F>& d_B, thrust::host_vector<F>& h_x, settings*,
 *       stats*, LD_M, LD_N) -- c++/src/gpugpower/gpu_sparse_PCA_solver.h:29-35
 * The C++ adapter in include/am24/sparse_PCA_solver.h keeps those exact
 * signatures on top of this ABI.
 *
 * Conventions (as in the reference): B is the m x n data matrix, m samples by
 * n features, column-major with leading dimension ldB >= m.  x receives the n
 * loadings of the best starting point, normalised to unit 2-norm.  Each
 * starting point is an n-vector; a batch of them is n x k column-major.
 *
 * Every call returns an am24_status; am24_last_error() describes the last
 * failure on the calling thread.  Handles are independent (one CUDA stream
 * each); one handle must not be used from two threads at once.
 */
#ifndef AM24_H
#define AM24_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AM24_ABI_VERSION 1

typedef enum {
  AM24_OK = 0,
  AM24_ERR_INVALID_ARG = 1,    /* bad size, pointer, formulation or parameter */
  AM24_ERR_OOM = 2,            /* device allocation failed */
  AM24_ERR_CUDA = 3,           /* CUDA runtime/driver error */
  AM24_ERR_DEVICE_TIMEOUT = 4, /* a bounded device-side wait gave up */
  AM24_ERR_UNSUPPORTED = 5,    /* device is not sm_100 or feature not built */
  AM24_ERR_DEGENERATE = 6,     /* informational: some start produced a NaN objective */
  AM24_ERR_ADMISSION_REJECTED = 7 /* a server's HBM budget cannot hold the matrix or request */
} am24_status;

/* SPCA_Formulation (c++/src/class/optimization_settings.h:27-37), same values. */
typedef enum {
  AM24_L0_CONSTRAINED_L2_PCA = 0,
  AM24_L0_CONSTRAINED_L1_PCA = 1,
  AM24_L1_CONSTRAINED_L2_PCA = 2,
  AM24_L1_CONSTRAINED_L1_PCA = 3,
  AM24_L0_PENALIZED_L2_PCA = 4,
  AM24_L0_PENALIZED_L1_PCA = 5,
  AM24_L1_PENALIZED_L2_PCA = 6,
  AM24_L1_PENALIZED_L1_PCA = 7
} am24_formulation;

/* Arithmetic of the two products (an extension: the reference computes in F).
 * FP32: FP32-accurate products every iteration (split FP16 operands with
 * power-of-two scales on batches of more than 128 starts, 3xTF32 on narrower
 * ones; the residual of each split is below 2^-22 of the value, or 2^-39 of its
 * row's largest).  MIXED: single-pass V = B^T Z (one FP16 MMA per product on
 * the scaled h0 / g0 planes, 11 significant bits per operand; single-pass BF16
 * with the environment switch AM24_MIXED_BF16=1) with FP32 accumulation while
 * the supports settle, then the FP32-accurate products from
 * the first iteration after which a share stable_share of the batch's starts
 * has kept the same support for stable_iterations iterations; the tolerance
 * test applies only from then on.  With lead_iterations = L > 0 the first L
 * iterations run the FP32-accurate products (their tolerance test applies)
 * before the single-pass phase begins.  MIXED needs batches of more than 128 starts
 * (CTA-pair tiles); smaller batches run FP32 throughout. */
typedef enum { AM24_PRECISION_FP32 = 0, AM24_PRECISION_MIXED = 1 } am24_precision;

/* How starting points are produced. */
typedef enum {
  AM24_START_REFERENCE = 0, /* the reference generator: rand_r seeded with the global
                               start index (c++/src/gpower/gpower_commons.h:22-47) */
  AM24_START_INJECTED = 1,  /* caller-supplied n x total_starts matrix */
  AM24_START_DEVICE_UNIFORM = 2 /* generated on the device: U[-1, 1] per entry from
                                   the splitmix64 mixer of (global start index, row),
                                   column normalised (batch mode only) */
} am24_start_mode;

/* L1-constraint projection (the soft-thresholding level w). */
typedef enum {
  AM24_L1_REFERENCE_SCAN = 0, /* the reference's first-break scan
                                 (c++/src/utils/thresh_functions.h:162-218) */
  AM24_L1_EXACT = 1           /* exact ||x||_1/||x||_2 = sqrt(s) projection */
} am24_l1_mode;

/* Mirror of OptimizationSettings (c++/src/class/optimization_settings.h:71-123),
 * fields the dense AM path reads, fixed-width.  am24_default_settings() gives the
 * reference's defaults.  total_starts, batch_size, constraint, total_batches and
 * store_all are rewritten by a solve exactly as the reference rewrites them. */
typedef struct {
  int32_t formulation;     /* am24_formulation */
  uint32_t constraint;     /* constraintParameter s (default 10) */
  double penalty;          /* penaltyParameter gamma (default 0) */
  double tolerance;        /* default 0.01 */
  int32_t max_iter;        /* maximumIterations (default 20) */
  int32_t total_starts;    /* totalStartingPoints (default 64) */
  int32_t batch_size;      /* batchSize (default 64) */
  int32_t use_otf;         /* useOTF (default 0) */
  int32_t use_sort_hard;   /* useSortForHardThresholding (default 0) */
  int32_t store_all;       /* storeIterationsForAllPoints (default 0) */
  uint32_t total_batches;  /* totalBatches: output */
  int32_t verbose;
  /* extensions */
  int32_t start_mode;      /* am24_start_mode (default AM24_START_REFERENCE) */
  int32_t l1_mode;         /* am24_l1_mode (default AM24_L1_REFERENCE_SCAN) */
  uint32_t timeout_ms;     /* bound on any device-side wait (default 5000) */
  int32_t precision;       /* am24_precision (default AM24_PRECISION_FP32) */
  uint32_t stable_iterations; /* AM24_PRECISION_MIXED: iterations a start's
                                 support must stay unchanged (default 5) ... */
  float stable_share;         /* ... in this share of the batch's starts before the
                                 batch refines (default 1: every start) */
  uint32_t lead_iterations;   /* AM24_PRECISION_MIXED: FP32-accurate iterations run
                                 before the single-pass phase starts (default 0);
                                 supports are counted stable only from then on */
  uint32_t reserved[3];
} am24_settings;

/* Mirror of OptimizationStatistics (c++/src/class/optimization_statistics.h:27-46).
 * The per-start arrays are caller-provided (NULL = not wanted) with capacity
 * per_start_capacity; they are filled when settings.store_all is set, as the
 * reference fills values/iters/cardinalities. */
typedef struct {
  uint32_t it;                         /* total (batch-)iterations */
  double fval;                         /* best objective (the return value) */
  double error;                        /* last batch-maximum relative change */
  double total_true_computation_time;  /* seconds spent iterating */
  double total_elapsed_time;           /* seconds for the whole call */
  uint32_t n;                          /* length of x */
  int32_t total_threads_used;          /* 1 (one device stream) */
  double *values;
  int32_t *iters;
  int32_t *cardinalities;
  uint32_t per_start_capacity;
  /* extensions */
  double explained_variance;  /* ||B x||_2^2 of the returned x, FP64 on the device */
  uint64_t start_iterations;  /* AM steps summed over starting points */
  int32_t degenerate_starts;  /* starts whose final objective was NaN */
  uint32_t low_precision_iterations; /* batch iterations run with single-pass operands */
  int32_t input_rounded_to_f32;       /* 1 when FP64 input was rounded to FP32 before
                                         the solve (am24_solve_dense_f64): the result is
                                         the FP32 solve of the rounded data */
  uint32_t reserved[5];
} am24_statistics;

typedef struct am24_handle_s *am24_handle;
typedef struct am24_matrix_s *am24_matrix;
typedef struct am24_batch_s *am24_batch;

/* ---- library / handle ---------------------------------------------------- */
uint32_t am24_abi_version(void);
const char *am24_last_error(void);
const char *am24_status_string(am24_status s);
void am24_default_settings(am24_settings *s);
/* chceckInputAndModifyIt (c++/src/class/optimization_settings.h:156-168):
 * s <= n, batch 0 -> total, total rounded up to whole batches. Host only. */
am24_status am24_check_input(am24_settings *s, uint32_t n);

/* A handle owns a stream on `device`.  Every entry point that takes a handle
 * (or a server) makes that device current on the calling thread
 * (cudaSetDevice) and leaves it current on return: a caller that drives other
 * devices from the same thread sets its own device again afterwards. */
am24_status am24_create(am24_handle *h, int device);
am24_status am24_destroy(am24_handle h);

/* ---- one-call solves (drop-in for denseDataSolver) ------------------------ */
/* Host B, host x.  start_points (n x total_starts after rounding, column-major)
 * is read when settings->start_mode == AM24_START_INJECTED, else ignored.
 * *fval_out (may be NULL) receives the returned objective. */
am24_status am24_solve_dense_f32(am24_handle h, const float *B, int32_t ldB, float *x,
                                 uint32_t m, uint32_t n, am24_settings *settings,
                                 am24_statistics *stats, const float *start_points,
                                 float *fval_out);
/* Same with B already in device memory (the reference GPU console's entry,
 * c++/src/gpugpower/gpu_sparse_PCA_solver.h:29-35): d_B column-major with
 * leading dimension ldB (the reference pads it to 128 B: LD_M). */
am24_status am24_solve_device_f32(am24_handle h, const float *d_B, int32_t ldB, float *x,
                                  uint32_t m, uint32_t n, am24_settings *settings,
                                  am24_statistics *stats, const float *start_points,
                                  float *fval_out);

/* FP64 host data (the reference's denseDataSolver<double> call).  There is no
 * FP64 arithmetic on this path: B, x and the injected starts are rounded to
 * FP32 (relative error up to 2^-24 per entry) and solved as
 * am24_solve_dense_f32 does; x and *fval_out are returned in double and
 * stats->input_rounded_to_f32 is set to 1, so a caller that asked for double
 * can tell.  The objective and explained variance then differ from an FP64
 * solve of the unrounded data by the rounding's effect (about 1e-7 relative on
 * well-conditioned data). */
am24_status am24_solve_dense_f64(am24_handle h, const double *B, int32_t ldB, double *x,
                                 uint32_t m, uint32_t n, am24_settings *settings,
                                 am24_statistics *stats, const double *start_points,
                                 double *fval_out);

/* ---- resident data matrices ---------------------------------------------- */
/* Copies B (host, or device when on_device != 0) into the handle's layout and
 * keeps it until am24_matrix_destroy. */
am24_status am24_matrix_create_f32(am24_handle h, const float *B, int32_t ldB, uint32_t m,
                                   uint32_t n, int32_t on_device, am24_matrix *out);
/* A resident matrix from compressed sparse columns, the input of the
 * reference's sparse solver (sparse_PCA_solver_CSC, c++/src/gpower/
 * sparse_PCA_solver_for_CSC.h:111-117): vals and row_ind (col_ptr[n] entries,
 * 0-based rows, at most one entry per row within a column) and col_ptr (n + 1,
 * col_ptr[0] = 0), host arrays.  means (n floats) and row_means (m floats) are
 * optional (NULL: no correction) and stand for its doMean / doRowMean: the
 * matrix solved is B - 1 means^T - row_means 1^T.  Here it is densified on the
 * device with the corrections applied to every entry ((b - means_c) -
 * row_means_i in FP32), after which every solve runs on the dense tensor-core
 * path.  Malformed CSC arrays are rejected on the host before anything is
 * copied.  The dense matrix must fit in device memory (AM24_ERR_OOM). */
am24_status am24_matrix_create_csc_f32(am24_handle h, const float *vals, const int32_t *row_ind,
                                       const int32_t *col_ptr, uint32_t m, uint32_t n,
                                       const float *means, const float *row_means,
                                       am24_matrix *out);
/* The same input kept compressed on the device, for matrices whose dense form
 * does not fit (or is mostly zeros): the reference's sparse_PCA_solver_CSC
 * (c++/src/gpower/sparse_PCA_solver_for_CSC.h:111-117) holds B only as CSC
 * too.  Device memory is 16 bytes per non-zero (CSC plus a CSR copy built on
 * the host) and the centring vectors; a solve adds 4 (3 n + 2 m) bytes per
 * start of its batch.  The centring is applied implicitly as rank-one
 * corrections of both products (the reference's doMean / doRowMean arithmetic,
 * :223-248, :277-309, here with the corrections' sums in FP64).  Rows within a
 * column need not be sorted: such columns are sorted on the host and duplicate
 * (row, column) entries added up in entry order.  Such a matrix is solved by
 * am24_solve_resident_f32 (batch mode: the dense path's iteration, both
 * products as FP32 kernels on the compressed arrays, AM24_PRECISION_MIXED runs
 * as FP32; use_otf returns AM24_ERR_UNSUPPORTED).  am24_matrix_deflate records
 * each x as the next factor of B (I - x_1 x_1^T) ... (I - x_C x_C^T) (at most
 * 32), applied to the loadings before Z = B V and to B^T Z after it, so the
 * arrays stay as uploaded; the batch, group and read entry points return
 * AM24_ERR_UNSUPPORTED for such a matrix. */
am24_status am24_matrix_create_csc_sparse_f32(am24_handle h, const float *vals,
                                              const int32_t *row_ind, const int32_t *col_ptr,
                                              uint32_t m, uint32_t n, const float *means,
                                              const float *row_means, am24_matrix *out);
am24_status am24_matrix_destroy(am24_handle h, am24_matrix mat);
am24_status am24_solve_resident_f32(am24_handle h, am24_matrix mat, float *x,
                                    am24_settings *settings, am24_statistics *stats,
                                    const float *start_points, float *fval_out);
/* Deflation for the next component: B <- B (I - x x^T) on the device, the
 * update the reference's multi-component driver applies between solves
 * (c++/matlab/run_example.m:33-34, in double).  Here y = B x is summed in
 * FP64 and each entry becomes (float)(b - y_i x_c) in FP64.  x (n floats, host
 * or device when on_device != 0) is normally the last solve's unit loading.
 * Every layout the matrix holds is rebuilt in place, so batches created on it
 * stay valid; work already queued on the handle's stream sees the old B, work
 * queued after it the new one, and work on other handles must not use the
 * matrix meanwhile.  A sparse-resident matrix keeps its arrays and records x as
 * the next factor instead (am24_matrix_create_csc_sparse_f32). */
am24_status am24_matrix_deflate(am24_handle h, am24_matrix mat, const float *x,
                                int32_t on_device);
/* Copies the matrix's current B (m x n, column-major, leading dimension ldB >=
 * m) to host memory: the data as uploaded, or as deflated. */
am24_status am24_matrix_read_f32(am24_handle h, am24_matrix mat, float *B, int32_t ldB);

/* ---- batch stepping (one AM iteration at a time) -------------------------- */
/* A batch of batch_size starting points on a resident matrix.  `settings` must
 * already have passed am24_check_input. */
am24_status am24_batch_create(am24_handle h, am24_matrix mat, const am24_settings *settings,
                              uint32_t batch_size, am24_batch *out);
am24_status am24_batch_destroy(am24_handle h, am24_batch b);
/* Loads n x batch_size starting points (host, or device when on_device != 0)
 * and resets the per-start values to 0 (ValueCoordinateHolder::reset). */
am24_status am24_batch_load(am24_handle h, am24_batch b, const float *V, int32_t on_device);
/* Runs `iterations` AM steps with iteration indices it0, it0+1, ... on the
 * handle's stream.  When max_error is non-NULL the call synchronizes and
 * stores the batch-maximum relative change of the last step there. */
am24_status am24_batch_iterate(am24_handle h, am24_batch b, int32_t it0, int32_t iterations,
                               float *max_error);
/* Copies the current state to the host (any pointer may be NULL): loadings
 * V (n x batch_size), per-start objective val, relative change err and
 * number of non-zero loadings nnz. */
am24_status am24_batch_read(am24_handle h, am24_batch b, float *V, float *val, float *err,
                            uint32_t *nnz);
/* No counterpart in the reference.  The step of am24_batch_iterate, with the
 * split-K partial sums of the dense Z = B V product kept in a file-scope device
 * array of AM24_STATIC_WS_BYTES inside the library instead of the batch's own
 * workspace; the call allocates no memory.  Batches whose workspace is larger
 * (splits x ceil(m/128) x ceil(batch_size/bn) x bn x 128 floats, bn the GEMM
 * N tile) are rejected with AM24_ERR_INVALID_ARG.  The array needs no
 * initial contents.  There is one array per device: calls that overlap in time
 * on one device, from any handle or thread, race on it.  The first call on a
 * device looks up the array's address (set-up); make it before any stream
 * capture. */
#define AM24_STATIC_WS_BYTES (16u << 20)
am24_status am24_batch_iterate_static_ws(am24_handle h, am24_batch b, int32_t it0,
                                         int32_t iterations, float *max_error);
/* AM24_PRECISION_MIXED batches: *refining = 0 while the batch's next step
 * uses single-pass operands, 1 when it runs the FP32-accurate products (the
 * lead-in steps, and every step after the switch); FP32 batches report 1.
 * Synchronizes the handle's stream. */
am24_status am24_batch_phase(am24_handle h, am24_batch b, int32_t *refining);
/* Number of kernel launches one am24_batch_iterate step issues. */
am24_status am24_batch_launches_per_step(am24_handle h, am24_batch b, int32_t *launches);
/* Diagnostic of the device-side timeouts: runs a kernel whose wait nothing
 * satisfies, bounded by timeout_us.  It gives up, reports as a timed-out solve
 * does (returns AM24_ERR_DEVICE_TIMEOUT, the expected outcome) and leaves the
 * handle usable.  Synchronizes the handle's stream. */
am24_status am24_selftest_bounded_wait(am24_handle h, uint32_t timeout_us);
/* Synchronizes the handle's stream. */
am24_status am24_sync(am24_handle h);
/* The handle's CUDA stream (a cudaStream_t), for callers that record their own
 * events around library work. */
void *am24_stream(am24_handle h);

/* ---- serving: resident matrices, continuous batching of solve requests ---- */
/* No counterpart in the reference.  A server owns a handle on `device` and one
 * engine thread that serves requests with a group (am24_group_*): requests
 * are admitted, oldest first, into the running group at step boundaries
 * (every AM24_SERVER_CHUNK grouped steps) while their device memory fits the
 * budget left beside the resident matrices and the requests already on the
 * device; every admitted request steps together with the others, and leaves
 * as soon as its own batch loop ends (its x, statistics and memory are then
 * released).  Each request is one batch of all its starting points
 * (batchSize = totalStartingPoints) that stops on its own largest change, as a
 * reference batch does, with tiles and reduction order of its own: its result
 * is the same bit for bit whatever else is served beside it.  Matrices are
 * admitted while their device layouts fit hbm_budget_bytes.
 * settings->use_otf and store_all are not supported by the server. */
#define AM24_SERVER_WORKERS 1 /* engine threads per server */
#define AM24_SERVER_CHUNK 4   /* grouped steps between admissions */
typedef struct am24_server_s *am24_server;
am24_status am24_server_create(int device, uint64_t hbm_budget_bytes, am24_server *out);
/* Finishes queued requests, then frees everything the server holds. */
am24_status am24_server_destroy(am24_server s);
/* Copies B (host, or device when on_device != 0) into a resident matrix;
 * AM24_ERR_ADMISSION_REJECTED when its layouts do not fit the budget left. */
am24_status am24_server_add_matrix_f32(am24_server s, const float *B, int32_t ldB, uint32_t m,
                                       uint32_t n, int32_t on_device, uint32_t *matrix_id);
/* Frees a resident matrix; AM24_ERR_INVALID_ARG while requests for it are pending. */
am24_status am24_server_remove_matrix(am24_server s, uint32_t matrix_id);
/* Queues a solve of `settings` (copied, after am24_check_input) on a resident
 * matrix; start_points (n x total_starts, copied) is read for
 * AM24_START_INJECTED.  AM24_ERR_ADMISSION_REJECTED when the request's batch
 * can never fit the budget.  Returns at once with a ticket. */
am24_status am24_submit(am24_server s, uint32_t matrix_id, const am24_settings *settings,
                        const float *start_points, uint64_t *ticket);
/* Non-blocking: *done = 1 once the request finished, then x (n floats) and
 * stats (may be NULL) are filled, the ticket is released and the request's own
 * status is returned; *done = 0 otherwise.  stats->total_elapsed_time is the
 * time from submission to completion. */
am24_status am24_poll(am24_server s, uint64_t ticket, float *x, am24_statistics *stats,
                      int32_t *done);
/* Blocking form of am24_poll. */
am24_status am24_wait(am24_server s, uint64_t ticket, float *x, am24_statistics *stats);

/* ---- groups: many independent problems in one set of launches per step --- */
/* No counterpart in the reference, which solves one problem per call; its
 * batch loop (c++/src/gpower/sparse_PCA_solver.h:171-232) is what each
 * problem of a group runs.  A group holds up to `capacity` problems of uneven
 * shape: each is one batch of starting points on a resident matrix with its
 * own settings (formulation, s or gamma, tolerance, max_iter, precision).  A
 * run repeats one grouped AM step for every problem that still iterates --
 * one plan kernel, then each product of all problems' tiles as one persistent
 * grouped tensor-core kernel (CTA pairs, split FP16 operands, or single-pass
 * BF16 in a MIXED problem's first phase) and every per-start pass as one
 * kernel over all problems' starts -- inside one captured CUDA graph whose
 * WHILE node loops on the device until every problem has stopped, with no
 * host round trip per step.  Each problem stops as a reference batch does
 * (it > 0, largest change below the tolerance, in the refinement phase; or
 * max_iter steps).  Its tiles, split-K and reduction order depend on it
 * alone, so its result is the same bit for bit alone and among others.
 * A group belongs to one handle and runs on its stream; destroy it before the
 * handle, and remove a matrix's problems (or destroy the group) before the
 * matrix. */
typedef struct am24_group_s *am24_group;
am24_status am24_group_create(am24_handle h, uint32_t capacity, am24_group *out);
/* Waits for the handle's stream, then frees every problem and the group. */
am24_status am24_group_destroy(am24_group g);
/* Adds one problem on resident matrix `mat` (which must outlive it): all of
 * settings->total_starts starting points (after am24_check_input) form one
 * batch.  start_mode REFERENCE, INJECTED (start_points: n x total_starts host
 * floats, copied) or DEVICE_UNIFORM; use_otf and store_all are not supported.
 * The problem's device memory comes from the handle's stream-ordered pool.
 * *problem receives its id (a slot index below capacity). */
am24_status am24_group_add(am24_group g, am24_matrix mat, const am24_settings *settings,
                           const float *start_points, uint32_t *problem);
/* Runs grouped steps of every added problem that has not stopped, until all
 * have stopped, or for at most max_steps steps when max_steps > 0.  One graph
 * launch; synchronizes the stream.  *device_ms (may be NULL) receives the
 * launch's device time (CUDA events on the handle's stream). */
am24_status am24_group_run(am24_group g, uint32_t max_steps, float *device_ms);
/* *stopped = 1 once the problem has stopped iterating, *steps its steps. */
am24_status am24_group_state(am24_group g, uint32_t problem, int32_t *stopped, uint32_t *steps);
/* The problem's best start (the largest objective, the first on ties),
 * normalised, into x (n floats), and its statistics (it = steps, fval, error,
 * explained_variance in FP64 on the device, start_iterations,
 * low_precision_iterations, degenerate_starts; times are the last run's). */
am24_status am24_group_result(am24_group g, uint32_t problem, float *x, am24_statistics *stats);
/* As am24_batch_read: the problem's loadings (n x k), objectives, changes and
 * non-zero counts (any pointer may be NULL). */
am24_status am24_group_read(am24_group g, uint32_t problem, float *V, float *val, float *err,
                            uint32_t *nnz);
/* Frees the problem's slot and device memory. */
am24_status am24_group_remove(am24_group g, uint32_t problem);
/* With on != 0, problems added from now on take tiles chosen by timing: the N
 * tile of both products (64, 128 or 256) and the split-K factor of the dense
 * Z = B V.  Problems fall into buckets of half an octave in m, n and k per
 * formulation mode; the first problem of a bucket is timed in a scratch group
 * under each candidate (three steps each, from device-generated starts) and
 * the fastest is kept in a process-wide table that every later problem of the
 * bucket uses.  Off (the default), the tiles come from a fixed cost model.
 * A problem's result depends on its tiles only through FP32 summation order. */
am24_status am24_group_set_autotune(am24_group g, int32_t on);
/* The autotuner's table: written to / merged from a text file (one line per
 * bucket), or emptied. */
am24_status am24_autotune_save(const char *path);
am24_status am24_autotune_load(const char *path);
am24_status am24_autotune_clear(void);

/* Kernel kinds reported by am24_batch_step_timed. */
typedef enum {
  AM24_KERNEL_GEMM_BV = 0,   /* Z = B V, tensor cores, split-K partial tiles */
  AM24_KERNEL_Z_REDUCE = 1,  /* split-K sum, sign / norm / normalise of Z */
  AM24_KERNEL_GEMM_BTZ = 2,  /* V = B^T Z, tensor cores (+ penalty epilogue) */
  AM24_KERNEL_SELECT = 3,    /* top-s select or L1-ball level, normalise (constrained) */
  AM24_KERNEL_FINALIZE = 4,  /* per-start objective, change, logs, batch maximum */
  AM24_KERNEL_GATHER_BV = 5, /* Z = B V as a gather over V's non-zeros (sparse steps) */
  AM24_KERNEL_DENSIFY = 6,   /* dense planes of V (FP16 or TF32) for the tensor-core Z = B V */
  AM24_KERNEL_GEMM_BTZ_LOW = 7, /* V = B^T Z with single-pass operands (MIXED's first
                                   phase: FP16, or BF16 with AM24_MIXED_BF16=1) */
  AM24_KERNEL_GEMM_BTZ_BF16 = 7, /* the same kind under its earlier name */
  AM24_KERNEL_SUPPORT = 8,   /* support-stability count and phase switch (MIXED) */
  AM24_KERNEL_GATHER_BV_GROUP = 9, /* the gather for four starts per block (few non-zeros) */
  AM24_KERNEL_SKIPPED = 0x100 /* or-ed into a kind: the launch returned at once */
} am24_kernel_kind;
/* One AM step like am24_batch_iterate(h, b, it, 1, NULL), with a CUDA event
 * recorded on the handle's stream before and after every kernel.  Synchronizes,
 * then writes each launch's duration (ms) to ms[i] and its am24_kernel_kind to
 * kinds[i] (both with room for 16) and the number of launches to *count.  Z = B V
 * has two paths per step (gather; or densify + tensor-core GEMM + reduction);
 * the kernels of the path the step does not need return at once. */
am24_status am24_batch_step_timed(am24_handle h, am24_batch b, int32_t it, float *ms,
                                  int32_t *kinds, int32_t *count);

#ifdef __cplusplus
}
#endif
#endif /* AM24_H */
