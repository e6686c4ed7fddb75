// Internal declarations shared by the kernels (am24_kernels.cu) and the host
// driver (am24_api.cu).  Not part of the public ABI.
#pragma once
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

namespace am24 {

// GEMM tiling: M tile is fixed at 128 (one TMEM lane per accumulator row).
constexpr int BM = 128;
// K slab per pipeline stage: 32 (128-byte rows, 128B swizzle, fewer deeper
// stages) or 16 (64-byte rows, 64B swizzle, twice the stages).
constexpr int BK_DEFAULT = 16;
constexpr int PAIR_BK_TF32 = 16;  // K elements per 64-byte row: TF32 pair scheme
constexpr int PAIR_BK_BF16 = 32;  // and BF16 pair scheme

// Formulation helpers (c++/src/class/optimization_settings.h:125-153).
inline bool is_constrained(int f) { return f >= 0 && f <= 3; }
inline bool is_l1_constrained(int f) { return f == 2 || f == 3; }
inline bool is_l1_variance(int f) { return f == 1 || f == 3 || f == 5 || f == 7; }
inline bool is_l1_penalized(int f) { return f == 6 || f == 7; }

// Layout of one resident data matrix.  B (m x n) is kept as FP32 in Bc, and
// the products' operand planes are made from it in two K-major orientations
// when a batch first needs them:
//   Bc: n rows (features) of m samples, leading dimension ldm  -> A of V = B^T Z
//   Bt: m rows (samples) of n features, leading dimension ldn  -> A of Z = B V
struct MatrixDev {
  int m, n, ldm, ldn;
  // TF32 hi/lo planes of Bc and Bt for the 3xTF32 products; made when a batch
  // first needs them (null before)
  float *Bc_hi, *Bc_lo, *Bt_hi, *Bt_lo;
  float *Bc;  // plain FP32 B, n rows of ldm samples (pad rows zero): the gather
              // Z = B V, the explained variance and every other layout read it
  // Three BF16 planes of Bc (plane p at Bc_b3 + p * n * ldm) with
  // x = b0 + b1 + b2 exactly; made when a batch of an L1-variance form first
  // needs them (null before).
  uint16_t *Bc_b3;
  int bf16_planes;  // planes Bc_b3 holds: 1 (b0 alone) or 3
  // Two FP16 planes of Bc scaled per feature (plane p at Bc_h2 + p * n * ldm):
  // x * 2^s_c = h0 + h1 (+ under 2^-22 |x|), row_scale[c] = 2^-s_c; made when a
  // batch first runs V = B^T Z on FP16 operands (null before).
  uint16_t *Bc_h2;
  float *row_scale;
  // The same for B^T (Z = B V): two FP16 planes of each sample's row of Bt,
  // scaled per sample (plane p at Bt_h2 + p * m * ldn), bt_row_scale[i] = 2^-s_i.
  uint16_t *Bt_h2;
  float *bt_row_scale;
};

// Per-batch device state for k starting points.
struct BatchDev {
  int k;          // starting points in the batch
  int bn1, bn2;   // GEMM N tiles (Z = B V and V = B^T Z)
  int bk;         // GEMM K slab (16 or 32)
  int splits1;    // split-K factor of Z = B V
  int kbps1;      // K blocks per split of Z = B V
  int m_tiles1, n_tiles1, m_tiles2, n_tiles2;
  int pair2;      // V = B^T Z runs on CTA pairs (256-row tiles; B maps of bn2/2 rows)
  int bf16_2;     // ... with the exact BF16 operands of the L1-variance forms
  int fp16_2;     // ... with the split FP16 operands (preferred over bf16_2 and TF32)
  int fp16_1;     // Z = B V on CTA pairs with split FP16 operands (split-K, splits1p)
  int splits1p;   // its split-K factor
  uint16_t *V_h;  // its B operand: two k x ldn FP16 planes (second at V_h + k * ldn)
                  // of v * 2^s_j, written by densify_fp16_kernel
  float *v_scale;            // per start 2^-s_j
  const float *bt_row_scale;  // the matrix's FP16 row scales of B^T
  size_t ws_len;  // floats in ws (the larger split-K layout)
  uint32_t *ctl;  // CTL_WORDS run-ahead control words
  // constrained forms: k x (ldn/32) words, the candidates of the hinted select
  // that V = B^T Z's epilogue marks (|v| at or above the bound of the column's
  // previous level)
  uint32_t *cmask;
  uint16_t *Z_h;  // FP16 Z for fp16_2: sgn(B V) exactly (one k x ldm plane, L1-variance
                  // forms), or two planes (second at Z_h + k * ldm) of z * 2^s_j
  float *z_scale;    // per start 2^-s_j (L2-variance forms with fp16_2)
  const float *row_scale;  // the matrix's FP16 row scales (fp16_2)
  uint16_t *Z_b;  // k x ldm BF16 Z: sgn(B V) exactly (L1-variance forms with bf16_2),
                  // or Z rounded to BF16 (MIXED); else null
  int mixed;             // MIXED precision: single-pass V = B^T Z until supports settle ...
  int mixed_fp16;        // ... on FP16 operands (the scaled h0 / g0 planes); else BF16
  uint32_t k_stable;     // steps of unchanged support a start needs ...
  uint32_t need_stable;  // ... in this many starts before the batch refines
  uint32_t lead;         // FP32-accurate steps before the single-pass phase
  uint32_t *vmask_prev;  // k x (ldn/32): the previous step's non-zero masks (MIXED)
  uint32_t *stable;      // per start: consecutive steps with an unchanged support (MIXED)
  uint32_t *phase;       // [0] 0 = BF16 phase, 1 = refinement (sticky), >= 2 the FP32
                         // lead-in ([0] - 1 steps left); [1] the step's count of
                         // stable starts; [2] blocks done (MIXED)
  float *Vx;            // k x ldn loadings; entry i of a column is defined only
                        // where its vmask bit is set (zero elsewhere)
  float *V_hi, *V_lo;   // k x ldn dense TF32 hi/lo planes of V: the B operand of the
                        // one-CTA tensor-core Z = B V, filled on dense steps only
                        // (null when Z = B V runs on the FP16 pairs)
  float *Z_hi, *Z_lo;   // k x ldm sample-space vectors z = hi + lo (the TF32 B
                        // operand of V = B^T Z, and the store the reductions re-read)
  float *Vraw;          // k x ldn raw B^T Z (constrained forms)
  float *ws;            // split-K partial tiles of Z = B V
  float *fz;            // per start: ||y||_2 or ||y||_1 from the Z reduction
  float *obj_part;      // per start x (m_tiles2*4): penalized objective partials
  float *nnz_part;      // per start x (m_tiles2*4): penalized non-zero partials
  uint32_t *nnz;        // per start: non-zeros after thresholding
  float *sel_hint;      // per start: last threshold level (0 = none), a search hint
  uint32_t *vmask;      // k x (ldn/32): bit r of word w set iff V[32w + r] != 0
  uint32_t *max_nnz;    // largest non-zero count of the last step (0xFFFFFFFF: dense V)
  uint32_t sparse_cap;  // Z = B V runs as a gather when max_nnz <= sparse_cap
  uint32_t *planes_nnz; // the max_nnz the previous step's penalty epilogue saw: above
                        // sparse_cap it wrote V_hi / V_lo (0 for constrained forms
                        // and after starts are loaded)
  float *val, *err;     // ValueCoordinateHolder val / current_error
  float *max_err;       // batch maximum relative change (1 float)
  int *iters, *cards;   // storeIterationsForAllPoints logs (total_starts each)
  int log_capacity;
  int *status;          // device status word (bounded-wait timeouts)
};

struct StepParams {
  int formulation;
  unsigned constraint;
  double penalty;
  double tolerance;
  int use_sort_hard;
  int l1_mode;
  int store_all;
  int it;             // iteration index within the batch (termination_criteria)
  int log_shift;      // batch shift of the per-start logs
  unsigned long long timeout_ns;
  int stop_check = 0;  // the step sets the stop word when the batch loop would end
};

// The sparse Z = B V runs four starts per block while no column has more
// than this many non-zeros (and the sparse bound allows the gather at all).
constexpr uint32_t GATHER_GROUP_MAX_NNZ = 1024;

// Run-ahead control words of a batch (BatchDev::ctl).  Every step kernel
// returns at once while ctl[CTL_STOP] is set, so a driver can queue steps
// ahead of the convergence test; a load clears the words.
enum : int {
  CTL_STOP = 0,       // set by the step that ends the batch loop (or a device timeout)
  CTL_STEPS = 1,      // steps executed since the load
  CTL_LOW_STEPS = 2,  // ... of them in the BF16 phase (MIXED)
  CTL_MAX_ERR = 3,    // the last executed step's largest change (float bits)
  CTL_BLOCKS = 4,     // finalize's block counter (scratch)
  CTL_WORDS = 8
};

struct TensorMaps {
  CUtensorMap a1_hi, a1_lo, b1_hi, b1_lo;  // Z = B V :  A = Bt, B = V
  CUtensorMap a2_hi, a2_lo, b2_hi, b2_lo;  // V = B^T Z: A = Bc, B = Z
  CUtensorMap a2_b0, a2_b1, a2_b2, b2_b;   // V = B^T Z, BF16: A = Bc_b3, B = Z_b
  CUtensorMap a2_h0, a2_h1, b2_h0, b2_h1;  // V = B^T Z, FP16: A = Bc_h2, B = Z_h
  CUtensorMap a1_h0, a1_h1, b1_h0, b1_h1;  // Z = B V, FP16: A = Bt_h2, B = V_h
};

// ---- grouped steps: many independent problems, one set of launches per step
//
// A problem is one batch of starting points on one resident matrix (its own
// formulation, s or gamma, tolerance, max_iter and precision).  Its device
// state is a GProblem; every kernel of a grouped step reads the list of the
// problems it serves from a GPlan that the step's first kernel writes, and
// loops over their work items (columns, groups of columns or GEMM tiles) with
// a grid sized to the GPU, not to the problems.  Every problem's arithmetic is
// a function of that problem alone (its own tiles, split-K and reduction
// order), so its result is the same bit for bit whatever else runs beside it.
enum GList : int {
  GL_GG0 = 0,  // sparse V with at most 1024 non-zeros: ceil(k / 4) items, by mode 0..2
  GL_GG1,
  GL_GG2,
  GL_GA0,      // sparse V with more non-zeros: k items, by mode
  GL_GA1,
  GL_GA2,
  GL_DN0,      // dense V (densify, then the split-K reduction): k items, by mode
  GL_DN1,
  GL_DN2,
  GL_SEL_HARD,   // k (top-s)
  GL_SEL_SCAN,   // k (L1 ball, the reference's scan)
  GL_SEL_EXACT,  // k (L1 ball, exact)
  GL_SUPPORT,    // k (MIXED support stability)
  GL_FIN,        // ceil(k / 8)
  GL_GEMM1_64,   // units of Z = B V on dense steps, by N tile (64, 128, 256)
  GL_GEMM1_128,
  GL_GEMM1_256,
  GL_RAW_64,     // units of V = B^T Z, by epilogue (raw: the constraints; L1 / L0
  GL_RAW_128,    // penalty) and N tile
  GL_RAW_256,
  GL_PL1_64,
  GL_PL1_128,
  GL_PL1_256,
  GL_PL0_64,
  GL_PL0_128,
  GL_PL0_256,
  GL_COUNT
};
// Epilogue of a grouped product's launch.
enum GEpi : int { GE_PARTIAL = 0, GE_RAW = 1, GE_PL1 = 2, GE_PL0 = 3 };
constexpr int FIN_STARTS = 8;  // starts per finalize item (a warp each)

// Operand schemes of the grouped V = B^T Z, chosen per problem and step.
enum GScheme : int { GS_FP16X3 = 0, GS_FP16X2A = 1, GS_FP16X1 = 2 };

// The tensor maps of one problem (a separate, 64-byte aligned table).
struct alignas(64) GMaps {
  CUtensorMap a1_h0, a1_h1, b1_h0, b1_h1;  // Z = B V: Bt FP16 planes, V FP16 planes
  CUtensorMap a2_h0, a2_h1, b2_h0, b2_h1;  // V = B^T Z: Bc FP16 planes, Z FP16 planes
};

struct GProblem {
  int live;  // 0: a free slot
  // matrix
  int m, n, ldm, ldn;
  const float *Bc;
  const float *row_scale, *bt_row_scale;  // FP16 plane scales of Bc (features), Bt (samples)
  // settings
  int k, formulation, mode;  // mode: 0 L2-variance constrained, 1 L1 variance, 2 L2 penalized
  int l1_exact, mixed, max_iter;
  unsigned constraint;
  float gamma;
  double tolerance;
  uint32_t sparse_cap, k_stable, need_stable;
  // tiles
  int bn;                          // N tile of both products (64, 128 or 256)
  int m_tiles1, n_tiles1, splits1, kb_per_split1;  // Z = B V (pair tiles, K blocks of 32)
  int m_tiles2, n_tiles2;          // V = B^T Z
  int parts;                       // m_tiles2 * 4 penalty partials per start
  // state
  float *Vx, *Vraw, *sel_hint, *Z_hi, *Z_lo, *fz, *obj_part, *nnz_part, *val, *err, *max_err;
  float *z_scale, *v_scale, *ws;
  uint32_t *vmask, *cmask, *nnz, *ctl, *stable, *phase;
  uint64_t *mask_hash;  // MIXED: per start, a hash of the last step's support
  uint16_t *Z_h, *Z_b, *V_h;
  size_t zplane;  // k * ldm: the second FP16 plane of Z
  int *status;
};

// Per-problem control words (GProblem::ctl), beyond the run-ahead words.
enum : int {
  GCTL_GATE = 8,     // the largest non-zero count of the previous step (this step's gate)
  GCTL_NEXT = 9,     // ... of this step, formed by finalize
  GCTL_SCHEME = 10,  // this step's GScheme for V = B^T Z
  GCTL_SUPPORT = 11, // MIXED: this step's stable starts (scratch)
  GCTL_SBLOCKS = 12, // MIXED: support items done (scratch)
  GCTL_WORDS = 16
};

// GPlan::status when a grouped work item named a slot out of range, a problem
// not live or an item past its problem's count (the item is skipped)
constexpr int DEV_ERR_GROUP_ITEM = 0x201;

struct GPlan {
  int n[GL_COUNT];      // problems in each list
  int total[GL_COUNT];  // work items in each list
  int active;           // problems that ran this step
  int loops;            // steps run since the last launch began
  int loop_cap;         // the launch stops after this many steps
  int status;           // a device-side wait of a grouped kernel gave up
  // per list, the next item a per-column kernel's block takes; the dense lists
  // are walked twice a step (densify, then the split-K reduction), which the
  // last three counters serve
  int next[GL_COUNT + 3];
};

// Device arrays of a group, sized for `cap` problems.
struct GroupDev {
  int cap;
  GProblem *probs;
  const GMaps *maps;
  GPlan *plan;
  int *prob;  // [GL_COUNT][cap]: the problems of each list
  int *pref;  // [GL_COUNT][cap + 1]: exclusive prefix of their items
  uint32_t *done;  // per slot after each step: 0 free, 1 iterating, 2 stopped
  const int *order;  // [cap]: the slots in the order the plan lists them (widest first)
  unsigned long long timeout_ns;
};

// One grouped AM step of every live, unstopped problem; the plan kernel first.
// grids: per-kernel persistent grid sizes (from grouped_grids()).
struct GroupGrids {
  int plan_threads, col, select_hard, select_soft, gather, gather_group, fin, pairs;
};
cudaError_t grouped_grids(GroupGrids *g);
cudaError_t launch_grouped_step(const GroupDev &g, const GroupGrids &grids, cudaStream_t st);
// Sets the WHILE condition of a captured loop: 1 while some problem is live and
// unstopped, the plan's loop count is below its cap and no wait gave up.
cudaError_t launch_grouped_condition(const GroupDev &g, unsigned long long handle,
                                     cudaStream_t st, bool in_graph = true);

// ---- sparse-resident matrices (am24_matrix_create_csc_sparse_f32)
// Outer entries (CSC columns, CSR rows) longer than SP_LONG entries are summed
// in segments of SP_SEG entries, many warps per entry, then combined in
// segment order: one very long column (a common term of a corpus) would
// otherwise hold a single warp for the whole product.
constexpr int SP_LONG = 1024;
constexpr int SP_SEG = 1024;
struct SparseLong {
  int count = 0;                // outer entries longer than SP_LONG
  int segs = 0;                 // their segments
  int32_t *outer = nullptr;     // count: the outer entries
  int32_t *seg_first = nullptr; // count + 1: each one's first segment
  int32_t *seg_e0 = nullptr;    // segs: entry range [seg_e0, seg_e1) of each segment
  int32_t *seg_e1 = nullptr;
};

// The data matrix in compressed form: CSC for V = B^T Z, CSR for Z = B V,
// and the optional implicit centring B - 1 means^T - row_means 1^T.
struct SparseDev {
  int m = 0, n = 0;
  int64_t nnz = 0;
  int32_t *col_ptr = nullptr, *row_ind = nullptr;  // CSC: n + 1, nnz (rows ascending)
  float *cvals = nullptr;
  int32_t *row_ptr = nullptr, *col_ind = nullptr;  // CSR: m + 1, nnz (columns ascending)
  float *rvals = nullptr;
  float *means = nullptr;      // n floats, or null
  float *row_means = nullptr;  // m floats, or null
  SparseLong long_cols, long_rows;  // of the CSC and the CSR arrays
  // deflation (am24_matrix_deflate): B <- B (I - x_1 x_1^T) ... (I - x_C x_C^T),
  // applied to V before Z = B V and to B^T Z after it, never to the arrays
  int comps = 0;
  const float *defl = nullptr;     // comps x n: x_1 .. x_C in call order
  const double *gram = nullptr;    // SP_DEFL_MAX x SP_DEFL_MAX: x_a^T x_b
  const double *defl_sum = nullptr;  // comps: 1^T x_c
  const double *defl_mu = nullptr;   // comps: means^T x_c (0 without means)
};
constexpr int SP_DEFL_MAX = 32;  // deflations a sparse-resident matrix takes

// A batch of k starts on a sparse matrix.  Start-major planes have columns of
// ldn (features) or ldm (samples) floats; the row-major planes Vt (n rows) and
// Zt (m rows) hold kp = round_up(k, 32) floats per row.
struct SparseBatchDev {
  int k = 0, kp = 0, ldn = 0, ldm = 0;
  float *Vx = nullptr;       // k x ldn loadings, defined where vmask is set
  uint32_t *vmask = nullptr; // k x ldn / 32
  float *Vraw = nullptr;     // k x ldn raw V = B^T Z (and the staging of loads)
  float *Vt = nullptr;       // n x kp
  float *Zs = nullptr;       // k x ldm
  float *Zt = nullptr;       // m x kp
  float *fz = nullptr, *val = nullptr, *err = nullptr, *max_err = nullptr;
  float *sel_hint = nullptr, *obj_part = nullptr, *nnz_part = nullptr;
  uint32_t *nnz = nullptr, *max_nnz = nullptr;
  uint32_t *ctl = nullptr;  // CTL_WORDS
  double *sum_v = nullptr, *dot_mu = nullptr, *zsum = nullptr, *zdot = nullptr;  // per start
  float *part_cols = nullptr, *part_rows = nullptr;  // segments x kp partial sums
  unsigned long long *work = nullptr;  // matrix entries in the supports' columns (this step)
  uint32_t *zgate = nullptr;           // this step's Z = B V path: 0 scatter, 1 CSR product
  double *defl_a = nullptr;            // k x SP_DEFL_MAX: V's deflation coefficients
  int *status = nullptr;
  int *iters = nullptr, *cards = nullptr;
  int log_capacity = 0;
};

// ---- launchers (am24_kernels.cu); all enqueue on `st` and return the CUDA error
// One AM step of a sparse batch (the dense step's iteration, with both
// products on the compressed matrix); sets the stop word as finalize does.
cudaError_t launch_sparse_step(const SparseDev &S, const SparseBatchDev &b, const StepParams &p,
                               cudaStream_t st);
// ||(B - centring) x||^2 in FP64 into *out; scratch: sparse_ev_scratch(S) doubles.
cudaError_t launch_sparse_ev(const SparseDev &S, const float *x, double *scratch, double *out,
                             cudaStream_t st);
inline size_t sparse_ev_scratch(const SparseDev &S) { return (size_t)(S.m + 255) / 256 + 2; }
int num_sms();
// Fills M's TF32 planes (Bc_hi/lo, Bt_hi/lo) from M.Bc.
cudaError_t launch_prep_tf32_planes(MatrixDev &M, cudaStream_t st);
// Fills M.Bc_b3 from M.Bc (its M.bf16_planes planes).
cudaError_t launch_prep_bf16x3(const MatrixDev &M, cudaStream_t st);
// Fills M.Bc_h2 and M.row_scale from M.Bc.
cudaError_t launch_prep_fp16x2(const MatrixDev &M, cudaStream_t st);
// Fills M.Bt_h2 and M.bt_row_scale from M.Bc; key: m words of scratch.
cudaError_t launch_prep_bt_fp16x2(const MatrixDev &M, uint32_t *key, cudaStream_t st);
// Loadings of `cols` columns from src (rows entries each) into dst and their
// non-zero masks (mask + c * (ld_dst / 32) per column).
cudaError_t launch_load_columns(const float *src, int ld_src, int rows, int cols, float *dst,
                                int ld_dst, uint32_t *mask, cudaStream_t st);
// dst[c][i] = mask bit i of column c ? Vx[c][i] : 0 for i < rows.
// Columns [0, cols) of V (leading dimension ld): device uniform starts for the
// global start indices first, first + 1, ... (AM24_START_DEVICE_UNIFORM).
cudaError_t launch_uniform_starts(float *V, int ld, int rows, int cols, uint32_t first,
                                  cudaStream_t st);
cudaError_t launch_masked_copy(const float *Vx, const uint32_t *mask, int ld, int rows, int cols,
                               float *dst, int ld_dst, cudaStream_t st);
// ev (optional, >= 17 events): ev[i] is recorded before launch i and
// ev[launches] after the last one; kinds[i] (optional) gets each launch's kind.
cudaError_t launch_am_step(const MatrixDev &M, BatchDev &b, const TensorMaps &tm,
                           const StepParams &p, cudaStream_t st, int *launches,
                           cudaEvent_t *ev = nullptr, int *kinds = nullptr);
cudaError_t launch_finalize_x(const float *v, int n, float *x, cudaStream_t st);
// A wait that nothing satisfies, bounded by timeout_ns; records the probe's
// timeout code in *status.
cudaError_t launch_bounded_wait_probe(unsigned long long timeout_ns, int *status,
                                      cudaStream_t st);
// M.Bc (zeroed) from device CSC arrays, then the optional centring
// (means: n floats, row_means: m floats, either may be null).
cudaError_t launch_csc_to_dense(MatrixDev &M, const float *vals, const int32_t *row_ind,
                               const int32_t *col_ptr, const float *means,
                               const float *row_means, cudaStream_t st);
// B <- B (I - x x^T) on M.Bc (device x; partial: ev_partial_len(M) doubles of
// scratch, y: m doubles).  The other layouts are not touched.
cudaError_t launch_deflate(MatrixDev &M, const float *x, double *partial, double *y,
                           cudaStream_t st);
// ||B x||^2 in FP64 into *out; partial: ev_partial_len(M) doubles of scratch.
cudaError_t launch_explained_variance(const MatrixDev &M, const float *x, double *partial,
                                      double *out, cudaStream_t st);
constexpr int EV_CHUNK = 512;  // features per partial sum of the explained variance
inline size_t ev_partial_len(const MatrixDev &M) {
  return (size_t)((M.n + EV_CHUNK - 1) / EV_CHUNK) * M.m;
}
int pick_bn(int k);
size_t ws_floats(int splits, int m_tiles, int n_tiles, int bn);

}  // namespace am24
