// Device kernels of one AM step and their launchers.
//
// One step for a batch of k starting points (reference:
// perform_one_iteration_for_{constrained,penalized}_pca,
// c++/src/gpower/gpower_commons.h:68-177):
//
//   1. gemm1     Z = B V            tcgen05 3xTF32, split-K partial tiles
//   2. z_reduce  sum the split partials; L1 variance: ||z||_1 and z <- sgn(z);
//                L2 variance: ||z||_2 (constrained) or z <- z/||z|| (penalized);
//                writes Z as TF32 hi/lo planes for gemm2
//   3. gemm2     V = B^T Z          tcgen05 3xTF32; penalized forms apply the
//                threshold, the per-start objective and non-zero count in the
//                epilogue; constrained forms store raw V
//   4. select    constrained only: per-start radix select of the s-th largest
//                |v| (L0) or the L1-ball level w (L1), normalisation
//   5. finalize  per-start objective, relative change, logs, batch maximum
//
// Every reduction has a fixed order, so a step is bitwise reproducible.
#include <cfloat>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <climits>
#include <cstdio>
#include <map>
#include <mutex>
#include <utility>

#include "am24_internal.h"
#include "gemm_tf32x3.cuh"
#include "gemm_pair.cuh"

namespace am24 {

namespace {

constexpr unsigned FULL = 0xffffffffu;
// K elements accumulated in TMEM before promotion to registers
constexpr int GEMM_PROMO_K = 128;

// x rounded to the nearest TF32 value (low 13 mantissa bits zero).  With
// lo = x - hi exact in FP32, x = hi + lo bit for bit, and lo takes either sign,
// so whatever the tensor core does with lo's low bits is unbiased.
__device__ __forceinline__ float tf32_hi(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}
__device__ __forceinline__ void split_store(float x, float *hi, float *lo) {
  const float h = tf32_hi(x);
  *hi = h;
  *lo = x - h;
}
// sgn with sgn(0) = 0 (c++/src/utils/various.h:44-46)
__device__ __forceinline__ float sgnf(float v) { return (float)((v > 0.f) - (v < 0.f)); }
// x rounded to the nearest BF16, as bits.
__device__ __forceinline__ uint16_t bf16_bits(float x) {
  return __bfloat16_as_ushort(__float2bfloat16_rn(x));
}
// sgn(v) as BF16 bits: +1 0x3F80, -1 0xBF80, 0 (and NaN) 0.
__device__ __forceinline__ uint16_t bf16_sign(float v) {
  return v > 0.f ? (uint16_t)0x3F80u : (v < 0.f ? (uint16_t)0xBF80u : (uint16_t)0u);
}
__device__ __forceinline__ uint32_t abs_key(float v) { return __float_as_uint(v) & 0x7FFFFFFFu; }
// sgn(v) as FP16 bits: +1 0x3C00, -1 0xBC00, 0 (and NaN) 0.
__device__ __forceinline__ uint16_t f16_sign(float v) {
  return v > 0.f ? (uint16_t)0x3C00u : (v < 0.f ? (uint16_t)0xBC00u : (uint16_t)0u);
}
// 2^e for e in [-126, 127], exactly.
__device__ __forceinline__ float pow2f(int e) { return __int_as_float((e + 127) << 23); }
// The shift s in [-113, 126] that puts a positive bound on |x| into
// [2^14, 2^15) (bounds below 2^-112 stay below that range); 0 for zero, NaN or
// infinite bounds.  x * 2^s then splits into FP16 planes without overflow
// (FP16's largest finite value is 65504).
__device__ __forceinline__ int fp16_shift(float bound) {
  const uint32_t eb = (__float_as_uint(bound) >> 23) & 0xFFu;
  if (!(bound > 0.f) || eb == 0xFFu) return 0;
  const int e = max((int)eb, 1) - 127;  // floor(log2(bound)) for normal bounds
  return min(14 - e, 126);
}
// x = h0 + h1 + r: h0 = fp16_rn(x), h1 = fp16_rn(x - h0) (the difference is
// exact in FP32), |r| <= 2^-11 |x - h0| for FP16-normal x - h0, else <= 2^-25.
__device__ __forceinline__ void fp16_split(float x, uint16_t *h0, uint16_t *h1) {
  const __half a = __float2half_rn(x);
  *h0 = __half_as_ushort(a);
  *h1 = __half_as_ushort(__float2half_rn(x - __half2float(a)));
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}

// Block-wide sum, result valid in every thread.  `red` holds >= 32 T.
template <typename T>
__device__ T block_sum(T v, T *red) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  T r = (lane < nw) ? red[lane] : T(0);
  if (w == 0) r = warp_sum(r);
  if (threadIdx.x == 0) red[0] = r;
  __syncthreads();
  r = red[0];
  __syncthreads();
  return r;
}

// Transposes the 32 x 32 bit matrix held by a warp: lane L passes bit j of
// x = A[L][j]; lane j gets the word whose bit L is A[L][j].  Five butterfly
// stages, each swapping the off-diagonal s x s blocks of every 2s x 2s block.
__device__ __forceinline__ uint32_t bit_transpose32(uint32_t x, int lane) {
  const uint32_t masks[5] = {0x0000FFFFu, 0x00FF00FFu, 0x0F0F0F0Fu, 0x33333333u, 0x55555555u};
#pragma unroll
  for (int k = 0; k < 5; k++) {
    const int sft = 16 >> k;
    const uint32_t m = masks[k];
    const uint32_t y = __shfl_xor_sync(FULL, x, sft);
    x = (lane & sft) ? ((x & ~m) | ((y >> sft) & m)) : ((x & m) | ((y << sft) & ~m));
  }
  return x;
}

// 32 lanes each hold v[0..31] (one per column); afterwards lane L returns the
// sum over all lanes of v[L].  31 shuffles instead of 32 x 5.
__device__ __forceinline__ float transpose_reduce32(float (&v)[32], int lane) {
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) {
    const bool upper = (lane & off) != 0;
#pragma unroll
    for (int i = 0; i < off; i++) {
      const float send = upper ? v[i] : v[i + off];
      const float keep = upper ? v[i + off] : v[i];
      v[i] = keep + __shfl_xor_sync(FULL, send, off);
    }
  }
  return v[0];
}

// fraction of the previous level used as the gather bound of the hinted searches
constexpr float HINT_FRACTION = 0.9f;
// The hinted bound on |v| keys of a column whose previous level was `hint` (> 0).
__device__ __forceinline__ uint32_t hinted_bound(float hint) {
  return max(1u, abs_key(HINT_FRACTION * hint));
}

// ------------------------------------------------------------ GEMM epilogues
// Z = B V split-K partial tile: ws[unit][col][row], whole 128 x bn tile.
struct EpiPartial {
  float *ws;
  int bn, m_tiles, n_tiles;  // m_tiles: 128-row blocks of C
  __device__ void setup() {}
  __device__ void unit_begin(const Unit &, int, int) {}
  __device__ void chunk(const Unit &t, int, int, int row, int col0, float (&r)[32]) {
    if (t.m0 >= m_tiles * BM) return;  // a 2-CTA tile's second half can lie past the last block
    const size_t slot = ((size_t)t.split * m_tiles + t.m0 / BM) * n_tiles + t.nt;
    float *base = ws + slot * ((size_t)bn * BM) + row;
#pragma unroll
    for (int j = 0; j < 32; j++) base[(size_t)(col0 + j) * BM] = r[j];
  }
};

// V = B^T Z raw output (constrained forms): out[col * ld + row].  With a
// candidate mask (cmask != null) it also does the selects' hinted gather: bit
// r of column col's mask (ld / 32 words per column, like vmask) is set when
// the column has a previous level hint[col] > 0 and |V[r, col]|'s key is at
// least hinted_bound(hint).  Every launch rewrites every word of rows < ld, so
// nothing needs clearing; the select kernels list the set bits instead of
// streaming the column.
struct EpiRaw {
  float *out;
  int ld, M, N, bn;
  const float *hint = nullptr;
  uint32_t *cmask = nullptr;
  // per unit: lane L holds the bound of column col_base + 32 c + L in bl[c]
  // (0xFFFFFFFF: the column has no level and lists nothing)
  int col_base = 0;
  uint32_t bl[4] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu};
  __device__ void setup() {}
  __device__ void unit_begin(const Unit &t, int lane, int cb) {
    if (!cmask) return;
    col_base = cb;
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const int col = t.nt * bn + cb + c * 32 + lane;
      const float h = col < N ? __ldg(hint + col) : 0.f;
      bl[c] = h > 0.f ? hinted_bound(h) : 0xFFFFFFFFu;
    }
  }
  __device__ void chunk(const Unit &t, int q, int lane, int row, int col0, float (&r)[32]) {
    if (t.m0 >= M) return;  // uniform: a 2-CTA tile's second half past the last row
    const int gi = t.m0 + row;
    const bool rv = gi < M;
    const int c0 = t.nt * bn + col0;
    if (rv) {
#pragma unroll
      for (int j = 0; j < 32; j++)
        if (c0 + j < N) out[(size_t)(c0 + j) * ld + gi] = r[j];
    }
    if (!cmask) return;
    // lane L: the rows of column c0 + L at or above its bound, as one mask word
    const int cl = c0 + lane;
    const int ci = ((col0 - col_base) >> 5) & 3;  // selects, not a local-memory index
    const uint32_t bound = ci == 0 ? bl[0] : ci == 1 ? bl[1] : ci == 2 ? bl[2] : bl[3];
    uint32_t mine = 0u;
#pragma unroll
    for (int j = 0; j < 32; j++) {
      const uint32_t bj = __shfl_sync(FULL, bound, j);
      const uint32_t bal = __ballot_sync(FULL, rv && bj != 0xFFFFFFFFu && abs_key(r[j]) >= bj);
      if (lane == j) mine = bal;
    }
    const int w = (t.m0 >> 5) + q;
    if (cl < N && w < (ld >> 5)) cmask[(size_t)cl * (ld >> 5) + w] = mine;
  }
};

// V = B^T Z with the penalty threshold fused (penalized forms).
//   L1 (c++/src/gpower/sparse_PCA_thresholding.h:26-47): d = |v| - gamma,
//      x = sgn(v) d if d > 0, objective term d^2.
//   L0 (:68-87): d = v^2 - gamma, x = v if d > 0, objective term d.
// The reference subtracts a double gamma; here d is the FP32 difference with
// gamma rounded to FP32 (they differ only where |v| or v^2 is within an ulp
// of gamma, a decision that the FP32 products feeding it already leave open).
// Writes the non-zero x and the non-zero bitmask and, per start and per
// (128-row block, warp), the partial objective and non-zero count, summed in
// fixed order by the finalize kernel.  When the previous step was dense
// (*max_nnz > cap), the next step most likely is too, so the epilogue also
// writes x as the TF32 hi/lo planes the tensor-core Z = B V reads (zeros
// included), which spares that step the densify pass.
template <bool L1>
struct EpiPenalty {
  float *Vx;
  float *obj_part, *nnz_part;
  int ld, M, N, bn, parts;  // parts = m_tiles * 4
  float gamma;
  uint32_t *vmask;  // non-zero bitmask words, ld / 32 per column
  float *V_hi, *V_lo;
  const uint32_t *max_nnz;  // the previous step's largest non-zero count
  uint32_t cap;             // ... above which Z = B V runs dense
  bool planes = false;      // this launch writes V_hi / V_lo (set by setup)
  __device__ void setup() { planes = V_hi != nullptr && *max_nnz > cap; }
  __device__ void unit_begin(const Unit &, int, int) {}
  // r holds this thread's 32 values (row `row`, columns col0..col0+31) and is
  // overwritten with the objective terms.
  __device__ void chunk(const Unit &t, int q, int lane, int row, int col0, float (&r)[32]) {
    if (planes)
      body<true>(t, q, lane, row, col0, r);
    else
      body<false>(t, q, lane, row, col0, r);
  }
  template <bool PLANES>
  __device__ void body(const Unit &t, int q, int lane, int row, int col0, float (&r)[32]) {
    if (t.m0 >= M) return;  // a 2-CTA tile's second half can lie past the last row
    const int gi = t.m0 + row;
    const bool rv = gi < M;
    const int mb = t.m0 / BM;  // 128-row block
    const int c0 = t.nt * bn + col0;
    const int ncols = rv ? min(32, N - c0) : 0;  // valid columns of this row
    uint32_t bits = 0u;  // bit j: (row, column c0 + j) is a non-zero
#pragma unroll
    for (int j = 0; j < 32; j++) {
      const float v = r[j];
      const bool valid = j < ncols;
      float d, o, x;
      if (L1) {
        d = __fsub_rn(fabsf(v), gamma);
        o = __fmul_rn(d, d);
        x = v > 0.f ? d : -d;
      } else {
        d = __fsub_rn(__fmul_rn(v, v), gamma);
        o = d;
        x = v;
      }
      const bool keep = valid && d > 0.f;
      r[j] = keep ? o : 0.f;
      const bool nz = keep && v != 0.f;
      bits |= (uint32_t)nz << j;
      if (nz) Vx[(size_t)(c0 + j) * ld + gi] = x;  // zeros live in the mask
      if (PLANES && valid) {
        const size_t o = (size_t)(c0 + j) * ld + gi;
        split_store(nz ? x : 0.f, V_hi + o, V_lo + o);
      }
    }
    const uint32_t word = bit_transpose32(bits, lane);  // lane j: column c0 + j, bit = row
    const float so = transpose_reduce32(r, lane);
    const int col = c0 + lane;
    if (col < N) {
      obj_part[(size_t)col * parts + mb * 4 + q] = so;
      nnz_part[(size_t)col * parts + mb * 4 + q] = (float)__popc(word);
      if (mb * 4 + q < (ld >> 5)) vmask[(size_t)col * (ld >> 5) + mb * 4 + q] = word;
    }
  }
};

// ------------------------------------------------------------ operand prep
// Bc[c * ldm + r] = split(B[c * ldB + r]): one block per feature column.
__global__ void prep_copy_kernel(const float *__restrict__ B, int ldB, int m, float *__restrict__ hi,
                                 float *__restrict__ lo, float *__restrict__ full, int ldm) {
  const size_t c = blockIdx.x;
  for (int r = threadIdx.x; r < m; r += blockDim.x) {
    const float v = B[c * ldB + r];
    split_store(v, hi + c * ldm + r, lo + c * ldm + r);
    if (full) full[c * ldm + r] = v;
  }
}

// Three BF16 planes with x = b0 + b1 + b2 exactly: b0 = bf16_rn(x),
// b1 = bf16_rn(x - b0), b2 = x - b0 - b1.  Each difference is exact in FP32
// (its operands are within a factor of two), the first remainder has at most
// 16 significant bits and the second at most 8, so b2 is a BF16 value.  (FP32
// subnormals below 2^-126 aside, where a tensor core may flush b2.)
__global__ void prep_bf16x3_kernel(const float *__restrict__ Bc, int ldm, int m, size_t plane,
                                   int planes, uint16_t *__restrict__ out) {
  const size_t c = blockIdx.x;
  for (int r = threadIdx.x; r < m; r += blockDim.x) {
    const size_t o = c * ldm + r;
    const float x = Bc[o];
    const __nv_bfloat16 b0 = __float2bfloat16_rn(x);
    const float r1 = x - __bfloat162float(b0);
    const __nv_bfloat16 b1 = __float2bfloat16_rn(r1);
    const __nv_bfloat16 b2 = __float2bfloat16_rn(r1 - __bfloat162float(b1));
    out[o] = __bfloat16_as_ushort(b0);
    if (planes == 3) {
      out[plane + o] = __bfloat16_as_ushort(b1);
      out[2 * plane + o] = __bfloat16_as_ushort(b2);
    }
  }
}

// Two FP16 planes of each feature of B with a power-of-two scale per feature:
// x * 2^s = h0 + h1 (fp16_split), s from the feature's largest |x| so that it
// lands in [2^14, 2^15); row_scale[c] = 2^-s undoes it in the GEMM epilogue.
__global__ void __launch_bounds__(256) prep_fp16x2_kernel(const float *__restrict__ Bc, int ldm,
                                                          int m, size_t plane,
                                                          uint16_t *__restrict__ out,
                                                          float *__restrict__ row_scale) {
  __shared__ uint32_t red[8];
  const size_t c = blockIdx.x;
  uint32_t mx = 0;
  for (int r = threadIdx.x; r < m; r += blockDim.x) mx = max(mx, abs_key(Bc[c * ldm + r]));
  mx = __reduce_max_sync(FULL, mx);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  mx = 0;
#pragma unroll
  for (int w = 0; w < 8; w++) mx = max(mx, red[w]);
  const int s = fp16_shift(__uint_as_float(mx));
  const float sc = pow2f(s);
  if (threadIdx.x == 0) row_scale[c] = pow2f(-s);
  for (int r = threadIdx.x; r < m; r += blockDim.x) {
    const size_t o = c * ldm + r;
    fp16_split(Bc[o] * sc, out + o, out + plane + o);
  }
}

// Per sample i, the largest |B[i, c]| over the features as a key, for the
// FP16 planes of B^T: blocks of SAMPLE_MAX_CHUNK features, threads over samples
// (coalesced reads of B's columns), atomicMax into key[i] (zeroed before).
constexpr int SAMPLE_MAX_CHUNK = 64;
__global__ void __launch_bounds__(256) sample_max_kernel(const float *__restrict__ Bc, int ldm,
                                                         int m, int n, uint32_t *__restrict__ key) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int c0 = blockIdx.y * SAMPLE_MAX_CHUNK, c1 = min(n, c0 + SAMPLE_MAX_CHUNK);
  uint32_t mx = 0;
  for (int c = c0; c < c1; c++) mx = max(mx, abs_key(Bc[(size_t)c * ldm + i]));
  atomicMax(key + i, mx);
}

// As prep_fp16x2_kernel for the rows of B^T: out[i * ldn + c] (second plane at
// out + plane) split from B[i, c] * 2^s_i, s_i from key[i]; row_scale[i] = 2^-s_i.
// 32 x 32 tiles through shared memory; columns [n, ldn) are left as they are.
__global__ void prep_bt_fp16x2_kernel(const float *__restrict__ Bc, int ldm, int m, int n,
                                      const uint32_t *__restrict__ key, int ldn, size_t plane,
                                      uint16_t *__restrict__ out, float *__restrict__ row_scale) {
  __shared__ float tile[32][33];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;  // features, samples
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int c = c0 + y, r = r0 + threadIdx.x;
    tile[y][threadIdx.x] = (c < n && r < m) ? Bc[(size_t)c * ldm + r] : 0.f;
  }
  __syncthreads();
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int r = r0 + y, c = c0 + threadIdx.x;
    if (r >= m) continue;
    const int s = fp16_shift(__uint_as_float(key[r]));
    if (c < n) {
      const size_t o = (size_t)r * ldn + c;
      fp16_split(tile[threadIdx.x][y] * pow2f(s), out + o, out + plane + o);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) row_scale[r] = pow2f(-s);
  }
}

// Bt[r * ldn + c] = split(B[c * ldB + r]): 32 x 32 tiles through shared memory.
__global__ void prep_transpose_kernel(const float *__restrict__ B, int ldB, int m, int n,
                                      float *__restrict__ hi, float *__restrict__ lo, int ldn) {
  __shared__ float tile[32][33];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int c = c0 + y, r = r0 + threadIdx.x;
    tile[y][threadIdx.x] = (c < n && r < m) ? B[(size_t)c * ldB + r] : 0.f;
  }
  __syncthreads();
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int r = r0 + y, c = c0 + threadIdx.x;
    if (r < m && c < n) {
      const size_t off = (size_t)r * ldn + c;
      split_store(tile[threadIdx.x][y], hi + off, lo + off);
    }
  }
}

// One block per column: dst = src (rows entries, zero up to ld_dst) and the
// column's non-zero bitmask (ld_dst / 32 words).
__global__ void load_columns_kernel(const float *__restrict__ src, int ld_src, int rows,
                                    float *__restrict__ dst, int ld_dst,
                                    uint32_t *__restrict__ mask) {
  const size_t c = blockIdx.x;
  const int lane = threadIdx.x & 31;
  for (int base = threadIdx.x & ~31; base < ld_dst; base += blockDim.x) {
    const int r = base + lane;
    const float v = (r < rows) ? src[c * ld_src + r] : 0.f;
    dst[c * ld_dst + r] = v;
    const unsigned nz = __ballot_sync(FULL, v != 0.f);
    if (lane == 0) mask[c * (ld_dst >> 5) + (base >> 5)] = nz;
  }
}

__global__ void masked_copy_kernel(const float *__restrict__ Vx, const uint32_t *__restrict__ mask,
                                   int ld, int rows, float *__restrict__ dst, int ld_dst) {
  const size_t c = blockIdx.x;
  for (int r = threadIdx.x; r < rows; r += blockDim.x) {
    const bool on = (mask[c * (ld >> 5) + (r >> 5)] >> (r & 31)) & 1u;
    dst[c * ld_dst + r] = on ? Vx[c * ld + r] : 0.f;
  }
}

// Dense TF32 hi/lo planes of V for the tensor-core Z = B V; does nothing on
// steps where the gather kernel takes Z = B V (*gate <= gate_max), and on
// dense steps whose planes the previous step's penalty epilogue already wrote
// (*planes > gate_max: the count that epilogue saw).
__global__ void densify_kernel(const float *__restrict__ Vx, const uint32_t *__restrict__ mask,
                               int ld, int rows, float *__restrict__ V_hi,
                               float *__restrict__ V_lo, const uint32_t *gate,
                               const uint32_t *planes, uint32_t gate_max,
                               const uint32_t *stop) {
  if (*stop || *gate <= gate_max || *planes > gate_max) return;
  const size_t c = blockIdx.x;
  for (int r = threadIdx.x; r < ld; r += blockDim.x) {
    const bool on = r < rows && ((mask[c * (ld >> 5) + (r >> 5)] >> (r & 31)) & 1u);
    split_store(on ? Vx[c * ld + r] : 0.f, V_hi + c * ld + r, V_lo + c * ld + r);
  }
}

// Dense FP16 planes of V for the CTA-pair Z = B V (split FP16 operands): on
// dense steps only (*gate > gate_max), one block per start, v * 2^s = h0 + h1
// with s from the column's largest |v|, v_scale[c] = 2^-s.
// The body for start c (one 256-thread block); densify_fp16_kernel runs it for
// blockIdx.x, the grouped steps for every start of their dense problems.
__device__ __forceinline__ void densify_fp16_body(const float *__restrict__ Vx,
                                                  const uint32_t *__restrict__ mask, int ld,
                                                  int rows, uint16_t *__restrict__ Vh,
                                                  size_t plane, float *__restrict__ v_scale,
                                                  const uint32_t *gate, uint32_t gate_max,
                                                  const uint32_t *stop, size_t c) {
  __shared__ uint32_t red[32];
  if (*stop || *gate <= gate_max) return;
  const uint32_t *mk = mask + c * (ld >> 5);
  const float4 *vx4 = reinterpret_cast<const float4 *>(Vx + c * ld);
  // four consecutive rows per thread and pass (ld is a multiple of 32)
  auto quad = [&](int q, float (&v)[4]) {
    const float4 x = vx4[q];
    const uint32_t bits = mk[q >> 3] >> ((4 * q) & 31);
    v[0] = ((bits & 1u) && 4 * q < rows) ? x.x : 0.f;
    v[1] = ((bits & 2u) && 4 * q + 1 < rows) ? x.y : 0.f;
    v[2] = ((bits & 4u) && 4 * q + 2 < rows) ? x.z : 0.f;
    v[3] = ((bits & 8u) && 4 * q + 3 < rows) ? x.w : 0.f;
  };
  const int quads = ld >> 2;
  uint32_t mx = 0;
#pragma unroll 8
  for (int q = threadIdx.x; q < quads; q += blockDim.x) {
    float v[4];
    quad(q, v);
    mx = max(mx, max(max(abs_key(v[0]), abs_key(v[1])), max(abs_key(v[2]), abs_key(v[3]))));
  }
  mx = __reduce_max_sync(FULL, mx);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  mx = 0;
  for (int w = 0; w < (int)(blockDim.x >> 5); w++) mx = max(mx, red[w]);
  const int s = fp16_shift(__uint_as_float(mx));
  const float sc = pow2f(s);
  if (threadIdx.x == 0) v_scale[c] = pow2f(-s);
  uint2 *h0 = reinterpret_cast<uint2 *>(Vh + c * ld);
  uint2 *h1 = reinterpret_cast<uint2 *>(Vh + plane + c * ld);
#pragma unroll 4
  for (int q = threadIdx.x; q < quads; q += blockDim.x) {
    float v[4];
    quad(q, v);
    uint16_t a[4], b[4];
#pragma unroll
    for (int i = 0; i < 4; i++) fp16_split(v[i] * sc, &a[i], &b[i]);
    h0[q] = make_uint2(a[0] | ((uint32_t)a[1] << 16), a[2] | ((uint32_t)a[3] << 16));
    h1[q] = make_uint2(b[0] | ((uint32_t)b[1] << 16), b[2] | ((uint32_t)b[3] << 16));
  }
}
// Persistent over the k columns with DENSIFY_BLOCKS_PER_SM blocks of 512
// threads per SM: a column's first pass (its largest |v|) streams it from HBM,
// and with this few columns in flight (2 x 148 x 4 B x p, 59 MB at p = 50000)
// the second pass finds it in L2, so V crosses HBM once.
constexpr int DENSIFY_THREADS = 512, DENSIFY_BLOCKS_PER_SM = 2;
__global__ void __launch_bounds__(DENSIFY_THREADS, DENSIFY_BLOCKS_PER_SM) densify_fp16_kernel(
    const float *__restrict__ Vx, const uint32_t *__restrict__ mask, int ld, int rows,
    uint16_t *__restrict__ Vh, size_t plane, float *__restrict__ v_scale, const uint32_t *gate,
    uint32_t gate_max, const uint32_t *stop, int k) {
  for (int c = blockIdx.x; c < k; c += gridDim.x) {
    densify_fp16_body(Vx, mask, ld, rows, Vh, plane, v_scale, gate, gate_max, stop, c);
    __syncthreads();  // red[] is reused by the next column
  }
}

// ------------------------------------------------------------ Z reduction
// MODE 0: L2 variance, constrained  -> z = y, fz = ||y||_2  (gpower_commons.h:100)
// MODE 1: L1 variance               -> z = sgn(y), fz = ||y||_1 (:85-86, :156)
// MODE 2: L2 variance, penalized    -> z = y * (1/||y||_2)     (:163-164)
template <int MODE>
__device__ __forceinline__ void z_reduce_body(const float *__restrict__ ws, int splits,
                                              int m_tiles, int n_tiles, int bn, int m,
                                              float *__restrict__ Z_hi, float *__restrict__ Z_lo,
                                              int ldm, float *__restrict__ fz,
                                              const uint32_t *gate, uint32_t gate_max,
                                              uint16_t *__restrict__ Zb,
                                              uint16_t *__restrict__ Zh, size_t zplane,
                                              float *__restrict__ zscale, const uint32_t *stop,
                                              int j) {
  __shared__ double red[32];
  if (*stop || *gate <= gate_max) return;  // the gather kernel produced Z this step
  const int nt = j / bn, c = j - nt * bn;
  const size_t unit_stride = (size_t)bn * BM;
  float *zh = Z_hi + (size_t)j * ldm;
  float *zl = Z_lo + (size_t)j * ldm;
  double acc = 0.0;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    const int mt = i >> 7, r = i & 127;
    float y = 0.f;
    for (int s = 0; s < splits; s++) {
      const size_t u = ((size_t)s * m_tiles + mt) * n_tiles + nt;
      y += ws[u * unit_stride + (size_t)c * BM + r];
    }
    if (MODE == 1) {
      acc += (double)fabsf(y);
      zh[i] = sgnf(y);
      zl[i] = 0.f;
      if (Zb) Zb[(size_t)j * ldm + i] = bf16_sign(y);
      if (Zh) Zh[(size_t)j * ldm + i] = f16_sign(y);
    } else {
      acc += (double)y * (double)y;
      split_store(y, zh + i, zl + i);
      if (MODE == 0 && Zb) Zb[(size_t)j * ldm + i] = bf16_bits(y);
    }
  }
  const double tot = block_sum(acc, red);
  if (MODE == 2 || (MODE == 0 && Zh)) {
    // second pass: MODE 2 normalises; both write the FP16 planes of z * 2^s,
    // s from a bound on |z| (||y||_2, or 1 for the normalised z)
    const float inv = MODE == 2 ? 1.0f / (float)sqrt(tot) : 1.0f;
    const int s = fp16_shift(MODE == 2 ? 1.0f : (float)sqrt(tot));
    const float sc = pow2f(s);
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
      const float y = zh[i] + zl[i];  // exact: this thread wrote both planes
      const float z = MODE == 2 ? y * inv : y;
      if (MODE == 2) {
        split_store(z, zh + i, zl + i);
        if (Zb) Zb[(size_t)j * ldm + i] = bf16_bits(z);
      }
      if (Zh) fp16_split(z * sc, Zh + (size_t)j * ldm + i, Zh + zplane + (size_t)j * ldm + i);
    }
    if (Zh && threadIdx.x == 0) zscale[j] = pow2f(-s);
  }
  if (MODE != 2 && threadIdx.x == 0) fz[j] = (MODE == 1) ? (float)tot : (float)sqrt(tot);
}
template <int MODE>
__global__ void __launch_bounds__(256) z_reduce_kernel(const float *__restrict__ ws, int splits,
                                                       int m_tiles, int n_tiles, int bn, int m,
                                                       float *__restrict__ Z_hi,
                                                       float *__restrict__ Z_lo, int ldm,
                                                       float *__restrict__ fz,
                                                       const uint32_t *gate, uint32_t gate_max,
                                                       uint16_t *__restrict__ Zb,
                                                       uint16_t *__restrict__ Zh, size_t zplane,
                                                       float *__restrict__ zscale,
                                                       const uint32_t *stop) {
  z_reduce_body<MODE>(ws, splits, m_tiles, n_tiles, bn, m, Z_hi, Z_lo, ldm, fz, gate, gate_max,
                      Zb, Zh, zplane, zscale, stop, blockIdx.x);
}

// ------------------------------------------------------------ sparse Z = B V
constexpr int GATHER_THREADS = 256;

// MIXED phase word after a step: the lead-in counts down to the single-pass
// phase 0, which switches to refinement (1, sticky) once enough starts are stable.
__device__ __forceinline__ uint32_t mixed_next_phase(uint32_t ph, bool stable_enough) {
  if (ph >= 2u) return ph == 2u ? 0u : ph - 1u;
  return (ph == 0u && stable_enough) ? 1u : ph;
}
constexpr int GATHER_ROWS = 8;  // samples per thread per pass
constexpr int GATHER_CAP = 4096;

// MIXED precision bookkeeping, after the step's non-zero masks are written:
// per start, the number of consecutive steps whose support (non-zero mask)
// equals the previous step's.  When at least `need` starts of the batch have
// kept their support for k_stable steps, phase[0] switches to refinement for
// good; the last block to finish decides, keeps the phase the step ran in as
// phase[3] and resets the step's scratch words.  phase[0] >= 2 is the FP32
// lead-in (phase[0] - 1 accurate steps left, no start counted stable); its
// last step hands over to the single-pass phase 0.
__global__ void __launch_bounds__(256) support_kernel(const uint32_t *__restrict__ vmask,
                                                      const uint32_t *__restrict__ prev, int words,
                                                      uint32_t *stable, uint32_t *phase,
                                                      uint32_t k_stable, uint32_t need,
                                                      const uint32_t *stop) {
  if (*stop) return;
  const int j = blockIdx.x;
  const uint32_t *a = vmask + (size_t)j * words, *b = prev + (size_t)j * words;
  int diff = 0;
  for (int w = threadIdx.x; w < words; w += blockDim.x) diff |= (a[w] != b[w]);
  diff = __syncthreads_or(diff);
  if (threadIdx.x == 0) {
    // read before this block's arrival: the last block rewrites phase[0] only
    // after every block has arrived
    const bool lead = *reinterpret_cast<volatile uint32_t *>(phase) >= 2u;
    const uint32_t st = (diff || lead) ? 0u : min(stable[j] + 1u, 0x7FFFFFFFu);
    stable[j] = st;
    if (st >= k_stable) atomicAdd(&phase[1], 1u);
    __threadfence();
    if (atomicAdd(&phase[2], 1u) == gridDim.x - 1) {
      __threadfence();
      const uint32_t count = atomicExch(&phase[1], 0u);
      const uint32_t ph = phase[0];
      phase[3] = ph;
      phase[0] = mixed_next_phase(ph, count >= need);
      phase[2] = 0u;
    }
  }
}

// Z = B V for one start when V's column has few non-zeros: runs instead of
// gemm1 + z_reduce when the previous step left at most gate_max non-zeros in
// every column (*gate).  The column's non-zero rows are listed in index order
// from its bitmask, then z = sum_q v_q B[:, q] is accumulated with FP32 FMAs in
// that fixed order (deterministic), and the same sign / norm / normalise
// step as z_reduce_kernel<MODE> finishes the column.
template <int MODE>
__device__ __forceinline__ void gather_bv_body(
    const float *__restrict__ Bc, int ldm, int m, int ldn,
    const float *__restrict__ Vx, const uint32_t *__restrict__ vmask, float *__restrict__ Z_hi,
    float *__restrict__ Z_lo, float *__restrict__ fz, const uint32_t *gate, uint32_t gate_max,
    uint16_t *__restrict__ Zb, uint16_t *__restrict__ Zh, size_t zplane,
    float *__restrict__ zscale, const uint32_t *stop, int j) {
  __shared__ int idx[GATHER_CAP];
  __shared__ float val[GATHER_CAP];
  __shared__ uint32_t wsum[GATHER_THREADS / 32];
  __shared__ double red[32];
  // dense V (gemm1 + z_reduce), or few enough non-zeros for gather_bv_group_kernel
  if (*stop || *gate > gate_max || *gate <= min(gate_max, GATHER_GROUP_MAX_NNZ)) return;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int words = ldn >> 5;
  const uint32_t *mk = vmask + (size_t)j * words;
  // each thread owns a contiguous run of mask words, so the block-wide
  // exclusive scan of their popcounts lists rows in index order
  const int per = (words + GATHER_THREADS - 1) / GATHER_THREADS;
  const int w0 = min(words, threadIdx.x * per), w1 = min(words, w0 + per);
  uint32_t cnt = 0;
  for (int q = w0; q < w1; q++) cnt += __popc(mk[q]);
  uint32_t incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(FULL, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) wsum[w] = incl;
  __syncthreads();
  uint32_t off = incl - cnt;
  for (int i = 0; i < w; i++) off += wsum[i];
  uint32_t total = 0;
  for (int i = 0; i < GATHER_THREADS / 32; i++) total += wsum[i];
  if (total > (uint32_t)GATHER_CAP) total = GATHER_CAP;  // cannot happen below the gate
  const float *vx = Vx + (size_t)j * ldn;
  for (int q = w0; q < w1; q++) {
    uint32_t bits = mk[q];
    while (bits) {
      const int b = __ffs(bits) - 1;
      bits &= bits - 1;
      const int r = q * 32 + b;
      if (off < (uint32_t)GATHER_CAP) {
        idx[off] = r;
        val[off] = vx[r];
      }
      off++;
    }
  }
  __syncthreads();
  // Each thread accumulates 2 x 4 consecutive samples per pass (16-byte loads);
  // the rows of four non-zeros are loaded before their FMAs, which still run in
  // index order per sample.  Samples in [m, ldm) read B's zero padding.
  constexpr int G4 = GATHER_ROWS / 4;
  double acc = 0.0;
  float4 y[G4];
  float *zh = Z_hi + (size_t)j * ldm;
  float *zl = Z_lo + (size_t)j * ldm;
  uint16_t *zb = Zb ? Zb + (size_t)j * ldm : nullptr;
  uint16_t *zh0 = Zh ? Zh + (size_t)j * ldm : nullptr;
  const int chunk = GATHER_THREADS * GATHER_ROWS;
  const int ld4 = ldm >> 2;
  const bool one_pass = m <= chunk;
  auto sample = [&](int base, int r) { return base + 4 * (r * GATHER_THREADS + (int)threadIdx.x); };
  auto fma4 = [](float v, const float4 &b, float4 &acc4) {
    acc4.x = fmaf(v, b.x, acc4.x);
    acc4.y = fmaf(v, b.y, acc4.y);
    acc4.z = fmaf(v, b.z, acc4.z);
    acc4.w = fmaf(v, b.w, acc4.w);
  };
  // the final value of sample i (c of the float4), stored as Z needs it
  auto emit = [&](int i, float yv) {
    if (MODE == 1) {
      acc += (double)fabsf(yv);
      zh[i] = sgnf(yv);
      zl[i] = 0.f;
      if (zb) zb[i] = bf16_sign(yv);
      if (zh0) zh0[i] = f16_sign(yv);
    } else {
      acc += (double)yv * (double)yv;
      if (!(MODE == 2 && one_pass)) split_store(yv, zh + i, zl + i);
      if (MODE == 0 && zb) zb[i] = bf16_bits(yv);
    }
  };
  for (int base = 0; base < m; base += chunk) {
    int i4[G4];
    bool ok[G4];
#pragma unroll
    for (int r = 0; r < G4; r++) {
      y[r] = make_float4(0.f, 0.f, 0.f, 0.f);
      i4[r] = sample(base, r) >> 2;
      ok[r] = i4[r] < ld4;
    }
    uint32_t q = 0;
    for (; q + 4 <= total; q += 4) {
      float4 bq[4][G4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const float4 *row4 = reinterpret_cast<const float4 *>(Bc + (size_t)idx[q + u] * ldm);
#pragma unroll
        for (int r = 0; r < G4; r++)
          bq[u][r] = ok[r] ? __ldg(row4 + i4[r]) : make_float4(0.f, 0.f, 0.f, 0.f);
      }
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const float v = val[q + u];
#pragma unroll
        for (int r = 0; r < G4; r++) fma4(v, bq[u][r], y[r]);
      }
    }
    for (; q < total; q++) {
      const float4 *row4 = reinterpret_cast<const float4 *>(Bc + (size_t)idx[q] * ldm);
      const float v = val[q];
#pragma unroll
      for (int r = 0; r < G4; r++)
        if (ok[r]) fma4(v, __ldg(row4 + i4[r]), y[r]);
    }
#pragma unroll
    for (int r = 0; r < G4; r++) {
      const int i = sample(base, r);
      const float e[4] = {y[r].x, y[r].y, y[r].z, y[r].w};
#pragma unroll
      for (int c = 0; c < 4; c++)
        if (i + c < m) emit(i + c, e[c]);
    }
  }
  const double tot = block_sum(acc, red);
  if (MODE == 2 || (MODE == 0 && zh0)) {
    // as in z_reduce_kernel: MODE 2 normalises, both write the FP16 planes
    const float inv = MODE == 2 ? 1.0f / (float)sqrt(tot) : 1.0f;
    const int s = fp16_shift(MODE == 2 ? 1.0f : (float)sqrt(tot));
    const float sc = pow2f(s);
    for (int base = 0; base < m; base += chunk) {
#pragma unroll
      for (int r = 0; r < G4; r++) {
        const int i = sample(base, r);
        const float e[4] = {y[r].x, y[r].y, y[r].z, y[r].w};
#pragma unroll
        for (int c = 0; c < 4; c++) {
          if (i + c >= m) continue;
          // one pass: the sums are still in registers; else re-read what this
          // thread wrote (hi + lo is exact)
          const float v = one_pass ? e[c] : zh[i + c] + zl[i + c];
          const float z = MODE == 2 ? v * inv : v;
          if (MODE == 2) {
            split_store(z, zh + i + c, zl + i + c);
            if (zb) zb[i + c] = bf16_bits(z);
          }
          if (zh0) fp16_split(z * sc, zh0 + i + c, zh0 + zplane + i + c);
        }
      }
    }
    if (zh0 && threadIdx.x == 0) zscale[j] = pow2f(-s);
  }
  if (MODE != 2 && threadIdx.x == 0) fz[j] = (MODE == 1) ? (float)tot : (float)sqrt(tot);
}
template <int MODE>
__global__ void __launch_bounds__(GATHER_THREADS) gather_bv_kernel(
    const float *__restrict__ Bc, int ldm, int m, int ldn,
    const float *__restrict__ Vx, const uint32_t *__restrict__ vmask, float *__restrict__ Z_hi,
    float *__restrict__ Z_lo, float *__restrict__ fz, const uint32_t *gate, uint32_t gate_max,
    uint16_t *__restrict__ Zb, uint16_t *__restrict__ Zh, size_t zplane,
    float *__restrict__ zscale, const uint32_t *stop) {
  gather_bv_body<MODE>(Bc, ldm, m, ldn, Vx, vmask, Z_hi, Z_lo, fz, gate, gate_max, Zb, Zh, zplane,
                       zscale, stop, blockIdx.x);
}

// The sparse Z = B V for GATHER_GROUP starts per block, while every column
// has at most GATHER_CAP / GATHER_GROUP non-zeros (*gate): the block lists the
// union of the group's non-zero rows in index order, loads each row once, and
// adds it to the sums of the starts it belongs to.  Every start's FMAs still
// run over its own non-zeros in index order, so the result is bit for bit that
// of gather_bv_kernel, with a quarter of the row loads where supports overlap.
// Above the group bound this kernel returns at once and gather_bv_kernel runs.
constexpr int GATHER_GROUP = 4;
static_assert(GATHER_GROUP_MAX_NNZ == GATHER_CAP / GATHER_GROUP, "group bound");
constexpr size_t GATHER_GROUP_SMEM =
    (size_t)GATHER_CAP * (sizeof(int) + GATHER_GROUP * sizeof(float) + 1);

template <int MODE>
__device__ __forceinline__ void gather_bv_group_body(
    const float *__restrict__ Bc, int ldm, int m, int ldn, int k,
    const float *__restrict__ Vx, const uint32_t *__restrict__ vmask, float *__restrict__ Z_hi,
    float *__restrict__ Z_lo, float *__restrict__ fz, const uint32_t *gate, uint32_t gate_max,
    uint16_t *__restrict__ Zb, uint16_t *__restrict__ Zh, size_t zplane,
    float *__restrict__ zscale, const uint32_t *stop, int group) {
  constexpr int G = GATHER_GROUP;
  extern __shared__ __align__(16) uint8_t gsm[];
  int *idx = reinterpret_cast<int *>(gsm);                                  // GATHER_CAP
  float *val = reinterpret_cast<float *>(gsm + sizeof(int) * GATHER_CAP);   // G x GATHER_CAP
  uint8_t *memb = gsm + (sizeof(int) + G * sizeof(float)) * GATHER_CAP;     // GATHER_CAP
  __shared__ uint32_t wsum[GATHER_THREADS / 32];
  __shared__ double red[32];
  // dense V (gemm1 + z_reduce), or gather_bv_kernel's case
  if (*stop || *gate > min(gate_max, GATHER_GROUP_MAX_NNZ)) return;
  const int j0 = group * G;
  const int ng = min(G, k - j0);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int words = ldn >> 5;
  const uint32_t *mk[G];
  const float *vx[G];
#pragma unroll
  for (int g = 0; g < G; g++) {
    const int j = j0 + min(g, ng - 1);  // past the last start: a repeat, never a member
    mk[g] = vmask + (size_t)j * words;
    vx[g] = Vx + (size_t)j * ldn;
  }
  auto word = [&](int g, int q) { return g < ng ? mk[g][q] : 0u; };
  // the union's rows in index order: an exclusive scan over threads' word runs
  const int per = (words + GATHER_THREADS - 1) / GATHER_THREADS;
  const int w0 = min(words, threadIdx.x * per), w1 = min(words, w0 + per);
  uint32_t cnt = 0;
  for (int q = w0; q < w1; q++) {
    uint32_t u = 0;
#pragma unroll
    for (int g = 0; g < G; g++) u |= word(g, q);
    cnt += __popc(u);
  }
  uint32_t incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(FULL, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) wsum[w] = incl;
  __syncthreads();
  uint32_t off = incl - cnt;
  for (int i = 0; i < w; i++) off += wsum[i];
  uint32_t total = 0;
  for (int i = 0; i < GATHER_THREADS / 32; i++) total += wsum[i];
  if (total > (uint32_t)GATHER_CAP) total = GATHER_CAP;  // cannot happen below the gate
  for (int q = w0; q < w1; q++) {
    uint32_t wg[G], u = 0;
#pragma unroll
    for (int g = 0; g < G; g++) {
      wg[g] = word(g, q);
      u |= wg[g];
    }
    while (u) {
      const int b = __ffs(u) - 1;
      u &= u - 1;
      const int r = q * 32 + b;
      if (off < (uint32_t)GATHER_CAP) {
        idx[off] = r;
        uint32_t mb = 0;
#pragma unroll
        for (int g = 0; g < G; g++) {
          const bool in = (wg[g] >> b) & 1u;
          mb |= (uint32_t)in << g;
          val[g * GATHER_CAP + off] = in ? vx[g][r] : 0.f;
        }
        memb[off] = (uint8_t)mb;
      }
      off++;
    }
  }
  __syncthreads();
  constexpr int G4 = GATHER_ROWS / 4;
  double acc[G];
  float4 y[G][G4];
  const int chunk = GATHER_THREADS * GATHER_ROWS;
  const int ld4 = ldm >> 2;
  const bool one_pass = m <= chunk;
  auto sample = [&](int base, int r) { return base + 4 * (r * GATHER_THREADS + (int)threadIdx.x); };
  auto fma4 = [](float v, const float4 &b, float4 &acc4) {
    acc4.x = fmaf(v, b.x, acc4.x);
    acc4.y = fmaf(v, b.y, acc4.y);
    acc4.z = fmaf(v, b.z, acc4.z);
    acc4.w = fmaf(v, b.w, acc4.w);
  };
#pragma unroll
  for (int g = 0; g < G; g++) acc[g] = 0.0;
  // sample i of start g, as gather_bv_kernel's emit stores it
  auto emit = [&](int g, int i, float yv) {
    const size_t o = (size_t)(j0 + g) * ldm + i;
    if (MODE == 1) {
      acc[g] += (double)fabsf(yv);
      Z_hi[o] = sgnf(yv);
      Z_lo[o] = 0.f;
      if (Zb) Zb[o] = bf16_sign(yv);
      if (Zh) Zh[o] = f16_sign(yv);
    } else {
      acc[g] += (double)yv * (double)yv;
      if (!(MODE == 2 && one_pass)) split_store(yv, Z_hi + o, Z_lo + o);
      if (MODE == 0 && Zb) Zb[o] = bf16_bits(yv);
    }
  };
  for (int base = 0; base < m; base += chunk) {
    int i4[G4];
    bool ok[G4];
#pragma unroll
    for (int r = 0; r < G4; r++) {
      i4[r] = sample(base, r) >> 2;
      ok[r] = i4[r] < ld4;
#pragma unroll
      for (int g = 0; g < G; g++) y[g][r] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    uint32_t q = 0;
    for (; q + 4 <= total; q += 4) {
      float4 bq[4][G4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const float4 *row4 = reinterpret_cast<const float4 *>(Bc + (size_t)idx[q + u] * ldm);
#pragma unroll
        for (int r = 0; r < G4; r++)
          bq[u][r] = ok[r] ? __ldg(row4 + i4[r]) : make_float4(0.f, 0.f, 0.f, 0.f);
      }
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const uint32_t mb = memb[q + u];
#pragma unroll
        for (int g = 0; g < G; g++) {
          if (!((mb >> g) & 1u)) continue;
          const float v = val[g * GATHER_CAP + q + u];
#pragma unroll
          for (int r = 0; r < G4; r++) fma4(v, bq[u][r], y[g][r]);
        }
      }
    }
    for (; q < total; q++) {
      const float4 *row4 = reinterpret_cast<const float4 *>(Bc + (size_t)idx[q] * ldm);
      const uint32_t mb = memb[q];
      float4 b[G4];
#pragma unroll
      for (int r = 0; r < G4; r++) b[r] = ok[r] ? __ldg(row4 + i4[r]) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
      for (int g = 0; g < G; g++) {
        if (!((mb >> g) & 1u)) continue;
        const float v = val[g * GATHER_CAP + q];
#pragma unroll
        for (int r = 0; r < G4; r++)
          if (ok[r]) fma4(v, b[r], y[g][r]);
      }
    }
#pragma unroll
    for (int g = 0; g < G; g++) {
      if (g >= ng) continue;
#pragma unroll
      for (int r = 0; r < G4; r++) {
        const int i = sample(base, r);
        const float e[4] = {y[g][r].x, y[g][r].y, y[g][r].z, y[g][r].w};
#pragma unroll
        for (int c = 0; c < 4; c++)
          if (i + c < m) emit(g, i + c, e[c]);
      }
    }
  }
#pragma unroll
  for (int g = 0; g < G; g++) {
    if (g >= ng) continue;  // uniform over the block
    const int j = j0 + g;
    const double tot = block_sum(acc[g], red);
    float *zh = Z_hi + (size_t)j * ldm, *zl = Z_lo + (size_t)j * ldm;
    uint16_t *zb = Zb ? Zb + (size_t)j * ldm : nullptr;
    uint16_t *zh0 = Zh ? Zh + (size_t)j * ldm : nullptr;
    if (MODE == 2 || (MODE == 0 && zh0)) {
      const float inv = MODE == 2 ? 1.0f / (float)sqrt(tot) : 1.0f;
      const int s = fp16_shift(MODE == 2 ? 1.0f : (float)sqrt(tot));
      const float sc = pow2f(s);
      for (int base = 0; base < m; base += chunk) {
#pragma unroll
        for (int r = 0; r < G4; r++) {
          const int i = sample(base, r);
          const float e[4] = {y[g][r].x, y[g][r].y, y[g][r].z, y[g][r].w};
#pragma unroll
          for (int c = 0; c < 4; c++) {
            if (i + c >= m) continue;
            const float v = one_pass ? e[c] : zh[i + c] + zl[i + c];
            const float z = MODE == 2 ? v * inv : v;
            if (MODE == 2) {
              split_store(z, zh + i + c, zl + i + c);
              if (zb) zb[i + c] = bf16_bits(z);
            }
            if (zh0) fp16_split(z * sc, zh0 + i + c, zh0 + zplane + i + c);
          }
        }
      }
      if (zh0 && threadIdx.x == 0) zscale[j] = pow2f(-s);
    }
    if (MODE != 2 && threadIdx.x == 0) fz[j] = (MODE == 1) ? (float)tot : (float)sqrt(tot);
  }
}
template <int MODE>
__global__ void __launch_bounds__(GATHER_THREADS) gather_bv_group_kernel(
    const float *__restrict__ Bc, int ldm, int m, int ldn, int k,
    const float *__restrict__ Vx, const uint32_t *__restrict__ vmask, float *__restrict__ Z_hi,
    float *__restrict__ Z_lo, float *__restrict__ fz, const uint32_t *gate, uint32_t gate_max,
    uint16_t *__restrict__ Zb, uint16_t *__restrict__ Zh, size_t zplane,
    float *__restrict__ zscale, const uint32_t *stop) {
  gather_bv_group_body<MODE>(Bc, ldm, m, ldn, k, Vx, vmask, Z_hi, Z_lo, fz, gate, gate_max, Zb,
                             Zh, zplane, zscale, stop, blockIdx.x);
}

// ------------------------------------------------------------ radix select
struct SelResult {
  uint32_t key;  // bit pattern of |v| at the requested descending rank
  uint32_t gt;   // number of keys strictly greater
  uint32_t eq;   // number of keys equal
};


// Key of descending rank `rank` (1 = largest) among |col[0..n)|, by three
// histogram passes over 11, 11 and 9 key bits.  All threads of the block
// call it; hist has 2048 entries, res 4.
// Readers of the values a selection walks: a column of V (read-only in the
// kernel) or a list of keys the kernel wrote itself (read through L2, never the
// non-coherent path).
struct ColumnSrc {
  const float *__restrict__ p;
  __device__ __forceinline__ float operator()(int i) const { return p[i]; }
};
struct ListSrc {
  const float *p;
  __device__ __forceinline__ float operator()(int i) const { return __ldcg(p + i); }
};

template <class Src>
__device__ SelResult block_select_src(Src colg, int n, uint32_t rank, uint32_t *hist,
                                      uint32_t *res);
__device__ __forceinline__ SelResult block_select(const float *__restrict__ colg, int n,
                                                  uint32_t rank, uint32_t *hist, uint32_t *res) {
  return block_select_src(ColumnSrc{colg}, n, rank, hist, res);
}
template <class Src>
__device__ SelResult block_select_src(Src colg, int n, uint32_t rank, uint32_t *hist,
                                      uint32_t *res) {
  uint32_t prefix = 0, pmask = 0, gt = 0, need = rank, eq = 0;
#pragma unroll 1
  for (int lvl = 0; lvl < 3; lvl++) {
    const int sh = (lvl == 0) ? 20 : (lvl == 1) ? 9 : 0;
    const uint32_t nb = (lvl == 2) ? 512u : 2048u;
    const uint32_t bmask = nb - 1;
    for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) hist[b] = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const uint32_t key = abs_key(colg(i));
      if ((key & pmask) == prefix) {
        const uint32_t bin = (key >> sh) & bmask;
        const unsigned peers = __match_any_sync(__activemask(), bin);
        if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&hist[bin], __popc(peers));
      }
    }
    __syncthreads();
    if (threadIdx.x < 32) {
      const int lane = threadIdx.x;
      uint32_t running = 0, fbin = 0, fcum = 0, feq = 0;
      bool found = false;
      for (int base = (int)nb - 32; base >= 0 && !found; base -= 32) {
        const uint32_t b = base + 31 - lane;
        const uint32_t c = hist[b];
        uint32_t incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t t = __shfl_up_sync(FULL, incl, o);
          if (lane >= o) incl += t;
        }
        const uint32_t total = __shfl_sync(FULL, incl, 31);
        if (running + total >= need) {
          const unsigned ballot = __ballot_sync(FULL, running + incl >= need);
          const int f = __ffs(ballot) - 1;
          const uint32_t inc_f = __shfl_sync(FULL, incl, f);
          const uint32_t c_f = __shfl_sync(FULL, c, f);
          fbin = base + 31 - f;
          fcum = running + inc_f - c_f;
          feq = c_f;
          found = true;
        } else {
          running += total;
        }
      }
      if (lane == 0) {
        res[0] = fbin;
        res[1] = fcum;
        res[2] = feq;
      }
    }
    __syncthreads();
    const uint32_t bin = res[0];
    gt += res[1];
    need -= res[1];
    eq = res[2];
    prefix |= bin << sh;
    pmask |= bmask << sh;
    __syncthreads();
  }
  return SelResult{prefix, gt, eq};
}

// x_i = f(v_i) for a column in global memory: the non-zero x_i are stored
// (only they are defined; the bitmask says which) and the column's non-zero
// bitmask is written.  Entries up to the next multiple of 32 are read; they lie
// in the column's zero padding.
template <class Fn>
__device__ __forceinline__ void write_column_global(const float *__restrict__ colg, int n,
                                                    float *vx, uint32_t *mask, Fn fn) {
  const int lane = threadIdx.x & 31;
  const int n32 = (n + 31) & ~31;
  for (int base = threadIdx.x & ~31; base < n32; base += blockDim.x) {
    const int i = base + lane;
    const float x = fn(colg[i]);
    if (x != 0.f) vx[i] = x;
    const unsigned nz = __ballot_sync(FULL, x != 0.f);
    if (lane == 0) mask[base >> 5] = nz;
  }
}

// Warp 0 walks the histogram from the top bin down and finds the bin holding
// descending rank `need` (1-based): res[0] = bin, res[1] = count of keys in
// higher bins, res[2] = count in the bin.  All threads call; result after the
// trailing barrier.
__device__ void find_rank_bin(const uint32_t *hist, int nb, uint32_t need, uint32_t *res) {
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    uint32_t running = 0, fbin = 0, fcum = running, feq = 0;
    bool found = false;
    for (int base = nb - 32; base >= 0 && !found; base -= 32) {
      const uint32_t c = hist[base + 31 - lane];
      uint32_t incl = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += t;
      }
      const uint32_t total = __shfl_sync(FULL, incl, 31);
      if (running + total >= need) {
        const unsigned ballot = __ballot_sync(FULL, running + incl >= need);
        const int f = __ffs(ballot) - 1;
        const uint32_t inc_f = __shfl_sync(FULL, incl, f);
        const uint32_t c_f = __shfl_sync(FULL, c, f);
        fbin = base + 31 - f;
        fcum = running + inc_f - c_f;
        feq = c_f;
        found = true;
      } else {
        running += total;
      }
    }
    if (!found) {  // fewer than `need` keys: every bin lies above
      fbin = 0;
      fcum = running;
      feq = 0;
    }
    if (lane == 0) {
      res[0] = fbin;
      res[1] = fcum;
      res[2] = feq;
    }
  }
  __syncthreads();
}

// Top-11-bit histogram of |col| keys into hist[2048] (warp-aggregated adds).
__device__ void key_histogram(const float *__restrict__ colg, int n, uint32_t *hist) {
  for (int b = threadIdx.x; b < 2048; b += blockDim.x) hist[b] = 0;
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const uint32_t bin = abs_key(colg[i]) >> 20;
    const unsigned peers = __match_any_sync(__activemask(), bin);
    if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&hist[bin], __popc(peers));
  }
  __syncthreads();
}

// Descending bitonic sort of a[0..len), len a power of two.
template <typename T>
__device__ void bitonic_desc(T *a, int len) {
  for (int k = 2; k <= len; k <<= 1) {
    for (int jj = k >> 1; jj > 0; jj >>= 1) {
      for (int i = threadIdx.x; i < len; i += blockDim.x) {
        const int ixj = i ^ jj;
        if (ixj > i) {
          const T x = a[i], y = a[ixj];
          const bool first_block = (i & k) == 0;
          if (first_block ? (x < y) : (x > y)) {
            a[i] = y;
            a[ixj] = x;
          }
        }
      }
      __syncthreads();
    }
  }
}

// The (|v| key << 32 | ~index) pairs of the entries whose bit is set in a
// column's mask (words 32-bit words), the first `cap` of them in index order,
// into out; returns how many bits are set.  Each thread owns a contiguous run
// of words, so an exclusive scan of their counts places the entries in order.
// scratch: one word of shared memory per warp of the block.
__device__ uint32_t pairs_from_mask(const uint32_t *__restrict__ mk, int words,
                                    const float *__restrict__ colg, uint64_t *out, uint32_t cap,
                                    uint32_t *scratch) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int per = (words + blockDim.x - 1) / blockDim.x;
  const int w0 = min(words, (int)threadIdx.x * per), w1 = min(words, w0 + per);
  uint32_t cnt = 0;
  for (int q = w0; q < w1; q++) cnt += __popc(mk[q]);
  uint32_t incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(FULL, incl, o);
    if (lane >= o) incl += t;
  }
  __syncthreads();  // scratch may still be read by the caller's previous use
  if (lane == 31) scratch[w] = incl;
  __syncthreads();
  uint32_t off = incl - cnt, total = 0;
  for (int i = 0; i < nw; i++) {
    if (i < w) off += scratch[i];
    total += scratch[i];
  }
  for (int q = w0; q < w1; q++) {
    uint32_t bits = mk[q];
    while (bits) {
      const int b = __ffs(bits) - 1;
      bits &= bits - 1;
      const uint32_t i = (uint32_t)(q * 32 + b);
      if (off < cap) out[off] = ((uint64_t)abs_key(__ldg(colg + i)) << 32) | (uint32_t)~i;
      off++;
    }
  }
  __syncthreads();
  return total;
}

// ------------------------------------------------------------ L0 constraint
constexpr int HARD_THREADS = 256;
constexpr int HARD_CAND = 2048;  // hinted (key, index) candidates resolved in shared memory

// One streaming pass over a column in global memory (16-byte loads, four in
// flight per thread): the entries with |v| key >= bound go to cand as
// (key << 32 | ~index), the first `cap` of them in any order; returns how many
// there are (it may exceed cap) and leaves in counter[1] the largest key below
// the bound (0 if none).  Entries past n are not taken.
__device__ uint32_t gather_pairs_above(const float *__restrict__ colg, int n, uint32_t bound,
                                       uint64_t *cand, uint32_t cap, uint32_t *counter) {
  if (threadIdx.x == 0) {
    counter[0] = 0;
    counter[1] = 0;
  }
  __syncthreads();
  uint32_t below = 0;
  const int lane = threadIdx.x & 31;
  const int n4 = (n + 3) >> 2;
  const float4 *c4 = reinterpret_cast<const float4 *>(colg);
  constexpr int U = 4;
  for (int base = (threadIdx.x & ~31); base < n4; base += U * blockDim.x) {
    float4 v[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int i = base + u * blockDim.x + lane;
      v[u] = (i < n4) ? __ldg(c4 + i) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int e0 = 4 * (base + u * blockDim.x + lane);
      const float x[4] = {v[u].x, v[u].y, v[u].z, v[u].w};
      uint32_t take = 0;
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const uint32_t key = abs_key(x[q]);
        const bool in = e0 + q < n;
        take |= (uint32_t)(in && key >= bound) << q;
        if (in && key < bound) below = max(below, key);
      }
      if (!__any_sync(FULL, take != 0)) continue;
      const uint32_t mine = __popc(take);
      uint32_t incl = mine;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += t;
      }
      uint32_t wbase = 0;
      if (lane == 31) wbase = atomicAdd(&counter[0], incl);
      wbase = __shfl_sync(FULL, wbase, 31);
      uint32_t pos = wbase + incl - mine;
#pragma unroll
      for (int q = 0; q < 4; q++)
        if (take & (1u << q)) {
          if (pos < cap)
            cand[pos] = ((uint64_t)abs_key(x[q]) << 32) | (uint32_t)~(uint32_t)(e0 + q);
          pos++;
        }
    }
  }
  below = __reduce_max_sync(FULL, below);
  if (lane == 0) atomicMax(&counter[1], below);
  __syncthreads();
  return counter[0];
}

// One streaming pass over a column: every |v| with key >= bound goes to
// list[] (global memory, room for n) as a float, in any order; returns how
// many, and leaves in counter[1] the largest key below the bound (0 if none).
__device__ uint32_t gather_keys_above(const float *__restrict__ colg, int n, uint32_t bound,
                                      float *list, uint32_t *counter) {
  if (threadIdx.x == 0) {
    counter[0] = 0;
    counter[1] = 0;
  }
  __syncthreads();
  uint32_t below = 0;
  const int lane = threadIdx.x & 31;
  for (int base = (threadIdx.x & ~31); base < n; base += blockDim.x) {
    const int i = base + lane;
    const uint32_t key = i < n ? abs_key(colg[i]) : 0u;
    const bool take = i < n && key >= bound;
    if (i < n && !take) below = max(below, key);
    const unsigned bal = __ballot_sync(FULL, take);
    if (!bal) continue;
    uint32_t wbase = 0;
    if (lane == 0) wbase = atomicAdd(&counter[0], (uint32_t)__popc(bal));
    wbase = __shfl_sync(FULL, wbase, 0);
    if (take) list[wbase + __popc(bal & ((1u << lane) - 1u))] = __uint_as_float(key);
  }
  below = __reduce_max_sync(FULL, below);
  if (lane == 0) atomicMax(&counter[1], below);
  __syncthreads();
  return counter[0];
}

// k_hard_thresholding (c++/src/utils/thresh_functions.h:121-145): level = the
// s-th largest |v| (with multiplicity, as the sorting variant :92-98 defines
// it), keep |v| >= level, then x <- x / ||x|| (c++/src/gpower/gpower_commons.h:111).
//
// One block per column, reading it from global memory.  (a) With the previous
// step's level as a hint, a streaming pass gathers the entries with
// |v| >= HINT_FRACTION * hint together with their indices; if fewer than s,
// a second pass gathers down to the largest key below that bound (exactly
// the kept set when one entry was missing).  When that holds s to HARD_CAND
// entries, sorting them gives the exact level, the norm and the kept entries,
// and the column is written sparsely (its mask words cleared, then the kept
// entries' bits and values set).  Otherwise (b) a histogram of the top 11 bits
// of |v| finds the bin holding rank s, keys above it are kept for sure, keys
// in it are gathered and sorted; a bin too full for shared memory falls back
// to (c) the exact three-level radix select; the column is then written by a
// full pass.
__device__ __forceinline__ void hard_select_body(
    const float *__restrict__ Vraw, int ldv, int n, unsigned s, float *__restrict__ Vx,
    uint32_t *__restrict__ nnz_out, int *status, uint32_t *__restrict__ vmask,
    float *__restrict__ hints, const uint32_t *stop, const uint32_t *__restrict__ cmask, int j) {
  if (*stop) return;
  __shared__ uint64_t cand[HARD_CAND];  // also 2 * HARD_CAND keys for (b)
  __shared__ uint32_t hist[2048];
  __shared__ uint32_t res[8];
  __shared__ double red[32];
  uint32_t *cand32 = reinterpret_cast<uint32_t *>(cand);
  const float *colg = Vraw + (size_t)j * ldv;
  float *vx = Vx + (size_t)j * ldv;
  uint32_t *mk = vmask + (size_t)j * (ldv >> 5);
  uint32_t thr = 0;
  double ss = 0.0, cnt = 0.0;
  bool done = false;
  const float hint = hints[j];
  uint32_t bound = hinted_bound(hint);
  for (int attempt = 0; attempt < 2 && hint > 0.f && !done; attempt++) {
    uint32_t c = 0, below = 0;
    bool listed = false;
    if (attempt == 0 && cmask) {
      // V = B^T Z's epilogue marked the entries at or above the same bound
      // (it keeps no largest key below the bound: with fewer than s entries the
      // column is gathered here as before)
      c = pairs_from_mask(cmask + (size_t)j * (ldv >> 5), ldv >> 5, colg, cand, HARD_CAND,
                          &res[0]);
      listed = c >= s;
    }
    if (!listed) {
      c = gather_pairs_above(colg, n, bound, cand, HARD_CAND, &res[0]);
      below = res[1];
    }
    if (c > (uint32_t)HARD_CAND) break;  // too many: the histogram path
    if (c < s) {
      // short by one: the s-th largest is the largest key below the bound, so
      // gathering down to it takes exactly the kept entries; otherwise widen
      bound = (s - c == 1) ? below : abs_key(HINT_FRACTION * __uint_as_float(below));
      if (bound == 0) break;
    } else {
      int len = 1;
      while (len < (int)c) len <<= 1;
      for (int q = c + threadIdx.x; q < len; q += blockDim.x) cand[q] = 0ull;
      __syncthreads();
      bitonic_desc(cand, len);
      thr = (uint32_t)(cand[s - 1] >> 32);
      // kept: the sorted prefix with key >= thr (ties with the s-th included)
      if (threadIdx.x == 0) res[1] = 0;
      __syncthreads();
      for (int q = threadIdx.x; q < (int)c; q += blockDim.x) {
        const uint32_t key = (uint32_t)(cand[q] >> 32);
        if (key >= thr && (q + 1 == (int)c || (uint32_t)(cand[q + 1] >> 32) < thr))
          res[1] = q + 1;
        if (key >= thr) {
          const double v = (double)__uint_as_float(key);
          ss += v * v;
        }
      }
      done = true;
    }
    __syncthreads();
  }
  if (done) {
    const uint32_t kept = res[1];
    ss = block_sum(ss, red);
    const float inv = 1.0f / (float)sqrt(ss);
    for (int w = threadIdx.x; w < (ldv >> 5); w += blockDim.x) mk[w] = 0u;
    __syncthreads();
    for (int q = threadIdx.x; q < (int)kept; q += blockDim.x) {
      const uint32_t i = ~(uint32_t)cand[q];
      vx[i] = __ldg(colg + i) * inv;
      atomicOr(&mk[i >> 5], 1u << (i & 31));
    }
    cnt = (double)kept;
  } else {
    // (b) histogram of the top 11 key bits, then the bin holding rank s
    key_histogram(colg, n, hist);
    find_rank_bin(hist, 2048, s, res);
    const uint32_t b1 = res[0], above = res[1], in_bin = res[2];
    __syncthreads();
    if (in_bin <= (uint32_t)(2 * HARD_CAND)) {
      if (threadIdx.x == 0) res[3] = 0;
      __syncthreads();
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const uint32_t key = abs_key(colg[i]);
        const uint32_t bin = key >> 20;
        if (bin > b1) {
          const double v = (double)__uint_as_float(key);
          ss += v * v;
          cnt += 1.0;
        } else if (bin == b1) {
          cand32[atomicAdd(&res[3], 1u)] = key;
        }
      }
      __syncthreads();
      const int nc = (int)res[3];
      int len = 1;
      while (len < nc) len <<= 1;
      for (int q = nc + threadIdx.x; q < len; q += blockDim.x) cand32[q] = 0u;
      __syncthreads();
      bitonic_desc(cand32, len);
      thr = cand32[s - above - 1];
      for (int q = threadIdx.x; q < nc; q += blockDim.x)
        if (cand32[q] >= thr) {
          const double v = (double)__uint_as_float(cand32[q]);
          ss += v * v;
          cnt += 1.0;
        }
    } else {
      // (c) exact radix select
      thr = block_select(colg, n, s, hist, res).key;
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const float v = colg[i];
        if (abs_key(v) >= thr) {
          ss += (double)v * (double)v;
          cnt += 1.0;
        }
      }
    }
    ss = block_sum(ss, red);
    cnt = block_sum(cnt, red);
    const float inv = 1.0f / (float)sqrt(ss);
    write_column_global(colg, n, vx, mk,
                        [=](float v) { return (abs_key(v) >= thr) ? v * inv : 0.f; });
  }
  if (threadIdx.x == 0) {
    hints[j] = __uint_as_float(thr);
    nnz_out[j] = (uint32_t)cnt;
  }
}
__global__ void __launch_bounds__(HARD_THREADS) hard_select_kernel(
    const float *__restrict__ Vraw, int ldv, int n, unsigned s, float *__restrict__ Vx,
    uint32_t *__restrict__ nnz_out, int *status, uint32_t *__restrict__ vmask,
    float *__restrict__ hints, const uint32_t *stop, const uint32_t *__restrict__ cmask) {
  hard_select_body(Vraw, ldv, n, s, Vx, nnz_out, status, vmask, hints, stop, cmask, blockIdx.x);
}

// ------------------------------------------------------------ L1 constraint
constexpr int SOFT_C = 1024;  // sorted-candidate chunk (power of two for the bitonic sort)
constexpr int SOFT_THREADS = 256;
// hinted candidates sorted at once (then scanned a chunk at a time)
constexpr int SOFT_HINT_CAP = 4096;
constexpr int SOFT_SMEM = 8 * SOFT_HINT_CAP + 4 * SOFT_C + 2 * 8 * SOFT_C;

// Unfused double arithmetic (no FMA contraction), as host C++ evaluates it.
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
// (S1 - t l) / sqrt(S2 - 2 l S1 + t l^2): ||(|v| - l)_+||_1 / ||(|v| - l)_+||_2 over the
// top t entries, in the reference's operation order (thresh_functions.h:193-204).
__device__ __forceinline__ double ratio_at(double S1, double S2, double t, double l) {
  const double num = dsub(S1, dmul(t, l));
  const double den = __dadd_rn(dsub(S2, dmul(dmul(2.0, l), S1)), dmul(dmul(t, l), l));
  return __ddiv_rn(num, __dsqrt_rn(den));
}

// Inclusive prefix sums of cand[0..total) (0 beyond), in double, offset by
// (o1, o2) for the values and their squares.  4 items per thread.
__device__ void block_scan2(const float *cand, int total, double o1, double o2, double *p1,
                            double *p2, double *red) {
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int base = t * (SOFT_C / SOFT_THREADS);
  double a[SOFT_C / SOFT_THREADS], b[SOFT_C / SOFT_THREADS];
  double s1 = 0, s2 = 0;
#pragma unroll
  for (int q = 0; q < SOFT_C / SOFT_THREADS; q++) {
    const double v = (base + q < total) ? (double)cand[base + q] : 0.0;
    s1 += v;
    s2 += v * v;
    a[q] = s1;
    b[q] = s2;
  }
  // exclusive scan of (s1, s2) over threads
  double x1 = s1, x2 = s2;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const double y1 = __shfl_up_sync(FULL, x1, o), y2 = __shfl_up_sync(FULL, x2, o);
    if (lane >= o) {
      x1 += y1;
      x2 += y2;
    }
  }
  __syncthreads();
  if (lane == 31) {
    red[w] = x1;
    red[16 + w] = x2;
  }
  __syncthreads();
  double w1 = 0, w2 = 0;
  for (int i = 0; i < w; i++) {
    w1 += red[i];
    w2 += red[16 + i];
  }
  const double e1 = o1 + w1 + x1 - s1, e2 = o2 + w2 + x2 - s2;
#pragma unroll
  for (int q = 0; q < SOFT_C / SOFT_THREADS; q++) {
    p1[base + q] = e1 + a[q];
    p2[base + q] = e2 + b[q];
  }
  __syncthreads();
}

__device__ void bitonic_sort_desc(float *a) {
  for (int k = 2; k <= SOFT_C; k <<= 1) {
    for (int jj = k >> 1; jj > 0; jj >>= 1) {
      for (int i = threadIdx.x; i < SOFT_C; i += blockDim.x) {
        const int ixj = i ^ jj;
        if (ixj > i) {
          const float x = a[i], y = a[ixj];
          const bool first_block = (i & k) == 0;
          if (first_block ? (x < y) : (x > y)) {
            a[i] = y;
            a[ixj] = x;
          }
        }
      }
      __syncthreads();
    }
  }
}

// Evaluates the reference scan's stopping predicates (or, EXACT, the exact
// projection's segment test) at chunk positions q in [0, E) of a descending
// sorted chunk; global rank index g = base + q.  p1/p2 are inclusive prefix
// sums including everything before the chunk (S1, S2).  The value below
// position q is cand[q + 1], or lo_after for the chunk's last position.
// Per thread: the smallest stopping g found and its level; w_last gets the
// '+' root at g = n - 1 (the reference's level when it never stops).
template <bool EXACT>
__device__ void eval_chunk(const float *cand, const double *p1, const double *p2, uint32_t total,
                           uint32_t E, uint32_t base, uint32_t n, double S1, double S2,
                           double lo_after, double sq, double sq2, double lim, uint32_t &best,
                           double &bw, double &w_last) {
  for (uint32_t q = threadIdx.x; q < E; q += blockDim.x) {
    const uint32_t g = base + q;
    const double t = (double)(g + 1);
    const double hi = (double)cand[q];
    const double lov = (q + 1 < total) ? (double)cand[q + 1] : lo_after;
    const double S1i = p1[q], S2i = p2[q];
    if (!EXACT) {
      // Same operations, order and (unfused) rounding as the reference's
      // expressions at thresh_functions.h:193-213; several of its stops are
      // decided by the last bit (e.g. a zero discriminant at the first step).
      const double S1p = q ? p1[q - 1] : S1, S2p = q ? p2[q - 1] : S2;
      const double left = ratio_at(S1i, S2i, t, hi);
      const double rprev = (g == 0) ? sq : ratio_at(S1p, S2p, t - 1.0, hi);
      const double a = dmul(t, dsub(t, sq2));
      const double b = dsub(dmul(dmul(2.0, S1i), sq2), dmul(dmul(2.0, t), S1i));
      const double c = dsub(dmul(S1i, S1i), dmul(sq2, S2i));
      const double disc = __dsqrt_rn(dsub(dmul(b, b), dmul(dmul(4.0, a), c)));
      const double wm = __ddiv_rn(dsub(-b, disc), dmul(2.0, a));
      const double wp = __ddiv_rn(__dadd_rn(-b, disc), dmul(2.0, a));
      if (g + 1 == n) w_last = wp;
      double cw = 0.0;
      bool hit = false;
      if (left > sq && rprev < sq) {
        hit = true;
        cw = hi;
      } else if (wm > lov && wm < hi) {
        hit = true;
        cw = wm;
      } else if (wp > lov && wp < hi && wp < lim) {
        hit = true;
        cw = wp;
      }
      if (hit && g < best) {
        best = g;
        bw = cw;
      }
    } else {
      const double rlo = (S1i - t * lov) / sqrt(S2i - 2.0 * lov * S1i + t * lov * lov);
      if (rlo >= sq && g < best) {
        const double a = t * (t - sq2);
        const double b = 2.0 * S1i * sq2 - 2.0 * t * S1i;
        const double c = S1i * S1i - sq2 * S2i;
        double lam;
        if (a == 0.0) {
          lam = -c / b;
        } else {
          const double disc = sqrt(fmax(b * b - 4.0 * a * c, 0.0));
          const double r1 = (-b - disc) / (2.0 * a), r2 = (-b + disc) / (2.0 * a);
          // the genuine root keeps every one of the t entries above it
          const bool ok1 = r1 >= lov && r1 <= hi, ok2 = r2 >= lov && r2 <= hi;
          lam = ok1 ? r1 : ok2 ? r2 : fmin(fmax(r1, lov), hi);
        }
        best = g;
        bw = lam;
      }
    }
  }
}

// Block minimum of the per-thread stopping rank; the owning thread publishes
// its level.  Returns the rank (0xFFFFFFFF when nobody stopped) and sets *w.
__device__ uint32_t resolve_stop(uint32_t best, double bw, uint32_t *res,
                                 volatile uint32_t *misc, double *w_sh, double *w) {
  uint32_t mb = best;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mb = min(mb, __shfl_xor_sync(FULL, mb, o));
  if ((threadIdx.x & 31) == 0) res[4 + (threadIdx.x >> 5)] = mb;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t m2 = 0xFFFFFFFFu;
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) m2 = min(m2, res[4 + i]);
    misc[1] = m2;
  }
  __syncthreads();
  const uint32_t brk = misc[1];
  if (brk != 0xFFFFFFFFu && best == brk) *w_sh = bw;
  __syncthreads();
  if (brk != 0xFFFFFFFFu) *w = *w_sh;
  __syncthreads();
  return brk;
}

// soft_thresholding (c++/src/utils/thresh_functions.h:162-254): the level w
// and x = sgn(v)(|v| - w)_+, then x <- x / ||x||.
//
// The reference sorts |v| and scans it from the top, stopping at the first
// index i where one of three predicates holds (:197-216).  Common case, three
// passes over the column: a histogram of the top 11 bits of |v| picks the
// highest bins holding at most SOFT_C values; one pass gathers them (and the
// largest value below them); they are sorted in shared memory, prefix sums
// in double give S1 and S2 at every rank, and all ranks' predicates are
// evaluated at once -- the smallest stopping rank wins, and the norm comes
// from the gathered values; a last pass writes the loadings.  When the stop
// lies deeper, the column is walked exactly a chunk of SOFT_C ranks at a time
// (radix select of each chunk boundary, ties by count); a column that never
// stops is walked to its end as in the reference (w is then the '+' root of
// the last step).
// EXACT: stop at the first segment whose lower knot already gives
// ||.||_1/||.||_2 >= sqrt(s) and take the root inside it -- the exact
// L1-ball / unit-sphere projection.
// The reference scan's exact walk over the values src(0..len) (all of a
// column's entries above some bound, or the whole column when len == n), a
// chunk of SOFT_C ranks at a time: each chunk's keys are found by a radix
// select of its lowest rank, gathered, sorted and scanned, and the stopping
// predicates evaluated rank by rank.  lo_end is the largest value below the
// set (0 for the whole column).  Returns the stopping rank and sets *w; NONE
// when the set ran out first (len < n), and the caller walks the column.
template <bool EXACT, class Src>
__device__ __noinline__ uint32_t exact_walk(Src src, uint32_t len, uint32_t n, double lo_end, float *cand,
                               double *p1, double *p2, uint32_t *hist, uint32_t *res,
                               double *red, volatile uint32_t *misc, double *w_sh, double sq,
                               double sq2, double *w) {
  const uint32_t NONE = 0xFFFFFFFFu;
  if (len == 0) return NONE;
  uint32_t brk = NONE;
  const SelResult top = block_select_src(src, (int)len, 1u, hist, res);
  const double lim = __dsub_rn((double)__uint_as_float(top.key), 0.000001);
  uint32_t consumed = 0, khi = NONE, ge_hi = 0;
  double S1 = 0.0, S2 = 0.0;
  while (true) {
    const uint32_t R = min(consumed + (uint32_t)SOFT_C, len);
    const uint32_t total = R - consumed;
    const SelResult lo = block_select_src(src, (int)len, R, hist, res);
    if (threadIdx.x == 0) misc[0] = 0;
    __syncthreads();
    if (lo.key == khi) {
      const float v = __uint_as_float(khi);
      for (uint32_t q = threadIdx.x; q < total; q += blockDim.x) cand[q] = v;
    } else {
      for (int i = threadIdx.x; i < (int)len; i += blockDim.x) {
        const uint32_t key = abs_key(src(i));
        if (key > lo.key && key < khi)
          cand[atomicAdd((uint32_t *)&misc[0], 1u)] = __uint_as_float(key);
      }
      __syncthreads();
      const uint32_t nb = misc[0];
      const uint32_t c_hi = ge_hi - consumed;
      const uint32_t c_lo = R - lo.gt;
      const float vhi = __uint_as_float(khi), vlo = __uint_as_float(lo.key);
      for (uint32_t q = threadIdx.x; q < c_hi + c_lo; q += blockDim.x)
        cand[nb + q] = (q < c_hi) ? vhi : vlo;
    }
    for (uint32_t q = total + threadIdx.x; q < (uint32_t)SOFT_C; q += blockDim.x) cand[q] = -1.f;
    __syncthreads();
    bitonic_sort_desc(cand);
    block_scan2(cand, (int)total, S1, S2, p1, p2, red);
    // the last position of a chunk waits for the next chunk's first value,
    // except at the end of the set, where the value below it is lo_end
    const uint32_t E = (R == len) ? total : total - 1;
    uint32_t best = NONE;
    double bw = 0.0, w_last = 0.0;
    eval_chunk<EXACT>(cand, p1, p2, total, E, consumed, n, S1, S2, lo_end, sq, sq2, lim, best, bw,
                      w_last);
    brk = resolve_stop(best, bw, res, misc, w_sh, w);
    if (brk != NONE) break;
    if (R == len) {
      if (len == n) {
        // never stopped: the reference keeps the '+' root of its last step;
        // the exact projection with ratio < sqrt(s) everywhere is lambda = 0
        if (!EXACT && consumed + E - 1 == n - 1 && threadIdx.x == (E - 1) % blockDim.x)
          *w_sh = w_last;
        if (EXACT && threadIdx.x == 0) *w_sh = 0.0;
        __syncthreads();
        *w = *w_sh;
        __syncthreads();
      }
      break;
    }
    consumed += E;
    S1 = p1[E - 1];
    S2 = p2[E - 1];
    khi = lo.key;
    ge_hi = lo.gt + lo.eq;
    __syncthreads();
  }
  return brk;
}

template <bool EXACT>
__device__ __forceinline__ void soft_select_body(
    const float *__restrict__ Vraw, int ldv, int n, unsigned s, float *__restrict__ Vx,
    uint32_t *__restrict__ nnz_out, int *status, uint32_t *__restrict__ vmask,
    float *__restrict__ hints, const uint32_t *stop, const uint32_t *__restrict__ cmask, int j) {
  if (*stop) return;
  // dynamic shared memory (SOFT_SMEM bytes): the hinted (key, index)
  // candidates, a chunk of sorted values and its prefix sums; the histogram
  // of the slower paths reuses the candidates' space (those paths run only
  // when the hinted one found no stop, and then its pairs are not needed)
  extern __shared__ __align__(16) uint8_t soft_smem[];
  uint64_t *pairs = reinterpret_cast<uint64_t *>(soft_smem);        // SOFT_HINT_CAP
  float *cand = reinterpret_cast<float *>(soft_smem + 8 * SOFT_HINT_CAP);  // SOFT_C
  double *p1 = reinterpret_cast<double *>(soft_smem + 8 * SOFT_HINT_CAP + 4 * SOFT_C);
  double *p2 = p1 + SOFT_C;
  uint32_t *hist = reinterpret_cast<uint32_t *>(soft_smem);           // 2048, over pairs
  __shared__ uint32_t res[32];
  __shared__ double red[32];
  __shared__ uint32_t misc_raw[16];
  __shared__ double w_shared;
  volatile uint32_t *misc = misc_raw;
  double *w_sh = &w_shared;

  const float *colg = Vraw + (size_t)j * ldv;
  // sqrt(s), sqrt(s)^2 as the double-precision reference forms them
  const double sq = __dsqrt_rn((double)s);
  const double sq2 = __dmul_rn(sq, sq);
  const uint32_t NONE = 0xFFFFFFFFu;

  double w = 0.0;
  uint32_t brk = NONE;
  bool have_norm = false;  // ss and cnt already summed over the gathered values
  bool sparse = false;     // ... and the gathered pairs hold every kept entry
  uint32_t c_pairs = 0;
  double ss = 0.0, cnt = 0.0;
  // ---- hinted path: gather (key, index) with |v| >= HINT_FRACTION * (previous level)
  const float hint = hints[j];
  uint32_t c_hint = 0;  // entries at or above the hinted bound
  if (hint > 0.f) {
    uint32_t c, below_key = 0;
    const bool listed = cmask != nullptr;
    if (listed) {  // marked by V = B^T Z's epilogue, with the same bound
      c = pairs_from_mask(cmask + (size_t)j * (ldv >> 5), ldv >> 5, colg, pairs, SOFT_HINT_CAP,
                          res);
    } else {
      c = gather_pairs_above(colg, n, hinted_bound(hint), pairs, SOFT_HINT_CAP, res);
      below_key = res[1];
    }
    c_hint = c;
    __syncthreads();
    if (c > 0 && c <= (uint32_t)SOFT_HINT_CAP) {
      int len = 1;
      while (len < (int)c) len <<= 1;
      for (int q = c + threadIdx.x; q < len; q += blockDim.x) pairs[q] = 0ull;
      __syncthreads();
      bitonic_desc(pairs, len);
      // the sorted set, a chunk of SOFT_C ranks at a time; every position sees
      // its next value in the set, except the set's last: for a listed set
      // (no largest value below it) that one is left to the paths below
      const double lim =
          __dsub_rn((double)__uint_as_float((uint32_t)(pairs[0] >> 32)), 0.000001);
      const double lo_after = (c == (uint32_t)n) ? 0.0 : (double)__uint_as_float(below_key);
      double S1 = 0.0, S2 = 0.0, w_last = 0.0;
      uint32_t q0 = 0;
      for (;;) {
        const uint32_t total = min((uint32_t)SOFT_C, c - q0);
        const bool last = q0 + total == c;
        for (uint32_t q = threadIdx.x; q < (uint32_t)SOFT_C; q += blockDim.x)
          cand[q] = (q < total) ? __uint_as_float((uint32_t)(pairs[q0 + q] >> 32)) : -1.f;
        __syncthreads();
        const double next =
            last ? lo_after : (double)__uint_as_float((uint32_t)(pairs[q0 + total] >> 32));
        const uint32_t E = (last && listed && c < (uint32_t)n) ? total - 1 : total;
        block_scan2(cand, (int)total, S1, S2, p1, p2, red);
        uint32_t best = NONE;
        double bw = 0.0;
        eval_chunk<EXACT>(cand, p1, p2, total, E, q0, (uint32_t)n, S1, S2, next, sq, sq2, lim,
                          best, bw, w_last);
        brk = resolve_stop(best, bw, res, misc, w_sh, &w);
        if (brk != NONE || last) break;
        S1 = p1[total - 1];
        S2 = p2[total - 1];
        q0 += total;
        __syncthreads();
      }
      if (brk == NONE && c == (uint32_t)n) {
        // never stopped: the '+' root at the column's last rank (evaluated by
        // the thread holding that position of the last chunk)
        if (!EXACT && threadIdx.x == (c - 1 - q0) % blockDim.x) *w_sh = w_last;
        if (EXACT && threadIdx.x == 0) *w_sh = 0.0;
        __syncthreads();
        w = *w_sh;
        brk = (uint32_t)n;
        __syncthreads();
      }
      if (brk != NONE) {
        // the level lies at or above every value outside the gathered set
        for (uint32_t q = threadIdx.x; q < c; q += blockDim.x) {
          const double d = (double)__uint_as_float((uint32_t)(pairs[q] >> 32)) - w;
          if (d > 0.0) {
            const double x = (double)(float)d;
            ss += x * x;
            cnt += 1.0;
          }
        }
        have_norm = true;
        sparse = true;
        c_pairs = c;
      }
    }
    __syncthreads();
  }

  // ---- more than SOFT_HINT_CAP entries above the hinted bound: the exact
  // walk over them alone (a compact list in this column of Vx, which the
  // writes below overwrite); it gives up if the stop lies below the bound
  if (brk == NONE && c_hint > (uint32_t)SOFT_HINT_CAP && c_hint < (uint32_t)n) {
    float *list = Vx + (size_t)j * ldv;
    const uint32_t cl = gather_keys_above(colg, n, hinted_bound(hint), list, res);
    const double lo_end = (double)__uint_as_float(res[1]);
    brk = exact_walk<EXACT>(ListSrc{list}, cl, (uint32_t)n, lo_end, cand, p1, p2, hist, res, red,
                            misc, w_sh, sq, sq2, &w);
  }

  // ---- fast path: the highest bins holding at most SOFT_C values
  uint32_t c = 0, bstar = 0;
  bool hist_ok = false;  // hist holds the column's top-bit histogram
  if (brk == NONE) {
    key_histogram(colg, n, hist);
    hist_ok = true;
    find_rank_bin(hist, 2048, (uint32_t)SOFT_C + 1u, res);
    const bool whole = (uint32_t)n <= (uint32_t)SOFT_C;
    bstar = whole ? 0u : res[0] + 1u;  // gather bins >= bstar
    c = whole ? (uint32_t)n : res[1];
    __syncthreads();
  }
  if (brk == NONE && c > 0) {
    if (threadIdx.x == 0) {
      misc[0] = 0;
      misc[2] = 0;
    }
    __syncthreads();
    uint32_t below = 0;  // largest key under the gathered bins
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const uint32_t key = abs_key(colg[i]);
      if ((key >> 20) >= bstar) cand[atomicAdd((uint32_t *)&misc[0], 1u)] = __uint_as_float(key);
      else below = max(below, key);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) below = max(below, __shfl_xor_sync(FULL, below, o));
    if ((threadIdx.x & 31) == 0) atomicMax((uint32_t *)&misc[2], below);
    for (uint32_t q = c + threadIdx.x; q < (uint32_t)SOFT_C; q += blockDim.x) cand[q] = -1.f;
    __syncthreads();
    const double lo_after = (c == (uint32_t)n) ? 0.0 : (double)__uint_as_float(misc[2]);
    bitonic_sort_desc(cand);
    block_scan2(cand, (int)c, 0.0, 0.0, p1, p2, red);
    const double lim = __dsub_rn((double)cand[0], 0.000001);  // ||v||_inf - 1e-6
    uint32_t best = NONE;
    double bw = 0.0, w_last = 0.0;
    eval_chunk<EXACT>(cand, p1, p2, c, c, 0, (uint32_t)n, 0.0, 0.0, lo_after, sq, sq2, lim, best,
                      bw, w_last);
    brk = resolve_stop(best, bw, res, misc, w_sh, &w);
    if (brk == NONE && c == (uint32_t)n) {
      // never stopped: the reference keeps the '+' root of its last step;
      // the exact projection with ratio < sqrt(s) everywhere is lambda = 0
      if (!EXACT && threadIdx.x == (c - 1) % blockDim.x) *w_sh = w_last;
      if (EXACT && threadIdx.x == 0) *w_sh = 0.0;
      __syncthreads();
      w = *w_sh;
      brk = (uint32_t)n;
      __syncthreads();
    }
    if (brk != NONE) {
      // every value above w sits in the gathered chunk
      for (uint32_t q = threadIdx.x; q < c; q += blockDim.x) {
        const double d = (double)cand[q] - w;
        if (d > 0.0) {
          const double x = (double)(float)d;
          ss += x * x;
          cnt += 1.0;
        }
      }
      have_norm = true;
    }
  }

  // ---- exact walk, a chunk of SOFT_C ranks at a time: over the entries in
  // the histogram's bins holding the top 8 * SOFT_C ranks first (a compact
  // list in this column of Vx), then, if the stop lies below them, over the
  // column
  if (brk == NONE && hist_ok && n > 8 * SOFT_C) {
    // the fast path's histogram: the bins holding the top 8 * SOFT_C ranks
    find_rank_bin(hist, 2048, 8u * (uint32_t)SOFT_C, res);
    const uint32_t bound = res[0] << 20;
    __syncthreads();
    float *list = Vx + (size_t)j * ldv;
    const uint32_t cl = gather_keys_above(colg, n, bound, list, res);
    if (cl < (uint32_t)n) {
      const double lo_end = (double)__uint_as_float(res[1]);
      brk = exact_walk<EXACT>(ListSrc{list}, cl, (uint32_t)n, lo_end, cand, p1, p2, hist, res,
                              red, misc, w_sh, sq, sq2, &w);
    }
  }
  if (brk == NONE)
    brk = exact_walk<EXACT>(ColumnSrc{colg}, (uint32_t)n, (uint32_t)n, 0.0, cand, p1, p2, hist,
                            res, red, misc, w_sh, sq, sq2, &w);

  if (threadIdx.x == 0) hints[j] = (float)w;
  // x = sgn(v)(|v| - w)_+ with w kept in double: a level that lands within
  // rounding of the largest |v| still leaves that entry non-zero, as in the
  // reference's double arithmetic.
  if (!have_norm) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const float v = colg[i];
      const double d = (double)fabsf(v) - w;
      if (d > 0.0) {
        const double x = (double)(float)d;
        ss += x * x;
        cnt += 1.0;
      }
    }
  }
  ss = block_sum(ss, red);
  cnt = block_sum(cnt, red);
  const float inv = 1.0f / (float)sqrt(ss);
  float *vx = Vx + (size_t)j * ldv;
  auto soft = [=](float v) {
    const double d = (double)fabsf(v) - w;
    return ((d > 0.0) ? (float)d * sgnf(v) : 0.f) * inv;
  };
  uint32_t *mk = vmask + (size_t)j * (ldv >> 5);
  if (sparse) {
    // every kept entry is a gathered pair: clear the mask, then set the kept
    for (int wd = threadIdx.x; wd < (ldv >> 5); wd += blockDim.x) mk[wd] = 0u;
    __syncthreads();
    for (uint32_t q = threadIdx.x; q < c_pairs; q += blockDim.x) {
      const uint32_t i = ~(uint32_t)pairs[q];
      const float x = soft(__ldg(colg + i));
      if (x != 0.f) {
        vx[i] = x;
        atomicOr(&mk[i >> 5], 1u << (i & 31));
      }
    }
  } else {
    write_column_global(colg, n, vx, mk, soft);
  }
  if (threadIdx.x == 0) {
    nnz_out[j] = (uint32_t)cnt;
  }
}
template <bool EXACT>
__global__ void __launch_bounds__(SOFT_THREADS, 4) soft_select_kernel(
    const float *__restrict__ Vraw, int ldv, int n, unsigned s, float *__restrict__ Vx,
    uint32_t *__restrict__ nnz_out, int *status, uint32_t *__restrict__ vmask,
    float *__restrict__ hints, const uint32_t *stop, const uint32_t *__restrict__ cmask) {
  soft_select_body<EXACT>(Vraw, ldv, n, s, Vx, nnz_out, status, vmask, hints, stop, cmask,
                          blockIdx.x);
}

// ------------------------------------------------------------ finalize
// Per start: objective f, relative change |f - f0| / f0
// (c++/src/utils/termination_criteria.h:30-36), the storeIterationsForAllPoints
// logs (c++/src/gpower/gpower_commons.h:120-130), and the batch maximum that
// ignores NaN changes (:132-133).  One block.
struct FinalizeArgs {
  int k, formulation, parts, it, store_all, log_shift, log_capacity;
  double tolerance;
  const float *fz;
  const float *obj_part, *nnz_part;
  const uint32_t *nnz_sel;
  float *val, *err, *max_err;
  uint32_t *max_nnz;
  int *iters, *cards;
  // run-ahead control (StepCtl words); stop_check: this step may stop the batch
  uint32_t *ctl;
  const uint32_t *phase;  // MIXED: phase[3] is the phase the step ran in; else null
  const int *status;
  int stop_check;
};

// One warp per start; the batch maximum is an atomicMax on the bit pattern
// of the (non-negative, non-NaN) changes, zeroed before the step -- max is
// order-independent, so the result is deterministic.
__device__ void finalize_start(const FinalizeArgs &a, int j, int lane);

// The last block to finish also closes the step for the run-ahead driver: it
// counts the step (and, MIXED, whether it ran in the BF16 phase), keeps the
// batch's largest change, and sets the stop word when the reference's batch
// loop would end here (it > 0, a refinement step, max change < tolerance) or
// a device-side wait gave up.
__global__ void __launch_bounds__(256) finalize_kernel(FinalizeArgs a) {
  if (a.ctl[CTL_STOP]) return;
  const int lane = threadIdx.x & 31;
  const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (j < a.k) finalize_start(a, j, lane);
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&a.ctl[CTL_BLOCKS], 1u) == gridDim.x - 1) {
      __threadfence();
      const float me = *reinterpret_cast<volatile float *>(a.max_err);
      const bool refined = a.phase == nullptr || a.phase[3] != 0u;
      a.ctl[CTL_STEPS] += 1u;
      if (!refined) a.ctl[CTL_LOW_STEPS] += 1u;
      a.ctl[CTL_MAX_ERR] = __float_as_uint(me);
      if ((a.stop_check && a.it > 0 && refined && (double)me < a.tolerance) ||
          *reinterpret_cast<const volatile int *>(a.status) != 0)
        a.ctl[CTL_STOP] = 1u;
      a.ctl[CTL_BLOCKS] = 0u;
    }
  }
}

// One start's objective, change and logs (one warp; lane 0 writes).
__device__ void finalize_start(const FinalizeArgs &a, int j, int lane) {
  const bool cons = a.formulation <= 3;
  const bool l1pen = a.formulation >= 6;
  float f;
  uint32_t nz;
  if (cons) {
    f = a.fz[j];
    nz = a.nnz_sel[j];
  } else {
    // fixed order: lane-strided partial sums, then a butterfly
    double acc = 0.0, c = 0.0;
    for (int q = lane; q < a.parts; q += 32) {
      acc += (double)a.obj_part[(size_t)j * a.parts + q];
      c += (double)a.nnz_part[(size_t)j * a.parts + q];
    }
    acc = warp_sum(acc);
    c = warp_sum(c);
    f = l1pen ? (float)sqrt(acc) : (float)acc;
    nz = (uint32_t)c;
  }
  if (lane != 0) return;
  atomicMax(a.max_nnz, nz);
  const float f0 = a.val[j];
  const float e = fabsf(f - f0) / f0;
  a.err[j] = e;
  a.val[j] = f;
  // the reference's `if (max < e) max = e`: NaN never wins
  if (e > 0.f) atomicMax(reinterpret_cast<unsigned int *>(a.max_err), __float_as_uint(e));
  if (a.store_all) {
    // the penalized thresholding calls log into slot j of every batch
    // (gpower_commons.h:170,173 leave the batch shift at 0)
    const int slot = cons ? a.log_shift + j : j;
    if (slot < a.log_capacity) {
      const bool done = a.it > 0 && (double)e < a.tolerance;
      if (done && a.iters[slot] == -1) {
        a.iters[slot] = a.it;
        a.cards[slot] = (int)nz;
      } else if (!done && a.iters[slot] != -1) {
        a.iters[slot] = -1;
      }
    }
  }
}

// x = v / ||v|| (c++/src/gpower/sparse_PCA_solver.h:236-237).
__global__ void finalize_x_kernel(const float *__restrict__ v, int n, float *__restrict__ x) {
  __shared__ double red[32];
  double ss = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) ss += (double)v[i] * (double)v[i];
  ss = block_sum(ss, red);
  const float inv = 1.0f / (float)sqrt(ss);
  for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = v[i] * inv;
}

// Partial sums of y_i = sum_c B[i, c] x_c in FP64 over chunks of EV_CHUNK
// features: partial[chunk * m + i], threads over samples (coalesced reads of
// B's columns), features with x_c = 0 skipped, a fixed order per chunk.
__global__ void __launch_bounds__(256) ev_partial_kernel(const float *__restrict__ Bc, int ldm,
                                                         int m, int n, const float *__restrict__ x,
                                                         double *__restrict__ partial) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int c0 = blockIdx.y * EV_CHUNK, c1 = min(n, c0 + EV_CHUNK);
  double acc = 0.0;
  for (int c = c0; c < c1; c++) {
    const float xc = x[c];
    if (xc != 0.f) acc += (double)Bc[(size_t)c * ldm + i] * (double)xc;
  }
  partial[(size_t)blockIdx.y * m + i] = acc;
}

// ||y||^2 with y_i the sum of its chunks' partials (in chunk order).
__global__ void ev_sum_kernel(const double *__restrict__ partial, int chunks, int m,
                              double *__restrict__ out) {
  __shared__ double red[32];
  double acc = 0.0;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    double y = 0.0;
    for (int c = 0; c < chunks; c++) y += partial[(size_t)c * m + i];
    acc += y * y;
  }
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) *out = acc;
}

// Compressed sparse columns into B's dense layout (zeroed before): one block
// per column.
__global__ void csc_scatter_kernel(const float *__restrict__ vals,
                                   const int32_t *__restrict__ row_ind,
                                   const int32_t *__restrict__ col_ptr, float *__restrict__ Bc,
                                   int ldm) {
  const size_t c = blockIdx.x;
  for (int q = col_ptr[c] + threadIdx.x; q < col_ptr[c + 1]; q += blockDim.x)
    Bc[c * ldm + row_ind[q]] = vals[q];
}

// The sparse solver's implicit centring made explicit:
// b <- (b - means[c]) - row_means[i] in FP32, either correction optional.
__global__ void center_kernel(float *__restrict__ Bc, int ldm, int m,
                              const float *__restrict__ means,
                              const float *__restrict__ row_means) {
  const size_t c = blockIdx.x;
  const float mc = means ? means[c] : 0.f;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    float b = Bc[c * ldm + i];
    if (means) b = b - mc;
    if (row_means) b = b - row_means[i];
    Bc[c * ldm + i] = b;
  }
}

// y_i = the sum of its chunks' partials (in chunk order), FP64.
__global__ void rowsum_kernel(const double *__restrict__ partial, int chunks, int m,
                              double *__restrict__ y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  double acc = 0.0;
  for (int c = 0; c < chunks; c++) acc += partial[(size_t)c * m + i];
  y[i] = acc;
}

// Deflation B <- B (I - x x^T) = B - y x^T with y = B x: every entry in FP64,
// rounded to FP32 once.  One block per feature, threads over samples.
__global__ void deflate_kernel(float *__restrict__ Bc, int ldm, int m,
                               const double *__restrict__ y, const float *__restrict__ x) {
  const size_t c = blockIdx.x;
  const double xc = (double)x[c];
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    const size_t o = c * ldm + i;
    Bc[o] = (float)((double)Bc[o] - y[i] * xc);
  }
}

// ------------------------------------------------------------ GEMM launch
struct GemmCfg {
  int bn, stages;
};

// Co-resident clusters of two CTAs for a pair kernel.
template <class K>
cudaError_t pair_clusters(K kern, int smem, int *out) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(2 * num_sms());
  cfg.blockDim = dim3(GEMM_THREADS);
  cfg.dynamicSmemBytes = smem;
  int n = 0;
  cudaError_t e = cudaOccupancyMaxActiveClusters(&n, (void *)kern, &cfg);
  if (e != cudaSuccess) return e;
  if (n < 1) return cudaErrorInvalidConfiguration;
  *out = n;
  return cudaSuccess;
}

// Launch set-up of a kernel on the current device, done once per (kernel,
// device) under a lock (serving runs several host threads, and a process may
// drive several devices): the dynamic shared-memory limit raised to smem and,
// for pair kernels, the number of co-resident clusters of two.
struct LaunchSetup {
  cudaError_t err;
  int clusters;
};
std::mutex g_setup_mu;
std::map<std::pair<const void *, int>, LaunchSetup> g_setup;

template <class K>
cudaError_t kernel_setup(K kern, int smem, bool pair, int *clusters = nullptr) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(g_setup_mu);
  const auto key = std::make_pair(reinterpret_cast<const void *>(kern), dev);
  auto it = g_setup.find(key);
  if (it == g_setup.end()) {
    LaunchSetup c{cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                  0};
    if (c.err == cudaSuccess && pair) c.err = pair_clusters(kern, smem, &c.clusters);
    it = g_setup.emplace(key, c).first;
  }
  if (clusters) *clusters = it->second.clusters;
  return it->second.err;
}

template <int BN, int BKT, int ST, class Epi>
cudaError_t run_gemm(const CUtensorMap &a_hi, const CUtensorMap &a_lo, const CUtensorMap &b_hi,
                     const CUtensorMap &b_lo, const GemmShape &sh, const Epi &epi,
                     cudaStream_t st) {
  using L = GemmSmem<BN, BKT, ST>;
  auto kern = gemm_tf32x3_kernel<BN, BKT, ST, GEMM_PROMO_K / BKT, Epi>;
  const cudaError_t e = kernel_setup(kern, L::TOTAL, false);
  if (e != cudaSuccess) return e;
  const int grid = sh.num_units < num_sms() ? sh.num_units : num_sms();
  kern<<<grid, GEMM_THREADS, L::TOTAL, st>>>(a_hi, a_lo, b_hi, b_lo, sh, epi);
  return cudaGetLastError();
}

// Stages per (N tile, K slab) fill ~192 KB of shared memory.
template <class S, int BN, int ST, class Epi>
cudaError_t run_gemm_pair(const CUtensorMap &m0, const CUtensorMap &m1, const CUtensorMap &m2,
                          const CUtensorMap &m3, const GemmShape &sh, const Epi &epi,
                          cudaStream_t st, int splits = 1) {
  using L = PairSmem<S, BN, ST>;
  auto kern = gemm_pair_kernel<S, BN, ST, S::PROMO_K / S::BK, Epi>;
  int clusters = 0;
  const cudaError_t e = kernel_setup(kern, L::TOTAL, true, &clusters);
  if (e != cudaSuccess) return e;
  GemmShape s2 = sh;  // K blocks of this scheme's BK; units are pair tiles x splits
  s2.kb_total = (sh.K + S::BK - 1) / S::BK;
  s2.kb_per_split = (s2.kb_total + splits - 1) / splits;
  s2.splits = (s2.kb_total + s2.kb_per_split - 1) / s2.kb_per_split;
  s2.num_units = s2.splits * ((sh.m_tiles + 1) / 2) * sh.n_tiles;
  const int pairs = s2.num_units < clusters ? s2.num_units : clusters;
  kern<<<2 * pairs, GEMM_THREADS, L::TOTAL, st>>>(m0, m1, m2, m3, s2, epi);
  return cudaGetLastError();
}

template <class Epi>
cudaError_t dispatch_gemm(int bn, int bk, const CUtensorMap &a_hi, const CUtensorMap &a_lo,
                          const CUtensorMap &b_hi, const CUtensorMap &b_lo, const GemmShape &sh,
                          const Epi &epi, cudaStream_t st) {
  if (bk == 32) {
    switch (bn) {
      case 256: return run_gemm<256, 32, 2>(a_hi, a_lo, b_hi, b_lo, sh, epi, st);
      case 128: return run_gemm<128, 32, 3>(a_hi, a_lo, b_hi, b_lo, sh, epi, st);
      case 64: return run_gemm<64, 32, 4>(a_hi, a_lo, b_hi, b_lo, sh, epi, st);
    }
  } else if (bk == 16) {
    switch (bn) {
      case 256: return run_gemm<256, 16, 4>(a_hi, a_lo, b_hi, b_lo, sh, epi, st);
      case 128: return run_gemm<128, 16, 6>(a_hi, a_lo, b_hi, b_lo, sh, epi, st);
      case 64: return run_gemm<64, 16, 8>(a_hi, a_lo, b_hi, b_lo, sh, epi, st);
    }
  }
  return cudaErrorInvalidValue;
}

// V = B^T Z: CTA pairs when the N tile is 256 (BF16 operands for the
// L1-variance forms when prepared), else the one-CTA kernel.
template <class Epi>
cudaError_t dispatch_gemm2(const BatchDev &b, const TensorMaps &tm, const GemmShape &sh,
                           const Epi &epi, bool l1_variance, cudaStream_t st) {
  if (b.pair2) {
    if (b.fp16_2) {
      GemmShape s2 = sh;
      s2.row_scale = b.row_scale;
      if (l1_variance)  // B = sgn(z), exact
        return run_gemm_pair<PairFP16x2A, 256, 8>(tm.a2_h0, tm.a2_h1, tm.b2_h0, tm.b2_h0, s2, epi,
                                                  st);
      s2.col_scale = b.z_scale;
      return run_gemm_pair<PairFP16x3, 256, 6>(tm.a2_h0, tm.a2_h1, tm.b2_h0, tm.b2_h1, s2, epi,
                                               st);
    }
    if (b.bf16_2 && l1_variance)
      return run_gemm_pair<PairBF16x3A, 256, 6>(tm.a2_b0, tm.a2_b1, tm.a2_b2, tm.b2_b, sh, epi,
                                                st);
    return run_gemm_pair<PairTF32x3, 256, 6>(tm.a2_hi, tm.a2_lo, tm.b2_hi, tm.b2_lo, sh, epi, st);
  }
  return dispatch_gemm(b.bn2, b.bk, tm.a2_hi, tm.a2_lo, tm.b2_hi, tm.b2_lo, sh, epi, st);
}


}  // namespace

int num_sms() {
  // SMs of the first device that asks (every device of a B200 node has 148);
  // a function-local static, initialised once however many threads ask
  static const int sms = [] {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 1;
  }();
  return sms;
}

int pick_bn(int k) { return k > 128 ? 256 : (k > 64 ? 128 : 64); }

size_t ws_floats(int splits, int m_tiles, int n_tiles, int bn) {
  return (size_t)splits * m_tiles * n_tiles * bn * BM;
}

cudaError_t launch_prep_bf16x3(const MatrixDev &M, cudaStream_t st) {
  prep_bf16x3_kernel<<<M.n, 256, 0, st>>>(M.Bc, M.ldm, M.m, (size_t)M.n * M.ldm, M.bf16_planes,
                                          M.Bc_b3);
  return cudaGetLastError();
}

cudaError_t launch_prep_fp16x2(const MatrixDev &M, cudaStream_t st) {
  prep_fp16x2_kernel<<<M.n, 256, 0, st>>>(M.Bc, M.ldm, M.m, (size_t)M.n * M.ldm, M.Bc_h2,
                                          M.row_scale);
  return cudaGetLastError();
}

cudaError_t launch_prep_bt_fp16x2(const MatrixDev &M, uint32_t *key, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(key, 0, sizeof(uint32_t) * M.m, st);
  if (e != cudaSuccess) return e;
  sample_max_kernel<<<dim3((M.m + 255) / 256, (M.n + SAMPLE_MAX_CHUNK - 1) / SAMPLE_MAX_CHUNK),
                      256, 0, st>>>(M.Bc, M.ldm, M.m, M.n, key);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  prep_bt_fp16x2_kernel<<<dim3((M.n + 31) / 32, (M.m + 31) / 32), dim3(32, 8), 0, st>>>(
      M.Bc, M.ldm, M.m, M.n, key, M.ldn, (size_t)M.m * M.ldn, M.Bt_h2, M.bt_row_scale);
  return cudaGetLastError();
}

cudaError_t launch_prep_tf32_planes(MatrixDev &M, cudaStream_t st) {
  prep_copy_kernel<<<M.n, 256, 0, st>>>(M.Bc, M.ldm, M.m, M.Bc_hi, M.Bc_lo, nullptr, M.ldm);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  dim3 grid((M.n + 31) / 32, (M.m + 31) / 32);
  prep_transpose_kernel<<<grid, dim3(32, 8), 0, st>>>(M.Bc, M.ldm, M.m, M.n, M.Bt_hi, M.Bt_lo,
                                                      M.ldn);
  return cudaGetLastError();
}

cudaError_t launch_load_columns(const float *src, int ld_src, int rows, int cols, float *dst,
                                int ld_dst, uint32_t *mask, cudaStream_t st) {
  if (cols <= 0) return cudaSuccess;
  load_columns_kernel<<<cols, 256, 0, st>>>(src, ld_src, rows, dst, ld_dst, mask);
  return cudaGetLastError();
}

// splitmix64's output mixer (Steele, Lea and Flood, "Fast splittable
// pseudorandom number generators", OOPSLA 2014): a bijection on 64-bit words.
__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Column c: U[-1, 1) from the top 24 bits of splitmix64((first + c) << 32 | i)
// for row i < rows, then scaled to unit 2-norm.
__global__ void __launch_bounds__(256) uniform_starts_kernel(float *__restrict__ V, int ld,
                                                             int rows, uint32_t first) {
  __shared__ double red[32];
  const size_t c = blockIdx.x;
  float *v = V + c * ld;
  const uint64_t key = (uint64_t)(first + (uint32_t)c) << 32;
  double ss = 0.0;
  for (int i = threadIdx.x; i < rows; i += blockDim.x) {
    const float u = (float)(splitmix64(key | (uint32_t)i) >> 40) * (2.0f / 16777216.0f) - 1.0f;
    v[i] = u;
    ss += (double)u * (double)u;
  }
  ss = block_sum(ss, red);
  const float inv = (float)(1.0 / sqrt(ss));
  for (int i = threadIdx.x; i < rows; i += blockDim.x) v[i] *= inv;
}

cudaError_t launch_uniform_starts(float *V, int ld, int rows, int cols, uint32_t first,
                                  cudaStream_t st) {
  if (cols <= 0) return cudaSuccess;
  uniform_starts_kernel<<<cols, 256, 0, st>>>(V, ld, rows, first);
  return cudaGetLastError();
}

cudaError_t launch_masked_copy(const float *Vx, const uint32_t *mask, int ld, int rows, int cols,
                               float *dst, int ld_dst, cudaStream_t st) {
  if (cols <= 0) return cudaSuccess;
  masked_copy_kernel<<<cols, 256, 0, st>>>(Vx, mask, ld, rows, dst, ld_dst);
  return cudaGetLastError();
}

// One warp waits, bounded by timeout_ns, on an mbarrier that nothing arrives
// on: the wait gives up, records DEV_ERR_TIMEOUT_PROBE in *status and the
// kernel returns, as every kernel's waits do when a partner never comes.
__global__ void bounded_wait_probe_kernel(unsigned long long timeout_ns, int *status) {
  __shared__ uint64_t bar;
  __shared__ int abort_flag;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    abort_flag = 0;
    fence_mbar_init();
  }
  __syncthreads();
  mbar_wait_bounded(&bar, 0, &abort_flag, status, DEV_ERR_TIMEOUT_PROBE, timeout_ns);
  __syncwarp();
}

cudaError_t launch_bounded_wait_probe(unsigned long long timeout_ns, int *status,
                                      cudaStream_t st) {
  bounded_wait_probe_kernel<<<1, 32, 0, st>>>(timeout_ns, status);
  return cudaGetLastError();
}

cudaError_t launch_finalize_x(const float *v, int n, float *x, cudaStream_t st) {
  finalize_x_kernel<<<1, 1024, 0, st>>>(v, n, x);
  return cudaGetLastError();
}

cudaError_t launch_explained_variance(const MatrixDev &M, const float *x, double *partial,
                                      double *out, cudaStream_t st) {
  const int chunks = (M.n + EV_CHUNK - 1) / EV_CHUNK;
  ev_partial_kernel<<<dim3((M.m + 255) / 256, chunks), 256, 0, st>>>(M.Bc, M.ldm, M.m, M.n, x,
                                                                     partial);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  ev_sum_kernel<<<1, 1024, 0, st>>>(partial, chunks, M.m, out);
  return cudaGetLastError();
}

cudaError_t launch_csc_to_dense(MatrixDev &M, const float *vals, const int32_t *row_ind,
                               const int32_t *col_ptr, const float *means,
                               const float *row_means, cudaStream_t st) {
  csc_scatter_kernel<<<M.n, 256, 0, st>>>(vals, row_ind, col_ptr, M.Bc, M.ldm);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || (!means && !row_means)) return e;
  center_kernel<<<M.n, 256, 0, st>>>(M.Bc, M.ldm, M.m, means, row_means);
  return cudaGetLastError();
}

cudaError_t launch_deflate(MatrixDev &M, const float *x, double *partial, double *y,
                           cudaStream_t st) {
  const int chunks = (M.n + EV_CHUNK - 1) / EV_CHUNK;
  ev_partial_kernel<<<dim3((M.m + 255) / 256, chunks), 256, 0, st>>>(M.Bc, M.ldm, M.m, M.n, x,
                                                                     partial);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  rowsum_kernel<<<(M.m + 255) / 256, 256, 0, st>>>(partial, chunks, M.m, y);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  deflate_kernel<<<M.n, 256, 0, st>>>(M.Bc, M.ldm, M.m, y, x);
  return cudaGetLastError();
}

template <int MODE>
cudaError_t launch_gather_group_mode(const MatrixDev &M, const BatchDev &b, size_t zplane,
                                     cudaStream_t st) {
  const cudaError_t e = kernel_setup(gather_bv_group_kernel<MODE>, (int)GATHER_GROUP_SMEM, false);
  if (e != cudaSuccess) return e;
  gather_bv_group_kernel<MODE><<<(b.k + GATHER_GROUP - 1) / GATHER_GROUP, GATHER_THREADS,
                                 GATHER_GROUP_SMEM, st>>>(
      M.Bc, M.ldm, M.m, M.ldn, b.k, b.Vx, b.vmask, b.Z_hi, b.Z_lo, b.fz, b.max_nnz,
      b.sparse_cap, b.Z_b, b.Z_h, zplane, b.z_scale, b.ctl);
  return cudaGetLastError();
}

cudaError_t launch_gather_group(const MatrixDev &M, const BatchDev &b, int mode, size_t zplane,
                                cudaStream_t st) {
  if (mode == 0) return launch_gather_group_mode<0>(M, b, zplane, st);
  if (mode == 1) return launch_gather_group_mode<1>(M, b, zplane, st);
  return launch_gather_group_mode<2>(M, b, zplane, st);
}

cudaError_t launch_am_step(const MatrixDev &M, BatchDev &b, const TensorMaps &tm,
                           const StepParams &p, cudaStream_t st, int *launches, cudaEvent_t *ev,
                           int *kinds) {
  cudaError_t e;
  int nl = 0;
  const int f = p.formulation;
  auto mark = [&](int kind) -> cudaError_t {
    if (kinds) kinds[nl] = kind;
    return ev ? cudaEventRecord(ev[nl], st) : cudaSuccess;
  };
  if ((e = cudaMemsetAsync(b.max_err, 0, sizeof(float), st)) != cudaSuccess) return e;
  if (b.mixed &&  // the support this step starts from, for the stability count
      (e = cudaMemcpyAsync(b.vmask_prev, b.vmask, sizeof(uint32_t) * (size_t)b.k * (M.ldn / 32),
                           cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
    return e;
  // 1. Z = B V (split-K partials)
  GemmShape g1;
  g1.M = M.m;
  g1.N = b.k;
  g1.K = M.n;
  g1.m_tiles = b.m_tiles1;
  g1.n_tiles = b.n_tiles1;
  g1.kb_total = (M.n + b.bk - 1) / b.bk;
  g1.kb_per_split = b.kbps1;
  g1.splits = b.splits1;
  g1.num_units = g1.splits * g1.m_tiles * g1.n_tiles;
  g1.timeout_ns = p.timeout_ns;
  g1.status = b.status;
  g1.stop = b.ctl;
  g1.gate = b.max_nnz;  // dense steps only
  g1.gate_min = b.sparse_cap + 1;
  g1.gate_max = 0xFFFFFFFFu;
  const int mode = is_l1_variance(f) ? 1 : (is_constrained(f) ? 0 : 2);
  const size_t zplane = (size_t)b.k * M.ldm;  // second FP16 plane of Z
  // 1a. sparse V (every column <= sparse_cap non-zeros last step): gather
  if ((e = mark(9)) != cudaSuccess) return e;
  if ((e = launch_gather_group(M, b, mode, zplane, st)) != cudaSuccess) return e;
  nl++;
  if ((e = mark(5)) != cudaSuccess) return e;
  if (mode == 0)
    gather_bv_kernel<0><<<b.k, GATHER_THREADS, 0, st>>>(M.Bc, M.ldm, M.m, M.ldn,
                                                        b.Vx, b.vmask, b.Z_hi, b.Z_lo, b.fz,
                                                        b.max_nnz, b.sparse_cap, b.Z_b, b.Z_h, zplane, b.z_scale,
                                                        b.ctl);
  else if (mode == 1)
    gather_bv_kernel<1><<<b.k, GATHER_THREADS, 0, st>>>(M.Bc, M.ldm, M.m, M.ldn,
                                                        b.Vx, b.vmask, b.Z_hi, b.Z_lo, b.fz,
                                                        b.max_nnz, b.sparse_cap, b.Z_b, b.Z_h, zplane, b.z_scale,
                                                        b.ctl);
  else
    gather_bv_kernel<2><<<b.k, GATHER_THREADS, 0, st>>>(M.Bc, M.ldm, M.m, M.ldn,
                                                        b.Vx, b.vmask, b.Z_hi, b.Z_lo, b.fz,
                                                        b.max_nnz, b.sparse_cap, b.Z_b, b.Z_h, zplane, b.z_scale,
                                                        b.ctl);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  nl++;
  // 1b. dense V: TF32 hi/lo planes, tensor-core Z = B V (split-K partials) ...
  if ((e = mark(6)) != cudaSuccess) return e;
  if (b.fp16_1)
    densify_fp16_kernel<<<std::min(b.k, DENSIFY_BLOCKS_PER_SM * num_sms()), DENSIFY_THREADS, 0,
                          st>>>(b.Vx, b.vmask, M.ldn, M.n, b.V_h, (size_t)b.k * M.ldn, b.v_scale,
                                b.max_nnz, b.sparse_cap, b.ctl, b.k);
  else
    densify_kernel<<<b.k, 256, 0, st>>>(b.Vx, b.vmask, M.ldn, M.n, b.V_hi, b.V_lo, b.max_nnz,
                                        b.planes_nnz, b.sparse_cap, b.ctl);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  nl++;
  EpiPartial ep{b.ws, b.bn1, b.m_tiles1, b.n_tiles1};
  if ((e = mark(0)) != cudaSuccess) return e;
  if (b.fp16_1) {
    GemmShape gp = g1;
    gp.row_scale = b.bt_row_scale;
    gp.col_scale = b.v_scale;
    e = run_gemm_pair<PairFP16x3, 256, 6>(tm.a1_h0, tm.a1_h1, tm.b1_h0, tm.b1_h1, gp, ep, st,
                                          b.splits1p);
  } else {
    e = dispatch_gemm(b.bn1, b.bk, tm.a1_hi, tm.a1_lo, tm.b1_hi, tm.b1_lo, g1, ep, st);
  }
  if (e != cudaSuccess) return e;
  nl++;
  // 2. ... then reduce + sign / normalise
  const int splits1 = b.fp16_1 ? b.splits1p : b.splits1;
  if ((e = mark(1)) != cudaSuccess) return e;
  if (mode == 0)
    z_reduce_kernel<0><<<b.k, 256, 0, st>>>(b.ws, splits1, b.m_tiles1, b.n_tiles1, b.bn1, M.m,
                                             b.Z_hi, b.Z_lo, M.ldm, b.fz, b.max_nnz, b.sparse_cap,
                                             b.Z_b, b.Z_h, zplane, b.z_scale, b.ctl);
  else if (mode == 1)
    z_reduce_kernel<1><<<b.k, 256, 0, st>>>(b.ws, splits1, b.m_tiles1, b.n_tiles1, b.bn1, M.m,
                                             b.Z_hi, b.Z_lo, M.ldm, b.fz, b.max_nnz, b.sparse_cap,
                                             b.Z_b, b.Z_h, zplane, b.z_scale, b.ctl);
  else
    z_reduce_kernel<2><<<b.k, 256, 0, st>>>(b.ws, splits1, b.m_tiles1, b.n_tiles1, b.bn1, M.m,
                                             b.Z_hi, b.Z_lo, M.ldm, b.fz, b.max_nnz, b.sparse_cap,
                                             b.Z_b, b.Z_h, zplane, b.z_scale, b.ctl);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  nl++;
  // 3. V = B^T Z
  GemmShape g2;
  g2.M = M.n;
  g2.N = b.k;
  g2.K = M.m;
  g2.m_tiles = b.m_tiles2;
  g2.n_tiles = b.n_tiles2;
  g2.kb_total = (M.m + b.bk - 1) / b.bk;
  g2.kb_per_split = g2.kb_total;
  g2.splits = 1;
  g2.num_units = g2.m_tiles * g2.n_tiles;
  g2.timeout_ns = p.timeout_ns;
  g2.status = b.status;
  g2.stop = b.ctl;
  g2.gate = nullptr;
  g2.gate_min = 0;
  g2.gate_max = 0;
  const int parts = b.m_tiles2 * 4;
  // MIXED: the single-pass BF16 product runs while phase[0] == 0, the
  // FP32-accurate one from then on; each launch returns at once in the other phase
  auto gemm2 = [&](const auto &epi) -> cudaError_t {
    cudaError_t e2;
    if (b.mixed) {
      GemmShape gl = g2;
      gl.gate = b.phase;
      gl.gate_min = 0;
      gl.gate_max = 0;
      if ((e2 = mark(7)) != cudaSuccess) return e2;
      if (b.mixed_fp16) {
        gl.row_scale = b.row_scale;
        gl.col_scale = is_l1_variance(f) ? nullptr : b.z_scale;  // sgn(z) is exact
        e2 = run_gemm_pair<PairFP16x1, 256, 12>(tm.a2_h0, tm.b2_h0, tm.a2_h0, tm.b2_h0, gl, epi,
                                                st);
      } else {
        e2 = run_gemm_pair<PairBF16x1, 256, 12>(tm.a2_b0, tm.b2_b, tm.a2_b0, tm.b2_b, gl, epi,
                                                st);
      }
      if (e2 != cudaSuccess) return e2;
      nl++;
      g2.gate = b.phase;
      g2.gate_min = 1;
      g2.gate_max = 0xFFFFFFFFu;
    }
    if ((e2 = mark(2)) != cudaSuccess) return e2;
    if ((e2 = dispatch_gemm2(b, tm, g2, epi, is_l1_variance(f), st)) != cudaSuccess) return e2;
    nl++;
    return cudaSuccess;
  };
  // the penalty epilogue writes the next dense step's TF32 planes of V
  // (unless that step's Z = B V takes FP16 planes from densify_fp16_kernel)
  float *vhi = b.fp16_1 ? nullptr : b.V_hi;
  if (is_constrained(f)) {
    EpiRaw er{b.Vraw, M.ldn, M.n, b.k, b.bn2};
    if (b.cmask) {  // the selects' hinted gather, done while V is in registers
      er.hint = b.sel_hint;
      er.cmask = b.cmask;
    }
    e = gemm2(er);
  } else if (is_l1_penalized(f)) {
    EpiPenalty<true> pe{b.Vx,       b.obj_part, b.nnz_part, M.ldn,    M.n,
                        b.k,        b.bn2,      parts,      (float)p.penalty,
                        b.vmask,    vhi,        b.V_lo,     b.max_nnz, b.sparse_cap};
    e = gemm2(pe);
  } else {
    EpiPenalty<false> pe{b.Vx,       b.obj_part, b.nnz_part, M.ldn,    M.n,
                         b.k,        b.bn2,      parts,      (float)p.penalty,
                         b.vmask,    vhi,        b.V_lo,     b.max_nnz, b.sparse_cap};
    e = gemm2(pe);
  }
  if (e != cudaSuccess) return e;
  // 4. constrained: selection / projection + normalisation
  if (is_constrained(f)) {
    if ((e = mark(3)) != cudaSuccess) return e;
    if (!is_l1_constrained(f)) {
      hard_select_kernel<<<b.k, HARD_THREADS, 0, st>>>(b.Vraw, M.ldn, M.n, p.constraint, b.Vx,
                                                        b.nnz, b.status, b.vmask, b.sel_hint,
                                                        b.ctl, b.cmask);
      e = cudaGetLastError();
    } else {
      if (p.l1_mode == 0) {
        if ((e = kernel_setup(soft_select_kernel<false>, SOFT_SMEM, false)) != cudaSuccess)
          return e;
        soft_select_kernel<false><<<b.k, SOFT_THREADS, SOFT_SMEM, st>>>(
            b.Vraw, M.ldn, M.n, p.constraint, b.Vx, b.nnz, b.status, b.vmask, b.sel_hint, b.ctl,
            b.cmask);
      } else {
        if ((e = kernel_setup(soft_select_kernel<true>, SOFT_SMEM, false)) != cudaSuccess)
          return e;
        soft_select_kernel<true><<<b.k, SOFT_THREADS, SOFT_SMEM, st>>>(
            b.Vraw, M.ldn, M.n, p.constraint, b.Vx, b.nnz, b.status, b.vmask, b.sel_hint, b.ctl,
            b.cmask);
      }
      e = cudaGetLastError();
    }
    if (e != cudaSuccess) return e;
    nl++;
  }
  // 4b. MIXED: support stability and the phase switch
  if (b.mixed) {
    if ((e = mark(8)) != cudaSuccess) return e;
    support_kernel<<<b.k, 256, 0, st>>>(b.vmask, b.vmask_prev, M.ldn / 32, b.stable, b.phase,
                                        b.k_stable, b.need_stable, b.ctl);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    nl++;
  }
  // 5. finalize
  FinalizeArgs fa;
  fa.k = b.k;
  fa.formulation = f;
  fa.parts = parts;
  fa.it = p.it;
  fa.store_all = p.store_all;
  fa.log_shift = p.log_shift;
  fa.log_capacity = b.log_capacity;
  fa.tolerance = p.tolerance;
  fa.fz = b.fz;
  fa.obj_part = b.obj_part;
  fa.nnz_part = b.nnz_part;
  fa.nnz_sel = b.nnz;
  fa.val = b.val;
  fa.err = b.err;
  fa.max_err = b.max_err;
  fa.iters = b.iters;
  fa.cards = b.cards;
  fa.max_nnz = b.max_nnz;
  fa.ctl = b.ctl;
  fa.phase = b.mixed ? b.phase : nullptr;
  fa.status = b.status;
  fa.stop_check = p.stop_check;
  // Z = B V of this step has read max_nnz; finalize sets it for the next step
  // penalized forms: the count this step's epilogue saw (whether it wrote the
  // dense planes), for the next step's densify gate
  if (!is_constrained(f) && !b.fp16_1 &&
      (e = cudaMemcpyAsync(b.planes_nnz, b.max_nnz, sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                           st)) != cudaSuccess)
    return e;
  if ((e = cudaMemsetAsync(b.max_nnz, 0, sizeof(uint32_t), st)) != cudaSuccess) return e;
  if ((e = mark(4)) != cudaSuccess) return e;
  finalize_kernel<<<(b.k + 7) / 8, 256, 0, st>>>(fa);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  nl++;
  if (ev && (e = cudaEventRecord(ev[nl], st)) != cudaSuccess) return e;
  if (launches) *launches = nl;
  return cudaSuccess;
}

// ------------------------------------------------------------ grouped steps
#include "gemm_pair_grouped.cuh"
#include "am24_group_kernels.cuh"

namespace {

template <class K>
cudaError_t persistent_grid(K kern, int threads, int smem, int *grid) {
  int per = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (void *)kern, threads, smem);
  if (e != cudaSuccess) return e;
  *grid = num_sms() * (per > 0 ? per : 1);
  return cudaSuccess;
}

template <int BN, int EPI>
cudaError_t grouped_gemm_setup(int *clusters) {
  return kernel_setup(gemm_pair_grouped_kernel<BN, EPI>, GPairSmem<BN>::TOTAL, true, clusters);
}

template <int BN, int EPI>
cudaError_t launch_grouped_gemm(const GroupDev &g, int list, cudaStream_t st) {
  int clusters = 0;
  const cudaError_t e = grouped_gemm_setup<BN, EPI>(&clusters);
  if (e != cudaSuccess) return e;
  gemm_pair_grouped_kernel<BN, EPI>
      <<<2 * clusters, GEMM_THREADS, GPairSmem<BN>::TOTAL, st>>>(g, list);
  return cudaGetLastError();
}

// The three N tiles of one epilogue, lists l64, l64 + 1, l64 + 2.
template <int EPI>
cudaError_t launch_grouped_gemms(const GroupDev &g, int l64, cudaStream_t st) {
  cudaError_t e;
  if ((e = launch_grouped_gemm<64, EPI>(g, l64, st)) ||
      (e = launch_grouped_gemm<128, EPI>(g, l64 + 1, st)) ||
      (e = launch_grouped_gemm<256, EPI>(g, l64 + 2, st)))
    return e;
  return cudaSuccess;
}

template <int EPI>
cudaError_t grouped_gemms_setup(int *c) {
  cudaError_t e;
  if ((e = grouped_gemm_setup<64, EPI>(c)) || (e = grouped_gemm_setup<128, EPI>(c)) ||
      (e = grouped_gemm_setup<256, EPI>(c)))
    return e;
  return cudaSuccess;
}

}  // namespace

cudaError_t grouped_grids(GroupGrids *gr) {
  cudaError_t e;
  if ((e = kernel_setup(g_gather_group_kernel<0>, (int)GATHER_GROUP_SMEM, false)) ||
      (e = kernel_setup(g_gather_group_kernel<1>, (int)GATHER_GROUP_SMEM, false)) ||
      (e = kernel_setup(g_gather_group_kernel<2>, (int)GATHER_GROUP_SMEM, false)))
    return e;
  int c = 0;
  if ((e = grouped_gemms_setup<GE_PARTIAL>(&c)) || (e = grouped_gemms_setup<GE_RAW>(&c)) ||
      (e = grouped_gemms_setup<GE_PL1>(&c)) || (e = grouped_gemms_setup<GE_PL0>(&c)))
    return e;
  gr->plan_threads = PLAN_THREADS;
  gr->pairs = c;
  if ((e = persistent_grid(g_z_reduce_kernel<0>, 256, 0, &gr->col)) ||
      (e = persistent_grid(g_hard_select_kernel, HARD_THREADS, 0, &gr->select_hard)) ||
      (e = kernel_setup(g_soft_select_kernel<false>, SOFT_SMEM, false)) ||
      (e = kernel_setup(g_soft_select_kernel<true>, SOFT_SMEM, false)) ||
      (e = persistent_grid(g_soft_select_kernel<false>, SOFT_THREADS, SOFT_SMEM,
                           &gr->select_soft)) ||
      (e = persistent_grid(g_gather_kernel<0>, GATHER_THREADS, 0, &gr->gather)) ||
      (e = persistent_grid(g_gather_group_kernel<0>, GATHER_THREADS, (int)GATHER_GROUP_SMEM,
                           &gr->gather_group)) ||
      (e = persistent_grid(g_finalize_kernel, 256, 0, &gr->fin)))
    return e;
  return cudaSuccess;
}

cudaError_t launch_grouped_step(const GroupDev &g, const GroupGrids &gr, cudaStream_t st) {
  cudaError_t e;
  group_plan_kernel<<<1, PLAN_THREADS, 0, st>>>(g);
  if ((e = cudaGetLastError())) return e;
  // Z = B V: the sparse gathers (by mode), or the dense path
  g_gather_group_kernel<0><<<gr.gather_group, GATHER_THREADS, GATHER_GROUP_SMEM, st>>>(g);
  g_gather_group_kernel<1><<<gr.gather_group, GATHER_THREADS, GATHER_GROUP_SMEM, st>>>(g);
  g_gather_group_kernel<2><<<gr.gather_group, GATHER_THREADS, GATHER_GROUP_SMEM, st>>>(g);
  g_gather_kernel<0><<<gr.gather, GATHER_THREADS, 0, st>>>(g);
  g_gather_kernel<1><<<gr.gather, GATHER_THREADS, 0, st>>>(g);
  g_gather_kernel<2><<<gr.gather, GATHER_THREADS, 0, st>>>(g);
  for (int mode = 0; mode < 3; mode++)
    g_densify_kernel<<<DENSIFY_BLOCKS_PER_SM * num_sms(), DENSIFY_THREADS, 0, st>>>(g, mode);
  if ((e = cudaGetLastError())) return e;
  if ((e = launch_grouped_gemms<GE_PARTIAL>(g, GL_GEMM1_64, st))) return e;
  g_z_reduce_kernel<0><<<gr.col, 256, 0, st>>>(g);
  g_z_reduce_kernel<1><<<gr.col, 256, 0, st>>>(g);
  g_z_reduce_kernel<2><<<gr.col, 256, 0, st>>>(g);
  if ((e = cudaGetLastError())) return e;
  // V = B^T Z with the penalty fused or the raw output marked for the selects
  if ((e = launch_grouped_gemms<GE_RAW>(g, GL_RAW_64, st)) ||
      (e = launch_grouped_gemms<GE_PL1>(g, GL_PL1_64, st)) ||
      (e = launch_grouped_gemms<GE_PL0>(g, GL_PL0_64, st)))
    return e;
  g_hard_select_kernel<<<gr.select_hard, HARD_THREADS, 0, st>>>(g);
  g_soft_select_kernel<false><<<gr.select_soft, SOFT_THREADS, SOFT_SMEM, st>>>(g);
  g_soft_select_kernel<true><<<gr.select_soft, SOFT_THREADS, SOFT_SMEM, st>>>(g);
  g_support_kernel<<<gr.col, 256, 0, st>>>(g);
  g_finalize_kernel<<<gr.fin, 256, 0, st>>>(g);
  return cudaGetLastError();
}

cudaError_t launch_grouped_condition(const GroupDev &g, unsigned long long handle,
                                     cudaStream_t st, bool in_graph) {
  g_condition_kernel<<<1, 256, 0, st>>>(g, (cudaGraphConditionalHandle)handle, in_graph);
  return cudaGetLastError();
}

// ------------------------------------------------------------ sparse steps
#include "am24_sparse_kernels.cuh"

namespace {
// One product on the compressed arrays: the tile kernel for the outer entries
// of at most SP_LONG entries, the segment and combine kernels for the others.
// gate (may be null): the launches do their work only when *gate >= gate_min.
void sparse_product(const int32_t *ptr, const int32_t *idx, const float *val, int ncols,
                    const SparseLong &L, const float *X, float *part, const SparseBatchDev &b,
                    float *out, int ld_out, const float *cvec, const double *a, const double *bv,
                    const uint32_t *gate, uint32_t gate_min, cudaStream_t st) {
  sp_spmm_kernel<<<dim3((ncols + SP_TILE - 1) / SP_TILE, b.kp / SP_TILE), SP_THREADS, 0, st>>>(
      ptr, idx, val, ncols, X, b.kp, b.k, out, ld_out, cvec, a, bv, b.ctl, gate, gate_min);
  if (L.count == 0) return;
  constexpr int WARPS = SP_THREADS / 32;
  sp_spmm_seg_kernel<<<dim3((L.segs + WARPS - 1) / WARPS, b.kp / SP_TILE), SP_THREADS, 0, st>>>(
      L.seg_e0, L.seg_e1, L.segs, idx, val, X, b.kp, part, b.ctl, gate, gate_min);
  sp_spmm_long_kernel<<<dim3(L.count, b.kp / SP_TILE), SP_TILE, 0, st>>>(
      L.outer, L.seg_first, part, b.kp, b.k, out, ld_out, cvec, a, bv, b.ctl, gate, gate_min);
}
}  // namespace

cudaError_t launch_sparse_step(const SparseDev &S, const SparseBatchDev &b, const StepParams &p,
                               cudaStream_t st) {
  cudaError_t e;
  const int f = p.formulation;
  const bool centred = S.means || S.row_means;
  if ((e = cudaMemsetAsync(b.max_err, 0, sizeof(float), st))) return e;
  // 1. Z = (B - 1 mu^T - r 1^T) V: CSR rows against V transposed
  // the centring's sums, and the entries a scatter of the supports would touch
  if ((e = cudaMemsetAsync(b.work, 0, sizeof(unsigned long long), st))) return e;
  sp_vstats_kernel<<<b.k, SP_THREADS, 0, st>>>(b.Vx, b.vmask, b.ldn, S.n, S.means,
                                               centred ? b.sum_v : nullptr, b.dot_mu, S.col_ptr,
                                               b.work, b.ctl);
  // the scatter of each support when the previous step left at most
  // SP_SCATTER_CAP loadings in every start and the scatter touches fewer
  // entries than the CSR product steps through; else the CSR product
  // deflated: the projected loadings P v are dense, so the CSR product runs
  if (S.comps > 0)
    sp_defl_coef_kernel<<<b.k, SP_THREADS, 0, st>>>(
        b.Vx, b.vmask, b.ldn, S.n, S.defl, S.comps, S.gram, S.defl_sum, S.defl_mu, b.defl_a,
        centred ? b.sum_v : nullptr, b.dot_mu, b.ctl);
  sp_zgate_kernel<<<1, 1, 0, st>>>(
      b.max_nnz, (uint32_t)SP_SCATTER_CAP, b.work,
      S.comps > 0 ? -1.0 : SP_SCATTER_PER_STEP * (double)S.nnz * (double)(b.kp / 32), b.zgate,
      b.ctl);
  sp_transpose_v_kernel<<<dim3((S.n + SP_TILE - 1) / SP_TILE, b.kp / SP_TILE), SP_THREADS, 0,
                          st>>>(b.Vx, b.vmask, b.ldn, S.n, b.k, b.Vt, b.kp, b.ctl, b.zgate, 1u,
                                S.defl, S.comps, b.defl_a);
  sparse_product(S.row_ptr, S.col_ind, S.rvals, S.m, S.long_rows, b.Vt, b.part_rows, b, b.Zs,
                 b.ldm, S.row_means, S.row_means ? b.sum_v : nullptr,
                 S.means ? b.dot_mu : nullptr, b.zgate, 1u, st);
  sp_scatter_z_kernel<<<b.k, SP_THREADS, 0, st>>>(
      S.col_ptr, S.row_ind, S.cvals, b.Vx, b.vmask, b.ldn, b.Zs, b.ldm, S.m, S.row_means,
      S.row_means ? b.sum_v : nullptr, S.means ? b.dot_mu : nullptr, b.zgate, 0u, b.ctl);
  // 2. the formulation's sign / norm of z, and the sums V's correction needs
  sp_zreduce_kernel<<<b.k, SP_THREADS, 0, st>>>(b.Zs, b.ldm, S.m, f, b.fz, S.row_means,
                                                centred ? b.zsum : nullptr, b.zdot, b.ctl);
  sp_transpose_z_kernel<<<dim3((S.m + SP_TILE - 1) / SP_TILE, b.kp / SP_TILE), SP_THREADS, 0,
                          st>>>(b.Zs, b.ldm, S.m, b.k, b.Zt, b.kp, b.ctl);
  // 3. V = (B - 1 mu^T - r 1^T)^T Z: CSC columns against Z transposed
  sparse_product(S.col_ptr, S.row_ind, S.cvals, S.n, S.long_cols, b.Zt, b.part_cols, b, b.Vraw,
                 b.ldn, S.means, S.means ? b.zsum : nullptr, S.row_means ? b.zdot : nullptr,
                 nullptr, 0, st);
  if (S.comps > 0)
    sp_defl_vraw_kernel<<<b.k, SP_THREADS, 0, st>>>(b.Vraw, b.ldn, S.n, S.defl, S.comps, S.gram,
                                                    b.ctl);
  if ((e = cudaGetLastError())) return e;
  // 4. thresholds: the dense path's selects (own candidate gather), or the penalties
  if (is_constrained(f)) {
    if (!is_l1_constrained(f)) {
      hard_select_kernel<<<b.k, HARD_THREADS, 0, st>>>(b.Vraw, b.ldn, S.n, p.constraint, b.Vx,
                                                        b.nnz, b.status, b.vmask, b.sel_hint,
                                                        b.ctl, nullptr);
    } else if (p.l1_mode == 0) {
      if ((e = kernel_setup(soft_select_kernel<false>, SOFT_SMEM, false))) return e;
      soft_select_kernel<false><<<b.k, SOFT_THREADS, SOFT_SMEM, st>>>(
          b.Vraw, b.ldn, S.n, p.constraint, b.Vx, b.nnz, b.status, b.vmask, b.sel_hint, b.ctl,
          nullptr);
    } else {
      if ((e = kernel_setup(soft_select_kernel<true>, SOFT_SMEM, false))) return e;
      soft_select_kernel<true><<<b.k, SOFT_THREADS, SOFT_SMEM, st>>>(
          b.Vraw, b.ldn, S.n, p.constraint, b.Vx, b.nnz, b.status, b.vmask, b.sel_hint, b.ctl,
          nullptr);
    }
  } else if (is_l1_penalized(f)) {
    sp_penalty_kernel<true><<<b.k, SP_THREADS, 0, st>>>(b.Vraw, b.ldn, S.n, (float)p.penalty,
                                                        b.Vx, b.vmask, b.obj_part, b.nnz_part,
                                                        b.ctl);
  } else {
    sp_penalty_kernel<false><<<b.k, SP_THREADS, 0, st>>>(b.Vraw, b.ldn, S.n, (float)p.penalty,
                                                         b.Vx, b.vmask, b.obj_part, b.nnz_part,
                                                         b.ctl);
  }
  if ((e = cudaGetLastError())) return e;
  // 5. objective, change, logs and the batch loop's termination test
  FinalizeArgs fa;
  fa.k = b.k;
  fa.formulation = f;
  fa.parts = 1;
  fa.it = p.it;
  fa.store_all = p.store_all;
  fa.log_shift = p.log_shift;
  fa.log_capacity = b.log_capacity;
  fa.tolerance = p.tolerance;
  fa.fz = b.fz;
  fa.obj_part = b.obj_part;
  fa.nnz_part = b.nnz_part;
  fa.nnz_sel = b.nnz;
  fa.val = b.val;
  fa.err = b.err;
  fa.max_err = b.max_err;
  fa.iters = b.iters;
  fa.cards = b.cards;
  fa.max_nnz = b.max_nnz;
  fa.ctl = b.ctl;
  fa.phase = nullptr;
  fa.status = b.status;
  fa.stop_check = p.stop_check;
  if ((e = cudaMemsetAsync(b.max_nnz, 0, sizeof(uint32_t), st))) return e;
  finalize_kernel<<<(b.k + 7) / 8, 256, 0, st>>>(fa);
  return cudaGetLastError();
}

cudaError_t launch_sparse_ev(const SparseDev &S, const float *x, double *scratch, double *out,
                             cudaStream_t st) {
  const int blocks = (S.m + SP_THREADS - 1) / SP_THREADS;
  double *xs = scratch, *partial = scratch + 2;
  sp_ev_xstats_kernel<<<1, SP_THREADS, 0, st>>>(x, S.n, S.means, xs);
  sp_ev_rows_kernel<<<blocks, SP_THREADS, 0, st>>>(S.row_ptr, S.col_ind, S.rvals, S.m, x,
                                                   S.row_means, xs, partial);
  sp_ev_sum_kernel<<<1, SP_THREADS, 0, st>>>(partial, blocks, out);
  return cudaGetLastError();
}

}  // namespace am24
