// Persistent tcgen05 GEMM for the two AM products, FP32-accurate via 3xTF32.
//
//   C[M x N] = A[M x K] * B[N x K]^T   (both operands K-major in global memory)
//
// Every FP32 operand is stored as two planes, hi = x rounded to the nearest
// TF32 value and lo = x - hi (exact in FP32), so x = hi + lo bit for bit.  The
// product is accumulated in FP32 in tensor memory as lo*hi + hi*lo + hi*hi;
// the dropped lo*lo term and the TF32 view of lo are each below 2^-21 of
// |a*b| and of either sign, so the result carries near-FP32 error at 3 TF32
// MMAs per K step.
//
// Tensor-core FP32 accumulation does not round to nearest, so a long K run
// inside TMEM drifts (measured ~1e-5 relative at K = 1000).  The accumulator is
// therefore promoted: the MMA fills a TMEM buffer for PROMO K slabs only, and
// the epilogue warps add each such chunk into a register accumulator with
// ordinary round-to-nearest FP32 adds.
//
// One CTA per SM, 10 warps:
//   warp 0      TMA producer (one lane): loads A_hi, A_lo, B_hi, B_lo K-slabs
//               into a STAGES-deep shared-memory ring (128-byte swizzle).
//   warp 1      MMA issuer (one lane): tcgen05.mma.kind::tf32, M=128, N=BN,
//               one K chunk into one of two TMEM buffers, then the other.
//   warps 2..9  accumulators: warp w reads TMEM lanes [32(w%4), 32(w%4)+32)
//               (the quarter its index allows) and columns of half (w-2)/4,
//               keeps BN/2 running sums per thread, and at the end of a work
//               unit hands them to the Epi functor.
// Two TMEM buffers let the drain of one chunk overlap the MMAs of the next.
// A work unit is (split, m-tile, n-tile) with the n-tile varying fastest, so
// CTAs running at the same time share A tiles (and, for split-K, B slabs)
// through L2.  Every barrier wait is bounded: on timeout the kernel records a
// DEV_ERR_TIMEOUT_* code in *status and all roles drain out.
#pragma once
#include "ptx.cuh"

namespace am24 {

constexpr int GEMM_BM = 128;
constexpr int GEMM_THREADS = 320;
constexpr int GEMM_EPI_THREADS = 256;

enum DeviceError : int {
  DEV_OK = 0,
  DEV_ERR_TIMEOUT_PRODUCER = 0x101,
  DEV_ERR_TIMEOUT_MMA_SMEM = 0x102,
  DEV_ERR_TIMEOUT_MMA_TMEM = 0x103,
  DEV_ERR_TIMEOUT_EPILOGUE = 0x104,
  DEV_ERR_TIMEOUT_PROBE = 0x1FF,  // the bounded-wait self-test (expected)
};

struct GemmShape {
  int M, N, K;
  int m_tiles, n_tiles;
  int kb_total;      // ceil(K / BK)
  int kb_per_split;  // K blocks per split; every split is non-empty
  int splits;
  int num_units;     // splits * m_tiles * n_tiles
  unsigned long long timeout_ns;
  int *status;
  // Optional gate: when gate != nullptr the launch does its work only if
  // gate_min <= *gate <= gate_max (otherwise another kernel of the step covers it).
  const uint32_t *gate;
  uint32_t gate_min, gate_max;
  // Optional output scaling (FP16 schemes): C[i][j] is multiplied by
  // row_scale[i] * col_scale[j] (either may be absent), powers of two that undo
  // the operands' range scaling exactly.
  const float *row_scale = nullptr;
  const float *col_scale = nullptr;
  const uint32_t *stop = nullptr;  // the launch returns at once while *stop is set
};

// One work unit as an epilogue sees it: rows [m0, m0 + 128) of C (this CTA's
// accumulator lanes), columns [nt * BN, nt * BN + BN), K blocks [kb0, kb1) of
// split `split`.
struct Unit {
  int mt, nt, split, kb0, kb1, index;
  int m0;
};

__device__ __forceinline__ Unit decode_unit(const GemmShape &s, int u) {
  Unit r;
  const int tiles = s.m_tiles * s.n_tiles;
  r.split = u / tiles;
  const int t = u - r.split * tiles;
  r.mt = t / s.n_tiles;
  r.nt = t - r.mt * s.n_tiles;
  r.kb0 = r.split * s.kb_per_split;
  r.kb1 = min(s.kb_total, r.kb0 + s.kb_per_split);
  r.index = u;
  r.m0 = r.mt * GEMM_BM;
  return r;
}

template <int BN, int BK, int STAGES>
struct GemmSmem {
  static constexpr int A_BYTES = GEMM_BM * BK * 4;
  static constexpr int B_BYTES = BN * BK * 4;
  static constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
  static constexpr int BAR_BYTES = 256;
  // + 1024 so the ring can be aligned to 1024 B inside the dynamic allocation
  static constexpr int TOTAL = STAGES * STAGE_BYTES + BAR_BYTES + 1024;
};

// Warp-uniform bounded wait: every lane waits, then the warp agrees.
__device__ __forceinline__ bool warp_wait(uint64_t *bar, uint32_t parity, volatile int *abort,
                                          int *status, int code, unsigned long long tmo) {
  bool ok = mbar_wait_bounded(bar, parity, abort, status, code, tmo);
  return __all_sync(0xffffffffu, ok);
}

template <int BN, int BK, int STAGES, int PROMO, class Epi>
__global__ void __launch_bounds__(GEMM_THREADS, 1)
    gemm_tf32x3_kernel(const __grid_constant__ CUtensorMap tmA_hi,
                       const __grid_constant__ CUtensorMap tmA_lo,
                       const __grid_constant__ CUtensorMap tmB_hi,
                       const __grid_constant__ CUtensorMap tmB_lo, const GemmShape shape,
                       Epi epi) {
  using L = GemmSmem<BN, BK, STAGES>;
  static_assert(BK == 32 || BK == 16, "BK must be 32 (128B swizzle) or 16 (64B swizzle)");
  static_assert(BN % 32 == 0 && BN >= 32 && BN <= 256, "BN must be a multiple of 32 in [32,256]");
  constexpr uint32_t SWZ = (BK == 32) ? 2u : 4u;  // descriptor swizzle mode: 128B / 64B
  constexpr uint32_t SBO = BK * 4 * 8;            // bytes between 8-row core-matrix groups
  constexpr uint32_t TMEM_COLS = (2 * BN <= 32) ? 32 : (2 * BN <= 64) ? 64 : (2 * BN <= 128) ? 128
                                 : (2 * BN <= 256) ? 256 : 512;
  constexpr uint32_t IDESC = make_idesc(GEMM_BM, BN, 2u, 2u);

  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = reinterpret_cast<uint8_t *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + STAGES * L::STAGE_BYTES);
  uint64_t *empty = full + STAGES;
  uint64_t *tfull = empty + STAGES;
  uint64_t *tempty = tfull + 2;
  uint64_t *drain = tempty + 2;
  uint32_t *tmem_holder = reinterpret_cast<uint32_t *>(drain + 1);
  volatile int *abort = reinterpret_cast<volatile int *>(tmem_holder + 1);

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  if ((shape.stop && *shape.stop) ||
      (shape.gate && (*shape.gate < shape.gate_min || *shape.gate > shape.gate_max)))
    return;  // uniform over the grid

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; a++) {
      mbar_init(&tfull[a], 1);
      mbar_init(&tempty[a], GEMM_EPI_THREADS);
    }
    mbar_init(drain, 1);
    *abort = 0;
    fence_mbar_init();
    tma_prefetch_desc(&tmA_hi);
    tma_prefetch_desc(&tmA_lo);
    tma_prefetch_desc(&tmB_hi);
    tma_prefetch_desc(&tmB_lo);
  }
  if (warp == 0) {
    __syncwarp();
    tmem_alloc(tmem_holder, TMEM_COLS);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_holder;
  const unsigned long long tmo = shape.timeout_ns;

  if (warp == 0) {
    if (lane == 0) {
      // ---------------------------------------------------------- producer
      int stage = 0;
      uint32_t phase = 0;
      uint32_t armed = 0;  // bit s: stage s has been armed at least once
      uint32_t armed_parity = 0;  // bit s: parity of the phase last armed on stage s
      for (int u = blockIdx.x; u < shape.num_units && !*abort; u += gridDim.x) {
        const Unit t = decode_unit(shape, u);
        for (int kb = t.kb0; kb < t.kb1; kb++) {
          if (!mbar_wait_bounded(&empty[stage], phase ^ 1u, abort, shape.status,
                                 DEV_ERR_TIMEOUT_PRODUCER, tmo))
            break;
          uint8_t *st = smem + stage * L::STAGE_BYTES;
          mbar_arrive_expect_tx(&full[stage], L::STAGE_BYTES);
          armed |= 1u << stage;
          armed_parity = (armed_parity & ~(1u << stage)) | (phase << stage);
          const int kx = kb * BK;
          tma_load_2d(st, &tmA_hi, &full[stage], kx, t.mt * GEMM_BM);
          tma_load_2d(st + L::A_BYTES, &tmA_lo, &full[stage], kx, t.mt * GEMM_BM);
          tma_load_2d(st + 2 * L::A_BYTES, &tmB_hi, &full[stage], kx, t.nt * BN);
          tma_load_2d(st + 2 * L::A_BYTES + L::B_BYTES, &tmB_lo, &full[stage], kx, t.nt * BN);
          if (++stage == STAGES) {
            stage = 0;
            phase ^= 1u;
          }
        }
      }
      if (*abort) {
        // Let loads already issued land before the CTA can exit (bounded).
        for (int s = 0; s < STAGES; s++) {
          if (!(armed & (1u << s))) continue;
          const uint32_t par = (armed_parity >> s) & 1u;
          const uint64_t t0 = global_timer_ns();
          while (!mbar_try_wait(&full[s], par) && global_timer_ns() - t0 < 100000000ull) {
          }
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // ---------------------------------------------------------- MMA issuer
      int stage = 0;
      uint32_t phase = 0;
      int acc = 0;
      uint32_t acc_phase = 0;
      bool ok = true;
      for (int u = blockIdx.x; ok && u < shape.num_units && !*abort; u += gridDim.x) {
        const Unit t = decode_unit(shape, u);
        for (int c0 = t.kb0; ok && c0 < t.kb1; c0 += PROMO) {
          const int c1 = min(t.kb1, c0 + PROMO);
          if (!mbar_wait_bounded(&tempty[acc], acc_phase ^ 1u, abort, shape.status,
                                 DEV_ERR_TIMEOUT_MMA_TMEM, tmo)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d_tmem = tmem_base + static_cast<uint32_t>(acc * BN);
          for (int kb = c0; kb < c1; kb++) {
            if (!mbar_wait_bounded(&full[stage], phase, abort, shape.status,
                                   DEV_ERR_TIMEOUT_MMA_SMEM, tmo)) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t a_hi = smem_u32(smem + stage * L::STAGE_BYTES);
            const uint32_t a_lo = a_hi + L::A_BYTES;
            const uint32_t b_hi = a_hi + 2 * L::A_BYTES;
            const uint32_t b_lo = b_hi + L::B_BYTES;
#pragma unroll
            for (int kk = 0; kk < BK / 8; kk++) {
              const uint32_t off = kk * 32;  // 8 TF32 elements of K per MMA
              const uint64_t dah = sdesc_kmajor(a_hi + off, SBO, SWZ);
              const uint64_t dal = sdesc_kmajor(a_lo + off, SBO, SWZ);
              const uint64_t dbh = sdesc_kmajor(b_hi + off, SBO, SWZ);
              const uint64_t dbl = sdesc_kmajor(b_lo + off, SBO, SWZ);
              mma_tf32(d_tmem, dal, dbh, IDESC, (kb > c0 || kk > 0) ? 1u : 0u);
              mma_tf32(d_tmem, dah, dbl, IDESC, 1u);
              mma_tf32(d_tmem, dah, dbh, IDESC, 1u);
            }
            mma_commit(&empty[stage]);
            if (++stage == STAGES) {
              stage = 0;
              phase ^= 1u;
            }
          }
          if (!ok) break;
          mma_commit(&tfull[acc]);
          if (++acc == 2) {
            acc = 0;
            acc_phase ^= 1u;
          }
        }
      }
      if (*abort) {
        // Wait (bounded) for MMAs already issued before TMEM is released.
        mma_commit(drain);
        const uint64_t t0 = global_timer_ns();
        while (!mbar_try_wait(drain, 0) && global_timer_ns() - t0 < 100000000ull) {
        }
      }
    }
  } else {
    // ------------------------------------------------------------ accumulate + epilogue
    constexpr int HALF = BN / 2;
    const int q = warp & 3;          // TMEM lanes [32q, 32q+32) are the ones this warp may read
    const int half = (warp - 2) >> 2;  // column half [half*HALF, half*HALF + HALF)
    const int row = q * 32 + lane;
    Epi ep = epi;  // per-launch state the epilogue reads once
    ep.setup();
    int acc = 0;
    uint32_t acc_phase = 0;
    bool ok = true;
    for (int u = blockIdx.x; ok && u < shape.num_units; u += gridDim.x) {
      const Unit t = decode_unit(shape, u);
      ep.unit_begin(t, lane, half * HALF);
      float sum[HALF];
#pragma unroll
      for (int i = 0; i < HALF; i++) sum[i] = 0.f;
      for (int c0 = t.kb0; c0 < t.kb1; c0 += PROMO) {
        if (__any_sync(0xffffffffu, *abort != 0) ||
            !warp_wait(&tfull[acc], acc_phase, abort, shape.status, DEV_ERR_TIMEOUT_EPILOGUE,
                       tmo)) {
          ok = false;
          break;
        }
        tc_fence_after();
#pragma unroll
        for (int c = 0; c < HALF / 32; c++) {
          uint32_t r[32];
          tmem_ld_32x32b_x32(tmem_base + (static_cast<uint32_t>(q * 32) << 16) +
                                 static_cast<uint32_t>(acc * BN + half * HALF + c * 32),
                             r);
          tmem_ld_wait();
#pragma unroll
          for (int j = 0; j < 32; j++) sum[c * 32 + j] += __uint_as_float(r[j]);
        }
        tc_fence_before();
        mbar_arrive(&tempty[acc]);
        if (++acc == 2) {
          acc = 0;
          acc_phase ^= 1u;
        }
      }
      if (!ok) break;
#pragma unroll
      for (int c = 0; c < HALF / 32; c++)
        ep.chunk(t, q, lane, row, half * HALF + c * 32,
                  *reinterpret_cast<float(*)[32]>(sum + c * 32));
    }
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem_base, TMEM_COLS);
}

}  // namespace am24
