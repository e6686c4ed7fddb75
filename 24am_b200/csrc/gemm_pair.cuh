// CTA-pair (cta_group::2) GEMM for V = B^T Z, FP32-accurate, in two operand
// schemes (the Scheme template parameter):
//
//   PairTF32x3   both operands as TF32 hi/lo planes (x = hi + lo exactly);
//                lo*hi + hi*lo + hi*hi per K step, as in gemm_tf32x3.cuh.
//   PairBF16x3A  A as three BF16 planes with x = b0 + b1 + b2 exactly (each a
//                round-to-nearest BF16 of the remainder of the previous ones),
//                B as one BF16 plane that must hold B exactly -- the L1-variance
//                forms, where Z = sgn(B V) has entries -1, 0, +1.  Every product
//                b_i * z is exact; b2*z + b1*z + b0*z per K step.  Half the
//                tensor-core time of PairTF32x3 (BF16 runs at twice the TF32
//                rate and needs 3 instead of 6 MMAs per 16 K elements).
//
// A cluster of two CTAs, on two SMs, computes a 256 x BN tile of C.  CTA rank r
// of the pair loads rows [r*128, r*128 + 128) of the tile's A rows and rows
// [r*BN/2, r*BN/2 + BN/2) of its B rows; the leader CTA (rank 0) issues
// tcgen05.mma.cta_group::2 with M = 256, which reads both CTAs' shared memory
// and accumulates 128 rows x BN columns into each CTA's tensor memory.  The
// tensor-core work per SM is that of a one-CTA kernel with a 128 x BN tile,
// but each SM streams 128 + BN/2 operand rows per K slab instead of 128 + BN.
// Shared-memory rows are 64 bytes of K (64-byte swizzle) in both schemes, so a
// stage is 32 KB either way.
//
// The tensor-core FP32 accumulation does not round to nearest; as in
// gemm_tf32x3.cuh each TMEM buffer takes PROMO K slabs (S::PROMO_K elements: 48
// MMA accumulations in both schemes) and the epilogue warps add it into
// round-to-nearest FP32 registers.
//
// Roles are the one-CTA kernel's (warp 0 TMA, warp 1 MMA, warps 2..9
// accumulate + epilogue), with the MMA warp active in the leader only.
// Barriers sit at the same shared-memory offsets in both CTAs:
//   full[s]   used in the leader: armed there with both CTAs' bytes; the TMA
//             loads of both CTAs complete on it.
//   empty[s]  both CTAs: the leader's commit arrives on both (multicast).
//   tfull[a]  both CTAs: accumulator buffer a is ready (multicast commit).
//   tempty[a] used in the leader: one arrival per epilogue warp of each CTA.
// Every wait is bounded as in the one-CTA kernel; a CTA that gives up raises
// its own abort flag, and its partner gives up at its next bounded wait.  Both
// CTAs meet at a cluster barrier before tensor memory is released.
#pragma once
#include "gemm_tf32x3.cuh"

namespace am24 {

// Work unit u of a pair launch, as CTA `rank` sees it: 128-row block
// mt = 2 * (pair tile) + rank.  The pair tiles are ceil(m_tiles / 2); with an
// odd m_tiles the last pair's second block lies past the matrix (its loads
// read the zero fill, and epilogues skip rows >= M).
__device__ __forceinline__ Unit decode_pair_unit(const GemmShape &s, int u, int rank) {
  Unit r;
  const int m_pairs = (s.m_tiles + 1) >> 1;
  const int tiles = m_pairs * s.n_tiles;
  r.split = u / tiles;
  const int t = u - r.split * tiles;
  const int mp = t / s.n_tiles;
  r.nt = t - mp * s.n_tiles;
  r.mt = 2 * mp + rank;
  r.m0 = r.mt * GEMM_BM;
  r.kb0 = r.split * s.kb_per_split;
  r.kb1 = min(s.kb_total, r.kb0 + s.kb_per_split);
  r.index = u;
  return r;
}

// Operand schemes.  NA + NB <= 4 planes, passed as the kernel's first tensor
// maps (A planes first; the others are not read); BK = K elements per 64-byte
// shared-memory row.
struct PairTF32x3 {
  static constexpr int NA = 2, NB = 2, BK = PAIR_BK_TF32;
  // K elements per TMEM chunk before the FP32 promotion: 48 MMAs accumulate
  // into a chunk (16 K steps of 3)
  static constexpr int PROMO_K = 128;
  // a[0] = hi, a[1] = lo; b[0] = hi, b[1] = lo.  One 16-element K block:
  // two K = 8 steps of lo*hi + hi*lo + hi*hi.
  template <uint32_t ID>
  __device__ static void k_block(uint32_t d, const uint32_t (&a)[2], const uint32_t (&b)[2],
                                 uint32_t sbo, bool first) {
#pragma unroll
    for (int kk = 0; kk < 2; kk++) {
      const uint32_t off = kk * 32;
      const uint64_t dah = sdesc_kmajor(a[0] + off, sbo, 4u);
      const uint64_t dal = sdesc_kmajor(a[1] + off, sbo, 4u);
      const uint64_t dbh = sdesc_kmajor(b[0] + off, sbo, 4u);
      const uint64_t dbl = sdesc_kmajor(b[1] + off, sbo, 4u);
      mma_tf32_pair(d, dal, dbh, ID, (first && kk == 0) ? 0u : 1u);
      mma_tf32_pair(d, dah, dbl, ID, 1u);
      mma_tf32_pair(d, dah, dbh, ID, 1u);
    }
  }
  static constexpr uint32_t FMT = 2u;
};
struct PairBF16x3A {
  static constexpr int NA = 3, NB = 1, BK = PAIR_BK_BF16;
  // the same 48 MMA accumulations per chunk as PairTF32x3 (16 K steps of 3)
  static constexpr int PROMO_K = 256;
  // a[0..2] = b0, b1, b2; b[0] = the exact BF16 operand.  One 32-element K
  // block: two K = 16 steps of b2*z + b1*z + b0*z.
  template <uint32_t ID>
  __device__ static void k_block(uint32_t d, const uint32_t (&a)[3], const uint32_t (&b)[1],
                                 uint32_t sbo, bool first) {
#pragma unroll
    for (int kk = 0; kk < 2; kk++) {
      const uint32_t off = kk * 32;
      const uint64_t db = sdesc_kmajor(b[0] + off, sbo, 4u);
      mma_bf16_pair(d, sdesc_kmajor(a[2] + off, sbo, 4u), db, ID, (first && kk == 0) ? 0u : 1u);
      mma_bf16_pair(d, sdesc_kmajor(a[1] + off, sbo, 4u), db, ID, 1u);
      mma_bf16_pair(d, sdesc_kmajor(a[0] + off, sbo, 4u), db, ID, 1u);
    }
  }
  static constexpr uint32_t FMT = 1u;
};

// FP16 operands, each split in two: x = h0 + h1 (+ a residual under 2^-22 |x|),
// h0 = fp16_rn(x), h1 = fp16_rn(x - h0), after a power-of-two scaling that puts
// the operand's largest magnitude just under 2^14 (FP16's range is narrow; the
// epilogue multiplies the scaling back out exactly).  h1*g0 + h0*g1 + h0*g0 per
// K step: the accuracy class of PairTF32x3 (FP16 holds TF32's 11 significant
// bits) at half its tensor time (FP16 runs at twice the TF32 rate, 3 instead of
// 6 MMAs per 16 K elements).
struct PairFP16x3 {
  static constexpr int NA = 2, NB = 2, BK = PAIR_BK_BF16;
  static constexpr int PROMO_K = 256;  // 48 MMA accumulations per chunk
  template <uint32_t ID>
  __device__ static void k_block(uint32_t d, const uint32_t (&a)[2], const uint32_t (&b)[2],
                                 uint32_t sbo, bool first) {
#pragma unroll
    for (int kk = 0; kk < 2; kk++) {
      const uint32_t off = kk * 32;
      const uint64_t da0 = sdesc_kmajor(a[0] + off, sbo, 4u);
      const uint64_t db0 = sdesc_kmajor(b[0] + off, sbo, 4u);
      mma_f16_pair(d, sdesc_kmajor(a[1] + off, sbo, 4u), db0, ID, (first && kk == 0) ? 0u : 1u);
      mma_f16_pair(d, da0, sdesc_kmajor(b[1] + off, sbo, 4u), ID, 1u);
      mma_f16_pair(d, da0, db0, ID, 1u);
    }
  }
  static constexpr uint32_t FMT = 0u;  // F16
};
// As PairFP16x3 with B exact in one FP16 plane (the L1-variance forms' sgn):
// h1*z + h0*z per K step, 2 MMAs per 16 K elements.
struct PairFP16x2A {
  static constexpr int NA = 2, NB = 1, BK = PAIR_BK_BF16;
  static constexpr int PROMO_K = 384;  // 48 MMA accumulations per chunk
  template <uint32_t ID>
  __device__ static void k_block(uint32_t d, const uint32_t (&a)[2], const uint32_t (&b)[1],
                                 uint32_t sbo, bool first) {
#pragma unroll
    for (int kk = 0; kk < 2; kk++) {
      const uint32_t off = kk * 32;
      const uint64_t db = sdesc_kmajor(b[0] + off, sbo, 4u);
      mma_f16_pair(d, sdesc_kmajor(a[1] + off, sbo, 4u), db, ID, (first && kk == 0) ? 0u : 1u);
      mma_f16_pair(d, sdesc_kmajor(a[0] + off, sbo, 4u), db, ID, 1u);
    }
  }
  static constexpr uint32_t FMT = 0u;
};

// Single-pass BF16 operands (A = b0 of the split, B = Z rounded to BF16) for
// the low-precision phase of the mixed mode: one MMA per 16 K elements, a
// work unit accumulated whole in tensor memory (no intermediate promotion).
struct PairBF16x1 {
  static constexpr int NA = 1, NB = 1, BK = PAIR_BK_BF16;
  static constexpr int PROMO_K = 1 << 20;
  template <uint32_t ID>
  __device__ static void k_block(uint32_t d, const uint32_t (&a)[1], const uint32_t (&b)[1],
                                 uint32_t sbo, bool first) {
#pragma unroll
    for (int kk = 0; kk < 2; kk++) {
      const uint32_t off = kk * 32;
      mma_bf16_pair(d, sdesc_kmajor(a[0] + off, sbo, 4u), sdesc_kmajor(b[0] + off, sbo, 4u), ID,
                    (first && kk == 0) ? 0u : 1u);
    }
  }
  static constexpr uint32_t FMT = 1u;
};

// Single-pass FP16 operands (A = h0 of B's scaled split, B = g0 of Z's, or
// the exact sign of the L1-variance forms) for the low-precision phase of the
// mixed mode: one MMA per 16 K elements, as PairBF16x1, with FP16's 11-bit
// significands where BF16 keeps 8 (the power-of-two scales of the FP16 planes
// keep every row and column in range), so each product carries about 2^-12
// relative error instead of 2^-9.  A work unit is accumulated whole in tensor
// memory.
struct PairFP16x1 {
  static constexpr int NA = 1, NB = 1, BK = PAIR_BK_BF16;
  static constexpr int PROMO_K = 1 << 20;
  template <uint32_t ID>
  __device__ static void k_block(uint32_t d, const uint32_t (&a)[1], const uint32_t (&b)[1],
                                 uint32_t sbo, bool first) {
#pragma unroll
    for (int kk = 0; kk < 2; kk++) {
      const uint32_t off = kk * 32;
      mma_f16_pair(d, sdesc_kmajor(a[0] + off, sbo, 4u), sdesc_kmajor(b[0] + off, sbo, 4u), ID,
                   (first && kk == 0) ? 0u : 1u);
    }
  }
  static constexpr uint32_t FMT = 0u;
};

template <class S, int BN, int STAGES>
struct PairSmem {
  static constexpr int ROW = 64;  // bytes of K per shared-memory row
  static constexpr int A_BYTES = GEMM_BM * ROW;
  static constexpr int B_BYTES = (BN / 2) * ROW;
  static constexpr int STAGE_BYTES = S::NA * A_BYTES + S::NB * B_BYTES;
  static constexpr int BAR_BYTES = 256;
  static constexpr int TOTAL = STAGES * STAGE_BYTES + BAR_BYTES + 1024;
};

constexpr int PAIR_EPI_WARPS = 2 * (GEMM_EPI_THREADS / 32);  // tempty arrivals per phase

template <class S, int BN, int STAGES, int PROMO, class Epi>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(GEMM_THREADS, 1)
    gemm_pair_kernel(const __grid_constant__ CUtensorMap tm0,
                     const __grid_constant__ CUtensorMap tm1,
                     const __grid_constant__ CUtensorMap tm2,
                     const __grid_constant__ CUtensorMap tm3, const GemmShape shape, Epi epi) {
  using L = PairSmem<S, BN, STAGES>;
  constexpr int BK = S::BK;
  static_assert(S::NA + S::NB <= 4, "at most four operand planes");
  static_assert(BN % 32 == 0 && BN >= 64 && BN <= 256, "BN must be a multiple of 32 in [64,256]");
  constexpr uint32_t SBO = L::ROW * 8;  // bytes between 8-row core-matrix groups
  constexpr uint32_t TMEM_COLS = (2 * BN <= 128) ? 128 : (2 * BN <= 256) ? 256 : 512;
  constexpr uint32_t IDESC = make_idesc(2 * GEMM_BM, BN, S::FMT, S::FMT);
  constexpr uint16_t BOTH = 0x3;
  const CUtensorMap *maps[4] = {&tm0, &tm1, &tm2, &tm3};

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
  const int rank = static_cast<int>(cluster_ctarank());
  const int pair = blockIdx.x >> 1;
  const int pairs = gridDim.x >> 1;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; a++) {
      mbar_init(&tfull[a], 1);
      mbar_init(&tempty[a], PAIR_EPI_WARPS);
    }
    mbar_init(drain, 1);
    *abort = 0;
    fence_mbar_init();
    for (int i = 0; i < 4; i++) tma_prefetch_desc(maps[i]);
  }
  if (warp == 0) {
    __syncwarp();
    tmem_alloc_pair(tmem_holder, TMEM_COLS);
    tmem_relinquish_pair();
  }
  tc_fence_before();
  cluster_sync_all();  // both CTAs' barriers initialised, tensor memory allocated
  tc_fence_after();
  const uint32_t tmem_base = *tmem_holder;
  const unsigned long long tmo = shape.timeout_ns;

  if (warp == 0) {
    if (lane == 0) {
      // ---------------------------------------------------------- producer (both CTAs)
      int stage = 0;
      uint32_t phase = 0;
      uint32_t armed = 0;
      uint32_t armed_parity = 0;
      for (int u = pair; u < shape.num_units && !*abort; u += pairs) {
        const Unit t = decode_pair_unit(shape, u, rank);
        for (int kb = t.kb0; kb < t.kb1; kb++) {
          if (!mbar_wait_bounded(&empty[stage], phase ^ 1u, abort, shape.status,
                                 DEV_ERR_TIMEOUT_PRODUCER, tmo))
            break;
          uint8_t *st = smem + stage * L::STAGE_BYTES;
          if (rank == 0) {
            mbar_arrive_expect_tx(&full[stage], 2 * L::STAGE_BYTES);
            armed |= 1u << stage;
            armed_parity = (armed_parity & ~(1u << stage)) | (phase << stage);
          }
          const uint32_t bar = mapa_shared(smem_u32(&full[stage]), 0);
          const int kx = kb * BK;
          const int yb = t.nt * BN + rank * (BN / 2);
#pragma unroll
          for (int i = 0; i < S::NA; i++)
            tma_load_2d_pair(st + i * L::A_BYTES, maps[i], bar, kx, t.m0);
#pragma unroll
          for (int i = 0; i < S::NB; i++)
            tma_load_2d_pair(st + S::NA * L::A_BYTES + i * L::B_BYTES, maps[S::NA + i], bar, kx,
                             yb);
          if (++stage == STAGES) {
            stage = 0;
            phase ^= 1u;
          }
        }
      }
      if (*abort) {
        // Loads already issued must land before either CTA exits: the leader
        // waits for the stages it armed (they count both CTAs' bytes), and
        // both CTAs give in-flight copies a further 2 ms.
        for (int s = 0; s < STAGES; s++) {
          if (!(armed & (1u << s))) continue;
          const uint32_t par = (armed_parity >> s) & 1u;
          const uint64_t t0 = global_timer_ns();
          while (!mbar_try_wait(&full[s], par) && global_timer_ns() - t0 < 100000000ull) {
          }
        }
        const uint64_t t0 = global_timer_ns();
        while (global_timer_ns() - t0 < 2000000ull) {
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0 && rank == 0) {
      // ---------------------------------------------------------- MMA issuer (leader)
      int stage = 0;
      uint32_t phase = 0;
      int acc = 0;
      uint32_t acc_phase = 0;
      bool ok = true;
      for (int u = pair; ok && u < shape.num_units && !*abort; u += pairs) {
        const Unit t = decode_pair_unit(shape, u, 0);
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
            const uint32_t base = smem_u32(smem + stage * L::STAGE_BYTES);
            uint32_t a[S::NA], b[S::NB];
#pragma unroll
            for (int i = 0; i < S::NA; i++) a[i] = base + i * L::A_BYTES;
#pragma unroll
            for (int i = 0; i < S::NB; i++) b[i] = base + S::NA * L::A_BYTES + i * L::B_BYTES;
            S::template k_block<IDESC>(d_tmem, a, b, SBO, kb == c0);
            mma_commit_pair(&empty[stage], BOTH);
            if (++stage == STAGES) {
              stage = 0;
              phase ^= 1u;
            }
          }
          if (!ok) break;
          mma_commit_pair(&tfull[acc], BOTH);
          if (++acc == 2) {
            acc = 0;
            acc_phase ^= 1u;
          }
        }
      }
      if (*abort) {
        mma_commit_pair(drain, 0x1);
        const uint64_t t0 = global_timer_ns();
        while (!mbar_try_wait(drain, 0) && global_timer_ns() - t0 < 100000000ull) {
        }
      }
    }
  } else {
    // ------------------------------------------------------------ accumulate + epilogue (both)
    constexpr int HALF = BN / 2;
    const int q = warp & 3;
    const int half = (warp - 2) >> 2;
    const int row = q * 32 + lane;
    Epi ep = epi;  // per-launch state the epilogue reads once
    ep.setup();
    int acc = 0;
    uint32_t acc_phase = 0;
    bool ok = true;
    for (int u = pair; ok && u < shape.num_units; u += pairs) {
      const Unit t = decode_pair_unit(shape, u, rank);
      // per-column data of this unit, one value per lane and 32 columns,
      // loaded before the drain so that their latency hides behind it
      ep.unit_begin(t, lane, half * HALF);
      float cs[HALF / 32];
#pragma unroll
      for (int c = 0; c < HALF / 32; c++)
        cs[c] = shape.col_scale ? __ldg(shape.col_scale +
                                        min(t.nt * BN + half * HALF + c * 32 + lane, shape.N - 1))
                                : 1.f;
      const float rs =
          shape.row_scale ? __ldg(shape.row_scale + min(t.m0 + row, shape.M - 1)) : 1.f;
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
        __syncwarp();
        if (lane == 0) mbar_arrive_cluster(mapa_shared(smem_u32(&tempty[acc]), 0));
        if (++acc == 2) {
          acc = 0;
          acc_phase ^= 1u;
        }
      }
      if (!ok) break;
      if (shape.row_scale) {  // exact: powers of two
#pragma unroll
        for (int i = 0; i < HALF; i++) sum[i] *= rs;
      }
      if (shape.col_scale) {
#pragma unroll
        for (int i = 0; i < HALF; i++) sum[i] *= __shfl_sync(0xffffffffu, cs[i >> 5], i & 31);
      }
#pragma unroll
      for (int c = 0; c < HALF / 32; c++)
        ep.chunk(t, q, lane, row, half * HALF + c * 32,
                  *reinterpret_cast<float(*)[32]>(sum + c * 32));
    }
  }

  tc_fence_before();
  cluster_sync_all();  // no remote barrier traffic and no MMA into either CTA after this
  tc_fence_after();
  if (warp == 0) tmem_dealloc_pair(tmem_base, TMEM_COLS);
}

}  // namespace am24
