// CTA-pair (cta_group::2) form of the 3xTF32 GEMM of gemm_tf32x3.cuh.
//
// A cluster of two CTAs, on two SMs, computes a 256 x BN tile of C.  CTA rank r
// of the pair loads rows [r*128, r*128 + 128) of the tile's A rows and rows
// [r*BN/2, r*BN/2 + BN/2) of its B rows; the leader CTA (rank 0) issues
// tcgen05.mma.cta_group::2 with M = 256, which reads both CTAs' shared memory
// and accumulates 128 rows x BN columns into each CTA's tensor memory.  The
// tensor-core work per SM is that of the one-CTA kernel with a 128 x BN tile,
// but each SM streams 128 + BN/2 operand rows per K slab instead of 128 + BN:
// for BN = 256 a third fewer bytes from L2 for the same FLOPs.
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

template <int BN, int BK, int STAGES>
struct PairSmem {
  static constexpr int A_BYTES = GEMM_BM * BK * 4;
  static constexpr int B_BYTES = (BN / 2) * BK * 4;
  static constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
  static constexpr int BAR_BYTES = 256;
  static constexpr int TOTAL = STAGES * STAGE_BYTES + BAR_BYTES + 1024;
};

constexpr int PAIR_EPI_WARPS = 2 * (GEMM_EPI_THREADS / 32);  // tempty arrivals per phase

template <int BN, int BK, int STAGES, int PROMO, class Epi>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(GEMM_THREADS, 1)
    gemm_tf32x3_pair_kernel(const __grid_constant__ CUtensorMap tmA_hi,
                            const __grid_constant__ CUtensorMap tmA_lo,
                            const __grid_constant__ CUtensorMap tmB_hi,
                            const __grid_constant__ CUtensorMap tmB_lo, const GemmShape shape,
                            Epi epi) {
  using L = PairSmem<BN, BK, STAGES>;
  static_assert(BK == 32 || BK == 16, "BK must be 32 (128B swizzle) or 16 (64B swizzle)");
  static_assert(BN % 32 == 0 && BN >= 64 && BN <= 256, "BN must be a multiple of 32 in [64,256]");
  constexpr uint32_t SWZ = (BK == 32) ? 2u : 4u;
  constexpr uint32_t SBO = BK * 4 * 8;
  constexpr uint32_t TMEM_COLS = (2 * BN <= 128) ? 128 : (2 * BN <= 256) ? 256 : 512;
  constexpr uint32_t IDESC = make_idesc(2 * GEMM_BM, BN, 2u, 2u);
  constexpr uint16_t BOTH = 0x3;

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
  if (shape.gate && *shape.gate <= shape.gate_max) return;  // uniform over the grid
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
    tma_prefetch_desc(&tmA_hi);
    tma_prefetch_desc(&tmA_lo);
    tma_prefetch_desc(&tmB_hi);
    tma_prefetch_desc(&tmB_lo);
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
          tma_load_2d_pair(st, &tmA_hi, bar, kx, t.m0);
          tma_load_2d_pair(st + L::A_BYTES, &tmA_lo, bar, kx, t.m0);
          tma_load_2d_pair(st + 2 * L::A_BYTES, &tmB_hi, bar, kx, yb);
          tma_load_2d_pair(st + 2 * L::A_BYTES + L::B_BYTES, &tmB_lo, bar, kx, yb);
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
            const uint32_t a_hi = smem_u32(smem + stage * L::STAGE_BYTES);
            const uint32_t a_lo = a_hi + L::A_BYTES;
            const uint32_t b_hi = a_hi + 2 * L::A_BYTES;
            const uint32_t b_lo = b_hi + L::B_BYTES;
#pragma unroll
            for (int kk = 0; kk < BK / 8; kk++) {
              const uint32_t off = kk * 32;
              const uint64_t dah = sdesc_kmajor(a_hi + off, SBO, SWZ);
              const uint64_t dal = sdesc_kmajor(a_lo + off, SBO, SWZ);
              const uint64_t dbh = sdesc_kmajor(b_hi + off, SBO, SWZ);
              const uint64_t dbl = sdesc_kmajor(b_lo + off, SBO, SWZ);
              mma_tf32_pair(d_tmem, dal, dbh, IDESC, (kb > c0 || kk > 0) ? 1u : 0u);
              mma_tf32_pair(d_tmem, dah, dbl, IDESC, 1u);
              mma_tf32_pair(d_tmem, dah, dbh, IDESC, 1u);
            }
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
    int acc = 0;
    uint32_t acc_phase = 0;
    bool ok = true;
    for (int u = pair; ok && u < shape.num_units; u += pairs) {
      const Unit t = decode_pair_unit(shape, u, rank);
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
      epi.begin(t, q, lane);
#pragma unroll
      for (int c = 0; c < HALF / 32; c++)
        epi.chunk(t, q, lane, row, half * HALF + c * 32,
                  *reinterpret_cast<float(*)[32]>(sum + c * 32));
      epi.end(t, q, lane);
    }
  }

  tc_fence_before();
  cluster_sync_all();  // no remote barrier traffic and no MMA into either CTA after this
  tc_fence_after();
  if (warp == 0) tmem_dealloc_pair(tmem_base, TMEM_COLS);
}

}  // namespace am24
