// Grouped CTA-pair GEMM: one persistent launch runs the tiles of many
// independent problems (a grouped AM step's Z = B V or V = B^T Z).
//
// The pipeline is gemm_pair_kernel's (gemm_pair.cuh): a cluster of two CTAs
// computes a 256 x BN tile with tcgen05.mma.cta_group::2, warp 0 loads K slabs
// with cp.async.bulk.tensor (no multicast), warp 1 of the leader issues the
// MMAs into one of two TMEM buffers, warps 2..9 of both CTAs drain them into
// round-to-nearest FP32 sums.  What changes is where a work unit comes from:
// the launch walks the units of one list of the step's plan (GPlan), whose
// problems and exclusive unit prefix the plan kernel wrote; unit u belongs to
// the problem whose prefix range holds it, and the three roles each look that
// up.  Per unit the problem supplies
//   * its tensor maps (a 64-byte aligned table in global memory; each load is
//     preceded by a tensormap acquire fence, as tables are rewritten between
//     launches when a serving loop admits new problems),
//   * its operand scheme (Z = B V: split FP16, three MMAs per 16 K; V = B^T Z:
//     that, or two MMAs for the L1-variance forms' exact sgn(z), or one FP16
//     MMA on the h0 / g0 planes in a MIXED problem's low-precision phase), the
//     scheme's promotion chunk and its output scales,
//   * its epilogue: split-K partial tiles (Z = B V), raw V with the selects'
//     candidate marks (constraints) or the fused L1 / L0 penalty.
// A stage holds the largest scheme's planes (two A, two B); smaller schemes
// load fewer bytes into the same layout.  All waits are bounded as in the
// one-problem kernel and record their code in the plan's status word.
//
// This file is included by am24_kernels.cu (namespace am24), after the
// epilogues (EpiPartial, EpiRaw, EpiPenalty) it uses.

// Index i of the list entry whose item range [pref[i], pref[i+1]) holds g.
__device__ __forceinline__ int find_item(const int *__restrict__ pref, int n, int g) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(pref + mid) <= g) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Before a TMA load reads a tensor map that a copy may have rewritten since the
// map was last used.
__device__ __forceinline__ void tensormap_acquire(const CUtensorMap *map) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(
                   reinterpret_cast<uint64_t>(map))
               : "memory");
}

template <int BN>
struct GPairSmem {
  static constexpr int ROW = 64;
  static constexpr int A_BYTES = GEMM_BM * ROW;
  static constexpr int B_BYTES = (BN / 2) * ROW;
  static constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
  static constexpr int STAGES_RAW = (200 * 1024) / STAGE_BYTES;
  static constexpr int STAGES = STAGES_RAW > 12 ? 12 : STAGES_RAW;
  static constexpr int BAR_BYTES = 256;
  static constexpr int TOTAL = STAGES * STAGE_BYTES + BAR_BYTES + 1024;
};

// One unit as a role sees it.
struct GUnit {
  int p;       // problem (slot)
  Unit t;
  int scheme;  // GScheme
  bool ok;     // the self-check passed (every role skips a unit that failed it)
};

template <bool Z1>
__device__ __forceinline__ GUnit grouped_unit(const GroupDev &g, int list, int np, int u,
                                              int rank) {
  const int *pref = g.pref + (size_t)list * (g.cap + 1);
  const int i = find_item(pref, np, u);
  GUnit r;
  r.p = __ldg(g.prob + (size_t)list * g.cap + i);
  const int local = u - __ldg(pref + i);
  r.ok = np > 0 && r.p >= 0 && r.p < g.cap && g.probs[r.p].live && local >= 0 &&
         local < __ldg(pref + i + 1) - __ldg(pref + i);
  if (!r.ok) {
    r.p = 0;
    r.scheme = GS_FP16X3;
    r.t = Unit{};
    if (rank == 0) atomicCAS(&g.plan->status, 0, (int)DEV_ERR_GROUP_ITEM);
    return r;
  }
  const GProblem &P = g.probs[r.p];
  GemmShape s;
  if (Z1) {
    s.m_tiles = P.m_tiles1;
    s.n_tiles = P.n_tiles1;
    s.kb_total = (P.n + PAIR_BK_BF16 - 1) / PAIR_BK_BF16;
    s.kb_per_split = P.kb_per_split1;
    r.scheme = GS_FP16X3;
  } else {
    s.m_tiles = P.m_tiles2;
    s.n_tiles = P.n_tiles2;
    s.kb_total = (P.m + PAIR_BK_BF16 - 1) / PAIR_BK_BF16;
    s.kb_per_split = s.kb_total;
    r.scheme = (int)*reinterpret_cast<volatile const uint32_t *>(P.ctl + GCTL_SCHEME);
  }
  r.t = decode_pair_unit(s, local, rank);
  return r;
}

__device__ __forceinline__ int scheme_na(int sc) { return sc == GS_FP16X1 ? 1 : 2; }
__device__ __forceinline__ int scheme_nb(int sc) { return sc == GS_FP16X3 ? 2 : 1; }
// K blocks (of 32) per TMEM chunk before the FP32 promotion: 48 MMA
// accumulations for the split schemes, the whole unit for single-pass BF16
__device__ __forceinline__ int scheme_promo(int sc) {
  return sc == GS_FP16X3 ? PairFP16x3::PROMO_K / PAIR_BK_BF16
                         : sc == GS_FP16X2A ? PairFP16x2A::PROMO_K / PAIR_BK_BF16 : 1 << 20;
}

// The drain of one unit into an epilogue: per-column data first, then each
// promotion chunk added into round-to-nearest sums, then the output scales and
// the epilogue's chunks of 32 columns.
template <int BN, class Epi>
__device__ __forceinline__ bool grouped_drain(Epi &ep, const Unit &t, int promo, int N, int M,
                                              const float *row_scale, const float *col_scale,
                                              uint32_t tmem_base, uint64_t *tfull,
                                              uint64_t *tempty, volatile int *abort, int *status,
                                              unsigned long long tmo, int &acc,
                                              uint32_t &acc_phase, int warp, int lane) {
  constexpr int HALF = BN / 2;
  const int q = warp & 3;
  const int half = (warp - 2) >> 2;
  const int row = q * 32 + lane;
  ep.setup();
  ep.unit_begin(t, lane, half * HALF);
  float cs[HALF / 32];
#pragma unroll
  for (int c = 0; c < HALF / 32; c++)
    cs[c] = col_scale ? __ldg(col_scale + min(t.nt * BN + half * HALF + c * 32 + lane, N - 1))
                      : 1.f;
  const float rs = row_scale ? __ldg(row_scale + min(t.m0 + row, M - 1)) : 1.f;
  float sum[HALF];
#pragma unroll
  for (int i = 0; i < HALF; i++) sum[i] = 0.f;
  for (int c0 = t.kb0; c0 < t.kb1; c0 += promo) {
    if (__any_sync(0xffffffffu, *abort != 0) ||
        !warp_wait(&tfull[acc], acc_phase, abort, status, DEV_ERR_TIMEOUT_EPILOGUE, tmo))
      return false;
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
  if (row_scale) {
#pragma unroll
    for (int i = 0; i < HALF; i++) sum[i] *= rs;
  }
  if (col_scale) {
#pragma unroll
    for (int i = 0; i < HALF; i++) sum[i] *= __shfl_sync(0xffffffffu, cs[i >> 5], i & 31);
  }
#pragma unroll
  for (int c = 0; c < HALF / 32; c++)
    ep.chunk(t, q, lane, row, half * HALF + c * 32, *reinterpret_cast<float(*)[32]>(sum + c * 32));
  return true;
}

// EPI == GE_PARTIAL: the split-K Z = B V of the list's dense problems
// (partial tiles); otherwise V = B^T Z of every problem in the list, whose
// formulations all take epilogue EPI (one epilogue per launch keeps the drain's
// registers those of the one-problem kernel).
template <int BN, int EPI>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(GEMM_THREADS, 1)
    gemm_pair_grouped_kernel(const GroupDev g, int list) {
  constexpr bool Z1 = EPI == GE_PARTIAL;
  using L = GPairSmem<BN>;
  constexpr int STAGES = L::STAGES;
  constexpr uint32_t SBO = L::ROW * 8;
  constexpr uint32_t TMEM_COLS = (2 * BN <= 128) ? 128 : (2 * BN <= 256) ? 256 : 512;
  constexpr uint32_t ID_F16 = make_idesc(2 * GEMM_BM, BN, 0u, 0u);
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
  const int num_units = g.plan->total[list];
  const int np = g.plan->n[list];
  if (num_units == 0) return;  // uniform over the grid
  const int rank = static_cast<int>(cluster_ctarank());
  const int pair = blockIdx.x >> 1;
  const int pairs = gridDim.x >> 1;
  int *status = &g.plan->status;
  const unsigned long long tmo = g.timeout_ns;

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
  }
  if (warp == 0) {
    __syncwarp();
    tmem_alloc_pair(tmem_holder, TMEM_COLS);
    tmem_relinquish_pair();
  }
  tc_fence_before();
  cluster_sync_all();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_holder;

  if (warp == 0) {
    if (lane == 0) {
      // ---------------------------------------------------------- producer (both CTAs)
      int stage = 0;
      uint32_t phase = 0;
      uint32_t armed = 0, armed_parity = 0;
      for (int u = pair; u < num_units && !*abort; u += pairs) {
        const GUnit gu = grouped_unit<Z1>(g, list, np, u, rank);
        if (!gu.ok) continue;
        const GMaps &mp = g.maps[gu.p];
        const CUtensorMap *ma[2], *mb[2];
        if (Z1) {
          ma[0] = &mp.a1_h0; ma[1] = &mp.a1_h1; mb[0] = &mp.b1_h0; mb[1] = &mp.b1_h1;
        } else {
          ma[0] = &mp.a2_h0; ma[1] = &mp.a2_h1; mb[0] = &mp.b2_h0; mb[1] = &mp.b2_h1;
        }
        const int na = scheme_na(gu.scheme), nb = scheme_nb(gu.scheme);
        for (int i = 0; i < na; i++) tensormap_acquire(ma[i]);
        for (int i = 0; i < nb; i++) tensormap_acquire(mb[i]);
        const uint32_t bytes = 2u * (uint32_t)(na * L::A_BYTES + nb * L::B_BYTES);
        const Unit &t = gu.t;
        for (int kb = t.kb0; kb < t.kb1; kb++) {
          if (!mbar_wait_bounded(&empty[stage], phase ^ 1u, abort, status,
                                 DEV_ERR_TIMEOUT_PRODUCER, tmo))
            break;
          uint8_t *st = smem + stage * L::STAGE_BYTES;
          if (rank == 0) {
            mbar_arrive_expect_tx(&full[stage], bytes);
            armed |= 1u << stage;
            armed_parity = (armed_parity & ~(1u << stage)) | (phase << stage);
          }
          const uint32_t bar = mapa_shared(smem_u32(&full[stage]), 0);
          const int kx = kb * PAIR_BK_BF16;
          const int yb = t.nt * BN + rank * (BN / 2);
          for (int i = 0; i < na; i++) tma_load_2d_pair(st + i * L::A_BYTES, ma[i], bar, kx, t.m0);
          for (int i = 0; i < nb; i++)
            tma_load_2d_pair(st + 2 * L::A_BYTES + i * L::B_BYTES, mb[i], bar, kx, yb);
          if (++stage == STAGES) {
            stage = 0;
            phase ^= 1u;
          }
        }
      }
      if (*abort) {
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
      for (int u = pair; ok && u < num_units && !*abort; u += pairs) {
        const GUnit gu = grouped_unit<Z1>(g, list, np, u, 0);
        if (!gu.ok) continue;
        const Unit &t = gu.t;
        const int promo = scheme_promo(gu.scheme);
        for (int c0 = t.kb0; ok && c0 < t.kb1; c0 += promo) {
          const int c1 = min(t.kb1, c0 + promo);
          if (!mbar_wait_bounded(&tempty[acc], acc_phase ^ 1u, abort, status,
                                 DEV_ERR_TIMEOUT_MMA_TMEM, tmo)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d_tmem = tmem_base + static_cast<uint32_t>(acc * BN);
          for (int kb = c0; kb < c1; kb++) {
            if (!mbar_wait_bounded(&full[stage], phase, abort, status, DEV_ERR_TIMEOUT_MMA_SMEM,
                                   tmo)) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t base = smem_u32(smem + stage * L::STAGE_BYTES);
            const uint32_t a[2] = {base, base + L::A_BYTES};
            const uint32_t bq = base + 2 * L::A_BYTES;
            const bool first = kb == c0;
            if (gu.scheme == GS_FP16X3) {
              const uint32_t b[2] = {bq, bq + L::B_BYTES};
              PairFP16x3::k_block<ID_F16>(d_tmem, a, b, SBO, first);
            } else if (gu.scheme == GS_FP16X2A) {
              const uint32_t b[1] = {bq};
              PairFP16x2A::k_block<ID_F16>(d_tmem, a, b, SBO, first);
            } else {
              const uint32_t a1[1] = {base}, b[1] = {bq};
              PairFP16x1::k_block<ID_F16>(d_tmem, a1, b, SBO, first);
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
    int acc = 0;
    uint32_t acc_phase = 0;
    for (int u = pair; u < num_units; u += pairs) {
      const GUnit gu = grouped_unit<Z1>(g, list, np, u, rank);
      if (!gu.ok) continue;
      const GProblem &P = g.probs[gu.p];
      const int promo = scheme_promo(gu.scheme);
      bool ok;
      if (Z1) {
        EpiPartial ep{P.ws, BN, P.m_tiles1, P.n_tiles1};
        ok = grouped_drain<BN>(ep, gu.t, promo, P.k, P.m, P.bt_row_scale, P.v_scale, tmem_base,
                               tfull, tempty, abort, status, tmo, acc, acc_phase, warp, lane);
      } else {
        // every scheme reads the scaled FP16 planes; Z's scale only where Z is
        // not an exact sign (the L1-variance forms)
        const float *rsc = P.row_scale;
        const float *csc = P.mode != 1 ? P.z_scale : nullptr;
        if (EPI == GE_RAW) {
          EpiRaw ep{P.Vraw, P.ldn, P.n, P.k, BN};
          ep.hint = P.sel_hint;
          ep.cmask = P.cmask;
          ok = grouped_drain<BN>(ep, gu.t, promo, P.k, P.n, rsc, csc, tmem_base, tfull, tempty,
                                 abort, status, tmo, acc, acc_phase, warp, lane);
        } else if (EPI == GE_PL1) {
          EpiPenalty<true> ep{P.Vx,  P.obj_part, P.nnz_part, P.ldn,   P.n,       P.k,
                              BN,    P.parts,    P.gamma,    P.vmask, nullptr,   nullptr,
                              P.ctl + GCTL_GATE, P.sparse_cap};
          ok = grouped_drain<BN>(ep, gu.t, promo, P.k, P.n, rsc, csc, tmem_base, tfull, tempty,
                                 abort, status, tmo, acc, acc_phase, warp, lane);
        } else {
          EpiPenalty<false> ep{P.Vx,  P.obj_part, P.nnz_part, P.ldn,   P.n,       P.k,
                               BN,    P.parts,    P.gamma,    P.vmask, nullptr,   nullptr,
                               P.ctl + GCTL_GATE, P.sparse_cap};
          ok = grouped_drain<BN>(ep, gu.t, promo, P.k, P.n, rsc, csc, tmem_base, tfull, tempty,
                                 abort, status, tmo, acc, acc_phase, warp, lane);
        }
      }
      if (!ok) break;
    }
  }

  tc_fence_before();
  cluster_sync_all();
  tc_fence_after();
  if (warp == 0) tmem_dealloc_pair(tmem_base, TMEM_COLS);
}
