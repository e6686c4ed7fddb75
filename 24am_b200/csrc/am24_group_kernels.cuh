// Kernels of the grouped AM step (many independent problems per launch).
//
// Included by am24_kernels.cu after its anonymous namespace: every kernel
// here runs the same per-column bodies as the one-problem step (gathers,
// densify, split-K reduction, selects, finalize), on the work items of one
// list of the step's plan, with a grid sized to the GPU (a block walks items
// blockIdx.x, blockIdx.x + gridDim.x, ...).  The plan kernel writes the lists
// at the start of each step from every live problem's control words, so the
// lists only hold problems that still iterate, and each problem lands in the
// lists of the path its previous step chose (sparse gather, dense product,
// which select, which operand scheme).

// ------------------------------------------------------------ plan
constexpr int PLAN_THREADS = 1024;

__device__ __forceinline__ int ceil_div(int a, int b) { return (a + b - 1) / b; }

// Work items of problem P in list l this step (0: not a member).  Also used
// by the host-side capacity checks through the same rules.
__device__ int plan_items(const GProblem &P, int l, uint32_t gate, uint32_t scheme) {
  const bool dense = gate > P.sparse_cap;
  const bool grouped = !dense && gate <= min(P.sparse_cap, GATHER_GROUP_MAX_NNZ);
  const int pairs1 = (P.m_tiles1 + 1) >> 1, pairs2 = (P.m_tiles2 + 1) >> 1;
  switch (l) {
    case GL_GG0: case GL_GG1: case GL_GG2:
      return (P.mode == l - GL_GG0 && grouped) ? ceil_div(P.k, GATHER_GROUP) : 0;
    case GL_GA0: case GL_GA1: case GL_GA2:
      return (P.mode == l - GL_GA0 && !dense && !grouped) ? P.k : 0;
    case GL_DN0: case GL_DN1: case GL_DN2:
      return (P.mode == l - GL_DN0 && dense) ? P.k : 0;
    case GL_SEL_HARD: return P.formulation <= 1 ? P.k : 0;
    case GL_SEL_SCAN: return (P.formulation == 2 || P.formulation == 3) && !P.l1_exact ? P.k : 0;
    case GL_SEL_EXACT: return (P.formulation == 2 || P.formulation == 3) && P.l1_exact ? P.k : 0;
    case GL_SUPPORT: return P.mixed ? P.k : 0;
    case GL_FIN: return ceil_div(P.k, FIN_STARTS);
    case GL_GEMM1_64: case GL_GEMM1_128: case GL_GEMM1_256:
      return (dense && P.bn == (64 << (l - GL_GEMM1_64))) ? P.splits1 * pairs1 * P.n_tiles1 : 0;
    case GL_RAW_64: case GL_RAW_128: case GL_RAW_256:
      return (P.formulation <= 3 && P.bn == (64 << (l - GL_RAW_64))) ? pairs2 * P.n_tiles2 : 0;
    case GL_PL1_64: case GL_PL1_128: case GL_PL1_256:
      return (P.formulation >= 6 && P.bn == (64 << (l - GL_PL1_64))) ? pairs2 * P.n_tiles2 : 0;
    case GL_PL0_64: case GL_PL0_128: case GL_PL0_256:
      return ((P.formulation == 4 || P.formulation == 5) && P.bn == (64 << (l - GL_PL0_64)))
                 ? pairs2 * P.n_tiles2 : 0;
  }
  return 0;
}

// One block.  For every live problem that has not stopped: its step
// set-up (this step's gate from the last step's count, the batch maximum
// cleared, the operand scheme of V = B^T Z from its MIXED phase), then its
// membership and items in every list, compacted in slot order with
// exclusive prefixes.  Counts the step and the problems that run it.
__global__ void __launch_bounds__(PLAN_THREADS) group_plan_kernel(GroupDev g) {
  __shared__ int wsum[GL_COUNT][PLAN_THREADS / 32];
  __shared__ int carry_n[GL_COUNT], carry_t[GL_COUNT];
  __shared__ int act_sum;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  if (tid < GL_COUNT) {
    carry_n[tid] = 0;
    carry_t[tid] = 0;
  }
  if (tid == 0) act_sum = 0;
  __syncthreads();
  for (int base = 0; base < g.cap; base += PLAN_THREADS) {
    const int p = base + tid < g.cap ? g.order[base + tid] : g.cap;
    int items[GL_COUNT];
    bool act = false;
    if (p < g.cap) {
      GProblem &P = g.probs[p];
      if (P.live && P.ctl[CTL_STOP] == 0u) {
        act = true;
        const uint32_t gate = P.ctl[GCTL_NEXT];
        P.ctl[GCTL_GATE] = gate;
        P.ctl[GCTL_NEXT] = 0u;
        *P.max_err = 0.f;
        const bool low = P.mixed && P.phase[0] == 0u;
        const uint32_t sc = low ? GS_FP16X1 : (P.mode == 1 ? GS_FP16X2A : GS_FP16X3);
        P.ctl[GCTL_SCHEME] = sc;
#pragma unroll
        for (int l = 0; l < GL_COUNT; l++) items[l] = plan_items(P, l, gate, sc);
      }
    }
    if (!act) {
#pragma unroll
      for (int l = 0; l < GL_COUNT; l++) items[l] = 0;
    }
    if (act) atomicAdd(&act_sum, 1);
    // per list: block-wide exclusive scans of membership and items
#pragma unroll 1
    for (int l = 0; l < GL_COUNT; l++) {
      const int mem = items[l] > 0 ? 1 : 0;
      // pack (membership, items) scans into two warp scans
      int in = mem, it = items[l];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int a = __shfl_up_sync(FULL, in, o), b = __shfl_up_sync(FULL, it, o);
        if (lane >= o) {
          in += a;
          it += b;
        }
      }
      if (lane == 31) wsum[l][w] = (in << 0);  // membership totals per warp
      __syncthreads();
      int off_n = 0;
      for (int i = 0; i < w; i++) off_n += wsum[l][i];
      int tot_n = 0;
      for (int i = 0; i < PLAN_THREADS / 32; i++) tot_n += wsum[l][i];
      __syncthreads();
      if (lane == 31) wsum[l][w] = it;
      __syncthreads();
      int off_t = 0;
      for (int i = 0; i < w; i++) off_t += wsum[l][i];
      int tot_t = 0;
      for (int i = 0; i < PLAN_THREADS / 32; i++) tot_t += wsum[l][i];
      if (mem) {
        const int pos = carry_n[l] + off_n + in - 1;
        g.prob[(size_t)l * g.cap + pos] = p;
        g.pref[(size_t)l * (g.cap + 1) + pos] = carry_t[l] + off_t + it - items[l];
      }
      __syncthreads();
      if (tid == 0) {
        carry_n[l] += tot_n;
        carry_t[l] += tot_t;
      }
      __syncthreads();
    }
  }
  if (tid < GL_COUNT + 3) g.plan->next[tid] = 0;
  if (tid < GL_COUNT) {
    g.plan->n[tid] = carry_n[tid];
    g.plan->total[tid] = carry_t[tid];
    g.pref[(size_t)tid * (g.cap + 1) + carry_n[tid]] = carry_t[tid];
  }
  if (tid == 0) {
    g.plan->active = act_sum;
    g.plan->loops += 1;
  }
}

// ------------------------------------------------------------ per-column kernels
// The item loop of one list: fn(problem, local item) for every item of list l.
// Blocks take items from the list's counter, so the widest problems' items
// (listed first) start first and no block idles while another holds a queue.
template <class Fn>
__device__ __forceinline__ void for_items(const GroupDev &g, int l, Fn fn, int counter = -1) {
  __shared__ int taken;
  const int total = g.plan->total[l];
  const int np = g.plan->n[l];
  const int *pref = g.pref + (size_t)l * (g.cap + 1);
  const int *prob = g.prob + (size_t)l * g.cap;
  for (;;) {
    if (threadIdx.x == 0) taken = atomicAdd(&g.plan->next[counter < 0 ? l : counter], 1);
    __syncthreads();
    const int it = taken;
    __syncthreads();
    if (it >= total) break;
    const int i = find_item(pref, np, it);
    const int p = __ldg(prob + i);
    const int local = it - __ldg(pref + i);
    // self-check: the plan only lists live problems' items
    if (np <= 0 || p < 0 || p >= g.cap || !g.probs[p].live || local < 0 ||
        local >= __ldg(pref + i + 1) - __ldg(pref + i)) {
      if (threadIdx.x == 0) atomicCAS(&g.plan->status, 0, (int)DEV_ERR_GROUP_ITEM);
      continue;  // uniform over the block
    }
    fn(g.probs[p], local);
    __syncthreads();  // shared memory is reused by the next item
  }
}

template <int MODE>
__global__ void __launch_bounds__(GATHER_THREADS) g_gather_group_kernel(GroupDev g) {
  for_items(g, GL_GG0 + MODE, [](const GProblem &P, int item) {
    gather_bv_group_body<MODE>(P.Bc, P.ldm, P.m, P.ldn, P.k, P.Vx, P.vmask, P.Z_hi, P.Z_lo, P.fz,
                               P.ctl + GCTL_GATE, P.sparse_cap, P.Z_b, P.Z_h, P.zplane,
                               P.z_scale, P.ctl + CTL_STOP, item);
  });
}

template <int MODE>
__global__ void __launch_bounds__(GATHER_THREADS) g_gather_kernel(GroupDev g) {
  for_items(g, GL_GA0 + MODE, [](const GProblem &P, int j) {
    gather_bv_body<MODE>(P.Bc, P.ldm, P.m, P.ldn, P.Vx, P.vmask, P.Z_hi, P.Z_lo, P.fz,
                         P.ctl + GCTL_GATE, P.sparse_cap, P.Z_b, P.Z_h, P.zplane, P.z_scale,
                         P.ctl + CTL_STOP, j);
  });
}

// dense steps before Z = B V: the FP16 planes of V (the problems of mode `mode`)
__global__ void __launch_bounds__(DENSIFY_THREADS, DENSIFY_BLOCKS_PER_SM)
    g_densify_kernel(GroupDev g, int mode) {
  for_items(g, GL_DN0 + mode, [](const GProblem &P, int j) {
    densify_fp16_body(P.Vx, P.vmask, P.ldn, P.n, P.V_h, (size_t)P.k * P.ldn, P.v_scale,
                      P.ctl + GCTL_GATE, P.sparse_cap, P.ctl + CTL_STOP, j);
  });
}

// dense steps after Z = B V: the split-K sum and the sign / norm / normalise
template <int MODE>
__global__ void __launch_bounds__(256) g_z_reduce_kernel(GroupDev g) {
  for_items(g, GL_DN0 + MODE, [](const GProblem &P, int j) {
    z_reduce_body<MODE>(P.ws, P.splits1, P.m_tiles1, P.n_tiles1, P.bn, P.m, P.Z_hi, P.Z_lo,
                        P.ldm, P.fz, P.ctl + GCTL_GATE, P.sparse_cap, P.Z_b, P.Z_h, P.zplane,
                        P.z_scale, P.ctl + CTL_STOP, j);
  }, GL_COUNT + MODE);
}

__global__ void __launch_bounds__(HARD_THREADS) g_hard_select_kernel(GroupDev g) {
  for_items(g, GL_SEL_HARD, [](const GProblem &P, int j) {
    hard_select_body(P.Vraw, P.ldn, P.n, P.constraint, P.Vx, P.nnz, P.status, P.vmask,
                     P.sel_hint, P.ctl + CTL_STOP, P.cmask, j);
  });
}

template <bool EXACT>
__global__ void __launch_bounds__(SOFT_THREADS, 4) g_soft_select_kernel(GroupDev g) {
  for_items(g, EXACT ? GL_SEL_EXACT : GL_SEL_SCAN, [](const GProblem &P, int j) {
    soft_select_body<EXACT>(P.Vraw, P.ldn, P.n, P.constraint, P.Vx, P.nnz, P.status, P.vmask,
                            P.sel_hint, P.ctl + CTL_STOP, P.cmask, j);
  });
}

// MIXED: per start, whether its support (non-zero mask) changed this step, by
// a 64-bit hash of the mask words (splitmix64 of (word index, word), summed,
// so that the order of the additions does not matter); then the stability
// count and, by the problem's last item, the phase switch (support_kernel's
// rule).  The hash of a column that changed equals the previous one with
// probability 2^-64.
__global__ void __launch_bounds__(256) g_support_kernel(GroupDev g) {
  __shared__ unsigned long long red[8];
  for_items(g, GL_SUPPORT, [&](const GProblem &P, int j) {
    const int words = P.ldn >> 5;
    const uint32_t *a = P.vmask + (size_t)j * words;
    unsigned long long h = 0ull;
    for (int wd = threadIdx.x; wd < words; wd += blockDim.x)
      h += splitmix64(((uint64_t)(uint32_t)wd << 32) | a[wd]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) h += __shfl_xor_sync(FULL, h, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = h;
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned long long t = 0ull;
      for (int i = 0; i < (int)(blockDim.x >> 5); i++) t += red[i];
      const bool same = P.mask_hash[j] == t;
      P.mask_hash[j] = t;
      // no start counts as stable during the FP32 lead-in (phase[0] >= 2)
      const bool lead = *reinterpret_cast<volatile uint32_t *>(P.phase) >= 2u;
      const uint32_t st = (same && !lead) ? min(P.stable[j] + 1u, 0x7FFFFFFFu) : 0u;
      P.stable[j] = st;
      if (st >= P.k_stable) atomicAdd(&P.ctl[GCTL_SUPPORT], 1u);
      __threadfence();
      if (atomicAdd(&P.ctl[GCTL_SBLOCKS], 1u) == (uint32_t)P.k - 1) {
        __threadfence();
        const uint32_t count = atomicExch(&P.ctl[GCTL_SUPPORT], 0u);
        const uint32_t ph = P.phase[0];
        P.phase[3] = ph;
        P.phase[0] = mixed_next_phase(ph, count >= P.need_stable);
        P.ctl[GCTL_SBLOCKS] = 0u;
      }
    }
  });
}

// Per start the objective, change and batch maximum (finalize_start); the
// problem's last item closes its step: counts it, keeps the largest change and
// sets the stop word after the step the reference's batch loop ends on (it > 0
// in the refinement phase with the largest change below the tolerance), after
// its max_iter-th step, or when a device-side wait gave up.
__global__ void __launch_bounds__(256) g_finalize_kernel(GroupDev g) {
  for_items(g, GL_FIN, [&](const GProblem &P, int item) {
    FinalizeArgs a;
    a.k = P.k;
    a.formulation = P.formulation;
    a.parts = P.parts;
    a.it = (int)P.ctl[CTL_STEPS];
    a.store_all = 0;
    a.log_shift = 0;
    a.log_capacity = 0;
    a.tolerance = P.tolerance;
    a.fz = P.fz;
    a.obj_part = P.obj_part;
    a.nnz_part = P.nnz_part;
    a.nnz_sel = P.nnz;
    a.val = P.val;
    a.err = P.err;
    a.max_err = P.max_err;
    a.max_nnz = P.ctl + GCTL_NEXT;
    a.iters = nullptr;
    a.cards = nullptr;
    a.ctl = P.ctl;
    a.phase = P.mixed ? P.phase : nullptr;
    a.status = P.status;
    a.stop_check = 1;
    const int j = item * FIN_STARTS + (threadIdx.x >> 5);
    if (j < P.k) finalize_start(a, j, threadIdx.x & 31);
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      const int items = ceil_div(P.k, FIN_STARTS);
      if (atomicAdd(&P.ctl[CTL_BLOCKS], 1u) == (uint32_t)items - 1) {
        __threadfence();
        const float me = *reinterpret_cast<volatile float *>(P.max_err);
        const bool refined = !P.mixed || P.phase[3] != 0u;
        const uint32_t steps = P.ctl[CTL_STEPS] + 1u;
        P.ctl[CTL_STEPS] = steps;
        if (!refined) P.ctl[CTL_LOW_STEPS] += 1u;
        P.ctl[CTL_MAX_ERR] = __float_as_uint(me);
        if ((a.it > 0 && refined && (double)me < P.tolerance) ||
            steps >= (uint32_t)P.max_iter ||
            *reinterpret_cast<const volatile int *>(P.status) != 0)
          P.ctl[CTL_STOP] = 1u;
        P.ctl[CTL_BLOCKS] = 0u;
      }
    }
  });
}

// The WHILE condition of a captured step loop: another step while some live
// problem has not stopped, the launch's step cap is not reached and no wait
// of a grouped product gave up.  Also writes every slot's state to g.done,
// which a host polls with one copy.
__global__ void __launch_bounds__(256) g_condition_kernel(GroupDev g,
                                                          cudaGraphConditionalHandle handle,
                                                          bool in_graph) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  for (int p = threadIdx.x; p < g.cap; p += blockDim.x) {
    const GProblem &P = g.probs[p];
    uint32_t d = 0u;
    if (P.live) {
      d = *reinterpret_cast<volatile const uint32_t *>(P.ctl + CTL_STOP) == 0u ? 1u : 2u;
      if (d == 1u) any = 1;
    }
    g.done[p] = d;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const GPlan &pl = *g.plan;
    const bool more = any && pl.loops < pl.loop_cap && pl.status == 0;
    if (in_graph) cudaGraphSetConditional(handle, more ? 1u : 0u);
  }
}
