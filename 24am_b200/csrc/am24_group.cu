// Host side of the grouped solves (am24_group_*, include/am24.h): many
// independent problems, each one reference batch (c++/src/gpower/
// sparse_PCA_solver.h:171-232) on its own resident matrix and settings, run
// together by one captured CUDA graph.  The graph holds a WHILE node whose
// body is one grouped AM step (launch_grouped_step: a plan kernel, then every
// product and per-start pass of all problems as one launch each) followed by
// the kernel that sets the loop's condition; so a run is one graph launch and
// the host never waits between steps.  Problems live in slots of device
// tables (descriptors and tensor maps) that the graph reads, so problems come
// and go between launches without rebuilding the graph.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <vector>

#include "am24.h"
#include "am24_host.h"
#include "am24_internal.h"

using namespace am24;
using namespace am24host;

namespace {

struct GroupSlot {
  bool used = false;
  am24_matrix mat = nullptr;
  am24_settings s{};
  GProblem P{};
  std::unique_ptr<Allocs> mem;
};

}  // namespace

struct am24_group_s {
  am24_handle h = nullptr;
  int cap = 0;
  Allocs mem;  // the tables (plain allocations: they outlive any one stream's work)
  GroupDev dev{};
  std::vector<GroupSlot> slots;
  GroupGrids grids{};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  float last_ms = 0.f;
  int autotune = 0;             // am24_group_set_autotune
  am24_group tuner = nullptr;   // the scratch group the tuner times candidates in
  ~am24_group_s() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  }
};

namespace {

// The plan's host-written words, before a launch.
struct PlanHead {
  int loops, loop_cap, status;
};

am24_status build_graph(am24_group g) {
  if (g->exec) return AM24_OK;
  const cudaStream_t st = g->h->stream;
  AM24_CUDA(grouped_grids(&g->grids));
  AM24_CUDA(cudaGraphCreate(&g->graph, 0));
  cudaGraphConditionalHandle cond;
  AM24_CUDA(cudaGraphConditionalHandleCreate(&cond, g->graph, 1, cudaGraphCondAssignDefault));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = cond;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  AM24_CUDA(cudaGraphAddNode(&node, g->graph, nullptr, 0, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  AM24_CUDA(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal));
  cudaError_t e = launch_grouped_step(g->dev, g->grids, st);
  if (e == cudaSuccess) e = launch_grouped_condition(g->dev, (unsigned long long)cond, st);
  cudaGraph_t captured = nullptr;
  const cudaError_t e2 = cudaStreamEndCapture(st, &captured);
  if (e != cudaSuccess || e2 != cudaSuccess) {
    cudaGetLastError();
    return fail(AM24_ERR_CUDA, std::string("grouped step capture: ") +
                                   cudaGetErrorString(e != cudaSuccess ? e : e2));
  }
  AM24_CUDA(cudaGraphInstantiate(&g->exec, g->graph, 0));
  return AM24_OK;
}

// AM24_GROUP_EAGER=1: runs step by step from the host instead of one graph
// launch (same kernels and results; for profilers).
bool eager_steps() {
  static const bool on = [] {
    const char *e = std::getenv("AM24_GROUP_EAGER");
    return e && e[0] == '1';
  }();
  return on;
}

am24_status check_slot(am24_group g, uint32_t problem) {
  if (!g) return fail(AM24_ERR_INVALID_ARG, "NULL group");
  if (problem >= (uint32_t)g->cap || !g->slots[problem].used)
    return fail(AM24_ERR_INVALID_ARG, "no such problem in the group");
  return AM24_OK;
}

// The control words of a problem (synchronizes the stream).
am24_status read_ctl(am24_group g, const GroupSlot &sl, uint32_t *ctl) {
  AM24_CUDA(cudaMemcpyAsync(ctl, sl.P.ctl, sizeof(uint32_t) * GCTL_WORDS,
                            cudaMemcpyDeviceToHost, g->h->stream));
  AM24_CUDA(cudaStreamSynchronize(g->h->stream));
  return AM24_OK;
}

// The order in which the plan lists the slots: live problems by descending
// feature count (their per-column passes are the longest, so their items go
// first), then the rest.  Written after every add and remove.
am24_status upload_order(am24_group g) {
  std::vector<int> order(g->cap);
  for (int i = 0; i < g->cap; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    const int na = g->slots[a].used ? g->slots[a].P.n : -1;
    const int nb = g->slots[b].used ? g->slots[b].P.n : -1;
    return na > nb;
  });
  AM24_CUDA(cudaMemcpyAsync(const_cast<int *>(g->dev.order), order.data(), sizeof(int) * g->cap,
                            cudaMemcpyHostToDevice, g->h->stream));
  AM24_CUDA(cudaStreamSynchronize(g->h->stream));
  return AM24_OK;
}

}  // namespace

namespace am24host {

uint64_t group_problem_bytes(int m, int n, int k, int formulation, bool mixed) {
  const uint64_t ldm = (uint64_t)(m + 31) / 32 * 32, ldn = (uint64_t)(n + 31) / 32 * 32;
  const uint64_t kv = (uint64_t)k * ldn, kz = (uint64_t)k * ldm, words = kv / 32;
  const int bn = pick_bn(k);
  const uint64_t m_tiles1 = (m + BM - 1) / BM, n_tiles = (k + bn - 1) / bn;
  int splits = 1, kbps = 1;
  choose_splits((int)(((m_tiles1 + 1) / 2) * n_tiles), (n + PAIR_BK_BF16 - 1) / PAIR_BK_BF16,
                std::max(1, num_sms() / 2), &splits, &kbps);
  const uint64_t parts = (uint64_t)((n + BM - 1) / BM) * 4;
  const uint64_t zh = is_l1_variance(formulation) ? 1 : 2;
  uint64_t b = kv * 4 * 2 + kv * 2 * 2 + words * 4 * (is_constrained(formulation) ? 2 : 1) +
               kz * (4 + 4 + 2 * zh) +
               (uint64_t)ws_floats(splits, (int)m_tiles1, (int)n_tiles, bn) * 4 +
               (uint64_t)k * (4 * 8 + parts * 8 + (mixed ? 16 : 0)) + 4096;
  return b;
}

am24_status group_done_flags(am24_group g, std::vector<uint32_t> &out) {
  out.resize(g->cap);
  AM24_CUDA(cudaMemcpyAsync(out.data(), g->dev.done, sizeof(uint32_t) * g->cap,
                            cudaMemcpyDeviceToHost, g->h->stream));
  AM24_CUDA(cudaStreamSynchronize(g->h->stream));
  return AM24_OK;
}

}  // namespace am24host

extern "C" {

am24_status am24_group_create(am24_handle h, uint32_t capacity, am24_group *out) {
  if (!h || !out) return fail(AM24_ERR_INVALID_ARG, "NULL argument");
  *out = nullptr;
  if (capacity == 0 || capacity > 65536)
    return fail(AM24_ERR_INVALID_ARG, "capacity must be in [1, 65536]");
  AM24_CUDA(cudaSetDevice(h->device));
  std::unique_ptr<am24_group_s> g(new am24_group_s());
  g->h = h;
  g->cap = (int)capacity;
  g->slots.resize(capacity);
  GroupDev &d = g->dev;
  d.cap = (int)capacity;
  d.timeout_ns = 5000ull * 1000000ull;
  GMaps *maps = nullptr;
  AM24_TRY(g->mem.get(&d.probs, capacity));
  AM24_TRY(g->mem.get(&maps, capacity));
  AM24_TRY(g->mem.get(&d.plan, 1));
  AM24_TRY(g->mem.get(&d.prob, (size_t)GL_COUNT * capacity));
  AM24_TRY(g->mem.get(&d.pref, (size_t)GL_COUNT * (capacity + 1)));
  AM24_TRY(g->mem.get(&d.done, capacity));
  int *order = nullptr;
  AM24_TRY(g->mem.get(&order, capacity));
  d.order = order;
  d.maps = maps;
  AM24_CUDA(cudaMemsetAsync(d.done, 0, sizeof(uint32_t) * capacity, h->stream));
  AM24_CUDA(cudaMemsetAsync(d.probs, 0, sizeof(GProblem) * capacity, h->stream));
  AM24_CUDA(cudaMemsetAsync(maps, 0, sizeof(GMaps) * capacity, h->stream));
  AM24_CUDA(cudaMemsetAsync(d.plan, 0, sizeof(GPlan), h->stream));
  AM24_TRY(upload_order(g.get()));
  AM24_CUDA(cudaEventCreate(&g->e0));
  AM24_CUDA(cudaEventCreate(&g->e1));
  AM24_CUDA(cudaStreamSynchronize(h->stream));
  *out = g.release();
  return AM24_OK;
}

am24_status am24_group_destroy(am24_group g) {
  if (!g) return AM24_OK;
  if (g->tuner) am24_group_destroy(g->tuner);
  cudaSetDevice(g->h->device);
  cudaStreamSynchronize(g->h->stream);
  for (auto &sl : g->slots) sl.mem.reset();  // stream-ordered frees
  cudaStreamSynchronize(g->h->stream);
  delete g;
  return AM24_OK;
}

}  // extern "C"

namespace {

// Tile choices of one problem: the N tile of both products and the split-K
// factor of Z = B V (0: the cost model's).
struct TileCfg {
  int bn = 0, splits = 0;
};

am24_status group_add_impl(am24_group g, am24_matrix mat, const am24_settings *settings,
                           const float *start_points, const TileCfg &cfg, uint32_t *problem);
am24_status autotune(am24_group g, am24_matrix mat, const am24_settings &s, TileCfg *out);

}  // namespace

extern "C" {

am24_status am24_group_add(am24_group g, am24_matrix mat, const am24_settings *settings,
                           const float *start_points, uint32_t *problem) {
  if (!g || !mat || !settings || !problem) return fail(AM24_ERR_INVALID_ARG, "NULL argument");
  AM24_TRY(validate_settings(settings));
  if (mat->sparse)
    return fail(AM24_ERR_UNSUPPORTED, "sparse-resident matrices are not grouped");
  TileCfg cfg;
  if (g->autotune) AM24_TRY(autotune(g, mat, *settings, &cfg));
  return group_add_impl(g, mat, settings, start_points, cfg, problem);
}

}  // extern "C"

namespace {

am24_status group_add_impl(am24_group g, am24_matrix mat, const am24_settings *settings,
                           const float *start_points, const TileCfg &cfg, uint32_t *problem) {
  AM24_TRY(validate_settings(settings));
  if (settings->use_otf || settings->store_all)
    return fail(AM24_ERR_INVALID_ARG, "a group supports neither use_otf nor store_all");
  if (settings->start_mode == AM24_START_INJECTED && !start_points)
    return fail(AM24_ERR_INVALID_ARG, "start_mode INJECTED needs start_points");
  am24_handle h = g->h;
  AM24_CUDA(cudaSetDevice(h->device));
  const MatrixDev &M = mat->d;
  am24_settings s = *settings;
  AM24_TRY(am24_check_input(&s, (uint32_t)M.n));
  s.batch_size = s.total_starts;
  s.total_batches = 1;
  const int k = s.total_starts;
  if (k < 1 || k > (1 << 20)) return fail(AM24_ERR_INVALID_ARG, "total_starts must be in [1, 2^20]");
  int slot = -1;
  for (int i = 0; i < g->cap; i++)
    if (!g->slots[i].used) {
      slot = i;
      break;
    }
  if (slot < 0) return fail(AM24_ERR_INVALID_ARG, "the group is full");
  const bool mixed = s.precision == AM24_PRECISION_MIXED;
  const int f = s.formulation;
  AM24_TRY(ensure_fp16_planes(h, mat));
  AM24_TRY(ensure_bt_fp16_planes(h, mat));

  GroupSlot &sl = g->slots[slot];
  GProblem P{};
  P.live = 1;
  P.m = M.m;
  P.n = M.n;
  P.ldm = M.ldm;
  P.ldn = M.ldn;
  P.Bc = M.Bc;
  P.row_scale = M.row_scale;
  P.bt_row_scale = M.bt_row_scale;
  P.k = k;
  P.formulation = f;
  P.mode = is_l1_variance(f) ? 1 : (is_constrained(f) ? 0 : 2);
  P.l1_exact = s.l1_mode == AM24_L1_EXACT;
  P.mixed = mixed;
  P.max_iter = s.max_iter;
  P.constraint = s.constraint;
  P.gamma = (float)s.penalty;
  P.tolerance = s.tolerance;
  P.sparse_cap = (uint32_t)std::min(4096, M.n / 32);
  P.k_stable = s.stable_iterations;
  P.need_stable =
      std::min((uint32_t)k, (uint32_t)std::max(1.0, std::ceil((double)s.stable_share * k - 1e-9)));
  P.bn = cfg.bn ? cfg.bn : pick_bn(k);
  P.m_tiles1 = (M.m + BM - 1) / BM;
  P.n_tiles1 = (k + P.bn - 1) / P.bn;
  const int kb1 = (M.n + PAIR_BK_BF16 - 1) / PAIR_BK_BF16;
  if (cfg.splits > 0) {
    P.kb_per_split1 = (kb1 + std::min(cfg.splits, kb1) - 1) / std::min(cfg.splits, kb1);
    P.splits1 = (kb1 + P.kb_per_split1 - 1) / P.kb_per_split1;  // every split non-empty
  } else {
    choose_splits(((P.m_tiles1 + 1) / 2) * P.n_tiles1, kb1, std::max(1, num_sms() / 2),
                  &P.splits1, &P.kb_per_split1);
  }
  P.m_tiles2 = (M.n + BM - 1) / BM;
  P.n_tiles2 = (k + P.bn - 1) / P.bn;
  P.parts = P.m_tiles2 * 4;
  const size_t kv = (size_t)k * M.ldn, kz = (size_t)k * M.ldm, words = kv / 32;
  const size_t zh_planes = P.mode == 1 ? 1 : 2;
  P.zplane = kz;

  std::unique_ptr<Allocs> A(new Allocs(h->stream));
  am24_status st;
  if ((st = A->get(&P.Vx, kv)) || (st = A->get(&P.vmask, words)) ||
      (st = A->get(&P.Vraw, kv)) || (st = A->get(&P.sel_hint, k)) || (st = A->get(&P.nnz, k)) ||
      (is_constrained(f) && (st = A->get(&P.cmask, words))) ||
      (st = A->get(&P.Z_hi, kz)) || (st = A->get(&P.Z_lo, kz)) ||
      (st = A->get(&P.Z_h, zh_planes * kz)) || (st = A->get(&P.z_scale, k)) ||
      (st = A->get(&P.V_h, 2 * kv)) ||
      (st = A->get(&P.v_scale, k)) ||
      (st = A->get(&P.ws, ws_floats(P.splits1, P.m_tiles1, P.n_tiles1, P.bn))) ||
      (st = A->get(&P.fz, k)) || (st = A->get(&P.val, k)) || (st = A->get(&P.err, k)) ||
      (st = A->get(&P.max_err, 1)) || (st = A->get(&P.obj_part, (size_t)k * P.parts)) ||
      (st = A->get(&P.nnz_part, (size_t)k * P.parts)) || (st = A->get(&P.ctl, GCTL_WORDS)) ||
      (st = A->get(&P.status, 1)) ||
      (mixed && ((st = A->get(&P.stable, k)) || (st = A->get(&P.phase, 4)) ||
                 (st = A->get(&P.mask_hash, k)))))
    return st;
  const cudaStream_t hs = h->stream;
  // every buffer starts zeroed, as a batch's do: a slot's memory may come back
  // from the pool holding an earlier problem's state
  AM24_CUDA(cudaMemsetAsync(P.Vx, 0, sizeof(float) * kv, hs));
  AM24_CUDA(cudaMemsetAsync(P.Vraw, 0, sizeof(float) * kv, hs));
  AM24_CUDA(cudaMemsetAsync(P.vmask, 0, sizeof(uint32_t) * words, hs));
  AM24_CUDA(cudaMemsetAsync(P.Z_hi, 0, sizeof(float) * kz, hs));
  AM24_CUDA(cudaMemsetAsync(P.Z_lo, 0, sizeof(float) * kz, hs));
  AM24_CUDA(cudaMemsetAsync(P.z_scale, 0, sizeof(float) * k, hs));
  AM24_CUDA(cudaMemsetAsync(P.v_scale, 0, sizeof(float) * k, hs));
  AM24_CUDA(cudaMemsetAsync(P.obj_part, 0, sizeof(float) * k * P.parts, hs));
  AM24_CUDA(cudaMemsetAsync(P.nnz_part, 0, sizeof(float) * k * P.parts, hs));
  AM24_CUDA(cudaMemsetAsync(P.max_err, 0, sizeof(float), hs));
  AM24_CUDA(cudaMemsetAsync(P.Z_h, 0, sizeof(uint16_t) * zh_planes * kz, hs));
  AM24_CUDA(cudaMemsetAsync(P.V_h, 0, sizeof(uint16_t) * 2 * kv, hs));
  if (P.cmask) AM24_CUDA(cudaMemsetAsync(P.cmask, 0, sizeof(uint32_t) * words, hs));
  AM24_CUDA(cudaMemsetAsync(P.sel_hint, 0, sizeof(float) * k, hs));
  AM24_CUDA(cudaMemsetAsync(P.val, 0, sizeof(float) * k, hs));
  AM24_CUDA(cudaMemsetAsync(P.err, 0, sizeof(float) * k, hs));
  AM24_CUDA(cudaMemsetAsync(P.nnz, 0, sizeof(uint32_t) * k, hs));
  AM24_CUDA(cudaMemsetAsync(P.fz, 0, sizeof(float) * k, hs));
  AM24_CUDA(cudaMemsetAsync(P.status, 0, sizeof(int), hs));
  if (mixed) {
    AM24_CUDA(cudaMemsetAsync(P.stable, 0, sizeof(uint32_t) * k, hs));
    const uint32_t words[4] = {mixed_first_phase(s.lead_iterations), 0u, 0u, 0u};
    AM24_CUDA(cudaMemcpyAsync(P.phase, words, sizeof words, cudaMemcpyHostToDevice, hs));
    AM24_CUDA(cudaMemsetAsync(P.mask_hash, 0, sizeof(uint64_t) * k, hs));
  }
  // control words: dense first step, and no step at all when max_iter is 0
  uint32_t ctl[GCTL_WORDS] = {};
  ctl[GCTL_NEXT] = 0xFFFFFFFFu;
  ctl[CTL_STOP] = s.max_iter <= 0 ? 1u : 0u;
  AM24_CUDA(cudaMemcpyAsync(P.ctl, ctl, sizeof ctl, cudaMemcpyHostToDevice, hs));
  // starting points staged in Vraw, then split into values and masks
  if (s.start_mode == AM24_START_DEVICE_UNIFORM) {
    AM24_CUDA(launch_uniform_starts(P.Vraw, M.ldn, M.n, k, 0, hs));
  } else {
    std::vector<float> staging;
    const float *src = start_points;
    if (s.start_mode != AM24_START_INJECTED) {
      std::vector<unsigned> gidx(k);
      for (int i = 0; i < k; i++) gidx[i] = (unsigned)i;
      host_starts(s, (unsigned)M.n, start_points, gidx.data(), k, staging);
      src = staging.data();
    }
    AM24_CUDA(cudaMemcpy2DAsync(P.Vraw, sizeof(float) * M.ldn, src, sizeof(float) * M.n,
                                sizeof(float) * M.n, k, cudaMemcpyHostToDevice, hs));
    AM24_CUDA(cudaStreamSynchronize(hs));  // `staging` goes out of scope
  }
  AM24_CUDA(launch_load_columns(P.Vraw, M.ldn, M.n, k, P.Vx, M.ldn, P.vmask, hs));
  // tensor maps
  GMaps maps;
  std::memset(&maps, 0, sizeof maps);
  const size_t pc = (size_t)M.n * M.ldm, pt = (size_t)M.m * M.ldn;
  if ((st = make_map_bf16(h, &maps.a1_h0, M.Bt_h2, M.n, M.m, M.ldn, BM, true)) ||
      (st = make_map_bf16(h, &maps.a1_h1, M.Bt_h2 + pt, M.n, M.m, M.ldn, BM, true)) ||
      (st = make_map_bf16(h, &maps.b1_h0, P.V_h, M.n, k, M.ldn, P.bn / 2, true)) ||
      (st = make_map_bf16(h, &maps.b1_h1, P.V_h + kv, M.n, k, M.ldn, P.bn / 2, true)) ||
      (st = make_map_bf16(h, &maps.a2_h0, M.Bc_h2, M.m, M.n, M.ldm, BM, true)) ||
      (st = make_map_bf16(h, &maps.a2_h1, M.Bc_h2 + pc, M.m, M.n, M.ldm, BM, true)) ||
      (st = make_map_bf16(h, &maps.b2_h0, P.Z_h, M.m, k, M.ldm, P.bn / 2, true)) ||
      (zh_planes == 2 &&
       (st = make_map_bf16(h, &maps.b2_h1, P.Z_h + kz, M.m, k, M.ldm, P.bn / 2, true))))
    return st;
  AM24_CUDA(cudaMemcpyAsync(const_cast<GMaps *>(g->dev.maps) + slot, &maps, sizeof maps,
                            cudaMemcpyHostToDevice, hs));
  AM24_CUDA(cudaMemcpyAsync(g->dev.probs + slot, &P, sizeof P, cudaMemcpyHostToDevice, hs));
  AM24_CUDA(cudaStreamSynchronize(hs));
  sl.used = true;
  sl.mat = mat;
  sl.s = s;
  sl.P = P;
  sl.mem = std::move(A);
  AM24_TRY(upload_order(g));
  *problem = (uint32_t)slot;
  return AM24_OK;
}

}  // namespace

extern "C" {

am24_status am24_group_run(am24_group g, uint32_t max_steps, float *device_ms) {
  if (!g) return fail(AM24_ERR_INVALID_ARG, "NULL group");
  am24_handle h = g->h;
  AM24_CUDA(cudaSetDevice(h->device));
  AM24_TRY(build_graph(g));
  int cap = 0;
  for (const auto &sl : g->slots)
    if (sl.used) cap = std::max(cap, sl.s.max_iter);
  PlanHead head{0, max_steps > 0 ? (int)max_steps : cap + 1, 0};
  // loops, loop_cap and status sit after the two count arrays and `active`
  static_assert(offsetof(GPlan, loop_cap) == offsetof(GPlan, loops) + sizeof(int) &&
                    offsetof(GPlan, status) == offsetof(GPlan, loops) + 2 * sizeof(int),
                "plan layout");
  AM24_CUDA(cudaMemcpyAsync(reinterpret_cast<char *>(g->dev.plan) + offsetof(GPlan, loops), &head,
                            sizeof head, cudaMemcpyHostToDevice, h->stream));
  AM24_CUDA(cudaEventRecord(g->e0, h->stream));
  if (eager_steps()) {
    // profiling aid: the same step kernels launched from a host loop, so that
    // a profiler sees each of them (kernel nodes of a graph with a conditional
    // node are not profiled one by one); one host round trip per step
    std::vector<uint32_t> flags;
    for (int i = 0; i < head.loop_cap; i++) {
      AM24_CUDA(launch_grouped_step(g->dev, g->grids, h->stream));
      AM24_CUDA(launch_grouped_condition(g->dev, 0ull, h->stream, false));
      GPlan pl;
      AM24_CUDA(cudaMemcpyAsync(&pl, g->dev.plan, sizeof pl, cudaMemcpyDeviceToHost, h->stream));
      AM24_TRY(group_done_flags(g, flags));
      if (pl.status != 0 || std::find(flags.begin(), flags.end(), 1u) == flags.end()) break;
    }
  } else {
    AM24_CUDA(cudaGraphLaunch(g->exec, h->stream));
  }
  AM24_CUDA(cudaEventRecord(g->e1, h->stream));
  GPlan plan;
  AM24_CUDA(cudaMemcpyAsync(&plan, g->dev.plan, sizeof plan, cudaMemcpyDeviceToHost, h->stream));
  AM24_CUDA(cudaStreamSynchronize(h->stream));
  AM24_CUDA(cudaEventElapsedTime(&g->last_ms, g->e0, g->e1));
  if (device_ms) *device_ms = g->last_ms;
  if (plan.status == (int)DEV_ERR_GROUP_ITEM)
    return fail(AM24_ERR_CUDA, "grouped step: a work list named a problem that is not live "
                               "(the items were skipped)");
  if (plan.status != 0) {
    char buf[96];
    snprintf(buf, sizeof buf, "device-side wait timed out (code 0x%x)", plan.status);
    return fail(AM24_ERR_DEVICE_TIMEOUT, buf);
  }
  return AM24_OK;
}

am24_status am24_group_state(am24_group g, uint32_t problem, int32_t *stopped, uint32_t *steps) {
  AM24_TRY(check_slot(g, problem));
  uint32_t ctl[GCTL_WORDS];
  AM24_TRY(read_ctl(g, g->slots[problem], ctl));
  if (stopped) *stopped = ctl[CTL_STOP] ? 1 : 0;
  if (steps) *steps = ctl[CTL_STEPS];
  return AM24_OK;
}

am24_status am24_group_read(am24_group g, uint32_t problem, float *V, float *val, float *err,
                            uint32_t *nnz) {
  AM24_TRY(check_slot(g, problem));
  const GroupSlot &sl = g->slots[problem];
  const GProblem &P = sl.P;
  const cudaStream_t hs = g->h->stream;
  AM24_CUDA(cudaSetDevice(g->h->device));
  const int k = P.k;
  if (V) {
    AM24_CUDA(launch_masked_copy(P.Vx, P.vmask, P.ldn, P.n, k, P.Vraw, P.ldn, hs));
    AM24_CUDA(cudaMemcpy2DAsync(V, sizeof(float) * P.n, P.Vraw, sizeof(float) * P.ldn,
                                sizeof(float) * P.n, k, cudaMemcpyDeviceToHost, hs));
  }
  if (val) AM24_CUDA(cudaMemcpyAsync(val, P.val, sizeof(float) * k, cudaMemcpyDeviceToHost, hs));
  if (err) AM24_CUDA(cudaMemcpyAsync(err, P.err, sizeof(float) * k, cudaMemcpyDeviceToHost, hs));
  if (nnz) {
    if (is_constrained(P.formulation)) {
      AM24_CUDA(cudaMemcpyAsync(nnz, P.nnz, sizeof(uint32_t) * k, cudaMemcpyDeviceToHost, hs));
    } else {
      std::vector<float> np((size_t)k * P.parts);
      AM24_CUDA(cudaMemcpyAsync(np.data(), P.nnz_part, sizeof(float) * np.size(),
                                cudaMemcpyDeviceToHost, hs));
      AM24_CUDA(cudaStreamSynchronize(hs));
      for (int j = 0; j < k; j++) {
        double c = 0;
        for (int q = 0; q < P.parts; q++) c += np[(size_t)j * P.parts + q];
        nnz[j] = (uint32_t)c;
      }
    }
  }
  AM24_CUDA(cudaStreamSynchronize(hs));
  return AM24_OK;
}

am24_status am24_group_result(am24_group g, uint32_t problem, float *x, am24_statistics *stats) {
  AM24_TRY(check_slot(g, problem));
  if (!x) return fail(AM24_ERR_INVALID_ARG, "NULL x");
  const GroupSlot &sl = g->slots[problem];
  const GProblem &P = sl.P;
  am24_handle h = g->h;
  const cudaStream_t hs = h->stream;
  AM24_CUDA(cudaSetDevice(h->device));
  uint32_t ctl[GCTL_WORDS];
  AM24_TRY(read_ctl(g, sl, ctl));
  int dev_status = 0;
  AM24_CUDA(cudaMemcpy(&dev_status, P.status, sizeof(int), cudaMemcpyDeviceToHost));
  if (dev_status != 0) {
    char buf[96];
    snprintf(buf, sizeof buf, "device-side wait timed out (code 0x%x)", dev_status);
    return fail(AM24_ERR_DEVICE_TIMEOUT, buf);
  }
  const int k = P.k, n = P.n;
  std::vector<float> val(k);
  AM24_CUDA(cudaMemcpyAsync(val.data(), P.val, sizeof(float) * k, cudaMemcpyDeviceToHost, hs));
  AM24_CUDA(cudaStreamSynchronize(hs));
  // the reference's choice (sparse_PCA_solver.h:212-231): the first largest objective
  int sel = 0, degenerate = std::isnan(val[0]) ? 1 : 0;
  float bv = val[0];
  for (int i = 1; i < k; i++) {
    degenerate += std::isnan(val[i]) ? 1 : 0;
    if (val[i] > bv) {
      bv = val[i];
      sel = i;
    }
  }
  Allocs local(hs);
  float *xb = nullptr, *x_dev = nullptr;
  double *ev_rows = nullptr;
  AM24_TRY(local.get(&xb, n));
  AM24_TRY(local.get(&x_dev, n));
  AM24_TRY(local.get(&ev_rows, ev_partial_len(sl.mat->d)));
  AM24_CUDA(launch_masked_copy(P.Vx + (size_t)sel * P.ldn, P.vmask + (size_t)sel * (P.ldn / 32),
                               P.ldn, n, 1, xb, n, hs));
  AM24_CUDA(launch_finalize_x(xb, n, x_dev, hs));
  AM24_CUDA(launch_explained_variance(sl.mat->d, x_dev, ev_rows, h->ev_out, hs));
  double ev = 0.0;
  AM24_CUDA(cudaMemcpyAsync(x, x_dev, sizeof(float) * n, cudaMemcpyDeviceToHost, hs));
  AM24_CUDA(cudaMemcpyAsync(&ev, h->ev_out, sizeof(double), cudaMemcpyDeviceToHost, hs));
  AM24_CUDA(cudaStreamSynchronize(hs));
  if (stats) {
    std::memset(stats, 0, sizeof *stats);
    stats->it = ctl[CTL_STEPS];
    stats->fval = bv;
    float me;
    std::memcpy(&me, &ctl[CTL_MAX_ERR], sizeof me);
    stats->error = me;
    stats->total_true_computation_time = g->last_ms * 1e-3;
    stats->total_elapsed_time = g->last_ms * 1e-3;
    stats->n = (uint32_t)n;
    stats->total_threads_used = 1;
    stats->explained_variance = ev;
    stats->start_iterations = (uint64_t)ctl[CTL_STEPS] * (uint64_t)k;
    stats->degenerate_starts = degenerate;
    stats->low_precision_iterations = ctl[CTL_LOW_STEPS];
  }
  return AM24_OK;
}

am24_status am24_group_remove(am24_group g, uint32_t problem) {
  AM24_TRY(check_slot(g, problem));
  GroupSlot &sl = g->slots[problem];
  AM24_CUDA(cudaSetDevice(g->h->device));
  // the slot is dead for the next launch before its memory goes back to the pool
  const int zero = 0;
  AM24_CUDA(cudaMemcpyAsync(reinterpret_cast<char *>(g->dev.probs + problem) +
                                offsetof(GProblem, live),
                            &zero, sizeof zero, cudaMemcpyHostToDevice, g->h->stream));
  AM24_CUDA(cudaStreamSynchronize(g->h->stream));
  sl.mem.reset();
  sl = GroupSlot{};
  return upload_order(g);
}

}  // extern "C"

// ---- autotuner ------------------------------------------------------------
// The N tile of a problem's products and the split-K factor of its dense
// Z = B V are chosen by timing.  Problems fall into buckets of half an octave
// in each of m, n and k, per formulation mode (L2-variance constrained, L1
// variance, L2-variance penalized: their operand schemes and selects differ);
// the first problem of a bucket is timed in a scratch group of its own under
// each candidate (N tile 64, 128 or 256 where it covers the starts in at most
// eight tiles; the cost model's split-K, half of it and twice it), three steps
// from device-generated starts with the tolerance test off, and the fastest
// (the cost model's choice unless another is more than 2% faster) is kept in a
// process-wide table for every later problem of the bucket.  A problem's tiles
// are then a function of its bucket and the table alone, so problems stay the
// same bit for bit alone and among others for as long as the table holds.
namespace {

struct TuneKey {
  int mode, bm, bn, bk;
  bool operator<(const TuneKey &o) const {
    return std::tie(mode, bm, bn, bk) < std::tie(o.mode, o.bm, o.bn, o.bk);
  }
};
std::mutex g_tune_mu;
std::map<TuneKey, TileCfg> g_tune;

int half_octave(int v) { return (int)std::lround(2.0 * std::log2((double)std::max(v, 1))); }

TuneKey tune_key(const MatrixDev &M, const am24_settings &s) {
  const int f = s.formulation;
  return TuneKey{is_l1_variance(f) ? 1 : (is_constrained(f) ? 0 : 2), half_octave(M.m),
                 half_octave(M.n), half_octave(std::max(s.total_starts, 1))};
}

am24_status autotune(am24_group g, am24_matrix mat, const am24_settings &s0, TileCfg *out) {
  const MatrixDev &M = mat->d;
  am24_settings s = s0;
  AM24_TRY(am24_check_input(&s, (uint32_t)M.n));
  const TuneKey key = tune_key(M, s);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) {
      *out = it->second;
      return AM24_OK;
    }
  }
  const int k = s.total_starts;
  const int kb1 = (M.n + PAIR_BK_BF16 - 1) / PAIR_BK_BF16;
  const int m_tiles1 = (M.m + BM - 1) / BM;
  std::vector<TileCfg> cands;
  for (int bn : {64, 128, 256}) {
    if (bn != pick_bn(k) && ((k + bn - 1) / bn > 8 || bn >= 2 * k)) continue;
    int s_model = 1, kbps = 1;
    choose_splits(((m_tiles1 + 1) / 2) * ((k + bn - 1) / bn), kb1, std::max(1, num_sms() / 2),
                  &s_model, &kbps);
    for (int sp : {s_model, std::max(1, s_model / 2), std::min(kb1, 2 * s_model)}) {
      bool dup = false;
      for (const auto &c : cands) dup = dup || (c.bn == bn && c.splits == sp);
      if (!dup) cands.push_back(TileCfg{bn, sp});
    }
  }
  TileCfg best{pick_bn(k), 0};
  if (cands.size() > 1) {
    if (!g->tuner) AM24_TRY(am24_group_create(g->h, 1, &g->tuner));
    am24_settings t = s;
    t.start_mode = AM24_START_DEVICE_UNIFORM;
    t.tolerance = 0.0;
    t.max_iter = 3;
    t.precision = AM24_PRECISION_FP32;
    double best_ms = 1e300, model_ms = 1e300;
    for (size_t i = 0; i <= cands.size(); i++) {
      const TileCfg &c = cands[i == 0 ? 0 : i - 1];  // the first one twice: warm-up
      uint32_t slot = 0;
      AM24_TRY(group_add_impl(g->tuner, mat, &t, nullptr, c, &slot));
      float ms = 0.f;
      const am24_status st = am24_group_run(g->tuner, 0, &ms);
      am24_group_remove(g->tuner, slot);
      AM24_TRY(st);
      if (i == 0) continue;
      if (c.bn == pick_bn(k) && c.splits == cands[0].splits) model_ms = ms;
      if (ms < best_ms) {
        best_ms = ms;
        best = c;
      }
    }
    if (model_ms <= 1.02 * best_ms) best = cands[0];
  } else if (!cands.empty()) {
    best = cands[0];
  }
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[key] = best;
  *out = best;
  return AM24_OK;
}

}  // namespace

extern "C" {

am24_status am24_group_set_autotune(am24_group g, int32_t on) {
  if (!g) return fail(AM24_ERR_INVALID_ARG, "NULL group");
  g->autotune = on ? 1 : 0;
  return AM24_OK;
}

am24_status am24_autotune_save(const char *path) {
  if (!path) return fail(AM24_ERR_INVALID_ARG, "NULL path");
  FILE *f = fopen(path, "w");
  if (!f) return fail(AM24_ERR_INVALID_ARG, std::string("cannot write ") + path);
  std::lock_guard<std::mutex> lk(g_tune_mu);
  fprintf(f, "# am24 autotune: mode m n k (half-octave buckets) -> n_tile splitk\n");
  for (const auto &kv : g_tune)
    fprintf(f, "%d %d %d %d %d %d\n", kv.first.mode, kv.first.bm, kv.first.bn, kv.first.bk,
            kv.second.bn, kv.second.splits);
  fclose(f);
  return AM24_OK;
}

am24_status am24_autotune_load(const char *path) {
  if (!path) return fail(AM24_ERR_INVALID_ARG, "NULL path");
  FILE *f = fopen(path, "r");
  if (!f) return fail(AM24_ERR_INVALID_ARG, std::string("cannot read ") + path);
  char line[256];
  std::map<TuneKey, TileCfg> add;
  while (fgets(line, sizeof line, f)) {
    if (line[0] == '#') continue;
    TuneKey k{};
    TileCfg c{};
    if (sscanf(line, "%d %d %d %d %d %d", &k.mode, &k.bm, &k.bn, &k.bk, &c.bn, &c.splits) != 6)
      continue;
    if ((c.bn != 64 && c.bn != 128 && c.bn != 256) || c.splits < 0) {
      fclose(f);
      return fail(AM24_ERR_INVALID_ARG, std::string("bad autotune entry in ") + path);
    }
    add[k] = c;
  }
  fclose(f);
  std::lock_guard<std::mutex> lk(g_tune_mu);
  for (const auto &kv : add) g_tune[kv.first] = kv.second;
  return AM24_OK;
}

am24_status am24_autotune_clear(void) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune.clear();
  return AM24_OK;
}

}  // extern "C"
