// The serving layer (am24_server_*, am24_submit / am24_poll / am24_wait):
// resident matrices under an HBM budget and continuous batching of solve
// requests on one grouped engine.
//
// One engine thread owns a handle and a group (am24_group_*).  It loops:
//   1. admit queued requests, oldest first, into free slots of the group while
//      the budget left beside the resident matrices and the requests already
//      admitted holds their device memory;
//   2. run up to SERVE_CHUNK grouped steps of every admitted request (one
//      graph launch; requests at different iterations step together);
//   3. finish the requests whose problem stopped: their best start, x, FP64
//      explained variance and statistics, then their slot and memory go back.
// So a request that arrives while others are on the device joins them at the
// next step boundary (at most SERVE_CHUNK steps later), and leaves as soon as
// its own batch loop ends.  Each request is its own problem of the group: its
// own batch of all its starts, stopping on its own largest change as the
// reference's batch loop does (c++/src/gpower/sparse_PCA_solver.h:192-212),
// with tiles and reduction order of its own, so its result is the same bit
// for bit whatever else is served beside it.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "am24.h"
#include "am24_host.h"
#include "am24_internal.h"

using namespace am24;
using namespace am24host;

namespace {

constexpr uint32_t SERVE_SLOTS = 1024;  // problems on the device at once
constexpr uint32_t SERVE_CHUNK = AM24_SERVER_CHUNK;  // grouped steps between admissions
constexpr uint32_t SERVE_MAX_STARTS = 8192;

struct ServeRequest {
  uint64_t ticket = 0;
  uint32_t matrix_id = 0;
  am24_settings s{};          // after am24_check_input, one batch of all starts
  std::vector<float> starts;  // n x total_starts (injected starts only)
  std::chrono::steady_clock::time_point submitted, admitted;
  uint64_t bytes = 0;
  uint32_t n = 0;  // the matrix's features (length of x)
  uint32_t slot = 0;
  bool done = false;
  am24_status status = AM24_OK;
  std::string error;
  std::vector<float> x;
  am24_statistics stats{};
};
using RequestPtr = std::shared_ptr<ServeRequest>;

// Device bytes of a matrix's layouts: FP32 B and the two FP16 planes of B and
// of B^T with their scales, all made when the matrix is added.
uint64_t matrix_bytes(uint32_t m, uint32_t n) {
  const uint64_t ldm = (m + 31) / 32 * 32, ldn = (n + 31) / 32 * 32;
  return 4ull * n * ldm + 2ull * 2 * n * ldm + 4ull * n + 2ull * 2 * m * ldn + 4ull * m +
         4ull * m;
}

}  // namespace

struct am24_server_s {
  am24_handle h = nullptr;         // the engine's handle (its stream runs the group)
  am24_handle upload_h = nullptr;  // matrix uploads from callers' threads
  am24_group g = nullptr;
  std::thread engine;
  std::mutex upload_mu;
  uint64_t budget = 0;
  std::mutex mu;  // everything below
  std::condition_variable cv_work, cv_done;
  struct Resident {
    am24_matrix mat;
    uint64_t bytes;
    uint32_t m, n;
    int pending;
  };
  std::map<uint32_t, Resident> matrices;
  uint64_t resident = 0;
  uint64_t inflight = 0;  // device bytes of the admitted requests
  uint32_t next_matrix = 1;
  uint64_t next_ticket = 1;
  std::deque<RequestPtr> queue;
  std::map<uint64_t, RequestPtr> tickets;
  bool stop = false;
  std::string stop_reason;  // why the engine stopped before destroy, for callers
};

namespace {

// Completes a request (engine thread): releases its budget and wakes waiters.
void complete(am24_server s, const RequestPtr &r, am24_status st, const std::string &err) {
  const auto now = std::chrono::steady_clock::now();
  std::lock_guard<std::mutex> lk(s->mu);
  r->status = st;
  r->error = err;
  r->stats.total_elapsed_time = std::chrono::duration<double>(now - r->submitted).count();
  r->done = true;
  s->inflight -= r->bytes;
  s->matrices.at(r->matrix_id).pending--;
  s->cv_done.notify_all();
}

void engine_loop(am24_server s) {
  cudaSetDevice(s->h->device);
  std::vector<RequestPtr> running(SERVE_SLOTS);
  uint32_t nrunning = 0;
  std::vector<uint32_t> flags;
  for (;;) {
    // 1. admission, oldest first, while slots and budget last
    std::vector<RequestPtr> admit;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      if (nrunning == 0)
        s->cv_work.wait(lk, [&] { return s->stop || !s->queue.empty(); });
      if (s->stop && s->queue.empty() && nrunning == 0) return;
      uint32_t free_slots = SERVE_SLOTS - nrunning;
      while (!s->queue.empty() && admit.size() < free_slots) {
        const RequestPtr &r = s->queue.front();
        const uint64_t used = s->resident + s->inflight;
        if (used + r->bytes > s->budget) break;  // waits for memory to come back
        s->inflight += r->bytes;
        admit.push_back(r);
        s->queue.pop_front();
      }
    }
    for (auto &r : admit) {
      am24_matrix mat;
      {
        std::lock_guard<std::mutex> lk(s->mu);
        mat = s->matrices.at(r->matrix_id).mat;
      }
      uint32_t slot = 0;
      const am24_status st = am24_group_add(s->g, mat, &r->s,
                                            r->starts.empty() ? nullptr : r->starts.data(), &slot);
      if (st != AM24_OK) {
        complete(s, r, st, g_last_error);
        continue;
      }
      r->slot = slot;
      r->admitted = std::chrono::steady_clock::now();
      r->starts.clear();
      r->starts.shrink_to_fit();
      running[slot] = r;
      nrunning++;
    }
    if (nrunning == 0) continue;
    // 2. a chunk of grouped steps
    float ms = 0.f;
    am24_status st = am24_group_run(s->g, SERVE_CHUNK, &ms);
    if (st == AM24_OK) st = group_done_flags(s->g, flags);
    if (st != AM24_OK) {
      // a failed run leaves the group's state unknown: fail what it held and
      // start a fresh group
      const std::string err = g_last_error;
      for (uint32_t i = 0; i < SERVE_SLOTS; i++)
        if (running[i]) {
          complete(s, running[i], st, err);
          running[i].reset();
        }
      nrunning = 0;
      am24_group_destroy(s->g);
      s->g = nullptr;
      if (am24_group_create(s->h, SERVE_SLOTS, &s->g) != AM24_OK) {
        const std::string create_err = g_last_error;
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;  // cannot serve any more: drain the queue with errors
        s->stop_reason = "a grouped run failed (" + err +
                         ") and the engine could not be restarted (" + create_err + ")";
        for (auto &r : s->queue) {
          r->status = AM24_ERR_CUDA;
          r->error = s->stop_reason;
          r->done = true;
          s->matrices.at(r->matrix_id).pending--;
        }
        s->queue.clear();
        s->cv_done.notify_all();
        return;
      }
      continue;
    }
    // 3. finished requests
    for (uint32_t i = 0; i < SERVE_SLOTS; i++) {
      if (!running[i] || flags[i] != 2u) continue;
      RequestPtr r = running[i];
      running[i].reset();
      nrunning--;
      r->x.assign(r->n, 0.f);
      am24_statistics stats{};
      am24_status rs = am24_group_result(s->g, i, r->x.data(), &stats);
      const std::string err = rs == AM24_OK ? std::string() : g_last_error;
      am24_group_remove(s->g, i);
      stats.total_true_computation_time =
          std::chrono::duration<double>(std::chrono::steady_clock::now() - r->admitted).count();
      r->stats = stats;
      complete(s, r, rs, err);
    }
  }
}

am24_status finish_ticket(am24_server s, const RequestPtr &r, float *x, am24_statistics *stats) {
  // caller holds s->mu; the request is done
  if (x && !r->x.empty()) std::memcpy(x, r->x.data(), sizeof(float) * r->x.size());
  if (stats) *stats = r->stats;
  s->tickets.erase(r->ticket);
  if (r->status != AM24_OK) return fail(r->status, r->error);
  return AM24_OK;
}

}  // namespace

extern "C" {

am24_status am24_server_create(int device, uint64_t hbm_budget_bytes, am24_server *out) {
  if (!out) return fail(AM24_ERR_INVALID_ARG, "NULL argument");
  *out = nullptr;
  std::unique_ptr<am24_server_s> s(new am24_server_s());
  s->budget = hbm_budget_bytes;
  am24_status st = am24_create(&s->upload_h, device);
  if (st == AM24_OK) st = am24_create(&s->h, device);
  if (st == AM24_OK) st = am24_group_create(s->h, SERVE_SLOTS, &s->g);
  if (st != AM24_OK) {
    if (s->g) am24_group_destroy(s->g);
    if (s->h) am24_destroy(s->h);
    if (s->upload_h) am24_destroy(s->upload_h);
    return st;
  }
  am24_server_s *raw = s.release();
  raw->engine = std::thread(engine_loop, raw);
  *out = raw;
  return AM24_OK;
}

am24_status am24_server_destroy(am24_server s) {
  if (!s) return AM24_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->engine.joinable()) s->engine.join();
  if (s->g) am24_group_destroy(s->g);
  for (auto &kv : s->matrices) am24_matrix_destroy(s->upload_h, kv.second.mat);
  am24_destroy(s->h);
  am24_destroy(s->upload_h);
  delete s;
  return AM24_OK;
}

am24_status am24_server_add_matrix_f32(am24_server s, const float *B, int32_t ldB, uint32_t m,
                                       uint32_t n, int32_t on_device, uint32_t *matrix_id) {
  if (!s || !B || !matrix_id) return fail(AM24_ERR_INVALID_ARG, "NULL argument");
  const uint64_t bytes = matrix_bytes(m, n);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->resident + bytes > s->budget)
      return fail(AM24_ERR_ADMISSION_REJECTED,
                  "matrix needs " + std::to_string(bytes) + " bytes, " +
                      std::to_string(s->budget - std::min(s->budget, s->resident)) +
                      " left in the budget");
    s->resident += bytes;  // reserved while uploading
  }
  am24_matrix mat = nullptr;
  am24_status st;
  {
    // the matrix and every layout a request may read, made before any
    // request can name it
    std::lock_guard<std::mutex> lk(s->upload_mu);
    st = am24_matrix_create_f32(s->upload_h, B, ldB, m, n, on_device, &mat);
    if (st == AM24_OK) st = ensure_fp16_planes(s->upload_h, mat);
    if (st == AM24_OK) st = ensure_bt_fp16_planes(s->upload_h, mat);
    if (st != AM24_OK && mat) {
      const std::string err = g_last_error;
      am24_matrix_destroy(s->upload_h, mat);
      g_last_error = err;
    }
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (st != AM24_OK) {
    s->resident -= bytes;
    return st;
  }
  const uint32_t id = s->next_matrix++;
  s->matrices[id] = am24_server_s::Resident{mat, bytes, m, n, 0};
  *matrix_id = id;
  return AM24_OK;
}

am24_status am24_server_remove_matrix(am24_server s, uint32_t matrix_id) {
  if (!s) return fail(AM24_ERR_INVALID_ARG, "NULL argument");
  am24_matrix mat = nullptr;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->matrices.find(matrix_id);
    if (it == s->matrices.end()) return fail(AM24_ERR_INVALID_ARG, "unknown matrix id");
    if (it->second.pending > 0)
      return fail(AM24_ERR_INVALID_ARG, "requests for this matrix are pending");
    mat = it->second.mat;
    s->resident -= it->second.bytes;
    s->matrices.erase(it);
  }
  std::lock_guard<std::mutex> lk(s->upload_mu);
  return am24_matrix_destroy(s->upload_h, mat);
}

am24_status am24_submit(am24_server s, uint32_t matrix_id, const am24_settings *settings,
                        const float *start_points, uint64_t *ticket) {
  if (!s || !settings || !ticket) return fail(AM24_ERR_INVALID_ARG, "NULL argument");
  AM24_TRY(validate_settings(settings));
  if (settings->use_otf || settings->store_all)
    return fail(AM24_ERR_INVALID_ARG, "the server supports neither use_otf nor store_all");
  if (settings->start_mode == AM24_START_INJECTED && !start_points)
    return fail(AM24_ERR_INVALID_ARG, "start_mode INJECTED needs start_points");
  auto r = std::make_shared<ServeRequest>();
  r->s = *settings;
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop)
    return fail(AM24_ERR_CUDA, "the server has stopped" +
                                   (s->stop_reason.empty() ? std::string()
                                                           : ": " + s->stop_reason));
  auto it = s->matrices.find(matrix_id);
  if (it == s->matrices.end()) return fail(AM24_ERR_INVALID_ARG, "unknown matrix id");
  const uint32_t n = it->second.n, m = it->second.m;
  AM24_TRY(am24_check_input(&r->s, n));
  r->s.batch_size = r->s.total_starts;
  r->s.total_batches = 1;
  if ((uint32_t)r->s.total_starts > SERVE_MAX_STARTS)
    return fail(AM24_ERR_ADMISSION_REJECTED, "more starts than the server's largest request");
  r->bytes = group_problem_bytes((int)m, (int)n, r->s.total_starts, r->s.formulation,
                                 r->s.precision == AM24_PRECISION_MIXED);
  if (s->resident + r->bytes > s->budget)
    return fail(AM24_ERR_ADMISSION_REJECTED, "the request does not fit the budget");
  if (r->s.start_mode == AM24_START_INJECTED)
    r->starts.assign(start_points, start_points + (size_t)n * r->s.total_starts);
  r->matrix_id = matrix_id;
  r->n = n;
  r->ticket = s->next_ticket++;
  r->submitted = std::chrono::steady_clock::now();
  it->second.pending++;
  s->tickets[r->ticket] = r;
  s->queue.push_back(r);
  *ticket = r->ticket;
  s->cv_work.notify_one();
  return AM24_OK;
}

am24_status am24_poll(am24_server s, uint64_t ticket, float *x, am24_statistics *stats,
                      int32_t *done) {
  if (!s || !done) return fail(AM24_ERR_INVALID_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return fail(AM24_ERR_INVALID_ARG, "unknown ticket");
  *done = it->second->done ? 1 : 0;
  if (!*done) return AM24_OK;
  return finish_ticket(s, it->second, x, stats);
}

am24_status am24_wait(am24_server s, uint64_t ticket, float *x, am24_statistics *stats) {
  if (!s) return fail(AM24_ERR_INVALID_ARG, "NULL argument");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return fail(AM24_ERR_INVALID_ARG, "unknown ticket");
  RequestPtr r = it->second;
  s->cv_done.wait(lk, [&] { return r->done; });
  return finish_ticket(s, r, x, stats);
}

}  // extern "C"
