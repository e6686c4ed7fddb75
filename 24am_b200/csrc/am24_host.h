// Host-side internals shared by the C ABI's translation units (am24_api.cu,
// am24_group.cu): the handle, matrix and batch objects, error reporting,
// stream-ordered allocation and the matrix-layout and tensor-map helpers.
// Not part of the public ABI.
#pragma once
#include <algorithm>
#include <string>
#include <vector>

#include <cudaTypedefs.h>

#include "am24.h"
#include "am24_internal.h"

namespace am24host {

using namespace am24;

// The last failure on the calling thread (am24_last_error).
extern thread_local std::string g_last_error;

inline am24_status fail(am24_status s, const std::string &msg) {
  g_last_error = msg;
  return s;
}

#define AM24_CUDA(expr)                                                                  \
  do {                                                                                   \
    cudaError_t e_ = (expr);                                                             \
    if (e_ != cudaSuccess) {                                                             \
      if (e_ == cudaErrorMemoryAllocation) {                                             \
        cudaGetLastError();                                                              \
        return fail(AM24_ERR_OOM, std::string(#expr) + ": " + cudaGetErrorString(e_));  \
      }                                                                                  \
      return fail(AM24_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_));   \
    }                                                                                    \
  } while (0)

#define AM24_TRY(expr)                   \
  do {                                   \
    am24_status s_ = (expr);             \
    if (s_ != AM24_OK) return s_;        \
  } while (0)

inline int round_up(int v, int a) { return (v + a - 1) / a * a; }

// Scoped device allocations of one object.  With a stream, stream-ordered
// (cudaMallocAsync / cudaFreeAsync on it, for memory only that stream uses):
// freeing then waits for no other stream, which matters when several handles
// work on one device at once.
struct Allocs {
  std::vector<void *> ptrs;
  cudaStream_t stream = nullptr;
  bool ordered = false;
  Allocs() = default;
  explicit Allocs(cudaStream_t st) : stream(st), ordered(true) {}
  ~Allocs() {
    for (void *p : ptrs) {
      if (ordered)
        cudaFreeAsync(p, stream);
      else
        cudaFree(p);
    }
  }
  template <typename T>
  am24_status get(T **out, size_t count) {
    void *p = nullptr;
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    cudaError_t e = ordered ? cudaMallocAsync(&p, bytes, stream) : cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(e == cudaErrorMemoryAllocation ? AM24_ERR_OOM : AM24_ERR_CUDA,
                  std::string("device allocation: ") + cudaGetErrorString(e));
    }
    ptrs.push_back(p);
    *out = static_cast<T *>(p);
    return AM24_OK;
  }
};

}  // namespace am24host

struct am24_handle_s {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t copy = nullptr;  // host-to-device copies that overlap work on `stream`
  // run-ahead batch loops: the stop word of each queued step lands in pinned
  // host memory, an event per slot
  static constexpr int AHEAD = 4;
  uint32_t *flags = nullptr;
  cudaEvent_t run_ev[AHEAD] = {};
  PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  am24host::Allocs scratch;  // small per-handle buffers
  double *ev_out = nullptr;
};

struct am24_matrix_s {
  am24::MatrixDev d{};  // sizes only (no layouts) when the matrix is sparse-resident
  am24host::Allocs mem;
  bool sparse = false;  // am24_matrix_create_csc_sparse_f32: kept compressed
  am24::SparseDev sp{};
  // sparse-resident deflations: host copies of what sp's device buffers hold
  std::vector<float> means_host;  // n, or empty
  std::vector<float> defl_host;   // comps x n
  std::vector<double> gram_host;  // SP_DEFL_MAX x SP_DEFL_MAX
  float *defl_dev = nullptr;
  double *gram_dev = nullptr, *defl_sum_dev = nullptr, *defl_mu_dev = nullptr;
};

struct am24_batch_s {
  am24::BatchDev d{};
  am24::TensorMaps tm{};
  am24_matrix mat = nullptr;
  am24_settings s{};
  int launches = 0;
  am24host::Allocs mem;
};


namespace am24host {

am24_status make_map(am24_handle h, CUtensorMap *map, const float *base, int K, int rows, int ld,
                     int box_rows, int bk);
am24_status make_map_bf16(am24_handle h, CUtensorMap *map, const uint16_t *base, int K, int rows,
                          int ld, int box_rows, bool fp16 = false);
am24_status ensure_bf16_planes(am24_handle h, am24_matrix mat, int planes);
am24_status ensure_tf32_planes(am24_handle h, am24_matrix mat);
am24_status ensure_fp16_planes(am24_handle h, am24_matrix mat);
am24_status ensure_bt_fp16_planes(am24_handle h, am24_matrix mat);
void choose_splits(int tiles, int kb_total, int sms, int *splits, int *kbps);
am24_status validate_settings(const am24_settings *s);
// The phase word a MIXED batch or problem starts in (lead_iterations > 0: the FP32 lead-in).
uint32_t mixed_first_phase(uint32_t lead);
// The kernels' parameters of step `it` of a batch whose first global start is `shift`.
StepParams step_params(const am24_settings &s, int it, int shift);
// Host check of compressed sparse columns (col_ptr n + 1 entries from 0,
// non-decreasing; row indices in [0, m)); the shared rule of both CSC entry points.
am24_status validate_csc(const float *vals, const int32_t *row_ind, const int32_t *col_ptr,
                         uint32_t m, uint32_t n);
// am24_matrix_deflate on a sparse-resident matrix: records x as the next factor
// (I - x x^T) of B's deflation.
am24_status deflate_sparse(am24_handle h, am24_matrix mat, const float *x, int32_t on_device);
// am24_solve_resident_f32 on a sparse-resident matrix (settings already checked).
am24_status solve_sparse(am24_handle h, am24_matrix mat, float *x, am24_settings &s,
                         am24_statistics *stats, const float *start_points, float *fval_out);
void reference_start(float *x, unsigned n, bool constrained, unsigned s, unsigned g);
void host_starts(const am24_settings &s, unsigned n, const float *start_points,
                 const unsigned *global_idx, int cols, std::vector<float> &out);

// Device bytes one problem of a group allocates (am24_group_add).
uint64_t group_problem_bytes(int m, int n, int k, int formulation, bool mixed);
// Every slot's state after the last step (0 free, 1 iterating, 2 stopped);
// synchronizes the group's stream.
am24_status group_done_flags(am24_group g, std::vector<uint32_t> &out);

}  // namespace am24host
