// Kernels of the sparse-resident AM step (included by am24_kernels.cu).
//
// The data matrix stays in compressed form on the device, as the reference's
// sparse solver keeps it (sparse_PCA_solver_CSC,
// c++/src/gpower/sparse_PCA_solver_for_CSC.h:111-508): CSC for V = B^T Z and
// CSR for Z = B V, with its implicit centring (doMean / doRowMean, :223-248,
// :277-309) folded into the products' epilogues as rank-one corrections:
//   Z = (B - 1 mu^T - r 1^T) V = B V - 1 (mu^T V) - r (1^T V)
//   V = (B - 1 mu^T - r 1^T)^T Z = B^T Z - mu (1^T Z) - 1 (r^T Z).
// Both products are the same tile kernel: for a compressed structure with
// `ncols` outer entries (CSR rows or CSC columns), out[j][c] = sum over the
// entries e of outer entry c of val[e] * X[idx[e]][j], X row-major with one
// row of kp floats per inner index (the starts side by side), out start-major.
// The per-column passes around them (selects, finalize) are the dense path's.

constexpr int SP_TILE = 32;        // outer entries x starts per tile
constexpr int SP_THREADS = 256;    // 8 warps, 4 outer entries each

// sum over entries e in [e0, e1) of val[e] * X[idx[e] * kp + j], in entry
// order with FP32 FMAs, for the lane's start j.  The warp loads 32 (index,
// value) pairs at once, one per lane, and broadcasts them, so the X loads of
// consecutive entries do not wait on one another.
__device__ __forceinline__ float sp_dot(const int32_t *__restrict__ idx,
                                        const float *__restrict__ val,
                                        const float *__restrict__ X, int kp, int j, int e0,
                                        int e1) {
  const int lane = threadIdx.x & 31;
  float acc = 0.f;
  for (int base = e0; base < e1; base += 32) {
    const int e = base + lane;
    int ii = 0;
    float vv = 0.f;
    if (e < e1) {
      ii = idx[e];
      vv = val[e];
    }
    const int cnt = min(32, e1 - base);
#pragma unroll 8
    for (int t = 0; t < cnt; t++) {
      const int i = __shfl_sync(0xFFFFFFFFu, ii, t);
      const float v = __shfl_sync(0xFFFFFFFFu, vv, t);
      acc = fmaf(v, X[(size_t)i * kp + j], acc);
    }
  }
  return acc;
}

// The rank-one centring of one output: acc - (cvec ? cvec[c] a[j] : 0) - (b ? b[j] : 0) in FP64.
__device__ __forceinline__ float sp_correct(float acc, int c, int j, const float *cvec,
                                            const double *a, const double *b) {
  if (!cvec && !b) return acc;
  double corr = 0.0;
  if (cvec) corr += (double)cvec[c] * a[j];
  if (b) corr += b[j];
  return (float)((double)acc - corr);
}

// out[j][c] (j < k, c < ncols) = sum_e val[e] X[idx[e] * kp + j]
//                                - (cvec ? cvec[c] * a[j] : 0) - (b ? b[j] : 0)
// One warp per outer entry, a lane per start: every entry reads one 128-byte
// row segment of X.  Each sum runs over the outer entry's entries in storage
// order with FP32 FMAs (deterministic); the correction is applied in FP64.
// Outer entries longer than SP_LONG are left to sp_spmm_seg_kernel and
// sp_spmm_long_kernel.
__global__ void __launch_bounds__(SP_THREADS) sp_spmm_kernel(
    const int32_t *__restrict__ ptr, const int32_t *__restrict__ idx,
    const float *__restrict__ val, int ncols, const float *__restrict__ X, int kp, int k,
    float *__restrict__ out, int ld_out, const float *__restrict__ cvec,
    const double *__restrict__ a, const double *__restrict__ b, const uint32_t *stop,
    const uint32_t *gate, uint32_t gate_min) {
  if (*stop || (gate && *gate < gate_min)) return;
  __shared__ float tile[SP_TILE][SP_TILE + 1];
  __shared__ int skip[SP_TILE];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int c0 = blockIdx.x * SP_TILE, j0 = blockIdx.y * SP_TILE;
  const int j = j0 + lane;  // < kp always (kp is a multiple of 32)
  for (int r = warp; r < SP_TILE; r += SP_THREADS / 32) {
    const int c = c0 + r;
    float acc = 0.f;
    bool own = false;
    if (c < ncols) {
      const int e0 = ptr[c], e1 = ptr[c + 1];
      own = e1 - e0 <= SP_LONG;
      if (own) {
        acc = sp_dot(idx, val, X, kp, j, e0, e1);
        if (j < k) acc = sp_correct(acc, c, j, cvec, a, b);
      }
    }
    tile[lane][r] = acc;
    if (lane == 0) skip[r] = !own;
  }
  __syncthreads();
  for (int r = warp; r < SP_TILE; r += SP_THREADS / 32) {
    const int jj = j0 + r, c = c0 + lane;
    if (jj < k && c < ncols && !skip[lane]) out[(size_t)jj * ld_out + c] = tile[r][lane];
  }
}

// Z = (B - centring) V once V is sparse (when sp_zgate_kernel chose this path:
// *gate <= cap), one block per start: the
// start's support listed in index order in shared memory, then z = sum over
// the support of v_q B[:, q], one CSC column at a time (its rows are distinct,
// so its entries add in parallel), and the centring as the CSR product applies
// it.  Row i's sum runs over the same columns in the same order as in the CSR
// product (whose other terms multiply v = 0), so the result is the same bit
// for bit (rows the CSR product sums in segments aside), at the cost of the
// support's entries instead of every row's.
constexpr int SP_SCATTER_CAP = 1024;
__global__ void __launch_bounds__(SP_THREADS) sp_scatter_z_kernel(
    const int32_t *__restrict__ col_ptr, const int32_t *__restrict__ row_ind,
    const float *__restrict__ cvals, const float *__restrict__ Vx,
    const uint32_t *__restrict__ vmask, int ldn, float *__restrict__ Zs, int ldm, int m,
    const float *__restrict__ row_means, const double *__restrict__ sum_v,
    const double *__restrict__ dot_mu, const uint32_t *gate, uint32_t cap, const uint32_t *stop) {
  if (*stop || *gate > cap) return;
  __shared__ int32_t list[SP_SCATTER_CAP];
  __shared__ uint32_t wsum[SP_THREADS / 32];
  const int j = blockIdx.x;
  const int words = ldn >> 5;
  const uint32_t *mk = vmask + (size_t)j * words;
  float *z = Zs + (size_t)j * ldm;
  for (int i = threadIdx.x; i < m; i += SP_THREADS) z[i] = 0.f;
  // the support in index order: a pass of SP_THREADS words at a time, each
  // thread's word expanded at its block-wide prefix of set bits
  int count = 0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int w0 = 0; w0 < words; w0 += SP_THREADS) {
    const int w = w0 + threadIdx.x;
    const uint32_t bits = w < words ? mk[w] : 0u;
    const uint32_t c = __popc(bits);
    uint32_t incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    uint32_t before = 0, total = 0;
    for (int x = 0; x < SP_THREADS / 32; x++) {
      if (x < warp) before += wsum[x];
      total += wsum[x];
    }
    uint32_t at = count + before + incl - c;
    for (uint32_t b = bits; b; b &= b - 1u) {
      if (at < (uint32_t)SP_SCATTER_CAP) list[at] = (w << 5) + (__ffs(b) - 1);
      at++;
    }
    count += (int)total;
    __syncthreads();
  }
  auto add_column = [&](int q) {
    const float v = Vx[(size_t)j * ldn + q];
    for (int e = col_ptr[q] + threadIdx.x; e < col_ptr[q + 1]; e += SP_THREADS) {
      const int i = row_ind[e];
      z[i] = fmaf(cvals[e], v, z[i]);
    }
    __syncthreads();
  };
  if (count <= SP_SCATTER_CAP) {
    for (int t = 0; t < count; t++) add_column(list[t]);
  } else {
    // more loadings than the list holds (the gate's count is the finalize
    // pass's, so this is not expected): the same order, read from the mask
    for (int w = 0; w < words; w++)
      for (uint32_t b = mk[w]; b; b &= b - 1u) add_column((w << 5) + (__ffs(b) - 1));
  }
  if (row_means || dot_mu) {
    for (int i = threadIdx.x; i < m; i += SP_THREADS)
      z[i] = sp_correct(z[i], i, j, row_means, sum_v, dot_mu);
  }
}

// Long outer entries, step 1: one warp per (segment, 32 starts), the
// segment's sum into part[s][j].
__global__ void __launch_bounds__(SP_THREADS) sp_spmm_seg_kernel(
    const int32_t *__restrict__ seg_e0, const int32_t *__restrict__ seg_e1, int segs,
    const int32_t *__restrict__ idx, const float *__restrict__ val,
    const float *__restrict__ X, int kp, float *__restrict__ part, const uint32_t *stop,
    const uint32_t *gate, uint32_t gate_min) {
  if (*stop || (gate && *gate < gate_min)) return;
  const int s = blockIdx.x * (SP_THREADS / 32) + (threadIdx.x >> 5);
  const int j = blockIdx.y * SP_TILE + (threadIdx.x & 31);
  if (s >= segs) return;  // whole warps leave together
  part[(size_t)s * kp + j] = sp_dot(idx, val, X, kp, j, seg_e0[s], seg_e1[s]);
}

// Long outer entries, step 2: per (entry, start) the segments' sums in
// segment order, then the centring, into out[j][c].
__global__ void __launch_bounds__(SP_TILE) sp_spmm_long_kernel(
    const int32_t *__restrict__ outer, const int32_t *__restrict__ seg_first,
    const float *__restrict__ part, int kp, int k, float *__restrict__ out, int ld_out,
    const float *__restrict__ cvec, const double *__restrict__ a, const double *__restrict__ b,
    const uint32_t *stop, const uint32_t *gate, uint32_t gate_min) {
  if (*stop || (gate && *gate < gate_min)) return;
  const int x = blockIdx.x;
  const int j = blockIdx.y * SP_TILE + threadIdx.x;
  if (j >= k) return;
  const int c = outer[x];
  float acc = 0.f;
  for (int s = seg_first[x]; s < seg_first[x + 1]; s++) acc += part[(size_t)s * kp + j];
  out[(size_t)j * ld_out + c] = sp_correct(acc, c, j, cvec, a, b);
}

// Vt[q][j] = V's column j at row q (zero where its mask bit is clear), for
// q < n, j < kp (columns k..kp-1 zero): the row-major X of Z = B V (dense
// steps only: *gate >= gate_min).
// With deflations (comps > 0) the column is the projected one,
// v - sum_c a[j][c] x_c (sp_defl_coef_kernel's coefficients).
__global__ void __launch_bounds__(SP_THREADS) sp_transpose_v_kernel(
    const float *__restrict__ Vx, const uint32_t *__restrict__ mask, int ldn, int n, int k,
    float *__restrict__ Vt, int kp, const uint32_t *stop, const uint32_t *gate,
    uint32_t gate_min, const float *__restrict__ defl, int comps,
    const double *__restrict__ defl_a) {
  if (*stop || *gate < gate_min) return;
  __shared__ float tile[SP_TILE][SP_TILE + 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int q0 = blockIdx.x * SP_TILE, j0 = blockIdx.y * SP_TILE;
  const int words = ldn >> 5;
  for (int r = warp; r < SP_TILE; r += SP_THREADS / 32) {
    const int j = j0 + r, q = q0 + lane;
    float v = 0.f;
    if (j < k && q < n) {
      const uint32_t w = mask[(size_t)j * words + (q >> 5)];
      if ((w >> (q & 31)) & 1u) v = Vx[(size_t)j * ldn + q];
      if (comps > 0) {
        double d = (double)v;
        for (int c = 0; c < comps; c++)
          d -= defl_a[(size_t)j * SP_DEFL_MAX + c] * (double)defl[(size_t)c * n + q];
        v = (float)d;
      }
    }
    tile[r][lane] = v;
  }
  __syncthreads();
  for (int r = warp; r < SP_TILE; r += SP_THREADS / 32) {
    const int q = q0 + r;
    if (q < n) Vt[(size_t)q * kp + j0 + lane] = tile[lane][r];
  }
}

// Zt[i][j] = Zs[j][i] for i < m, j < kp (columns k..kp-1 zero): the row-major
// X of V = B^T Z.
__global__ void __launch_bounds__(SP_THREADS) sp_transpose_z_kernel(
    const float *__restrict__ Zs, int ldm, int m, int k, float *__restrict__ Zt, int kp,
    const uint32_t *stop) {
  if (*stop) return;
  __shared__ float tile[SP_TILE][SP_TILE + 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int i0 = blockIdx.x * SP_TILE, j0 = blockIdx.y * SP_TILE;
  for (int r = warp; r < SP_TILE; r += SP_THREADS / 32) {
    const int j = j0 + r, i = i0 + lane;
    tile[r][lane] = (j < k && i < m) ? Zs[(size_t)j * ldm + i] : 0.f;
  }
  __syncthreads();
  for (int r = warp; r < SP_TILE; r += SP_THREADS / 32) {
    const int i = i0 + r;
    if (i < m) Zt[(size_t)i * kp + j0 + lane] = tile[lane][r];
  }
}

// Fixed-order block sum of one double per thread (SP_THREADS threads).
__device__ __forceinline__ double sp_block_sum(double v, double *red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
#pragma unroll
  for (int w = 0; w < SP_THREADS / 32; w++) t += red[w];
  __syncthreads();
  return t;
}

// Per start j (one block): sum_v[j] = sum_q v_q and dot_mu[j] = sum_q mu_q v_q
// over V's defined entries, in FP64 (the rank-one corrections of Z = B V, when
// sum_v is not null), and the number of matrix entries in the start's support
// columns, added to *work (what a scatter of the support would touch).
__global__ void __launch_bounds__(SP_THREADS) sp_vstats_kernel(
    const float *__restrict__ Vx, const uint32_t *__restrict__ mask, int ldn, int n,
    const float *__restrict__ means, double *__restrict__ sum_v, double *__restrict__ dot_mu,
    const int32_t *__restrict__ col_ptr, unsigned long long *work, const uint32_t *stop) {
  if (*stop) return;
  __shared__ double red[SP_THREADS / 32];
  const int j = blockIdx.x;
  const int words = ldn >> 5;
  double s = 0.0, d = 0.0, entries = 0.0;
  for (int q = threadIdx.x; q < n; q += SP_THREADS) {
    const uint32_t w = mask[(size_t)j * words + (q >> 5)];
    if ((w >> (q & 31)) & 1u) {
      const double v = (double)Vx[(size_t)j * ldn + q];
      s += v;
      if (means) d += (double)means[q] * v;
      entries += (double)(col_ptr[q + 1] - col_ptr[q]);
    }
  }
  entries = sp_block_sum(entries, red);
  if (sum_v) {
    s = sp_block_sum(s, red);
    d = sp_block_sum(d, red);
  }
  if (threadIdx.x == 0) {
    if (sum_v) {
      sum_v[j] = s;
      dot_mu[j] = d;
    }
    atomicAdd(work, (unsigned long long)entries);
  }
}

// The path of this step's Z = B V, into *zgate: 0 the scatter of each
// support, 1 the CSR product.  The scatter needs every start's support
// within its list (the previous step's largest count, *max_nnz, at most cap)
// and must touch fewer matrix entries (*work over all starts) than csr_steps:
// SP_SCATTER_PER_STEP times the steps of the CSR product's warps (nnz x k / 32,
// one 32-start row segment per entry and chunk of starts).  A scattered entry
// (a coalesced read of its row and value, one update of a z row that stays in
// cache) costs about a quarter of such a warp step: measured on B200 with
// 1024 starts, a support work of 1.4x the warp steps ran faster scattered
// (6.5 against 9.3 ms per step), while a corpus whose supports hold its most
// common terms (an estimated 5x) ran slower (26.9 against 24.0).
constexpr double SP_SCATTER_PER_STEP = 4.0;
__global__ void sp_zgate_kernel(const uint32_t *max_nnz, uint32_t cap,
                                const unsigned long long *work, double csr_steps,
                                uint32_t *zgate, const uint32_t *stop) {
  if (*stop) return;
  *zgate = (*max_nnz <= cap && (double)*work < csr_steps) ? 0u : 1u;
}

// Per start j (one block), on z = Zs[j] after the centred product:
//   constrained L2 variance (forms 0, 2): fz = ||z||_2, z kept;
//   constrained L1 variance (1, 3): fz = ||z||_1, z <- sgn z;
//   penalized L2 variance (4, 6): z <- z / ||z||_2;
//   penalized L1 variance (5, 7): z <- sgn z
// (gpower_commons.h:68-177 as the dense path runs it), then, when the matrix
// is centred, zsum[j] = sum_i z_i and zdot[j] = sum_i r_i z_i of the result
// (the corrections of V = B^T Z).  Norms and sums in FP64, fixed order.
__global__ void __launch_bounds__(SP_THREADS) sp_zreduce_kernel(
    float *__restrict__ Zs, int ldm, int m, int formulation, float *__restrict__ fz,
    const float *__restrict__ row_means, double *__restrict__ zsum, double *__restrict__ zdot,
    const uint32_t *stop) {
  if (*stop) return;
  __shared__ double red[SP_THREADS / 32];
  const int j = blockIdx.x;
  float *z = Zs + (size_t)j * ldm;
  const bool l1var = formulation == 1 || formulation == 3 || formulation == 5 || formulation == 7;
  const bool cons = formulation <= 3;
  float inv = 1.f;
  if (cons || !l1var) {
    double t = 0.0;
    for (int i = threadIdx.x; i < m; i += SP_THREADS) {
      const double v = (double)z[i];
      t += l1var ? fabs(v) : v * v;
    }
    t = sp_block_sum(t, red);
    if (cons && threadIdx.x == 0) fz[j] = l1var ? (float)t : (float)sqrt(t);
    if (!cons) inv = 1.0f / (float)sqrt(t);
  }
  double s = 0.0, d = 0.0;
  for (int i = threadIdx.x; i < m; i += SP_THREADS) {
    float v = z[i];
    if (l1var)
      v = (float)((v > 0.f) - (v < 0.f));
    else if (!cons)
      v *= inv;
    if (l1var || !cons) z[i] = v;
    if (zsum) {
      s += (double)v;
      if (row_means) d += (double)row_means[i] * (double)v;
    }
  }
  if (zsum) {
    s = sp_block_sum(s, red);
    d = sp_block_sum(d, red);
    if (threadIdx.x == 0) {
      zsum[j] = s;
      zdot[j] = d;
    }
  }
}

// Penalized thresholds on raw V (sparse_PCA_thresholding.h:26-102), per start
// j (one block): L1 (forms 6, 7) x = sgn(v)(|v| - gamma)_+ with objective
// sqrt(sum (|v| - gamma)_+^2); L0 (4, 5) x = v [v^2 > gamma] with objective
// sum (v^2 - gamma)_+, gamma rounded to FP32 as the dense epilogue rounds it.
// Writes x and its mask words, and the objective and non-zero count as the
// start's single partial (obj_part[j], nnz_part[j]) for finalize.
template <bool L1>
__global__ void __launch_bounds__(SP_THREADS) sp_penalty_kernel(
    const float *__restrict__ Vraw, int ldn, int n, float gamma, float *__restrict__ Vx,
    uint32_t *__restrict__ mask, float *__restrict__ obj_part, float *__restrict__ nnz_part,
    const uint32_t *stop) {
  if (*stop) return;
  __shared__ double red[SP_THREADS / 32];
  const int j = blockIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int words = ldn >> 5;
  const float *v = Vraw + (size_t)j * ldn;
  float *x = Vx + (size_t)j * ldn;
  double obj = 0.0, cnt = 0.0;
  for (int w = warp; w < words; w += SP_THREADS / 32) {
    const int q = (w << 5) + lane;
    bool keep = false;
    float xv = 0.f;
    if (q < n) {
      const float a = v[q];
      const float d = L1 ? fabsf(a) - gamma : a * a - gamma;
      keep = d > 0.f;
      if (keep) {
        xv = L1 ? copysignf(d, a) : a;
        obj += L1 ? (double)d * (double)d : (double)d;
        cnt += 1.0;
      }
    }
    const uint32_t bits = __ballot_sync(0xFFFFFFFFu, keep);
    x[q] = xv;  // q < ldn: the plane's padding takes zeros
    if (lane == 0) mask[(size_t)j * words + w] = bits;
  }
  obj = sp_block_sum(obj, red);
  cnt = sp_block_sum(cnt, red);
  if (threadIdx.x == 0) {
    obj_part[j] = (float)obj;
    nnz_part[j] = (float)cnt;
  }
}

// Deflation, V side (one block per start): with P = (I - x_1 x_1^T) ...
// (I - x_C x_C^T), Z = B P v applies the factors to v from the last to the
// first: a_c = x_c^T v - sum_{c' > c} a_c' (x_c^T x_c') for c = C .. 1, and
// P v = v - sum_c a_c x_c.  Stores a[j][c] for the transposition and corrects
// the centring sums (when sum_v is not null) to those of P v.
__global__ void __launch_bounds__(SP_THREADS) sp_defl_coef_kernel(
    const float *__restrict__ Vx, const uint32_t *__restrict__ mask, int ldn, int n,
    const float *__restrict__ defl, int comps, const double *__restrict__ gram,
    const double *__restrict__ defl_sum, const double *__restrict__ defl_mu,
    double *__restrict__ defl_a, double *sum_v, double *dot_mu, const uint32_t *stop) {
  if (*stop) return;
  __shared__ double red[SP_THREADS / 32];
  __shared__ double d[SP_DEFL_MAX];
  const int j = blockIdx.x;
  const int words = ldn >> 5;
  for (int c = 0; c < comps; c++) {
    double s = 0.0;
    for (int q = threadIdx.x; q < n; q += SP_THREADS) {
      const uint32_t w = mask[(size_t)j * words + (q >> 5)];
      if ((w >> (q & 31)) & 1u)
        s += (double)defl[(size_t)c * n + q] * (double)Vx[(size_t)j * ldn + q];
    }
    s = sp_block_sum(s, red);
    if (threadIdx.x == 0) d[c] = s;
  }
  if (threadIdx.x == 0) {
    double a[SP_DEFL_MAX];
    double ds = 0.0, dm = 0.0;
    for (int c = comps - 1; c >= 0; c--) {
      double v = d[c];
      for (int c2 = c + 1; c2 < comps; c2++) v -= a[c2] * gram[c * SP_DEFL_MAX + c2];
      a[c] = v;
      defl_a[(size_t)j * SP_DEFL_MAX + c] = v;
      ds += v * defl_sum[c];
      dm += v * defl_mu[c];
    }
    if (sum_v) {
      sum_v[j] -= ds;
      dot_mu[j] -= dm;
    }
  }
}

// Deflation, B^T Z side (one block per start): V = P^T B^T z applies the
// factors to u = B^T z from the first to the last: b_c = x_c^T u -
// sum_{c' < c} b_c' (x_c^T x_c'), then u <- u - sum_c b_c x_c, in place.
__global__ void __launch_bounds__(SP_THREADS) sp_defl_vraw_kernel(
    float *__restrict__ Vraw, int ldn, int n, const float *__restrict__ defl, int comps,
    const double *__restrict__ gram, const uint32_t *stop) {
  if (*stop) return;
  __shared__ double red[SP_THREADS / 32];
  __shared__ double b[SP_DEFL_MAX];
  const int j = blockIdx.x;
  float *u = Vraw + (size_t)j * ldn;
  for (int c = 0; c < comps; c++) {
    double s = 0.0;
    for (int q = threadIdx.x; q < n; q += SP_THREADS)
      s += (double)defl[(size_t)c * n + q] * (double)u[q];
    s = sp_block_sum(s, red);
    if (threadIdx.x == 0) b[c] = s;
  }
  if (threadIdx.x == 0) {
    for (int c = 0; c < comps; c++) {
      double v = b[c];
      for (int c2 = 0; c2 < c; c2++) v -= b[c2] * gram[c * SP_DEFL_MAX + c2];
      b[c] = v;
    }
  }
  __syncthreads();
  for (int q = threadIdx.x; q < n; q += SP_THREADS) {
    double v = (double)u[q];
    for (int c = 0; c < comps; c++) v -= b[c] * (double)defl[(size_t)c * n + q];
    u[q] = (float)v;
  }
}

// Explained variance ||(B - 1 mu^T - r 1^T) x||^2 of a unit loading in FP64:
// a thread per sample row, y_i = sum_e b_e x_col(e) - mu^T x - r_i 1^T x, each
// block's sum of y_i^2 into partial[block]; xs = {1^T x, mu^T x} precomputed.
__global__ void __launch_bounds__(SP_THREADS) sp_ev_rows_kernel(
    const int32_t *__restrict__ row_ptr, const int32_t *__restrict__ col_ind,
    const float *__restrict__ rvals, int m, const float *__restrict__ x,
    const float *__restrict__ row_means, const double *__restrict__ xs,
    double *__restrict__ partial) {
  __shared__ double red[SP_THREADS / 32];
  const int i = blockIdx.x * SP_THREADS + threadIdx.x;
  double y2 = 0.0;
  if (i < m) {
    double y = 0.0;
    for (int e = row_ptr[i]; e < row_ptr[i + 1]; e++) y += (double)rvals[e] * (double)x[col_ind[e]];
    y -= xs[1];
    if (row_means) y -= (double)row_means[i] * xs[0];
    y2 = y * y;
  }
  y2 = sp_block_sum(y2, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = y2;
}

// xs = {sum_q x_q, sum_q mu_q x_q} (one block), then, after sp_ev_rows_kernel,
// *out = the fixed-order sum of the partials (sp_ev_sum_kernel).
__global__ void __launch_bounds__(SP_THREADS) sp_ev_xstats_kernel(
    const float *__restrict__ x, int n, const float *__restrict__ means, double *__restrict__ xs) {
  __shared__ double red[SP_THREADS / 32];
  double s = 0.0, d = 0.0;
  for (int q = threadIdx.x; q < n; q += SP_THREADS) {
    s += (double)x[q];
    if (means) d += (double)means[q] * (double)x[q];
  }
  s = sp_block_sum(s, red);
  d = sp_block_sum(d, red);
  if (threadIdx.x == 0) {
    xs[0] = s;
    xs[1] = d;
  }
}
__global__ void __launch_bounds__(SP_THREADS) sp_ev_sum_kernel(const double *__restrict__ partial,
                                                               int count, double *__restrict__ out) {
  __shared__ double red[SP_THREADS / 32];
  double t = 0.0;
  for (int b = threadIdx.x; b < count; b += SP_THREADS) t += partial[b];
  t = sp_block_sum(t, red);
  if (threadIdx.x == 0) *out = t;
}
