/*
 * Precision-generic body of the oracle (see am_oracle.c).  Included twice,
 * with F = float / SUF = f32 and F = double / SUF = f64.
 *
 * Every function restates a piece of the reference's AM path and cites the
 * reference file:line it follows.  Arithmetic is written in the same order
 * and the same precision as the reference's C++ (including its int/double
 * promotions), and reductions run sequentially in index order like
 * oracle/shim/naive_cblas.c, so that with one thread this code reproduces the
 * reference build in oracle/_ref/ bit for bit.
 */
#define CAT2(a, b) a##_##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SUF)

/* |v| as the reference's myabs (c++/src/utils/various.h:47-50) and std::abs. */
static inline F FN(orc_abs)(F v) { return v > 0 ? v : -v; }
/* sgn with sgn(0) = 0 (c++/src/utils/various.h:44-46). */
static inline int FN(orc_sgn)(F v) { return (v > (F)0) - (v < (F)0); }

/* C = op(A) * B, column-major, beta = 0, sequential K sums
 * (the two cblas_?gemm calls at c++/src/gpower/gpower_commons.h:75,89). */
void FN(orc_gemm)(int transA, int M, int N, int K, const F *A, int lda, const F *B, int ldb,
                  F *C, int ldc) {
  for (int j = 0; j < N; j++)
    for (int i = 0; i < M; i++) {
      F acc = 0;
      for (int l = 0; l < K; l++) {
        F a = transA ? A[l + (long)i * lda] : A[i + (long)l * lda];
        acc += a * B[l + (long)j * ldb];
      }
      C[i + (long)j * ldc] = acc;
    }
}

static F FN(orc_nrm2)(int n, const F *x) {
  F s = 0;
  for (int i = 0; i < n; i++) s += x[i] * x[i];
  return (F)sqrt((double)s);
}
static F FN(orc_asum)(int n, const F *x) {
  F s = 0;
  for (int i = 0; i < n; i++) s += FN(orc_abs)(x[i]);
  return s;
}
static void FN(orc_scal)(int n, F *x, F a) {
  for (int i = 0; i < n; i++) x[i] *= a;
}

/* Relative change |f - f0| / f0 (c++/src/utils/termination_criteria.h:30-36). */
F FN(orc_error)(F f, F f0) { return FN(orc_abs)(f - f0) / f0; }
/* it > 0 && err < tol (c++/src/utils/termination_criteria.h:39-44). */
int FN(orc_terminated)(F err, int it, double tol) { return it > 0 && (double)err < tol; }

static int FN(cmp_abs_asc)(const void *a, const void *b) {
  F x = FN(orc_abs)(*(const F *)a), y = FN(orc_abs)(*(const F *)b);
  return (x > y) - (x < y);
}

/* Hard-threshold level by sorting: |x|_(len-k) of the ascending |x| order
 * (find_hard_treshHolding_parameter_with_sorting, c++/src/utils/thresh_functions.h:92-98). */
F FN(orc_hard_level_sort)(const F *x, unsigned len, unsigned k, F *buf) {
  memcpy(buf, x, sizeof(F) * len);
  qsort(buf, len, sizeof(F), FN(cmp_abs_asc));
  return FN(orc_abs)(buf[len - k]);
}

/* Hard-threshold level by the reference's default ordered-set scan
 * (find_hard_treshHolding_parameter_without_sorting, c++/src/utils/thresh_functions.h:101-118).
 * The set is keyed by value only (comparator :53-60), so equal values collapse
 * and the set can shrink below k; this keeps that behaviour.  buf (>= k+1
 * entries) holds the set in descending order. */
F FN(orc_hard_level_set)(const F *x, unsigned len, unsigned k, F *buf) {
  unsigned sz = 0;
#define SET_INSERT(v)                                                   \
  do {                                                                  \
    F v_ = (v);                                                         \
    unsigned p_ = 0;                                                    \
    while (p_ < sz && buf[p_] > v_) p_++;                               \
    if (p_ < sz && buf[p_] == v_) break; /* already present */         \
    memmove(&buf[p_ + 1], &buf[p_], sizeof(F) * (sz - p_));             \
    buf[p_] = v_;                                                       \
    sz++;                                                               \
  } while (0)
  for (unsigned j = 0; j < k && j < len; j++) SET_INSERT(FN(orc_abs)(x[j]));
  for (unsigned j = k; j < len; j++) {
    F tmp = FN(orc_abs)(x[j]);
    if (sz > 0 && tmp > buf[sz - 1]) {
      sz--; /* erase the smallest */
      SET_INSERT(tmp);
    }
  }
#undef SET_INSERT
  return sz > 0 ? buf[sz - 1] : (F)0;
}

/* Keep |x_i| >= level, zero the rest, return the 2-norm of what is kept
 * (k_hard_thresholding, c++/src/utils/thresh_functions.h:121-145). */
F FN(orc_hard_threshold)(F *x, unsigned len, unsigned k, int use_sort, F *buf) {
  F level = use_sort ? FN(orc_hard_level_sort)(x, len, k, buf)
                     : FN(orc_hard_level_set)(x, len, k, buf);
  F norm = 0;
  for (unsigned i = 0; i < len; i++) {
    F v = x[i];
    if (FN(orc_abs)(v) < level) x[i] = 0;
    else norm += v * v;
  }
  return (F)sqrt((double)norm);
}

/* Soft-threshold level w of the reference's L1-ball scan
 * (soft_thresholding, c++/src/utils/thresh_functions.h:162-218): walks the
 * |x| values in descending order keeping running sums S1 = sum|x|, S2 = sum x^2,
 * and stops at the first of three predicates.  Returns w; *brk gets the scan
 * index it stopped at (len when it never stopped, in which case w is the
 * '+' root of the last step, as in the reference). */
F FN(orc_soft_level)(const F *x, unsigned len, unsigned constrain, F *buf, unsigned *brk) {
  const F sq = (F)sqrt(constrain + 0.0);
  memcpy(buf, x, sizeof(F) * len);
  qsort(buf, len, sizeof(F), FN(cmp_abs_asc));
  const F linfty = FN(orc_abs)(buf[len - 1]);
  const F eps = (F)0.000001;
  F s1 = 0, s2 = 0, w = 0, lo, hi, sub_right_old = sq;
  int t = 0;
  unsigned i;
  for (i = 0; i < len; i++) {
    F tmp = FN(orc_abs)(buf[len - i - 1]);
    s1 += tmp;
    s2 += tmp * tmp;
    t++;
    hi = tmp;
    lo = (i < len - 1) ? FN(orc_abs)(buf[len - i - 2]) : (F)0;
    F sub_left = (s1 - t * tmp) / (F)sqrt(s2 - 2 * tmp * s1 + t * tmp * tmp);
    if (sub_left > sq && sub_right_old < sq) {
      w = tmp;
      break;
    }
    F sub_right = (s1 - t * lo) / (F)sqrt(s2 - 2 * lo * s1 + t * lo * lo);
    F a = t * (t - sq * sq);
    F b = 2 * s1 * sq * sq - 2 * t * s1;
    F c = s1 * s1 - sq * sq * s2;
    w = (-b - (F)sqrt(b * b - 4 * a * c)) / (2 * a);
    if (w > lo && w < hi) break;
    w = (-b + (F)sqrt(b * b - 4 * a * c)) / (2 * a);
    if (w > lo && w < hi && w < linfty - eps) break;
    sub_right_old = sub_right;
  }
  if (brk) *brk = i;
  return w;
}

/* x_i <- sgn(x_i)(|x_i| - w)_+ and return the 2-norm
 * (c++/src/utils/thresh_functions.h:226-253). */
F FN(orc_soft_threshold)(F *x, unsigned len, unsigned constrain, F *buf) {
  F w = FN(orc_soft_level)(x, len, constrain, buf, NULL);
  F norm = 0;
  for (unsigned i = 0; i < len; i++) {
    F v = x[i];
    F d = FN(orc_abs)(v) - w;
    if (d > 0) {
      F val = d * FN(orc_sgn)(v);
      x[i] = val;
      norm += val * val;
    } else {
      x[i] = 0;
    }
  }
  return (F)sqrt((double)norm);
}

/* L1 penalty: x = sgn(v)(|v| - gamma)_+, objective sqrt(sum (|v|-gamma)_+^2)
 * (L1_penalized_thresholding, c++/src/gpower/sparse_PCA_thresholding.h:26-47).
 * gamma is a double in the reference, so |v| - gamma is formed in double. */
F FN(orc_l1_penalty)(F *v, unsigned len, double gamma) {
  F f = 0;
  for (unsigned i = 0; i < len; i++) {
    F tmp = v[i];
    F d = (F)((double)FN(orc_abs)(tmp) - gamma);
    if (d > 0) {
      f += d * d;
      v[i] = d * FN(orc_sgn)(tmp);
    } else {
      v[i] = 0;
    }
  }
  return (F)sqrt((double)f);
}

/* L0 penalty: keep v_i where v_i^2 > gamma, objective sum (v_i^2 - gamma)_+
 * (L0_penalized_thresholding, c++/src/gpower/sparse_PCA_thresholding.h:68-87). */
F FN(orc_l0_penalty)(F *v, unsigned len, double gamma) {
  F f = 0;
  for (unsigned i = 0; i < len; i++) {
    F tmp = v[i];
    F d = (F)((double)(tmp * tmp) - gamma);
    if (d > 0) f += d;
    else v[i] = 0;
  }
  return f;
}

static unsigned FN(orc_nnz)(const F *x, unsigned n) {
  unsigned c = 0;
  for (unsigned i = 0; i < n; i++) c += x[i] != 0;
  return c;
}

/* Per-start bookkeeping of storeIterationsForAllPoints
 * (c++/src/gpower/gpower_commons.h:120-130, sparse_PCA_thresholding.h:51-63). */
static void FN(orc_log_start)(const orc_settings *s, F err, int it, int *iters, int *cards,
                              unsigned slot, const F *x, unsigned n) {
  if (!s->store_all) return;
  int done = FN(orc_terminated)(err, it, s->tolerance);
  if (done && iters[slot] == -1) {
    iters[slot] = it;
    cards[slot] = (int)FN(orc_nnz)(x, n);
  } else if (!done && iters[slot] != -1) {
    iters[slot] = -1;
  }
}

/* One AM iteration over a batch of bs starts, V (n x bs) in place, Z (m x bs)
 * scratch.  Constrained forms follow perform_one_iteration_for_constrained_pca
 * (c++/src/gpower/gpower_commons.h:68-136), penalized forms
 * perform_one_iteration_for_penalized_pca (:140-177).  val/tmpv/err are the
 * ValueCoordinateHolder fields val/tmp/current_error
 * (c++/src/utils/various.h:19-42).  Returns the batch's largest error, where
 * NaN errors never raise the maximum (c++/src/gpower/gpower_commons.h:132-133). */
F FN(orc_iteration)(const F *B, int ldB, unsigned m, unsigned n, unsigned bs, F *V, F *Z,
                    const orc_settings *s, F *val, F *tmpv, F *err, int it, unsigned shift,
                    int *iters, int *cards, F *buf) {
  const int form = s->formulation;
  const int l1var = (form == ORC_L0C_L1 || form == ORC_L1C_L1 || form == ORC_L0P_L1 ||
                     form == ORC_L1P_L1);
  F max_err = 0;
  FN(orc_gemm)(0, (int)m, (int)bs, (int)n, B, ldB, V, (int)n, Z, (int)m);
  if (orc_is_constrained(form)) {
    if (l1var)
      for (unsigned j = 0; j < bs; j++) {
        F *z = &Z[(size_t)m * j];
        tmpv[j] = FN(orc_asum)((int)m, z);
        for (unsigned i = 0; i < m; i++) z[i] = (F)FN(orc_sgn)(z[i]);
      }
    FN(orc_gemm)(1, (int)n, (int)bs, (int)m, B, ldB, Z, (int)m, V, (int)n);
    for (unsigned j = 0; j < bs; j++) {
      F *x = &V[(size_t)n * j];
      F f = 0;
      if (!l1var) f = FN(orc_nrm2)((int)m, &Z[(size_t)m * j]);
      F nx = (form == ORC_L1C_L2 || form == ORC_L1C_L1)
                 ? FN(orc_soft_threshold)(x, n, s->constraint, buf)
                 : FN(orc_hard_threshold)(x, n, s->constraint, s->use_sort_hard, buf);
      FN(orc_scal)((int)n, x, 1 / nx);
      if (l1var) f = tmpv[j];
      F e = FN(orc_error)(f, val[j]);
      err[j] = e;
      FN(orc_log_start)(s, e, it, iters, cards, shift + j, x, n);
      if (max_err < e) max_err = e;
      val[j] = f;
    }
  } else {
    for (unsigned j = 0; j < bs; j++) {
      F *z = &Z[(size_t)m * j];
      if (l1var) {
        for (unsigned i = 0; i < m; i++) z[i] = (F)FN(orc_sgn)(z[i]);
      } else {
        F nz = FN(orc_nrm2)((int)m, z);
        FN(orc_scal)((int)m, z, 1 / nz);
      }
    }
    FN(orc_gemm)(1, (int)n, (int)bs, (int)m, B, ldB, Z, (int)m, V, (int)n);
    for (unsigned j = 0; j < bs; j++) {
      F *x = &V[(size_t)n * j];
      F f = (form == ORC_L1P_L2 || form == ORC_L1P_L1) ? FN(orc_l1_penalty)(x, n, s->penalty)
                                                       : FN(orc_l0_penalty)(x, n, s->penalty);
      F e = FN(orc_error)(f, val[j]);
      err[j] = e;
      if (max_err < e) max_err = e;
      val[j] = f;
      /* the penalized thresholding calls at gpower_commons.h:170,173 leave the
       * batch shift at its default of 0, so every batch logs into slots 0..bs-1 */
      FN(orc_log_start)(s, e, it, iters, cards, j, x, n);
    }
  }
  return max_err;
}

/* The reference's own starting point for global start index g
 * (getSignleStartingPoint, c++/src/gpower/gpower_commons.h:22-47), written
 * into a zeroed column x of length n.  Constrained forms: s draws of
 * (index, value) from rand_r seeded with g, duplicates overwrite but still
 * count in the norm, then scaled by 1/sqrt(sum value^2).  Penalized forms:
 * U[-1, 1] entries, not normalised. */
void FN(orc_reference_start)(F *x, unsigned n, int constrained, unsigned s, unsigned g) {
  unsigned seed = g;
  if (constrained) {
    F norm = 0;
    for (unsigned i = 0; i < s; i++) {
      unsigned idx = (unsigned)(int)((F)n * (F)rand_r(&seed) / (F)RAND_MAX);
      if (idx == n) idx--;
      F tmp = (F)rand_r(&seed) / (F)RAND_MAX;
      x[idx] = tmp;
      norm += tmp * tmp;
    }
    FN(orc_scal)((int)n, x, (F)1 / (F)sqrt((double)norm));
  } else {
    for (unsigned i = 0; i < n; i++) {
      F tmp = (F)rand_r(&seed) / (F)RAND_MAX;
      tmp = -1 + 2 * tmp;
      x[i] = tmp;
    }
  }
}

/* denseDataSolver (c++/src/gpower/sparse_PCA_solver.h:36-243): settings are
 * adjusted as chceckInputAndModifyIt does (c++/src/class/optimization_settings.h:156-168),
 * then batches with batch-global termination (:171-232) or the on-the-fly
 * slot-refill loop (:83-168), best start by objective, x <- x/||x||.
 * Starting points come from V_all (n x total_starts, after rounding) when it
 * is non-NULL, else from orc_reference_start.  values/iters/cards may be NULL
 * unless store_all is set. */
F FN(orc_dense_solver)(const F *B, int ldB, F *x, unsigned m, unsigned n, orc_settings *s,
                       orc_stats *st, const F *V_all, double *values, int *iters, int *cards) {
  orc_check_input(s, n);
  const unsigned bs = (unsigned)s->batch_size;
  const int cons = orc_is_constrained(s->formulation);
  F *Z = (F *)calloc((size_t)m * bs, sizeof(F));
  F *V = (F *)calloc((size_t)n * bs, sizeof(F));
  F *val = (F *)calloc(bs, sizeof(F));
  F *tmpv = (F *)calloc(bs, sizeof(F));
  F *err = (F *)calloc(bs, sizeof(F));
  F *buf = (F *)calloc((size_t)n + 2, sizeof(F));
  if (s->store_all && !s->use_otf)
    for (int i = 0; i < s->total_starts; i++) {
      iters[i] = -1;
      cards[i] = -1;
      values[i] = -1;
    }
  F best = -1;
  unsigned total_it = 0;
  if (s->use_otf) {
    s->store_all = 0;
    unsigned *cur = (unsigned *)calloc(bs, sizeof(unsigned));
    unsigned *order = (unsigned *)calloc(bs, sizeof(unsigned));
    for (unsigned j = 0; j < bs; j++) {
      order[j] = j;
      if (V_all) memcpy(&V[(size_t)n * j], &V_all[(size_t)n * j], sizeof(F) * n);
      else FN(orc_reference_start)(&V[(size_t)n * j], n, cons, s->constraint, j);
    }
    unsigned generated = bs;
    int go = 1;
    while (go) {
      total_it++;
      FN(orc_iteration)(B, ldB, m, n, bs, V, Z, s, val, tmpv, err, 0, 0, iters, cards, buf);
      go = 0;
      for (unsigned i = 0; i < bs; i++) {
        cur[i]++;
        if (FN(orc_terminated)(err[i], (int)cur[i], s->tolerance) ||
            cur[i] >= (unsigned)s->max_iter) {
          if (best < val[i]) {
            best = val[i];
            memcpy(x, &V[(size_t)n * i], sizeof(F) * n);
          }
          if (generated < (unsigned)s->total_starts) {
            val[i] = 0;
            tmpv[i] = 0;
            order[i] = generated++;
            cur[i] = 0;
            go = 1;
          }
        } else {
          go = 1;
        }
      }
      for (unsigned j = 0; j < bs; j++)
        if (cur[j] == 0) {
          F *col = &V[(size_t)n * j];
          if (V_all) {
            memcpy(col, &V_all[(size_t)n * order[j]], sizeof(F) * n);
          } else {
            if (cons) FN(orc_scal)((int)n, col, (F)0);
            FN(orc_reference_start)(col, n, cons, s->constraint, order[j]);
          }
        }
    }
    free(cur);
    free(order);
  } else {
    for (unsigned b = 0; b < s->total_batches; b++) {
      unsigned shift = b * bs;
      /* scaling by zero (not memset) keeps a NaN left by the previous batch,
       * as cblas_vector_scale(.., 0) does at sparse_PCA_solver.h:175-176 */
      FN(orc_scal)((int)(n * bs), V, (F)0);
      for (unsigned j = 0; j < bs; j++) {
        if (V_all) memcpy(&V[(size_t)n * j], &V_all[(size_t)n * (shift + j)], sizeof(F) * n);
        else FN(orc_reference_start)(&V[(size_t)n * j], n, cons, s->constraint, shift + j);
        val[j] = 0;
        tmpv[j] = 0;
      }
      for (int it = 0; it < s->max_iter; it++) {
        total_it++;
        F e = FN(orc_iteration)(B, ldB, m, n, bs, V, Z, s, val, tmpv, err, it, shift, iters,
                                cards, buf);
        if (FN(orc_terminated)(e, it, s->tolerance)) break;
      }
      unsigned sel = 0;
      F bv = val[0];
      if (s->store_all) values[shift] = bv;
      for (unsigned i = 1; i < bs; i++) {
        if (s->store_all) values[shift + i] = val[i];
        if (val[i] > bv) {
          bv = val[i];
          sel = i;
        }
      }
      if (best < bv) {
        best = bv;
        memcpy(x, &V[(size_t)n * sel], sizeof(F) * n);
      }
    }
  }
  F nx = FN(orc_nrm2)((int)n, x);
  FN(orc_scal)((int)n, x, 1 / nx);
  st->it = total_it;
  st->fval = best;
  free(Z);
  free(V);
  free(val);
  free(tmpv);
  free(err);
  free(buf);
  return best;
}

#undef FN
#undef CAT
#undef CAT2
