/*
 * ORACLE -- test infrastructure, not product code.
 *
 * A plain-C restatement of the reference's (optml/24am) alternating-
 * maximization core for the 8 sparse-PCA formulations, used only by tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker of
 * the CUDA path.  The product library never links or calls it.
 *
 * Parity is pinned: with one thread and oracle/shim/naive_cblas.c, the
 * reference's own solver built by oracle/Makefile (oracle/_ref/libref24_naive.so)
 * and this restatement agree bit for bit on every formulation, in batch and
 * on-the-fly modes, with reference-generated and with injected starting
 * points (tests/test_oracle_vs_reference.py), and both are checked against the
 * committed fixtures in tests/golden/.
 *
 * Naming follows the reference: B (here `B`, column-major, ldB >= m) is the
 * m x n data matrix (m samples, n features), V holds one loading vector per
 * starting point (n x batch), Z one sample-space vector per start (m x batch).
 */
#define _DEFAULT_SOURCE
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "am_oracle.h"

int orc_is_constrained(int f) { return f >= ORC_L0C_L2 && f <= ORC_L1C_L1; }

/* chceckInputAndModifyIt (c++/src/class/optimization_settings.h:156-168). */
void orc_check_input(orc_settings *s, unsigned n) {
  if (s->constraint > n) s->constraint = n;
  if (s->batch_size == 0) s->batch_size = s->total_starts;
  s->total_batches = (unsigned)(s->total_starts / s->batch_size);
  if (s->total_batches * (unsigned)s->batch_size < (unsigned)s->total_starts) s->total_batches++;
  s->total_starts = (int)(s->total_batches * (unsigned)s->batch_size);
}

#define F float
#define SUF f32
#include "am_oracle_impl.h"
#undef F
#undef SUF

#define F double
#define SUF f64
#include "am_oracle_impl.h"
#undef F
#undef SUF
