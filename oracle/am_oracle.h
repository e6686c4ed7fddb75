/*
 * ORACLE -- test infrastructure, not product code.  Declarations for
 * am_oracle.c, the CPU restatement of the reference's AM core.
 */
#ifndef AM24_ORACLE_H
#define AM24_ORACLE_H

/* SPCA_Formulation values (c++/src/class/optimization_settings.h:27-37). */
enum {
  ORC_L0C_L2 = 0, /* L0_constrained_L2_PCA */
  ORC_L0C_L1 = 1, /* L0_constrained_L1_PCA */
  ORC_L1C_L2 = 2, /* L1_constrained_L2_PCA */
  ORC_L1C_L1 = 3, /* L1_constrained_L1_PCA */
  ORC_L0P_L2 = 4, /* L0_penalized_L2_PCA */
  ORC_L0P_L1 = 5, /* L0_penalized_L1_PCA */
  ORC_L1P_L2 = 6, /* L1_penalized_L2_PCA */
  ORC_L1P_L1 = 7  /* L1_penalized_L1_PCA */
};

/* The OptimizationSettings fields the AM path reads
 * (c++/src/class/optimization_settings.h:73-99); same layout as the
 * ref_settings struct of oracle/ref_harness.cpp. */
typedef struct {
  int formulation;
  unsigned constraint;
  double penalty;
  double tolerance;
  int max_iter;
  int total_starts;
  int batch_size;
  int use_otf;
  int use_sort_hard;
  int store_all;
  unsigned total_batches;
} orc_settings;

typedef struct {
  unsigned it;
  double fval;
  double compute_time;
  int threads;
} orc_stats;

int orc_is_constrained(int formulation);
void orc_check_input(orc_settings *s, unsigned n);

#endif
