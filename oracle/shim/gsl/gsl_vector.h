/* Stand-in for GSL's gsl_vector: only what c++/src/utils/gsl_helper.h:39-49 touches. */
#ifndef AM24_ORACLE_SHIM_GSL_VECTOR_H
#define AM24_ORACLE_SHIM_GSL_VECTOR_H
#include <stddef.h>
typedef struct { size_t size; size_t stride; double *data; } gsl_vector;
static inline double gsl_vector_get(const gsl_vector *v, size_t i) { return v->data[i * v->stride]; }
#endif
