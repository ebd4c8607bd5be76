/* Stand-in declarations for the GSL vector/matrix/permutation/linear-algebra
 * calls that only the reference's non-LTE solver reaches. The oracle harness
 * never enables non-LTE atoms; every call aborts loudly if reached. */
#ifndef ORACLE_SHIM_GSL_VECTOR_H
#define ORACLE_SHIM_GSL_VECTOR_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { size_t size; double* data; } gsl_vector;
typedef struct { size_t size1, size2; double* data; } gsl_matrix;
typedef struct { size_t size; size_t* data; } gsl_permutation;

gsl_vector* gsl_vector_calloc(size_t n);
void gsl_vector_set_zero(gsl_vector* v);
void gsl_vector_set(gsl_vector* v, size_t i, double x);
double gsl_vector_get(const gsl_vector* v, size_t i);
gsl_matrix* gsl_matrix_calloc(size_t n1, size_t n2);
void gsl_matrix_set_zero(gsl_matrix* m);
void gsl_matrix_set(gsl_matrix* m, size_t i, size_t j, double x);
double gsl_matrix_get(const gsl_matrix* m, size_t i, size_t j);
gsl_permutation* gsl_permutation_alloc(size_t n);
void gsl_permutation_init(gsl_permutation* p);
int gsl_linalg_LU_decomp(gsl_matrix* A, gsl_permutation* p, int* signum);
int gsl_linalg_LU_solve(const gsl_matrix* LU, const gsl_permutation* p, const gsl_vector* b, gsl_vector* x);

#ifdef __cplusplus
}
#endif
#endif
