/*
 * Numeric types of the phasing path, layout-compatible with the reference's
 * single-precision build (include/spimage/linear_alg.h:39-56,95-114).
 * Only the types and inline helpers the phasing API needs are declared here.
 */
#ifndef SPB_LINEAR_ALG_H
#define SPB_LINEAR_ALG_H 1

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mem_util.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef float real;                       /* _SP_SINGLE_PRECISION */
typedef struct { float re, im; } Complex; /* binary-compatible with fftwf_complex / float2 */

#define sp_real(a) (a).re
#define sp_imag(a) (a).im
#define REAL_MAX FLT_MAX
#define REAL_EPSILON FLT_EPSILON

typedef struct { unsigned int rows; unsigned int cols; real *data; } sp_matrix;
typedef sp_matrix SpRotation;
typedef struct { unsigned int size; real *data; } sp_vector;
typedef struct { unsigned int x; unsigned int y; unsigned int z; real *data; } sp_3matrix;
typedef struct { unsigned int x; unsigned int y; unsigned int z; int *data; } sp_i3matrix;
typedef struct { unsigned int x; unsigned int y; unsigned int z; Complex *data; } sp_c3matrix;

static inline Complex sp_cinit(real a, real b) { Complex r; r.re = a; r.im = b; return r; }
static inline real sp_cabs(Complex a) { return sqrt(a.im * a.im + a.re * a.re); }
static inline real sp_cabs2(Complex a) { return a.im * a.im + a.re * a.re; }
static inline real sp_min(real a, real b) { return a < b ? a : b; }
static inline real sp_max(real a, real b) { return a > b ? a : b; }

/* allocation, include/spimage/linear_alg.h:273-293 */
sp_3matrix *_sp_3matrix_alloc(unsigned int nx, unsigned int ny, unsigned int nz, const char *file, int line);
#define sp_3matrix_alloc(nx, ny, nz) _sp_3matrix_alloc(nx, ny, nz, __FILE__, __LINE__)
sp_i3matrix *_sp_i3matrix_alloc(unsigned int nx, unsigned int ny, unsigned int nz, const char *file, int line);
#define sp_i3matrix_alloc(nx, ny, nz) _sp_i3matrix_alloc(nx, ny, nz, __FILE__, __LINE__)
sp_c3matrix *_sp_c3matrix_alloc(unsigned int nx, unsigned int ny, unsigned int nz, const char *file, int line);
#define sp_c3matrix_alloc(nx, ny, nz) _sp_c3matrix_alloc(nx, ny, nz, __FILE__, __LINE__)
void _sp_3matrix_free(sp_3matrix *m, const char *file, int line);
#define sp_3matrix_free(m) _sp_3matrix_free(m, __FILE__, __LINE__)
void _sp_i3matrix_free(sp_i3matrix *m, const char *file, int line);
#define sp_i3matrix_free(m) _sp_i3matrix_free(m, __FILE__, __LINE__)
void _sp_c3matrix_free(sp_c3matrix *m, const char *file, int line);
#define sp_c3matrix_free(m) _sp_c3matrix_free(m, __FILE__, __LINE__)

#ifdef __cplusplus
}
#endif
#endif
