/*
 * FFTW3 single-precision API shim (oracle test infrastructure).
 *
 * Declares the subset of the FFTW 3.x interface that the reference's
 * src/fft.c:34-312 calls (fftwf_plan_dft_3d, fftwf_plan_many_dft,
 * fftwf_execute, fftwf_destroy_plan, fftwf_malloc/free, fftwf_init_threads,
 * fftwf_plan_with_nthreads) and runs them on oracle/cpufft (spfft).
 * Planning never touches the arrays (real FFTW_MEASURE planning overwrites
 * them the first time a problem is planned).
 */
#ifndef ORACLE_FFTW3_SHIM_H
#define ORACLE_FFTW3_SHIM_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

typedef float fftwf_complex[2];
typedef struct fftwf_plan_s *fftwf_plan;
typedef double fftw_complex[2];
typedef struct fftw_plan_s *fftw_plan;

fftwf_plan fftwf_plan_dft_3d(int n0, int n1, int n2, fftwf_complex *in, fftwf_complex *out, int sign,
                             unsigned flags);
fftwf_plan fftwf_plan_dft_2d(int n0, int n1, fftwf_complex *in, fftwf_complex *out, int sign, unsigned flags);
fftwf_plan fftwf_plan_dft_1d(int n0, fftwf_complex *in, fftwf_complex *out, int sign, unsigned flags);
fftwf_plan fftwf_plan_many_dft(int rank, const int *n, int howmany, fftwf_complex *in, const int *inembed,
                               int istride, int idist, fftwf_complex *out, const int *onembed, int ostride,
                               int odist, int sign, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_destroy_plan(fftwf_plan p);
void *fftwf_malloc(size_t n);
void fftwf_free(void *p);
int fftwf_init_threads(void);
void fftwf_plan_with_nthreads(int nthreads);
void fftwf_cleanup_threads(void);

#ifdef __cplusplus
}
#endif
#endif
