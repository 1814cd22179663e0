/*
 * spfft -- CPU single-precision FFT used by the oracle (test infrastructure only).
 *
 * The reference engine calls FFTW3 (single precision) through
 * src/fft.c:53-99,152-189 (fftwf_plan_dft_3d + fftwf_execute on every call).
 * FFTW is not installed here, so the oracle builds the reference's own
 * sources against an FFTW3-API shim (oracle/fftw_shim) that runs this FFT.
 *
 * Algorithm (fixed, so that other implementations can reproduce it bit for bit):
 *   - 1-D transform of length n: Stockham autosort, radix sequence from
 *     spfft_radix_plan() (16s first, then 8/4/2, then 3s, 5s, then other primes
 *     in ascending order; a trailing 2 after a 16 becomes 8*4).
 *   - Stage s with radix r and Ns = product of earlier radices, for every
 *     butterfly j in [0, n/r):  k = j % Ns;  a[m] = x[j + m*n/r];
 *     a[m] *= tw[m*k*(n/(Ns*r))] when m*k != 0;  a = DFT_r(a);
 *     y[(j/Ns)*Ns*r + k + m*Ns] = a[m].
 *   - tw[i] = ((float)cos(2*pi*i/n), (float)-sin(2*pi*i/n)) computed in double
 *     (conjugated for the backward transform).
 *   - Butterflies for r = 2,3,4,5,8,16 and a generic O(r^2) prime butterfly,
 *     all in float with every multiply and add rounded separately (the file is
 *     built with -ffp-contract=off; no fused multiply-add anywhere).
 *   - Multi-dimensional transforms are separable: the forward transform runs
 *     the fastest axis first (x, then y, then z); the backward transform runs
 *     the slowest axis first (z, then y, then x).  Both are unnormalised, with
 *     FFTW's sign convention (forward = exp(-2 pi i jk/n)).
 */
#ifndef SPFFT_H
#define SPFFT_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { float re, im; } spfft_cpx;

#define SPFFT_MAX_STAGES 48

typedef struct {
  int n;
  int nstages;
  int radix[SPFFT_MAX_STAGES];
  spfft_cpx *tw; /* n forward twiddles */
} spfft_plan;

/* Fills radix[] with the canonical radix sequence of n and returns its length. */
int spfft_radix_plan(int n, int *radix);
spfft_plan *spfft_plan_create(int n);
void spfft_plan_destroy(spfft_plan *p);

/* In-place transform of `howmany` lines of length p->n.  Element i of line h
 * sits at data[h*dist + i*stride] (units of complex elements).  sign = -1 is
 * forward, +1 backward.  nthreads >= 1 splits the lines over POSIX threads. */
void spfft_lines(const spfft_plan *p, int sign, spfft_cpx *data, long howmany,
                 long stride, long dist, int nthreads);

/* Row-major rank-d transform (dims[0] slowest).  in may equal out. */
void spfft_nd(int rank, const int *dims, int sign, const spfft_cpx *in,
              spfft_cpx *out, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
