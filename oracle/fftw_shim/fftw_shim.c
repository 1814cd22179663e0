/*
 * FFTW3 single-precision API shim over oracle/cpufft (spfft).  Test
 * infrastructure: it lets the reference's unmodified src/fft.c run without
 * libfftw3f.  Multi-dimensional plans follow FFTW's row-major convention
 * (n0 slowest); the transform is unnormalised like FFTW's.
 */
#include "fftw3.h"
#include "../cpufft/spfft.h"

#include <stdlib.h>
#include <string.h>

struct fftwf_plan_s {
  int kind; /* 0 = rank-d contiguous, 1 = many 1-D lines */
  int rank;
  int dims[3];
  int sign;
  spfft_cpx *in, *out;
  /* many */
  const spfft_plan *line;
  spfft_plan *owned;
  int howmany, istride, idist, ostride, odist;
  int nthreads;
};

static int g_nthreads = 1;

int fftwf_init_threads(void) { return 1; }
void fftwf_plan_with_nthreads(int nthreads) { g_nthreads = nthreads < 1 ? 1 : nthreads; }
void fftwf_cleanup_threads(void) { g_nthreads = 1; }

void *fftwf_malloc(size_t n) {
  void *p = NULL;
  if (posix_memalign(&p, 64, n ? n : 1)) return NULL;
  return p;
}
void fftwf_free(void *p) { free(p); }

static fftwf_plan make_nd(int rank, const int *dims, fftwf_complex *in, fftwf_complex *out, int sign) {
  fftwf_plan p = (fftwf_plan)calloc(1, sizeof(*p));
  p->kind = 0;
  p->rank = rank;
  for (int i = 0; i < rank; i++) p->dims[i] = dims[i];
  p->sign = sign;
  p->in = (spfft_cpx *)in;
  p->out = (spfft_cpx *)out;
  p->nthreads = g_nthreads;
  return p;
}

fftwf_plan fftwf_plan_dft_3d(int n0, int n1, int n2, fftwf_complex *in, fftwf_complex *out, int sign,
                             unsigned flags) {
  (void)flags;
  int d[3] = {n0, n1, n2};
  return make_nd(3, d, in, out, sign);
}
fftwf_plan fftwf_plan_dft_2d(int n0, int n1, fftwf_complex *in, fftwf_complex *out, int sign, unsigned flags) {
  (void)flags;
  int d[2] = {n0, n1};
  return make_nd(2, d, in, out, sign);
}
fftwf_plan fftwf_plan_dft_1d(int n0, fftwf_complex *in, fftwf_complex *out, int sign, unsigned flags) {
  (void)flags;
  return make_nd(1, &n0, in, out, sign);
}

fftwf_plan fftwf_plan_many_dft(int rank, const int *n, int howmany, fftwf_complex *in, const int *inembed,
                               int istride, int idist, fftwf_complex *out, const int *onembed, int ostride,
                               int odist, int sign, unsigned flags) {
  (void)inembed; (void)onembed; (void)flags;
  if (rank != 1) return NULL;
  fftwf_plan p = (fftwf_plan)calloc(1, sizeof(*p));
  p->kind = 1;
  p->rank = 1;
  p->dims[0] = n[0];
  p->sign = sign;
  p->in = (spfft_cpx *)in;
  p->out = (spfft_cpx *)out;
  p->owned = spfft_plan_create(n[0]);
  p->line = p->owned;
  p->howmany = howmany;
  p->istride = istride; p->idist = idist;
  p->ostride = ostride; p->odist = odist;
  p->nthreads = g_nthreads;
  return p;
}

void fftwf_execute(const fftwf_plan p) {
  if (!p) return;
  if (p->kind == 0) {
    spfft_nd(p->rank, p->dims, p->sign, p->in, p->out, p->nthreads);
    return;
  }
  const int n = p->dims[0];
  if (p->in != p->out) {
    for (long h = 0; h < p->howmany; h++)
      for (long i = 0; i < n; i++)
        p->out[h * p->odist + i * p->ostride] = p->in[h * p->idist + i * p->istride];
  }
  spfft_lines(p->line, p->sign, p->out, p->howmany, p->ostride, p->odist, p->nthreads);
}

void fftwf_destroy_plan(fftwf_plan p) {
  if (!p) return;
  spfft_plan_destroy(p->owned);
  free(p);
}
