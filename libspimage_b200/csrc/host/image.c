/*
 * Image and matrix lifecycle helpers of the phasing path (host C).
 * Behaviour follows the reference: src/linear_alg.c:84-125 (calloc'd
 * matrices), src/image_util.c:1223-1300 (alloc/duplicate/free),
 * :2322-2326 (memcpy), :1035-1067 (dephase/rephase), :120-127 (sp_srand,
 * p_drand48 over glibc rand()).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "spimage.h"

sp_3matrix *_sp_3matrix_alloc(unsigned int nx, unsigned int ny, unsigned int nz, const char *file, int line) {
  (void)file; (void)line;
  sp_3matrix *m = (sp_3matrix *)malloc(sizeof(sp_3matrix));
  m->x = nx; m->y = ny; m->z = nz;
  m->data = (real *)calloc((size_t)nx * ny * nz, sizeof(real));
  return m;
}

sp_i3matrix *_sp_i3matrix_alloc(unsigned int nx, unsigned int ny, unsigned int nz, const char *file, int line) {
  (void)file; (void)line;
  sp_i3matrix *m = (sp_i3matrix *)malloc(sizeof(sp_i3matrix));
  m->x = nx; m->y = ny; m->z = nz;
  m->data = (int *)calloc((size_t)nx * ny * nz, sizeof(int));
  return m;
}

sp_c3matrix *_sp_c3matrix_alloc(unsigned int nx, unsigned int ny, unsigned int nz, const char *file, int line) {
  (void)file; (void)line;
  sp_c3matrix *m = (sp_c3matrix *)malloc(sizeof(sp_c3matrix));
  m->x = nx; m->y = ny; m->z = nz;
  m->data = (Complex *)calloc((size_t)nx * ny * nz, sizeof(Complex));
  return m;
}

void _sp_3matrix_free(sp_3matrix *m, const char *file, int line) {
  (void)file; (void)line;
  if (!m) return;
  free(m->data);
  free(m);
}
void _sp_i3matrix_free(sp_i3matrix *m, const char *file, int line) {
  (void)file; (void)line;
  if (!m) return;
  free(m->data);
  free(m);
}
void _sp_c3matrix_free(sp_c3matrix *m, const char *file, int line) {
  (void)file; (void)line;
  if (!m) return;
  free(m->data);
  free(m);
}

Image *_sp_image_alloc(int x, int y, int z, const char *file, int line) {
  if (x < 1 || y < 1 || z < 1) {
    fprintf(stderr, "Dimensions must be positive integers\n");
    abort();
  }
  Image *r = (Image *)malloc(sizeof(Image));
  r->detector = (Detector *)calloc(1, sizeof(Detector));
  r->detector->image_center[0] = (x - 1) / 2.0;
  r->detector->image_center[1] = (y - 1) / 2.0;
  r->detector->image_center[2] = (z - 1) / 2.0;
  r->detector->orientation = NULL;
  r->mask = _sp_i3matrix_alloc(x, y, z, file, line);
  r->image = _sp_c3matrix_alloc(x, y, z, file, line);
  r->scaled = 0;
  r->shifted = 0;
  r->phased = 0;
  r->rec_coords = NULL;
  r->num_dimensions = z == 1 ? SP_2D : SP_3D;
  return r;
}

Image *_sp_image_duplicate(const Image *in, int flags, const char *file, int line) {
  Image *r = (Image *)malloc(sizeof(Image));
  memcpy(r, in, sizeof(Image));
  r->detector = (Detector *)malloc(sizeof(Detector));
  memcpy(r->detector, in->detector, sizeof(Detector));
  r->image = _sp_c3matrix_alloc(in->image->x, in->image->y, in->image->z, file, line);
  if (flags & SP_COPY_DATA)
    memcpy(r->image->data, in->image->data, sizeof(Complex) * (size_t)sp_image_size(in));
  r->mask = _sp_i3matrix_alloc(in->image->x, in->image->y, in->image->z, file, line);
  if (flags & SP_COPY_MASK) memcpy(r->mask->data, in->mask->data, sizeof(int) * (size_t)sp_image_size(in));
  return r;
}

void _sp_image_free(Image *in, const char *file, int line) {
  if (!in) return;
  _sp_c3matrix_free(in->image, file, line);
  _sp_i3matrix_free(in->mask, file, line);
  free(in->detector);
  free(in);
}

void sp_image_memcpy(Image *dst, const Image *src) {
  memcpy(dst->mask->data, src->mask->data, sizeof(int) * (size_t)sp_image_size(src));
  memcpy(dst->image->data, src->image->data, sizeof(Complex) * (size_t)sp_image_size(src));
  memcpy(dst->detector, src->detector, sizeof(Detector));
}

void sp_image_fill(Image *a, Complex value) {
  const long long n = sp_image_size(a);
  for (long long i = 0; i < n; i++) a->image->data[i] = value;
}

/* complex multiply by (value, 0), as src/image_util.c:1967-1970 */
void sp_image_scale(Image *img, real value) {
  const long long n = sp_image_size(img);
  for (long long i = 0; i < n; i++) {
    const Complex a = img->image->data[i];
    img->image->data[i].re = a.re * value - a.im * 0.0f;
    img->image->data[i].im = a.re * 0.0f + value * a.im;
  }
}

void sp_image_dephase(Image *img) {
  img->phased = 0;
  const long long n = sp_image_size(img);
  for (long long i = 0; i < n; i++) {
    img->image->data[i].re = sp_cabs(img->image->data[i]);
    img->image->data[i].im = 0;
  }
}

void sp_srand(int i) { srand((unsigned)i); }

real p_drand48(void) { return (real)(((double)rand()) / (double)RAND_MAX); }

/* n values of p_drand48() into out[], leaving the C library's rand() state
 * exactly where n calls of rand() would leave it.  glibc's rand() is its
 * random() generator: after srand() an additive feedback generator of degree
 * 31 and separation 3 (x[i] = x[i-31] + x[i-3] mod 2^32, output x[i] >> 1).
 * setstate() swaps in another state array and returns the current one, whose
 * leading word then encodes the generator type (mod 5) and the position of
 * its rear pointer (div 5).  When the current state has that form, the values
 * are generated here (no lock and call per value) and the advanced state is
 * handed back with setstate(); otherwise rand() is called n times.
 *
 * Two bulk draws never overlap: a process-wide mutex covers the span from
 * the first setstate() to the restoring one, so a second draw cannot take
 * the stand-in state for the real one and leave the generator on it.  If
 * setstate() nevertheless hands back the stand-in (another caller swapped
 * it in), the real state is not ours to restore and the per-value loop is
 * used.  Outside callers of rand()/srand() during a bulk draw act on the
 * stand-in (the drawn values and the final state are the ones above); such
 * concurrent use interleaves unpredictably with a per-value rand() loop
 * too.  The state layout is glibc's: other C libraries take the per-value
 * loop.  No thread of this library calls rand() (the server draws its
 * starts on the device). */
static void drand_fill(real *out, long long n) {
#if defined(__GLIBC__)
  enum { MAX_TYPES = 5, TYPE_3 = 3, DEG = 31, SEP = 3 };
  static pthread_mutex_t mu = PTHREAD_MUTEX_INITIALIZER;
  static int32_t holder[DEG + 2]; /* leading word 0: a valid degree-0 state while ours is out */
  pthread_mutex_lock(&mu);
  int32_t *cur = (int32_t *)setstate((char *)holder);
  if (cur && cur != holder) {
    const int32_t word = cur[0];
    if (word >= 0 && word % MAX_TYPES == TYPE_3 && word / MAX_TYPES < DEG) {
      int32_t *x = cur + 1;
      int r = word / MAX_TYPES, f = (r + SEP) % DEG;
      for (long long i = 0; i < n; i++) {
        const uint32_t val = (uint32_t)x[f] + (uint32_t)x[r];
        x[f] = (int32_t)val;
        out[i] = (real)(((double)(int)(val >> 1)) / (double)RAND_MAX);
        f = f + 1 == DEG ? 0 : f + 1;
        r = r + 1 == DEG ? 0 : r + 1;
      }
      cur[0] = MAX_TYPES * r + TYPE_3;
      setstate((char *)cur);
      pthread_mutex_unlock(&mu);
      return;
    }
    setstate((char *)cur);
  }
  pthread_mutex_unlock(&mu);
#endif
  for (long long i = 0; i < n; i++) out[i] = p_drand48();
}

/* Random-phase rephasing, split so that the libm work runs on several host
 * threads: the phases are drawn first, in pixel order from the one rand()
 * sequence as the reference draws them; then each pixel's
 * (cos(phase) * |v|, sin(phase) * |v|) is evaluated with the same double
 * libm calls and roundings, on whichever thread -- the same bits. */
typedef struct {
  Complex *data;
  const real *phase;
  long long i0, i1;
} rephase_span;

static void *rephase_worker(void *arg) {
  const rephase_span *s = (const rephase_span *)arg;
  for (long long i = s->i0; i < s->i1; i++) {
    const real phase = s->phase[i];
    const real amp = sp_cabs(s->data[i]);
    s->data[i].re = cos(phase) * amp;
    s->data[i].im = sin(phase) * amp;
  }
  return NULL;
}

#define REPHASE_MAX_THREADS 32
static void rephase_parallel(Complex *data, const real *phase, long long n) {
  long long nt = n >= (1 << 16) ? sysconf(_SC_NPROCESSORS_ONLN) : 1;
  if (nt < 1) nt = 1;
  if (nt > REPHASE_MAX_THREADS) nt = REPHASE_MAX_THREADS;
  pthread_t th[REPHASE_MAX_THREADS];
  rephase_span span[REPHASE_MAX_THREADS];
  int started[REPHASE_MAX_THREADS] = {0};
  for (long long t = 0; t < nt; t++) {
    span[t].data = data;
    span[t].phase = phase;
    span[t].i0 = n * t / nt;
    span[t].i1 = n * (t + 1) / nt;
    if (t > 0) started[t] = pthread_create(&th[t], NULL, rephase_worker, &span[t]) == 0;
  }
  rephase_worker(&span[0]);
  for (long long t = 1; t < nt; t++) {
    if (started[t]) pthread_join(th[t], NULL);
    else rephase_worker(&span[t]); /* no thread: do the span here */
  }
}

void sp_image_rephase(Image *img, int type) {
  img->phased = 1;
  const long long n = sp_image_size(img);
  if (type == SP_ZERO_PHASE) {
    for (long long i = 0; i < n; i++) img->image->data[i] = sp_cinit(sp_cabs(img->image->data[i]), 0);
  } else if (type == SP_RANDOM_PHASE) {
    real *phase = (real *)malloc(sizeof(real) * (size_t)(n > 0 ? n : 1));
    if (!phase) { /* no scratch: one pass, as the reference */
      for (long long i = 0; i < n; i++) {
        const real ph = p_drand48() * 3.14159265358979323846 * 2;
        const real amp = sp_cabs(img->image->data[i]);
        img->image->data[i].re = cos(ph) * amp;
        img->image->data[i].im = sin(ph) * amp;
      }
      return;
    }
    drand_fill(phase, n);
    for (long long i = 0; i < n; i++) phase[i] = phase[i] * 3.14159265358979323846 * 2;
    rephase_parallel(img->image->data, phase, n);
    free(phase);
  }
}

/* ---- FFI helpers: sp_smap's constructors are static inline in map.h, so a
 * foreign-function binding (ctypes, cffi) has no symbol to call; these give
 * it one. ---- */
sp_smap *spb_smap_create(int n, const real *keys, const real *values) {
  sp_smap *m = sp_smap_alloc(n > 0 ? (unsigned)n : 1u);
  for (int i = 0; i < n; i++) sp_smap_insert(m, keys[i], values[i]);
  return m;
}
void spb_smap_free(sp_smap *m) { sp_smap_free(m); }
real spb_smap_interpolate(sp_smap *m, real x) { return sp_smap_interpolate(m, x); }
