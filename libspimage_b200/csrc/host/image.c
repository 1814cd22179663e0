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
#include "host_internal.h"

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

/* glibc's rand() is its random() generator: after srand() an additive
 * feedback generator of degree 31 and separation 3 over 32-bit words,
 * x[k] = x[k-31] + x[k-3] (mod 2^32), whose output is x[k] >> 1.  Its state
 * is the last 31 words in a circular array with a front and a rear index;
 * setstate() swaps in another state array and returns the current one, whose
 * leading word then encodes the generator type (mod 5) and the rear index
 * (div 5).
 *
 * The recurrence is linear, so the word m steps after a window of 31
 * consecutive words w[0..30] is a fixed combination of them: with
 * z^m = c_0 + c_1 z + ... + c_30 z^30 modulo z^31 - z^28 - 1 (coefficients
 * mod 2^32), x[n+m] = sum_j c_j x[n+j].  A host thread can thus start
 * anywhere in the sequence: a random-phase start of n pixels is drawn by
 * several threads, each producing the words of its own span of pixels, and
 * the C library's state is advanced by n words -- the same values, in the
 * same pixel order, and the same state as n calls of rand(). */
enum { RNG_MAX_TYPES = 5, RNG_TYPE_3 = 3, RNG_DEG = 31, RNG_SEP = 3 };

/* a <- a * b mod (z^31 - z^28 - 1), coefficients mod 2^32 */
static void rng_poly_mulmod(uint32_t *a, const uint32_t *b) {
  uint32_t prod[2 * RNG_DEG - 1];
  memset(prod, 0, sizeof(prod));
  for (int i = 0; i < RNG_DEG; i++)
    for (int j = 0; j < RNG_DEG; j++) prod[i + j] += a[i] * b[j];
  /* z^k = z^(k-3) + z^(k-31) for k >= 31, highest terms first */
  for (int k = 2 * RNG_DEG - 2; k >= RNG_DEG; k--) {
    prod[k - RNG_SEP] += prod[k];
    prod[k - RNG_DEG] += prod[k];
  }
  memcpy(a, prod, sizeof(uint32_t) * RNG_DEG);
}

/* c <- c * z mod (z^31 - z^28 - 1) */
static void rng_poly_mulz(uint32_t *c) {
  const uint32_t top = c[RNG_DEG - 1];
  memmove(c + 1, c, sizeof(uint32_t) * (RNG_DEG - 1));
  c[0] = top;
  c[RNG_DEG - RNG_SEP] += top;
}

/* out[j] = x[n+m+j] (j = 0..30) from the window w[j] = x[n+j] */
static void rng_window_at(const uint32_t *w, long long m, uint32_t *out) {
  uint32_t c[RNG_DEG], base[RNG_DEG];
  memset(c, 0, sizeof(c));
  memset(base, 0, sizeof(base));
  c[0] = 1;    /* z^0 */
  base[1] = 1; /* z */
  for (long long e = m; e > 0; e >>= 1) {
    if (e & 1) rng_poly_mulmod(c, base);
    if (e > 1) {
      uint32_t sq[RNG_DEG];
      memcpy(sq, base, sizeof(sq));
      rng_poly_mulmod(base, sq);
    }
  }
  for (int j = 0; j < RNG_DEG; j++) {
    uint32_t v = 0;
    for (int i = 0; i < RNG_DEG; i++) v += c[i] * w[i];
    out[j] = v;
    rng_poly_mulz(c);
  }
}

/* Takes the C library's generator state when it has glibc's TYPE_3 form:
 * copies the window of its last 31 words into w[] and advances the state by
 * n words as n calls of rand() would.  Returns 0 (and leaves the state alone)
 * when the state has another form; the caller then calls rand() itself.
 *
 * A process-wide mutex covers the span from the first setstate() to the
 * restoring one, so two draws cannot take the stand-in state for the real one
 * and leave the generator on it.  If setstate() nevertheless hands back the
 * stand-in (another caller swapped it in), the real state is not ours to
 * advance and 0 is returned.  Outside callers of rand()/srand() during that
 * short span act on the stand-in; such concurrent use interleaves
 * unpredictably with a per-value rand() loop too.  No thread of this library
 * calls rand() (the server draws its starts on the device). */
static int rng_take(long long n, uint32_t *w) {
#if defined(__GLIBC__)
  static pthread_mutex_t mu = PTHREAD_MUTEX_INITIALIZER;
  static int32_t holder[RNG_DEG + 2]; /* leading word 0: a valid degree-0 state while ours is out */
  int ok = 0;
  pthread_mutex_lock(&mu);
  int32_t *cur = (int32_t *)setstate((char *)holder);
  if (cur && cur != holder) {
    const int32_t word = cur[0];
    if (word >= 0 && word % RNG_MAX_TYPES == RNG_TYPE_3 && word / RNG_MAX_TYPES < RNG_DEG) {
      int32_t *x = cur + 1;
      const int r = word / RNG_MAX_TYPES, f = (r + RNG_SEP) % RNG_DEG;
      /* slot f holds the oldest word, slot f + j the j-th after it */
      for (int j = 0; j < RNG_DEG; j++) w[j] = (uint32_t)x[(f + j) % RNG_DEG];
      /* after n words slot (f + n + j) holds the window at offset n */
      uint32_t fin[RNG_DEG];
      rng_window_at(w, n, fin);
      const int fn = (int)((f + n) % RNG_DEG);
      for (int j = 0; j < RNG_DEG; j++) x[(fn + j) % RNG_DEG] = (int32_t)fin[j];
      cur[0] = RNG_MAX_TYPES * (int32_t)((r + n) % RNG_DEG) + RNG_TYPE_3;
      ok = 1;
    }
    setstate((char *)cur);
  }
  pthread_mutex_unlock(&mu);
  return ok;
#else
  (void)n;
  (void)w;
  return 0;
#endif
}

/* ------------------------------------------------------------ host threads
 * Worker threads started on first use and kept for the process: a parallel
 * loop wakes them instead of creating threads per call (creating and joining
 * fifteen threads cost about 0.3 ms a call, several times per start).  One
 * loop at a time runs on the pool; a caller that finds it taken by another
 * host thread runs its spans on threads of its own.  The spans, and so the
 * results, are the same either way.  A child forked while the pool exists
 * starts with an empty one. */
#define SPB_POOL_MAX 32

static struct {
  pthread_mutex_t run; /* held by the caller whose loop is on the pool */
  pthread_mutex_t mu;
  pthread_cond_t go, done;
  int workers;                        /* started: ids 1..workers */
  unsigned long gen;                  /* loops posted */
  unsigned long born[SPB_POOL_MAX];   /* gen when worker id was started */
  int pending;                        /* workers still in the current loop */
  int nt;
  long long n;
  spb_span_fn fn;
  void *ctx;
} pool = {PTHREAD_MUTEX_INITIALIZER, PTHREAD_MUTEX_INITIALIZER, PTHREAD_COND_INITIALIZER,
          PTHREAD_COND_INITIALIZER, 0, 0, {0}, 0, 0, 0, NULL, NULL};

static void pool_after_fork_child(void) {
  pthread_mutex_init(&pool.run, NULL);
  pthread_mutex_init(&pool.mu, NULL);
  pthread_cond_init(&pool.go, NULL);
  pthread_cond_init(&pool.done, NULL);
  pool.workers = 0;
  pool.pending = 0;
}

static pthread_once_t pool_once = PTHREAD_ONCE_INIT;
static void pool_register_fork(void) { pthread_atfork(NULL, NULL, pool_after_fork_child); }

static void *pool_main(void *arg) {
  const int id = (int)(intptr_t)arg;
  pthread_mutex_lock(&pool.mu);
  unsigned long seen = pool.born[id];
  for (;;) {
    while (pool.gen == seen) pthread_cond_wait(&pool.go, &pool.mu);
    seen = pool.gen;
    if (id < pool.nt) {
      const spb_span_fn fn = pool.fn;
      void *ctx = pool.ctx;
      const long long n = pool.n, nt = pool.nt;
      pthread_mutex_unlock(&pool.mu);
      fn(ctx, id, n * id / nt, n * (id + 1) / nt);
      pthread_mutex_lock(&pool.mu);
      if (--pool.pending == 0) pthread_cond_signal(&pool.done);
    }
  }
  return NULL;
}

typedef struct {
  spb_span_fn fn;
  void *ctx;
  int t;
  long long i0, i1;
} par_span;

static void *par_worker(void *arg) {
  par_span *s = (par_span *)arg;
  s->fn(s->ctx, s->t, s->i0, s->i1);
  return NULL;
}

/* fn(ctx, t, i0, i1) for the nt contiguous spans of [0, n) */
static void run_spans(int nt, long long n, spb_span_fn fn, void *ctx) {
  if (nt <= 1) {
    fn(ctx, 0, 0, n);
    return;
  }
  if (nt > SPB_POOL_MAX) nt = SPB_POOL_MAX;
  if (pthread_mutex_trylock(&pool.run) == 0) {
    pthread_once(&pool_once, pool_register_fork);
    pthread_mutex_lock(&pool.mu);
    while (pool.workers < nt - 1) {
      pthread_t th;
      const int id = pool.workers + 1;
      pool.born[id] = pool.gen;
      if (pthread_create(&th, NULL, pool_main, (void *)(intptr_t)id) != 0) break;
      pthread_detach(th);
      pool.workers = id;
    }
    const int helpers = pool.workers < nt - 1 ? pool.workers : nt - 1;
    pool.nt = nt;
    pool.n = n;
    pool.fn = fn;
    pool.ctx = ctx;
    pool.pending = helpers;
    pool.gen++;
    pthread_cond_broadcast(&pool.go);
    pthread_mutex_unlock(&pool.mu);
    fn(ctx, 0, 0, n / nt);
    for (int t = helpers + 1; t < nt; t++) fn(ctx, t, n * t / nt, n * (t + 1) / nt); /* spans without a worker */
    pthread_mutex_lock(&pool.mu);
    while (pool.pending) pthread_cond_wait(&pool.done, &pool.mu);
    pthread_mutex_unlock(&pool.mu);
    pthread_mutex_unlock(&pool.run);
    return;
  }
  /* the pool is busy with another caller's loop */
  pthread_t th[SPB_POOL_MAX];
  par_span span[SPB_POOL_MAX];
  int started[SPB_POOL_MAX] = {0};
  for (int t = 0; t < nt; t++) {
    span[t].fn = fn;
    span[t].ctx = ctx;
    span[t].t = t;
    span[t].i0 = n * t / nt;
    span[t].i1 = n * (t + 1) / nt;
    if (t > 0) started[t] = pthread_create(&th[t], NULL, par_worker, &span[t]) == 0;
  }
  par_worker(&span[0]);
  for (int t = 1; t < nt; t++) {
    if (started[t]) pthread_join(th[t], NULL);
    else par_worker(&span[t]); /* no thread: run the span here */
  }
}

static int host_threads(long long n, long long min_n, int cap) {
  long long nt = n >= min_n ? sysconf(_SC_NPROCESSORS_ONLN) : 1;
  if (nt > cap) nt = cap;
  if (nt < 1) nt = 1;
  return (int)nt;
}

int spb_parallel_for(long long n, spb_span_fn fn, void *ctx) {
  const int nt = host_threads(n, 1 << 18, SPB_PAR_MAX);
  run_spans(nt, n, fn, ctx);
  return nt;
}

/* Random-phase rephasing of pixels [i0, i1): the words of draws i0.. come
 * from the window w of the 31 words before draw 0; each pixel's phase is
 * p_drand48() * 2 pi rounded to float and its value
 * (cos(phase) * |v|, sin(phase) * |v|) is evaluated with the same double libm
 * calls and roundings as the reference's loop -- on whichever thread, the
 * same bits. */
typedef struct {
  Complex *data;
  const uint32_t *w;
} rephase_job;

static void rephase_span(void *arg, int t, long long i0, long long i1) {
  (void)t;
  const rephase_job *s = (const rephase_job *)arg;
  uint32_t buf[RNG_DEG];
  rng_window_at(s->w, i0, buf); /* the 31 words before draw i0 */
  int f = 0, r = RNG_DEG - RNG_SEP;
  for (long long i = i0; i < i1; i++) {
    const uint32_t val = buf[f] + buf[r];
    buf[f] = val;
    f = f + 1 == RNG_DEG ? 0 : f + 1;
    r = r + 1 == RNG_DEG ? 0 : r + 1;
    const real u = (real)(((double)(int)(val >> 1)) / (double)RAND_MAX);
    const real phase = u * 3.14159265358979323846 * 2;
    const real amp = sp_cabs(s->data[i]);
    s->data[i].re = cos(phase) * amp;
    s->data[i].im = sin(phase) * amp;
  }
}

/* The phases alone: phase[i] = p_drand48() * 2 pi rounded to float, from the
 * same rand() words, in the same pixel order, leaving the generator where n
 * calls of rand() leave it -- the phases sp_image_rephase(SP_RANDOM_PHASE)
 * would use for an image of n pixels (drawn on all host threads). */
typedef struct {
  float *out;
  const uint32_t *w;
  int phases; /* 1: p_drand48() * 2 pi rounded to float, 0: p_drand48() */
} draw_job;

static void draw_span(void *arg, int t, long long i0, long long i1) {
  (void)t;
  const draw_job *s = (const draw_job *)arg;
  uint32_t buf[RNG_DEG];
  rng_window_at(s->w, i0, buf);
  int f = 0, r = RNG_DEG - RNG_SEP;
  for (long long i = i0; i < i1; i++) {
    const uint32_t val = buf[f] + buf[r];
    buf[f] = val;
    f = f + 1 == RNG_DEG ? 0 : f + 1;
    r = r + 1 == RNG_DEG ? 0 : r + 1;
    const real u = (real)(((double)(int)(val >> 1)) / (double)RAND_MAX);
    spb_stream_f32(&s->out[i], s->phases ? (real)(u * 3.14159265358979323846 * 2) : u);
  }
  spb_stream_fence(); /* the values are uploaded next */
}

/* n consecutive p_drand48() values (phases = 0) or phases (phases = 1) into
 * out[], drawn on the host threads from the words n calls of rand() would
 * return, the generator left where they leave it */
static void draw_parallel(float *out, long long n, int phases) {
  uint32_t w[RNG_DEG];
  if (n > 0 && rng_take(n, w)) {
    draw_job job = {out, w, phases};
    run_spans(host_threads(n, 1 << 18, SPB_POOL_MAX), n, draw_span, &job);
    return;
  }
  /* another generator layout: one rand() per value */
  for (long long i = 0; i < n; i++) {
    const real u = p_drand48();
    out[i] = phases ? (real)(u * 3.14159265358979323846 * 2) : u;
  }
}

void spb_random_uniforms(float *u, long long n) { draw_parallel(u, n, 0); }

void spb_random_phases(float *phase, long long n) { draw_parallel(phase, n, 1); }

void sp_image_rephase(Image *img, int type) {
  img->phased = 1;
  const long long n = sp_image_size(img);
  if (type == SP_ZERO_PHASE) {
    for (long long i = 0; i < n; i++) img->image->data[i] = sp_cinit(sp_cabs(img->image->data[i]), 0);
  } else if (type == SP_RANDOM_PHASE) {
    uint32_t w[RNG_DEG];
    if (n > 0 && rng_take(n, w)) {
      rephase_job job = {img->image->data, w};
      run_spans(host_threads(n, 1 << 16, SPB_POOL_MAX), n, rephase_span, &job);
      return;
    }
    /* another generator layout: one rand() per pixel, as the reference */
    for (long long i = 0; i < n; i++) {
      const real ph = p_drand48() * 3.14159265358979323846 * 2;
      const real amp = sp_cabs(img->image->data[i]);
      img->image->data[i].re = cos(ph) * amp;
      img->image->data[i].im = sin(ph) * amp;
    }
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
