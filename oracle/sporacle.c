/*
 * sporacle -- CPU restatement of the reference phasing engine (test
 * infrastructure; see sporacle.h).  Types follow the reference's
 * single-precision build: `real` is float, the reference's double-valued
 * library calls (sqrt, pow, exp, cos, sin) are kept double and rounded where
 * the reference assigns to float.  Built with -ffp-contract=off.
 */
#include "sporacle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MAXKEYS 64
#define MAXSUP 8

typedef struct {
  int n;
  float keys[MAXKEYS], values[MAXKEYS];
} smap;

typedef struct {
  int type;
  smap blur, sel;
  int close_size;        /* close: dilations, then as many erosions */
  float *tmpl_abs;       /* template: |blur of the initial support| per pixel */
  float *tmpl_sorted;    /* template: the same values, descending */
  float tmpl_area;       /* template: fraction of the initial support's pixels */
} supalg;

struct spo_phaser {
  int nx, ny, nz;
  long n;
  float *amp, *amp_min, *amp_max;
  spfft_cpx *phased_amp;
  int *flags;
  int objective;
  int alg, constraints;
  smap beta;
  float gamma1, gamma2;
  int nsup, sup_period;
  supalg sup[MAXSUP];
  int iteration;
  spfft_cpx *g0, *g1, *gp;
  int nthreads;
};

/* ---------- helpers ---------- */

/* glibc rand()-based uniform, src/image_util.c:120-127 (sp_srand, p_drand48) */
void spo_srand(int seed) { srand((unsigned)seed); }
static float drand(void) { return (float)(((double)rand()) / (double)RAND_MAX); }

/* sp_cabs, include/spimage/linear_alg.h:163-165 */
static inline float cabsf_ref(spfft_cpx a) { return (float)sqrt((double)(a.im * a.im + a.re * a.re)); }

/* sp_image_scale by (float)(1/N) as a complex multiply by (v,0),
 * src/image_util.c:1967-1970 + linear_alg.h:196-201,1435-1440 */
static void scale_cmul(spfft_cpx *a, long n, float v) {
  for (long i = 0; i < n; i++) {
    const float re = a[i].re, im = a[i].im;
    a[i].re = re * v - im * 0.0f;
    a[i].im = re * 0.0f + v * im;
  }
}

static void fft3(const spo_phaser *ph, int sign, const spfft_cpx *in, spfft_cpx *out) {
  const int dims[3] = {ph->nz, ph->ny, ph->nx};
  spfft_nd(3, dims, sign, in, out, ph->nthreads);
}

void spo_fft(int nx, int ny, int nz, int sign, const spfft_cpx *in, spfft_cpx *out) {
  const int dims[3] = {nz, ny, nx};
  spfft_nd(3, dims, sign, in, out, 1);
}

/* Cubic-Bezier schedule, include/spimage/map.h:103-141 and
 * src/support_update.c:402-440.  Same mixed float/double arithmetic. */
float spo_bezier(int nkeys, const float *keys, const float *values, float x) {
  int idx;
  for (idx = 0; idx < nkeys; idx++)
    if (x < keys[idx]) break;
  if (idx == 0) return values[0];
  if (idx == nkeys) return values[nkeys - 1];
  const float p0y = values[idx - 1], p0x = keys[idx - 1];
  const float p3y = values[idx], p3x = keys[idx];
  const double root =
      pow((double)pow(p0x - p3x, 4) * (6 * p0x * p3x - 16 * p0x * x - 16 * p3x * x + 5 * pow(p0x, 2) +
                                       5 * pow(p3x, 2) + 16 * pow(x, 2)),
          0.5);
  const double cub = 8 * p0x * p3x * x - 2 * p3x * pow(p0x, 2) - 4 * x * pow(p0x, 2) + 2 * pow(p0x, 3) -
                     2 * p0x * pow(p3x, 2) - 4 * x * pow(p3x, 2) + 2 * pow(p3x, 3) + root;
  const float t =
      (2 - 2 * (p0x - p3x) * pow(cub, -0.3333333333333333) + 2 * pow(p0x - p3x, -1) * pow(cub, 0.3333333333333333)) /
      4.;
  return 3 * p0y * t * pow(1 - t, 2) + p0y * pow(1 - t, 3) + 3 * p3y * (1 - t) * pow(t, 2) + p3y * pow(t, 3);
}

static float smap_at(const smap *m, int iteration) { return spo_bezier(m->n, m->keys, m->values, (float)iteration); }

static void smap_set(smap *m, int n, const float *k, const float *v) {
  if (n > MAXKEYS) n = MAXKEYS;
  m->n = n;
  for (int i = 0; i < n; i++) { m->keys[i] = k[i]; m->values[i] = v[i]; }
}

/* ---------- construction ---------- */

spo_phaser *spo_create(int nx, int ny, int nz) {
  spo_phaser *ph = (spo_phaser *)calloc(1, sizeof(spo_phaser));
  ph->nx = nx; ph->ny = ny; ph->nz = nz;
  ph->n = (long)nx * ny * nz;
  ph->flags = (int *)calloc((size_t)ph->n, sizeof(int));
  ph->nthreads = 1;
  return ph;
}

void spo_destroy(spo_phaser *ph) {
  if (!ph) return;
  spo_clear_support_updates(ph);
  free(ph->amp); free(ph->amp_min); free(ph->amp_max); free(ph->phased_amp);
  free(ph->flags); free(ph->g0); free(ph->g1); free(ph->gp);
  free(ph);
}

void spo_set_threads(spo_phaser *ph, int nthreads) { ph->nthreads = nthreads < 1 ? 1 : nthreads; }

/* sp_phaser_set_amplitudes, src/phasing.c:294-333 */
void spo_set_amplitudes(spo_phaser *ph, const float *amp, const int *mask) {
  if (!ph->amp) ph->amp = (float *)malloc(sizeof(float) * (size_t)ph->n);
  for (long i = 0; i < ph->n; i++) {
    ph->amp[i] = amp[i];
    if (mask[i]) ph->flags[i] |= SPO_MEASURED;
    else ph->flags[i] &= ~SPO_MEASURED;
  }
}

/* sp_phaser_set_amplitudes_margins, src/phasing.c:335-363 */
void spo_set_amplitudes_margins(spo_phaser *ph, const float *amp_min, const float *amp_max) {
  if (!ph->amp_min) ph->amp_min = (float *)malloc(sizeof(float) * (size_t)ph->n);
  if (!ph->amp_max) ph->amp_max = (float *)malloc(sizeof(float) * (size_t)ph->n);
  memcpy(ph->amp_min, amp_min, sizeof(float) * (size_t)ph->n);
  memcpy(ph->amp_max, amp_max, sizeof(float) * (size_t)ph->n);
}

/* sp_phaser_set_phased_amplitudes, src/phasing.c:235-269 */
void spo_set_phased_amplitudes(spo_phaser *ph, const spfft_cpx *pa, const int *mask) {
  if (!ph->phased_amp) ph->phased_amp = (spfft_cpx *)malloc(sizeof(spfft_cpx) * (size_t)ph->n);
  for (long i = 0; i < ph->n; i++) {
    ph->phased_amp[i] = pa[i];
    if (mask[i]) ph->flags[i] |= SPO_MEASURED;
    else ph->flags[i] &= ~SPO_MEASURED;
  }
}

void spo_set_objective(spo_phaser *ph, int objective) { ph->objective = objective; }

/* sp_phaser_set_support / sp_phaser_init_support with an image, src/phasing.c:207-232,728-743 */
void spo_set_support(spo_phaser *ph, const float *support_real) {
  for (long i = 0; i < ph->n; i++) {
    if (support_real[i] != 0.0f) ph->flags[i] |= SPO_INSIDE;
    else ph->flags[i] &= ~SPO_INSIDE;
  }
}

/* sp_c3matrix_max: first maximum of sp_cabs, include/spimage/linear_alg.h:1974-1989 */
static float max_abs(const spfft_cpx *a, long n) {
  float m = cabsf_ref(a[0]);
  for (long i = 1; i < n; i++) {
    const float v = cabsf_ref(a[i]);
    if (v > m) m = v;
  }
  return m;
}

/* SpSupportFromPatterson, src/phasing.c:744-763 */
void spo_init_support_patterson(spo_phaser *ph, float value) {
  spfft_cpx *tmp = (spfft_cpx *)malloc(sizeof(spfft_cpx) * (size_t)ph->n);
  for (long i = 0; i < ph->n; i++) { tmp[i].re = ph->amp[i] * ph->amp[i]; tmp[i].im = 0; }
  fft3(ph, +1, tmp, tmp);
  const float thr = max_abs(tmp, ph->n) * value;
  for (long i = 0; i < ph->n; i++) {
    if (cabsf_ref(tmp[i]) > thr) ph->flags[i] |= SPO_INSIDE;
    else ph->flags[i] &= ~SPO_INSIDE;
  }
  free(tmp);
}

/* sp_phasing_{hio,raar,er,diff_map}_alloc, src/phasing.c:16-76 */
void spo_set_algorithm(spo_phaser *ph, int type, int nbeta, const float *beta_keys, const float *beta_values,
                       float gamma1, float gamma2, int constraints) {
  ph->alg = type;
  ph->constraints = constraints;
  if (nbeta > 0) smap_set(&ph->beta, nbeta, beta_keys, beta_values);
  if (type == SPO_DIFFMAP) {
    if (isinf(gamma1)) {
      const float beta = smap_at(&ph->beta, 0);
      const float sigma = 0.1f;
      ph->gamma1 = -(4 + (2 + beta) * sigma + beta * sigma * sigma) / (beta * (4 - sigma + sigma * sigma));
      ph->gamma2 = (3 - beta) / (2 * beta);
    } else {
      ph->gamma1 = gamma1;
      ph->gamma2 = gamma2;
    }
  }
}

float spo_dm_gamma(spo_phaser *ph, int which) { return which == 1 ? ph->gamma1 : ph->gamma2; }

void spo_clear_support_updates(spo_phaser *ph) {
  for (int s = 0; s < ph->nsup; s++) {
    free(ph->sup[s].tmpl_abs);
    free(ph->sup[s].tmpl_sorted);
  }
  ph->nsup = 0;
}

/* sp_support_{threshold,area,static}_alloc + sp_support_array_{init,append},
 * src/support_update.c:7-42,95-108,458-487 */
void spo_add_support_update(spo_phaser *ph, int type, int period, int nblur, const float *blur_keys,
                            const float *blur_values, int nsel, const float *sel_keys, const float *sel_values) {
  if (ph->nsup >= MAXSUP) return;
  supalg *s = &ph->sup[ph->nsup++];
  memset(s, 0, sizeof(*s));
  s->type = type;
  if (nblur > 0) smap_set(&s->blur, nblur, blur_keys, blur_values);
  if (nsel > 0) smap_set(&s->sel, nsel, sel_keys, sel_values);
  ph->sup_period = period;
}

/* sp_support_close_alloc, src/support_update.c:110-125 */
void spo_add_support_close(spo_phaser *ph, int period, int size) {
  if (ph->nsup >= MAXSUP) return;
  supalg *s = &ph->sup[ph->nsup++];
  memset(s, 0, sizeof(*s));
  s->type = SPO_SUP_CLOSE;
  s->close_size = size;
  ph->sup_period = period;
}

/* sp_support_centre_image_alloc, src/support_update.c:44-49 */
void spo_add_support_centre(spo_phaser *ph, int period) {
  if (ph->nsup >= MAXSUP) return;
  supalg *s = &ph->sup[ph->nsup++];
  memset(s, 0, sizeof(*s));
  s->type = SPO_SUP_CENTRE;
  ph->sup_period = period;
}

static int desc_float(const void *a, const void *b) {
  const float x = *(const float *)a, y = *(const float *)b;
  return x < y ? 1 : (x == y ? 0 : -1);
}

/* sp_support_template_alloc, src/support_update.c:51-84: the initial support
 * blurred once; its |.| values kept in pixel order and sorted descending; the
 * fraction of nonzero support pixels accumulated in float. */
void spo_add_support_template(spo_phaser *ph, int period, const float *support_real, float blur_radius, int narea,
                              const float *area_keys, const float *area_values) {
  if (ph->nsup >= MAXSUP) return;
  const long n = ph->n;
  supalg *s = &ph->sup[ph->nsup++];
  memset(s, 0, sizeof(*s));
  s->type = SPO_SUP_TEMPLATE;
  smap_set(&s->sel, narea, area_keys, area_values);
  spfft_cpx *in = (spfft_cpx *)malloc(sizeof(spfft_cpx) * (size_t)n);
  spfft_cpx *blur = (spfft_cpx *)malloc(sizeof(spfft_cpx) * (size_t)n);
  float area = 0.0f;
  for (long i = 0; i < n; i++) {
    in[i].re = support_real[i];
    in[i].im = 0.0f;
    if (support_real[i] != 0.0f) area += 1.0f;
  }
  s->tmpl_area = area / (float)n;
  spo_gaussian_blur(ph->nx, ph->ny, ph->nz, in, blur_radius, blur);
  s->tmpl_abs = (float *)malloc(sizeof(float) * (size_t)n);
  s->tmpl_sorted = (float *)malloc(sizeof(float) * (size_t)n);
  for (long i = 0; i < n; i++) s->tmpl_abs[i] = s->tmpl_sorted[i] = cabsf_ref(blur[i]);
  qsort(s->tmpl_sorted, (size_t)n, sizeof(float), desc_float);
  free(in);
  free(blur);
  ph->sup_period = period;
}

/* ---------- model initialisation, src/phasing.c:606-724 ---------- */

static void alloc_iterates(spo_phaser *ph) {
  if (!ph->g0) ph->g0 = (spfft_cpx *)malloc(sizeof(spfft_cpx) * (size_t)ph->n);
  if (!ph->g1) ph->g1 = (spfft_cpx *)malloc(sizeof(spfft_cpx) * (size_t)ph->n);
  if (!ph->gp) ph->gp = (spfft_cpx *)malloc(sizeof(spfft_cpx) * (size_t)ph->n);
}

int spo_init_model(spo_phaser *ph, int flags, const spfft_cpx *user_model) {
  const long n = ph->n;
  spfft_cpx *model = (spfft_cpx *)calloc((size_t)n, sizeof(spfft_cpx));
  if (user_model) {
    memcpy(model, user_model, sizeof(spfft_cpx) * (size_t)n);
  } else if (flags & SPO_RANDOM_PHASES) {
    /* amplitudes with random phases (src/image_util.c:1044-1067), then IFFT / N */
    for (long i = 0; i < n; i++) {
      const float phase = drand() * 3.14159265358979323846 * 2;
      spfft_cpx a = {ph->amp[i], 0.0f};
      const float amp = cabsf_ref(a);
      model[i].re = cos(phase) * amp;
      model[i].im = sin(phase) * amp;
    }
    fft3(ph, +1, model, model);
    scale_cmul(model, n, (float)(1.0 / (double)n));
  } else if (flags & SPO_ZERO_PHASES) {
    for (long i = 0; i < n; i++) {
      spfft_cpx a = {ph->amp[i], 0.0f};
      model[i].re = cabsf_ref(a);
      model[i].im = 0.0f;
    }
    fft3(ph, +1, model, model);
    scale_cmul(model, n, (float)(1.0 / (double)n));
  } else if (flags & SPO_RANDOM_VALUES) {
    double sum = 0;
    for (long i = 0; i < n; i++) sum += ph->amp[i] * ph->amp[i];
    sum /= n;
    for (long i = 0; i < n; i++) {
      /* gcc evaluates sp_cinit(p_drand48()-0.5, p_drand48()-0.5) right to left */
      const float im = (float)(drand() - 0.5);
      const float re = (float)(drand() - 0.5);
      model[i].re = re;
      model[i].im = im;
    }
    double msum = 0;
    for (long i = 0; i < n; i++) msum += model[i].im * model[i].im + model[i].re * model[i].re;
    const float model_sum = (float)msum;
    scale_cmul(model, n, (float)sqrt(sum / model_sum));
  } else {
    free(model);
    return -3;
  }
  if (flags & SPO_MASKED_OUT_ZEROED) {
    fft3(ph, -1, model, model);
    for (long i = 0; i < n; i++)
      if ((ph->flags[i] & SPO_MEASURED) == 0) { model[i].re = 0; model[i].im = 0; }
    fft3(ph, +1, model, model);
    scale_cmul(model, n, (float)(1.0 / (double)n));
  }
  alloc_iterates(ph);
  memset(ph->g0, 0, sizeof(spfft_cpx) * (size_t)n);
  memcpy(ph->g1, model, sizeof(spfft_cpx) * (size_t)n);
  memset(ph->gp, 0, sizeof(spfft_cpx) * (size_t)n);
  free(model);
  return 0;
}

/* sp_phaser_set_model, src/phasing.c:189-204 */
void spo_set_model(spo_phaser *ph, const spfft_cpx *model) {
  alloc_iterates(ph);
  memcpy(ph->g1, model, sizeof(spfft_cpx) * (size_t)ph->n);
}

/* ---------- projections, src/phasing.c:1026-1109 ---------- */

static void apply_constraints(spo_phaser *ph, spfft_cpx *g, int c) {
  for (long i = 0; i < ph->n; i++) {
    if (!(ph->flags[i] & SPO_INSIDE)) continue;
    if (c & SPO_REAL) {
      g[i].im = 0;
    } else if (c & SPO_POS_REAL) {
      if (g[i].re < 0) g[i].re = (c & SPO_FLIP) ? fabsf(g[i].re) : 0;
      g[i].im = 0;
    } else if (c & SPO_POS_COMPLEX) {
      if (g[i].re < 0) g[i].re = (c & SPO_FLIP) ? fabsf(g[i].re) : 0;
      if (g[i].im < 0) g[i].im = (c & SPO_FLIP) ? fabsf(g[i].im) : 0;
    }
  }
}

static void fourier_constraints(spo_phaser *ph, spfft_cpx *G, int c) {
  if (c & SPO_CENTROSYM)
    for (long i = 0; i < ph->n; i++) G[i].im = 0;
}

static void module_projection(spo_phaser *ph, spfft_cpx *G, int c) {
  for (long i = 0; i < ph->n; i++) {
    if (!(ph->flags[i] & SPO_MEASURED)) continue;
    float m = 1.0f;
    if (!(c & SPO_MARGIN)) {
      m = ph->amp[i] / cabsf_ref(G[i]);
    } else {
      const float a = cabsf_ref(G[i]);
      if (a < ph->amp_min[i]) m = ph->amp_min[i] / a;
      else if (a > ph->amp_max[i]) m = ph->amp_max[i] / a;
    }
    if (isfinite(m)) {
      G[i].re = G[i].re * m;
      G[i].im = G[i].im * m;
    } else {
      G[i].re = ph->amp[i];
      G[i].im = 0;
    }
  }
}

/* the projection alone on caller arrays (element-level tests) */
void spo_module_projection(long n, spfft_cpx *G, const float *amp, const int *flags, int constraints) {
  spo_phaser tmp;
  memset(&tmp, 0, sizeof(tmp));
  tmp.n = n;
  tmp.amp = (float *)amp;
  tmp.flags = (int *)flags;
  module_projection(&tmp, G, constraints & ~SPO_MARGIN);
}

static void phased_amp_projection(spo_phaser *ph, spfft_cpx *G) {
  for (long i = 0; i < ph->n; i++)
    if (ph->flags[i] & SPO_MEASURED) G[i] = ph->phased_amp[i];
}

static void project_fourier(spo_phaser *ph, spfft_cpx *G) {
  if (ph->objective == 0) module_projection(ph, G, ph->constraints);
  else phased_amp_projection(ph, G);
}

static void swap_g(spo_phaser *ph) {
  spfft_cpx *t = ph->g0;
  ph->g0 = ph->g1;
  ph->g1 = t;
}

/* ER, HIO, RAAR: src/phasing.c:1111-1219 */
static void iterate_simple(spo_phaser *ph, int iterations) {
  const long n = ph->n;
  const float inv_n = (float)(1.0 / (double)n);
  for (int it = 0; it < iterations; it++) {
    const float beta = ph->alg == SPO_ER ? 0.0f : smap_at(&ph->beta, ph->iteration);
    swap_g(ph);
    fft3(ph, -1, ph->g0, ph->g1);
    fourier_constraints(ph, ph->g1, ph->constraints);
    project_fourier(ph, ph->g1);
    fft3(ph, +1, ph->g1, ph->gp);
    scale_cmul(ph->gp, n, inv_n);
    const float one_m2b = 1 - 2 * beta;
    for (long i = 0; i < n; i++) {
      if (ph->flags[i] & SPO_INSIDE) {
        ph->g1[i] = ph->gp[i];
      } else if (ph->alg == SPO_HIO) {
        ph->g1[i].re = ph->g0[i].re - ph->gp[i].re * beta;
        ph->g1[i].im = ph->g0[i].im - ph->gp[i].im * beta;
      } else if (ph->alg == SPO_RAAR) {
        ph->g1[i].re = ph->gp[i].re * one_m2b + ph->g0[i].re * beta;
        ph->g1[i].im = ph->gp[i].im * one_m2b + ph->g0[i].im * beta;
      } else {
        ph->g1[i].re = 0;
        ph->g1[i].im = 0;
      }
    }
    apply_constraints(ph, ph->g1, ph->constraints);
    ph->iteration++;
  }
}

/* Difference map: src/phasing.c:1222-1274 (+ f1 at :1262-1274) */
static void iterate_diff_map(spo_phaser *ph, int iterations) {
  const long n = ph->n;
  const float g1c = ph->gamma1, g2c = ph->gamma2;
  spfft_cpx *f1 = (spfft_cpx *)malloc(sizeof(spfft_cpx) * (size_t)n);
  for (int it = 0; it < iterations; it++) {
    const float beta = smap_at(&ph->beta, ph->iteration);
    swap_g(ph);
    fft3(ph, -1, ph->g0, ph->g1);
    fourier_constraints(ph, ph->g1, ph->constraints);
    for (long i = 0; i < n; i++) {
      if (ph->flags[i] & SPO_INSIDE) {
        f1[i] = ph->g0[i];
      } else {
        f1[i].re = -g1c * ph->g0[i].re;
        f1[i].im = -g1c * ph->g0[i].im;
      }
    }
    fft3(ph, -1, f1, f1);
    module_projection(ph, f1, ph->constraints);
    fft3(ph, +1, f1, f1);
    module_projection(ph, ph->g1, ph->constraints);
    fft3(ph, +1, ph->g1, ph->gp);
    const int size = (int)n;
    for (long i = 0; i < n; i++) {
      const spfft_cpx g0 = ph->g0[i], rho = ph->gp[i], pf = f1[i];
      spfft_cpx g;
      if (ph->flags[i] & SPO_INSIDE) {
        g.re = g0.re + (beta) * ((1 + g2c) * rho.re / size - g2c * g0.re);
        g.im = g0.im + (beta) * ((1 + g2c) * rho.im / size - g2c * g0.im);
      } else {
        g = g0;
      }
      g.re -= beta * pf.re / size;
      g.im -= beta * pf.im / size;
      ph->g1[i] = g;
    }
    apply_constraints(ph, ph->g1, ph->constraints);
    ph->iteration++;
  }
  free(f1);
}

/* ---------- support update, src/support_update.c + image_filter.c:80-90 ---------- */

/* dist_to_top_left, src/image_util.c:1012-1032 */
static float dist_top_left(long i, int nx, int ny, int nz) {
  const float z = (float)(i / ((long)ny * nx));
  const float y = (float)((i % ((long)ny * nx)) / nx);
  const float x = (float)(i % nx);
  float dx, dy, dz;
  if ((unsigned)nx - x < x) dx = (unsigned)nx - x; else dx = x;
  if ((unsigned)ny - y < y) dy = (unsigned)ny - y; else dy = y;
  if ((unsigned)nz - z < z) dz = (unsigned)nz - z; else dz = z;
  return (float)sqrt(pow(dx, 2) + pow(dy, 2) + pow(dz, 2));
}

/* sp_gaussian_blur, src/image_filter.c:80-90 */
void spo_gaussian_blur(int nx, int ny, int nz, const spfft_cpx *in, float radius, spfft_cpx *out) {
  const long n = (long)nx * ny * nz;
  const int dims[3] = {nz, ny, nx};
  spfft_nd(3, dims, -1, in, out, 1);
  for (long i = 0; i < n; i++) {
    const float cr = dist_top_left(i, nx, ny, nz) / ((float)nx);
    const float m = (float)(exp(-2. * pow(3.14159265358979323846, 2) * pow(cr, 2) * pow(radius, 2)) / ((float)n));
    const float re = out[i].re, im = out[i].im;
    out[i].re = re * m - im * 0.0f;
    out[i].im = re * 0.0f + m * im;
  }
  spfft_nd(3, dims, +1, out, out, 1);
}

static int desc_cmp(const void *a, const void *b) {
  const float x = *(const float *)a, y = *(const float *)b;
  return x < y ? 1 : (x == y ? 0 : -1);
}

/* area threshold: |blur| sorted descending, value at (int)(N*area),
 * src/support_update.c:143-144 */
float spo_area_threshold(long n, const spfft_cpx *blur, float area) {
  float *v = (float *)malloc(sizeof(float) * (size_t)n);
  for (long i = 0; i < n; i++) v[i] = cabsf_ref(blur[i]);
  qsort(v, (size_t)n, sizeof(float), desc_cmp);
  const float t = v[(int)((float)n * area)];
  free(v);
  return t;
}

static void support_from_threshold(spo_phaser *ph, const spfft_cpx *blur, float t) {
  for (long i = 0; i < ph->n; i++) {
    if (cabsf_ref(blur[i]) > t) ph->flags[i] |= SPO_INSIDE;
    else ph->flags[i] &= ~SPO_INSIDE;
  }
}

/* sp_support_close_update_support_cpu, src/support_update.c:225-290: `size`
 * dilations then `size` erosions of the support bit over the 6-neighbourhood;
 * neighbours outside the array are left out. */
static void support_close(spo_phaser *ph, int size) {
  const int nx = ph->nx, ny = ph->ny, nz = ph->nz;
  const long n = ph->n;
  int *a = (int *)malloc(sizeof(int) * (size_t)n), *b = (int *)malloc(sizeof(int) * (size_t)n);
  memcpy(a, ph->flags, sizeof(int) * (size_t)n);
  memcpy(b, ph->flags, sizeof(int) * (size_t)n);
  for (int pass = 0; pass < 2 * size; pass++) {
    const int dilate = pass < size;
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
          const long i = ((long)z * ny + y) * nx + x;
          int in;
          if (dilate) {
            in = (a[i] & SPO_INSIDE) || (x > 0 && (a[i - 1] & SPO_INSIDE)) || (x < nx - 1 && (a[i + 1] & SPO_INSIDE)) ||
                 (y > 0 && (a[i - nx] & SPO_INSIDE)) || (y < ny - 1 && (a[i + nx] & SPO_INSIDE)) ||
                 (z > 0 && (a[i - (long)nx * ny] & SPO_INSIDE)) || (z < nz - 1 && (a[i + (long)nx * ny] & SPO_INSIDE));
          } else {
            in = !(!(a[i] & SPO_INSIDE) || (x > 0 && !(a[i - 1] & SPO_INSIDE)) ||
                   (x < nx - 1 && !(a[i + 1] & SPO_INSIDE)) || (y > 0 && !(a[i - nx] & SPO_INSIDE)) ||
                   (y < ny - 1 && !(a[i + nx] & SPO_INSIDE)) || (z > 0 && !(a[i - (long)nx * ny] & SPO_INSIDE)) ||
                   (z < nz - 1 && !(a[i + (long)nx * ny] & SPO_INSIDE)));
          }
          b[i] = in ? (b[i] | SPO_INSIDE) : (b[i] & ~SPO_INSIDE);
        }
    int *t = a;
    a = b;
    b = t;
  }
  memcpy(ph->flags, a, sizeof(int) * (size_t)n);
  free(a);
  free(b);
}

/* sp_pixel_flags_translate_mask, src/image_util.c:3587-3611: the support bit
 * moves by (dx,dy,dz) with wrap-around, the other bits stay in place */
static void translate_support(spo_phaser *ph, int dx, int dy, int dz) {
  const int nx = ph->nx, ny = ph->ny, nz = ph->nz;
  int *t = (int *)calloc((size_t)ph->n, sizeof(int));
  while (dx < 0) dx += nx;
  while (dy < 0) dy += ny;
  while (dz < 0) dz += nz;
  for (int x = 0; x < nx; x++)
    for (int y = 0; y < ny; y++)
      for (int z = 0; z < nz; z++) {
        const int X = (x + dx) % nx, Y = (y + dy) % ny, Z = (z + dz) % nz;
        const int v1 = ph->flags[((long)z * ny + y) * nx + x];
        const long d = ((long)Z * ny + Y) * nx + X;
        const int v2 = ph->flags[d];
        t[d] = (v1 & SPO_INSIDE) ? (v2 | SPO_INSIDE) : (v2 & ~SPO_INSIDE);
      }
  memcpy(ph->flags, t, sizeof(int) * (size_t)ph->n);
  free(t);
}

static int inside_at(const spo_phaser *ph, int x, int y, int z) {
  return ph->flags[((long)z * ph->ny + y) * ph->nx + x] & SPO_INSIDE;
}

/* sp_support_centre_image_cpu, src/support_update.c:305-389.  The reference
 * also Fourier-translates ph->model, the phaser's cached host copy of the
 * model, which the next iteration does not read: only the support moves.
 * The centre of mass (src/linear_alg.c:444-473) is accumulated in float in
 * pixel order and truncated to int. */
static void support_centre(spo_phaser *ph) {
  const int nx = ph->nx, ny = ph->ny, nz = ph->nz;
  if (nz == 1) {
    for (int x = 0; x < nx; x++)
      if (inside_at(ph, x, (ny - 1) / 2, 0)) {
        translate_support(ph, 0, (ny - 1) / 2, 0);
        break;
      }
    for (int y = 0; y < ny; y++)
      if (inside_at(ph, (nx - 1) / 2, y, 0)) {
        translate_support(ph, (nx - 1) / 2, 0, 0);
        break;
      }
  } else {
    /* the break leaves only the inner loop */
    for (int y = 0; y < ny; y++)
      for (int z = 0; z < nz; z++)
        if (inside_at(ph, (nx - 1) / 2, y, z)) {
          translate_support(ph, (nx - 1) / 2, 0, 0);
          break;
        }
    for (int x = 0; x < nx; x++)
      for (int z = 0; z < nz; z++)
        if (inside_at(ph, x, (ny - 1) / 2, z)) {
          translate_support(ph, 0, (ny - 1) / 2, 0);
          break;
        }
    for (int x = 0; x < nx; x++)
      for (int y = 0; y < ny; y++)
        if (inside_at(ph, x, y, (nz - 1) / 2)) {
          translate_support(ph, 0, 0, (nz - 1) / 2);
          break;
        }
  }
  float c[3] = {0.0f, 0.0f, 0.0f};
  int sum = 0;
  long i = 0;
  for (int z = 0; z < nz; z++)
    for (int y = 0; y < ny; y++)
      for (int x = 0; x < nx; x++, i++)
        if (ph->flags[i] & SPO_INSIDE) {
          c[0] += (float)((x + (nx - 1) / 2) % nx);
          c[1] += (float)((y + (ny - 1) / 2) % ny);
          c[2] += (float)((z + (nz - 1) / 2) % nz);
          sum++;
        }
  if (sum) {
    c[0] /= (float)sum;
    c[1] /= (float)sum;
    c[2] /= (float)sum;
    c[0] -= (float)((nx - 1) / 2);
    c[1] -= (float)((ny - 1) / 2);
    c[2] -= (float)((nz - 1) / 2);
  }
  translate_support(ph, (int)(0 - c[0]), (int)(0 - c[1]), (int)(0 - c[2]));
}

/* sp_support_template_update_support_cpu, src/support_update.c:193-205: the
 * threshold is the sorted template value at (int)(N * area * original area)
 * (clamped to N-1 where the reference would read past the end) */
static void support_template(spo_phaser *ph, const supalg *a) {
  const float area = smap_at(&a->sel, ph->iteration);
  long k = (long)(int)((float)ph->n * area * a->tmpl_area);
  if (k >= ph->n) k = ph->n - 1;
  if (k < 0) k = 0;
  const float t = a->tmpl_sorted[k];
  for (long i = 0; i < ph->n; i++) {
    if (a->tmpl_abs[i] > t) ph->flags[i] |= SPO_INSIDE;
    else ph->flags[i] &= ~SPO_INSIDE;
  }
}

static void support_update(spo_phaser *ph) {
  const long n = ph->n;
  for (int s = 0; s < ph->nsup; s++) {
    const supalg *a = &ph->sup[s];
    if (a->type == SPO_SUP_CLOSE) {
      support_close(ph, a->close_size);
      continue;
    }
    if (a->type == SPO_SUP_CENTRE) {
      support_centre(ph);
      continue;
    }
    if (a->type == SPO_SUP_TEMPLATE) {
      support_template(ph, a);
      continue;
    }
    if (a->type != SPO_SUP_AREA && a->type != SPO_SUP_THRESHOLD) continue; /* static: nothing */
    const float radius = smap_at(&a->blur, ph->iteration);
    spfft_cpx *tmp = (spfft_cpx *)malloc(sizeof(spfft_cpx) * (size_t)n);
    spfft_cpx *blur = (spfft_cpx *)malloc(sizeof(spfft_cpx) * (size_t)n);
    for (long i = 0; i < n; i++) { tmp[i].re = cabsf_ref(ph->g1[i]); tmp[i].im = 0; }
    spo_gaussian_blur(ph->nx, ph->ny, ph->nz, tmp, radius, blur);
    float t;
    if (a->type == SPO_SUP_AREA) {
      const float area = smap_at(&a->sel, ph->iteration);
      t = spo_area_threshold(n, blur, area);
    } else {
      const float rel = smap_at(&a->sel, ph->iteration);
      t = max_abs(blur, n) * rel;
    }
    support_from_threshold(ph, blur, t);
    free(tmp);
    free(blur);
  }
}

/* sp_phaser_iterate, src/phasing.c:895-1024 */
int spo_iterate(spo_phaser *ph, int iterations) {
  if (!ph->alg) return -2;
  if (!ph->g1) return -3;
  if ((!ph->amp && ph->objective == 0) || (!ph->phased_amp && ph->objective == 1)) return -4;
  void (*step)(spo_phaser *, int) = ph->alg == SPO_DIFFMAP ? iterate_diff_map : iterate_simple;
  if (ph->nsup > 0) {
    while (iterations) {
      int to_update = ph->sup_period - 1 - ph->iteration % ph->sup_period;
      const int to_iterate = iterations < to_update ? iterations : to_update;
      step(ph, to_iterate);
      iterations -= to_iterate;
      to_update -= to_iterate;
      if (to_update == 0 && iterations > 0) {
        support_update(ph);
        ph->iteration++;
        iterations -= 1;
      }
    }
  } else if (iterations) {
    step(ph, iterations);
  }
  return 0;
}

int spo_iteration(const spo_phaser *ph) { return ph->iteration; }

void spo_get(const spo_phaser *ph, int which, spfft_cpx *out) {
  const spfft_cpx *src = which == 0 ? ph->g0 : (which == 1 ? ph->g1 : ph->gp);
  memcpy(out, src, sizeof(spfft_cpx) * (size_t)ph->n);
}

void spo_get_flags(const spo_phaser *ph, int *out) { memcpy(out, ph->flags, sizeof(int) * (size_t)ph->n); }

/* ---------- metrics, src/phasing.c:803-893 ---------- */

float spo_efourier(spo_phaser *ph, float *FcFo) {
  const long n = ph->n;
  spfft_cpx *F = (spfft_cpx *)malloc(sizeof(spfft_cpx) * (size_t)n);
  fft3(ph, -1, ph->g1, F);
  float den = 0, nom = 0, fden = 0, fnum = 0;
  for (long i = 0; i < n; i++) {
    const spfft_cpx a = {ph->amp[i], 0.0f};
    if (ph->flags[i] & SPO_MEASURED) {
      fnum += cabsf_ref(a);
      fden += cabsf_ref(F[i]);
      nom += pow(cabsf_ref(F[i]) - cabsf_ref(a), 2);
      den += pow(cabsf_ref(a), 2);
    } else {
      den += pow(cabsf_ref(F[i]), 2);
    }
  }
  free(F);
  if (FcFo) *FcFo = fnum / fden;
  return (float)sqrt(nom / den);
}

float spo_ereal(spo_phaser *ph) {
  float nom = 0, den = 0;
  for (long i = 0; i < ph->n; i++) {
    if (!(ph->flags[i] & SPO_INSIDE)) nom += pow(cabsf_ref(ph->gp[i]), 2);
    den += pow(cabsf_ref(ph->gp[i]), 2);
  }
  return (float)sqrt(nom / den);
}

float spo_support_fraction(spo_phaser *ph) {
  int c = 0;
  for (long i = 0; i < ph->n; i++)
    if (ph->flags[i] & SPO_INSIDE) c++;
  return (float)c / (float)ph->n;
}
