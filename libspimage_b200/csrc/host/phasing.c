/*
 * SpPhaser API (host C) over the device layer (include/spimage/spb_device.h).
 *
 * Mirrors the reference's src/phasing.c: same entry points, argument meaning,
 * return codes and caching of host-side images per iteration.  The phasing
 * engine is always the GPU one; host copies of the inputs (amplitudes, pixel
 * flags, ...) are kept like the reference does and uploaded lazily before
 * device work.  Device errors are reported by return code (-8) and by
 * sp_phaser_last_error() instead of exit()/abort().
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "spimage.h"
#include "spimage/spb_device.h"
#include "host_internal.h"

#define FLAG_BITS ((unsigned)(SpPixelInsideSupport | SpPixelMeasuredAmplitude))

typedef struct {
  spb_ctx *ctx;
  int starts; /* independent reconstructions in the context (0 = 1) */
  int amp_dirty, margins_dirty, pamp_dirty;
  /* Pixel flags live on the host (ph->pixel_flags) and on the device.  The
   * host edits whole bit classes (every pixel's measured bit, or every
   * pixel's support bit); support updates change support bits on the
   * device.  Each side tracks the bits it holds newer values of, so that only
   * those cross: host_bits go up before the device uses the flags, dev_bits
   * come down before the host reads them.  The two sets never overlap. */
  unsigned flags_host_bits;
  unsigned flags_dev_bits;
  void *pinned_amp;    /* ph->amplitudes->data when page-locked */
  void *pinned_model;  /* ph->model->image->data when page-locked */
  Image *spare_model, *spare_change; /* the previous start's images while a new start is made */
} dev_state;

static char g_last_err[512];

const char *sp_phaser_last_error(void) { return g_last_err; }

static int dev_error(const char *where) {
  snprintf(g_last_err, sizeof(g_last_err), "%s: %s", where, spb_error_string());
  fprintf(stderr, "spimage-b200: %s\n", g_last_err);
  return -8;
}

static dev_state *state(SpPhaser *ph) {
  if (!ph->device) ph->device = calloc(1, sizeof(dev_state));
  return (dev_state *)ph->device;
}

/* A new start takes the model and model-change images off the phaser (the
 * phaser has no model until the start succeeds, as in the reference, which
 * frees them) and keeps them to reuse: a fresh 1024^2 image costs page faults
 * on its first download every start. */
static void release_model_images(SpPhaser *ph) {
  dev_state *s = state(ph);
  if (ph->model) {
    if (s->spare_model) sp_image_free(s->spare_model);
    s->spare_model = ph->model;
    ph->model = NULL;
  }
  if (ph->model_change) {
    if (s->spare_change) sp_image_free(s->spare_change);
    s->spare_change = ph->model_change;
    ph->model_change = NULL;
  }
}

static void free_spare_model_images(SpPhaser *ph) {
  dev_state *s = state(ph);
  if (s->spare_model) {
    if (s->pinned_model == s->spare_model->image->data) {
      spb_host_unregister(s->pinned_model);
      s->pinned_model = NULL;
    }
    sp_image_free(s->spare_model);
    s->spare_model = NULL;
  }
  if (s->spare_change) {
    sp_image_free(s->spare_change);
    s->spare_change = NULL;
  }
}

static int ensure_ctx(SpPhaser *ph) {
  dev_state *s = state(ph);
  if (s->ctx) return 0;
  if (!ph->nx) {
    snprintf(g_last_err, sizeof(g_last_err), "phaser dimensions are not set");
    return -8;
  }
  if (spb_ctx_create_batch(&s->ctx, ph->nx, ph->ny, ph->nz, s->starts > 0 ? s->starts : 1))
    return dev_error("device context");
  s->amp_dirty = ph->amplitudes != NULL;
  s->flags_host_bits = ph->pixel_flags != NULL ? FLAG_BITS : 0u; /* a fresh context has none */
  s->flags_dev_bits = 0;
  s->margins_dirty = ph->amplitudes_min != NULL;
  s->pamp_dirty = ph->phased_amplitudes != NULL;
  return 0;
}

/* pull the flag bits the device changed before the host reads the flags */
static int sync_flags_to_host(SpPhaser *ph) {
  dev_state *s = state(ph);
  if (!s->ctx || !s->flags_dev_bits || !ph->pixel_flags) return 0;
  if (spb_ctx_get_flags_bits(s->ctx, ph->pixel_flags->data, (int)s->flags_dev_bits))
    return dev_error("download pixel flags");
  s->flags_dev_bits = 0;
  return 0;
}

/* the host has just rewritten `bits` of every pixel's flags */
static void host_wrote_flags(SpPhaser *ph, unsigned bits) {
  dev_state *s = state(ph);
  s->flags_host_bits |= bits;
  s->flags_dev_bits &= ~bits;
}

/* the device has changed `bits` of the flags (support updates) */
static void device_wrote_flags(SpPhaser *ph, unsigned bits) { state(ph)->flags_dev_bits |= bits; }

/* need_flags = 0: the caller's device work reads no pixel flags, so edited
 * flag bits may wait for a later call (a new start is typically followed by
 * a new support before the iterations) */
static int sync_to_device_for(SpPhaser *ph, int need_flags) {
  if (ensure_ctx(ph)) return -8;
  dev_state *s = state(ph);
  if (s->amp_dirty && ph->amplitudes) {
    if (spb_ctx_set_amplitudes(s->ctx, ph->amplitudes->data)) return dev_error("upload amplitudes");
    s->amp_dirty = 0;
  }
  if (s->flags_host_bits && ph->pixel_flags && need_flags) {
    if (spb_ctx_set_flags_bits(s->ctx, ph->pixel_flags->data, (int)s->flags_host_bits))
      return dev_error("upload pixel flags");
    s->flags_host_bits = 0;
  }
  if (s->margins_dirty && ph->amplitudes_min && ph->amplitudes_max) {
    if (spb_ctx_set_margins(s->ctx, ph->amplitudes_min->data, ph->amplitudes_max->data))
      return dev_error("upload amplitude margins");
    s->margins_dirty = 0;
  }
  if (s->pamp_dirty && ph->phased_amplitudes) {
    if (spb_ctx_set_phased_amplitudes(s->ctx, (const float *)ph->phased_amplitudes->data))
      return dev_error("upload phased amplitudes");
    s->pamp_dirty = 0;
  }
  return 0;
}

static int sync_to_device(SpPhaser *ph) { return sync_to_device_for(ph, 1); }

/* ------------------------------------------------------------- algorithms */

/* phasing.c:16-45: gamma1 = INFINITY selects Elser's optimal gammas at beta(0) */
SpPhasingAlgorithm *sp_phasing_diff_map_alloc(sp_smap *beta, real gamma1, real gamma2,
                                              SpPhasingConstraints constraints) {
  SpPhasingAlgorithm *ret = (SpPhasingAlgorithm *)malloc(sizeof(SpPhasingAlgorithm));
  SpPhasingDiffMapParameters *p = (SpPhasingDiffMapParameters *)malloc(sizeof(SpPhasingDiffMapParameters));
  ret->type = SpDiffMap;
  p->beta = beta;
  if (isinf(gamma1)) {
    const real b = sp_smap_interpolate(p->beta, 0);
    const real sigma = 0.1;
    p->gamma1 = -(4 + (2 + b) * sigma + b * sigma * sigma) / (b * (4 - sigma + sigma * sigma));
    p->gamma2 = (3 - b) / (2 * b);
  } else {
    p->gamma1 = gamma1;
    p->gamma2 = gamma2;
  }
  p->constraints = constraints;
  ret->params = p;
  return ret;
}

static SpPhasingAlgorithm *beta_alg(SpPhasingAlgorithmType type, sp_smap *beta, SpPhasingConstraints c) {
  SpPhasingAlgorithm *ret = (SpPhasingAlgorithm *)malloc(sizeof(SpPhasingAlgorithm));
  SpPhasingHIOParameters *p = (SpPhasingHIOParameters *)malloc(sizeof(SpPhasingHIOParameters));
  ret->type = type;
  p->beta = beta;
  p->constraints = c;
  ret->params = p;
  return ret;
}

SpPhasingAlgorithm *sp_phasing_raar_alloc(sp_smap *beta, SpPhasingConstraints constraints) {
  return beta_alg(SpRAAR, beta, constraints);
}

SpPhasingAlgorithm *sp_phasing_hio_alloc(sp_smap *beta, SpPhasingConstraints constraints) {
  return beta_alg(SpHIO, beta, constraints);
}

SpPhasingAlgorithm *sp_phasing_er_alloc(SpPhasingConstraints constraints) {
  SpPhasingAlgorithm *ret = (SpPhasingAlgorithm *)malloc(sizeof(SpPhasingAlgorithm));
  SpPhasingERParameters *p = (SpPhasingERParameters *)malloc(sizeof(SpPhasingERParameters));
  ret->type = SpER;
  p->constraints = constraints;
  ret->params = p;
  return ret;
}

/* ---------------------------------------------------------- construction */

SpPhaser *sp_phaser_alloc(void) {
  SpPhaser *ph = (SpPhaser *)calloc(1, sizeof(SpPhaser));
  ph->model_iteration = -1;
  ph->fmodel_iteration = -1;
  ph->model_before_projection_iteration = -1;
  ph->model_change_iteration = -1;
  ph->support_iteration = -1;
  ph->old_model_iteration = -1;
  ph->phasing_objective = SpRecoverPhases;
  return ph;
}

void sp_phaser_set_objective(SpPhaser *ph, SpPhasingObjective obj) { ph->phasing_objective = obj; }

void sp_phaser_free(SpPhaser *ph) {
  if (!ph) return;
  if (ph->device) {
    dev_state *s = (dev_state *)ph->device;
    free_spare_model_images(ph);
    spb_host_unregister(s->pinned_model);
    spb_host_unregister(s->pinned_amp);
    s->pinned_model = s->pinned_amp = NULL;
  }
  Image **imgs[] = {&ph->model, &ph->model_before_projection, &ph->model_change, &ph->amplitudes_image,
                    &ph->old_model, &ph->support, &ph->fmodel};
  for (size_t i = 0; i < sizeof(imgs) / sizeof(imgs[0]); i++)
    if (*imgs[i]) { sp_image_free(*imgs[i]); *imgs[i] = NULL; }
  if (ph->amplitudes) sp_3matrix_free(ph->amplitudes);
  if (ph->amplitudes_min) sp_3matrix_free(ph->amplitudes_min);
  if (ph->amplitudes_max) sp_3matrix_free(ph->amplitudes_max);
  if (ph->pixel_flags) sp_i3matrix_free(ph->pixel_flags);
  if (ph->phased_amplitudes) sp_c3matrix_free(ph->phased_amplitudes);
  if (ph->device) {
    dev_state *s = (dev_state *)ph->device;
    if (s->ctx) spb_ctx_destroy(s->ctx);
    free(s);
  }
  free(ph);
}

/* phasing.c:271-292: first image fixes the shape; a mismatch aborts */
static void phaser_check_dimensions(SpPhaser *ph, const Image *a) {
  if (!ph->nx) {
    ph->nx = sp_image_x(a);
    ph->ny = sp_image_y(a);
    ph->nz = sp_image_z(a);
    ph->image_size = ph->nx * ph->ny * ph->nz;
  }
  if (ph->nx != sp_image_x(a) || ph->ny != sp_image_y(a) || ph->nz != sp_image_z(a)) {
    fprintf(stderr, "spimage-b200: image shape %dx%dx%d does not match the phaser's %dx%dx%d\n", sp_image_x(a),
            sp_image_y(a), sp_image_z(a), ph->nx, ph->ny, ph->nz);
    abort();
  }
}

static void ensure_flags(SpPhaser *ph) {
  if (!ph->pixel_flags) ph->pixel_flags = sp_i3matrix_alloc(ph->nx, ph->ny, ph->nz);
}

/* phasing.c:189-204 */
void sp_phaser_set_model(SpPhaser *ph, const Image *model) {
  phaser_check_dimensions(ph, model);
  ph->model_iteration = -1;
  if (ensure_ctx(ph)) return;
  if (spb_ctx_set_model(state(ph)->ctx, (const float *)model->image->data, 0)) dev_error("set model");
}

/* phasing.c:207-232 */
/* the support bit of every pixel from a support image (on the host threads) */
typedef struct {
  SpPhaser *ph;
  const Image *support;
} support_job;

static void support_span(void *ctx, int t, long long i0, long long i1) {
  (void)t;
  const support_job *j = (const support_job *)ctx;
  for (long long i = i0; i < i1; i++) {
    if (sp_real(j->support->image->data[i])) j->ph->pixel_flags->data[i] |= SpPixelInsideSupport;
    else j->ph->pixel_flags->data[i] &= ~SpPixelInsideSupport;
  }
}

void sp_phaser_set_support(SpPhaser *ph, const Image *support) {
  phaser_check_dimensions(ph, support);
  ph->support_iteration = -1;
  ensure_flags(ph);
  support_job job = {ph, support}; /* every pixel's support bit: no need to fetch the device's first */
  spb_parallel_for(ph->image_size, support_span, &job);
  host_wrote_flags(ph, SpPixelInsideSupport);
}

/* phasing.c:235-269 */
void sp_phaser_set_phased_amplitudes(SpPhaser *ph, const Image *pa) {
  phaser_check_dimensions(ph, pa);
  if (!ph->phased_amplitudes) ph->phased_amplitudes = sp_c3matrix_alloc(ph->nx, ph->ny, ph->nz);
  ensure_flags(ph);
  for (int i = 0; i < ph->image_size; i++) {
    ph->phased_amplitudes->data[i] = pa->image->data[i];
    if (pa->mask->data[i]) ph->pixel_flags->data[i] |= SpPixelMeasuredAmplitude;
    else ph->pixel_flags->data[i] &= ~SpPixelMeasuredAmplitude;
  }
  state(ph)->pamp_dirty = 1;
  host_wrote_flags(ph, SpPixelMeasuredAmplitude);
}

/* phasing.c:294-333 */
/* amplitudes and measured bits from an amplitude image (on the host threads) */
typedef struct {
  SpPhaser *ph;
  const Image *img;
  long long masked[SPB_PAR_MAX];
} set_amp_job;

static void set_amp_span(void *ctx, int t, long long i0, long long i1) {
  set_amp_job *j = (set_amp_job *)ctx;
  long long masked = 0;
  for (long long i = i0; i < i1; i++) {
    spb_stream_f32(&j->ph->amplitudes->data[i], sp_real(j->img->image->data[i])); /* uploaded next */
    if (j->img->mask->data[i]) {
      j->ph->pixel_flags->data[i] |= SpPixelMeasuredAmplitude;
      masked++;
    } else {
      j->ph->pixel_flags->data[i] &= ~SpPixelMeasuredAmplitude;
    }
  }
  spb_stream_fence();
  j->masked[t] = masked;
}

void sp_phaser_set_amplitudes(SpPhaser *ph, const Image *amplitudes) {
  phaser_check_dimensions(ph, amplitudes);
  if (!ph->amplitudes) {
    ph->amplitudes = sp_3matrix_alloc(ph->nx, ph->ny, ph->nz);
    if (!spb_host_register(ph->amplitudes->data, sizeof(real) * (size_t)ph->image_size))
      state(ph)->pinned_amp = ph->amplitudes->data;
  }
  ensure_flags(ph);
  set_amp_job job = {ph, amplitudes, {0}}; /* every pixel's measured bit */
  const int spans = spb_parallel_for(ph->image_size, set_amp_span, &job);
  long long masked = 0;
  for (int t = 0; t < spans; t++) masked += job.masked[t];
  if (masked == 0) fprintf(stderr, "Amplitudes mask is all zeros!\n");
  state(ph)->amp_dirty = 1;
  host_wrote_flags(ph, SpPixelMeasuredAmplitude);
}

/* phasing.c:335-363 */
void sp_phaser_set_amplitudes_margins(SpPhaser *ph, const Image *amin, const Image *amax) {
  phaser_check_dimensions(ph, amin);
  phaser_check_dimensions(ph, amax);
  if (!ph->amplitudes_min) ph->amplitudes_min = sp_3matrix_alloc(ph->nx, ph->ny, ph->nz);
  if (!ph->amplitudes_max) ph->amplitudes_max = sp_3matrix_alloc(ph->nx, ph->ny, ph->nz);
  for (int i = 0; i < ph->image_size; i++) {
    ph->amplitudes_min->data[i] = sp_real(amin->image->data[i]);
    ph->amplitudes_max->data[i] = sp_real(amax->image->data[i]);
  }
  state(ph)->margins_dirty = 1;
}

/* ------------------------------------------------------------- accessors */

const Image *sp_phaser_amplitudes(SpPhaser *ph) {
  if (!ph->amplitudes_image) {
    ph->amplitudes_image = sp_image_alloc(ph->nx, ph->ny, ph->nz);
    sync_flags_to_host(ph);
    for (int i = 0; i < ph->image_size; i++) {
      ph->amplitudes_image->image->data[i] = sp_cinit(ph->amplitudes->data[i], 0);
      ph->amplitudes_image->mask->data[i] = (ph->pixel_flags->data[i] & SpPixelMeasuredAmplitude) ? 1 : 0;
    }
  }
  return ph->amplitudes_image;
}

static Image *fetch(SpPhaser *ph, Image **slot, int *slot_iteration, int which) {
  if (*slot_iteration != ph->iteration || !*slot) {
    if (!*slot) *slot = sp_image_alloc(ph->nx, ph->ny, ph->nz);
    if (ensure_ctx(ph)) return NULL;
    if (spb_ctx_get_image(state(ph)->ctx, which, (float *)(*slot)->image->data)) {
      dev_error("download image");
      return NULL;
    }
    *slot_iteration = ph->iteration;
  }
  return *slot;
}

static Image *model_nc(SpPhaser *ph) { return fetch(ph, &ph->model, &ph->model_iteration, SPB_G1); }

const Image *sp_phaser_model(SpPhaser *ph) { return model_nc(ph); }

const Image *sp_phaser_model_before_projection(SpPhaser *ph) {
  return fetch(ph, &ph->model_before_projection, &ph->model_before_projection_iteration, SPB_GP);
}

const Image *sp_phaser_old_model(SpPhaser *ph) {
  return fetch(ph, &ph->old_model, &ph->old_model_iteration, SPB_G0);
}

static Image *fmodel_nc(SpPhaser *ph) {
  Image *f = fetch(ph, &ph->fmodel, &ph->fmodel_iteration, SPB_FMODEL);
  if (f) f->phased = 1;
  return f;
}

const Image *sp_phaser_fmodel(SpPhaser *ph) { return fmodel_nc(ph); }

const Image *sp_phaser_fmodel_with_mask(SpPhaser *ph) {
  Image *f = fmodel_nc(ph);
  const Image *amp = sp_phaser_amplitudes(ph);
  if (f) memcpy(f->mask->data, amp->mask->data, sizeof(int) * (size_t)ph->image_size);
  return f;
}

/* phasing.c:532-554: model - old model */
Image *sp_phaser_model_change(SpPhaser *ph) {
  Image *m = model_nc(ph);
  if (!m) return NULL;
  if (ph->model_change_iteration != ph->iteration) {
    const Image *old = sp_phaser_old_model(ph);
    if (!old) return NULL;
    ph->model_change_iteration = ph->iteration;
    for (int i = 0; i < ph->image_size; i++) {
      ph->model_change->image->data[i].re = m->image->data[i].re - old->image->data[i].re;
      ph->model_change->image->data[i].im = m->image->data[i].im - old->image->data[i].im;
    }
  }
  return ph->model_change;
}

const Image *sp_phaser_support(SpPhaser *ph) {
  if (!ph->support) ph->support = sp_image_alloc(ph->nx, ph->ny, ph->nz);
  if (ph->iteration != ph->support_iteration) {
    if (sync_flags_to_host(ph)) return NULL;
    ph->support_iteration = ph->iteration;
    sp_image_fill(ph->support, sp_cinit(0, 0));
    for (int i = 0; i < ph->image_size; i++)
      if (ph->pixel_flags->data[i] & SpPixelInsideSupport) ph->support->image->data[i].re = 1;
  }
  return ph->support;
}

const Image *sp_phaser_model_with_support(SpPhaser *ph) {
  Image *m = model_nc(ph);
  const Image *s = sp_phaser_support(ph);
  if (!m || !s) return m;
  for (int i = 0; i < ph->image_size; i++)
    m->mask->data[i] = (s->image->data[i].re == 0.0 && s->image->data[i].im == 0.0) ? 0 : 1;
  return m;
}

/* ------------------------------------------------------------- init/run */

/* phasing.c:558-586; this library has only the GPU engine */
int sp_phaser_init(SpPhaser *ph, SpPhasingAlgorithm *alg, SpSupportArray *sup_alg, SpPhasingEngine engine) {
  if (!ph) {
    fprintf(stderr, "Phaser is NULL!\n");
    return -1;
  }
  if (!alg) {
    fprintf(stderr, "Algorithm is NULL!\n");
    return -2;
  }
  ph->algorithm = alg;
  ph->sup_algorithm = sup_alg;
  ph->iteration = 0;
  if (engine == SpEngineCPU) {
    snprintf(g_last_err, sizeof(g_last_err), "SpEngineCPU requested: this library runs phasing on the GPU only");
    fprintf(stderr, "spimage-b200: %s\n", g_last_err);
    return -3;
  }
  if (spb_device_count() < 1) {
    snprintf(g_last_err, sizeof(g_last_err), "no CUDA device available for the GPU phasing engine");
    fprintf(stderr, "spimage-b200: %s\n", g_last_err);
    return -3;
  }
  ph->engine = SpEngineCUDA;
  return 0;
}

int sp_phaser_set_phasing_algorithm(SpPhaser *ph, SpPhasingAlgorithm *alg) {
  if (!alg) {
    fprintf(stderr, "Algorithm is NULL!\n");
    return -2;
  }
  ph->algorithm = alg;
  return 0;
}

int sp_phaser_set_support_algorithm(SpPhaser *ph, SpSupportArray *alg) {
  if (!alg) {
    fprintf(stderr, "Phasing algorithm is NULL!\n");
    return -2;
  }
  ph->sup_algorithm = alg;
  return 0;
}

static int draw_start(SpPhaser *ph, int flags, Image *m);
static int finish_init_model(SpPhaser *ph, int flags, int rc);

/* phasing.c:606-724 with the CPU engine's semantics: the starting model is
 * derived from the host RNG (glibc rand(), as p_drand48) exactly like the
 * reference CPU engine, then transformed on the GPU. */
int sp_phaser_init_model(SpPhaser *ph, const Image *user_model, int flags) {
  if (!ph) return -1;
  if (ph->engine != SpEngineCUDA) {
    snprintf(g_last_err, sizeof(g_last_err), "sp_phaser_init must succeed before sp_phaser_init_model");
    return -3;
  }
  release_model_images(ph);
  if (!user_model && !(flags & (SpModelRandomPhases | SpModelZeroPhases | SpModelRandomValues))) return -3;
  if (user_model) phaser_check_dimensions(ph, user_model);
  /* only a masked-out start reads the pixel flags */
  if (sync_to_device_for(ph, (flags & SpModelMaskedOutZeroed) != 0)) return -8;
  spb_ctx *ctx = state(ph)->ctx;
  int rc = 0;
  if (user_model) {
    rc = spb_ctx_set_model(ctx, (const float *)user_model->image->data, 1);
  } else if (flags & SpModelRandomPhases) {
    /* the phases from rand() on the host, the trigonometry on the device */
    if (!ph->amplitudes) {
      snprintf(g_last_err, sizeof(g_last_err), "sp_phaser_init_model: set the amplitudes before a random-phase start");
      return -3;
    }
    float *phases = (float *)spb_ctx_host_stage(ctx, sizeof(float) * (size_t)ph->image_size);
    if (!phases) return dev_error("init model");
    spb_random_phases(phases, ph->image_size);
    rc = spb_ctx_models_from_phases(ctx, phases, ph->amplitudes->data, 1, 1);
  } else {
    Image *m = sp_image_alloc(ph->nx, ph->ny, ph->nz);
    if (draw_start(ph, flags, m)) rc = spb_ctx_model_from_fourier(ctx, (const float *)m->image->data, 1);
    else rc = spb_ctx_set_model(ctx, (const float *)m->image->data, 1);
    sp_image_free(m);
  }
  return finish_init_model(ph, flags, rc);
}

/* Fills `m` from the host RNG as the reference's CPU engine does for `flags`;
 * returns 1 when `m` is a Fourier-space start (random or zero phases on the
 * amplitudes), 0 when it is a real-space model (random values). */
static int draw_start(SpPhaser *ph, int flags, Image *m) {
  const int n = ph->image_size;
  if (flags & (SpModelRandomPhases | SpModelZeroPhases)) {
    for (int i = 0; i < n; i++) m->image->data[i] = sp_cinit(ph->amplitudes->data[i], 0);
    sp_image_rephase(m, (flags & SpModelRandomPhases) ? SP_RANDOM_PHASE : SP_ZERO_PHASE);
    return 1;
  }
  /* SpModelRandomValues: uniform (re, im) in [-0.5, 0.5) scaled so that the
   * squared norm matches the amplitudes' (phasing.c:674-690) */
  double sum = 0;
  for (int i = 0; i < n; i++) sum += ph->amplitudes->data[i] * ph->amplitudes->data[i];
  sum /= n;
  /* the reference's sp_cinit(p_drand48()-0.5, p_drand48()-0.5) draws the
   * imaginary part first under gcc's argument evaluation order: pixel i takes
   * draws 2i (imaginary) and 2i + 1 (real) */
  float *u = (float *)malloc(sizeof(float) * 2 * (size_t)n);
  if (u) {
    spb_random_uniforms(u, 2 * (long long)n);
    for (int i = 0; i < n; i++) {
      const real im = u[2 * (size_t)i] - 0.5;
      const real re = u[2 * (size_t)i + 1] - 0.5;
      m->image->data[i] = sp_cinit(re, im);
    }
    free(u);
  } else {
    for (int i = 0; i < n; i++) {
      const real im = p_drand48() - 0.5;
      const real re = p_drand48() - 0.5;
      m->image->data[i] = sp_cinit(re, im);
    }
  }
  double msum = 0;
  for (int i = 0; i < n; i++) msum += sp_cabs2(m->image->data[i]);
  const real model_sum = (real)msum;
  sp_image_scale(m, sqrt(sum / model_sum));
  return 0;
}

static int finish_init_model(SpPhaser *ph, int flags, int rc) {
  if (!rc && (flags & SpModelMaskedOutZeroed)) rc = spb_ctx_mask_out_unmeasured(state(ph)->ctx);
  if (rc) {
    free_spare_model_images(ph);
    return dev_error("init model");
  }
  /* host copy is fetched on the first sp_phaser_model() (model_iteration -1);
   * the images of the previous start are reused (same dimensions) */
  dev_state *s = state(ph);
  ph->model = s->spare_model ? s->spare_model : sp_image_alloc(ph->nx, ph->ny, ph->nz);
  ph->model_change = s->spare_change ? s->spare_change : sp_image_alloc(ph->nx, ph->ny, ph->nz);
  s->spare_model = s->spare_change = NULL;
  if (!s->pinned_model &&
      !spb_host_register(ph->model->image->data, sizeof(Complex) * (size_t)ph->image_size))
    s->pinned_model = ph->model->image->data;
  ph->model->phased = 1;
  ph->model_iteration = -1;
  ph->model_change_iteration = -1;
  return 0;
}

static int init_models_check(SpPhaser *ph, int flags) {
  if (!ph) return -1;
  if (ph->engine != SpEngineCUDA) {
    snprintf(g_last_err, sizeof(g_last_err), "sp_phaser_init must succeed before sp_phaser_init_model");
    return -3;
  }
  release_model_images(ph);
  if (!(flags & (SpModelRandomPhases | SpModelZeroPhases | SpModelRandomValues))) return -3;
  if (!ph->amplitudes) return -3;
  if (sync_to_device_for(ph, (flags & SpModelMaskedOutZeroed) != 0)) return -8;
  return 0;
}

int sp_phaser_init_models(SpPhaser *ph, int flags, const int *seeds) {
  const int rc0 = init_models_check(ph, flags);
  if (rc0) return rc0;
  spb_ctx *ctx = state(ph)->ctx;
  const int nb = sp_phaser_starts(ph);
  const size_t n = (size_t)ph->image_size;
  Image *m = sp_image_alloc(ph->nx, ph->ny, ph->nz);
  int rc = 0;
  if (flags & SpModelRandomPhases) {
    /* nb starts' phases from rand() on the host (start b after sp_srand(seeds[b])),
       the trigonometry and the transforms on the device */
    float *phases = (float *)malloc(sizeof(float) * n * (size_t)nb);
    if (!phases) {
      sp_image_free(m);
      return -8;
    }
    for (int b = 0; b < nb; b++) {
      if (seeds) sp_srand(seeds[b]);
      spb_random_phases(phases + n * (size_t)b, (long long)n);
    }
    rc = spb_ctx_models_from_phases(ctx, phases, ph->amplitudes->data, 0, 1);
    free(phases);
  } else if (flags & SpModelZeroPhases) {
    /* nb Fourier-space starts, transformed together on the device */
    float *all = (float *)malloc(sizeof(float) * 2 * n * (size_t)nb);
    for (int b = 0; b < nb; b++) {
      if (seeds) sp_srand(seeds[b]);
      draw_start(ph, flags, m);
      memcpy(all + 2 * n * (size_t)b, m->image->data, sizeof(float) * 2 * n);
    }
    rc = spb_ctx_models_from_fourier(ctx, all, 1);
    free(all);
  } else {
    for (int b = 0; b < nb && !rc; b++) {
      if (seeds) sp_srand(seeds[b]);
      draw_start(ph, flags, m);
      rc = spb_ctx_set_start_model(ctx, b, (const float *)m->image->data, b == 0);
    }
  }
  sp_image_free(m);
  return finish_init_model(ph, flags, rc);
}

int sp_phaser_init_models_device(SpPhaser *ph, int flags, const unsigned long long *seeds) {
  const int rc0 = init_models_check(ph, flags | SpModelRandomPhases);
  if (rc0) return rc0;
  const int rc = spb_ctx_random_phase_models(state(ph)->ctx, seeds, 1);
  return finish_init_model(ph, flags, rc);
}

int sp_phaser_starts(const SpPhaser *ph) {
  const dev_state *s = (const dev_state *)ph->device;
  return (s && s->starts > 0) ? s->starts : 1;
}

int sp_phaser_set_starts(SpPhaser *ph, int starts) {
  if (!ph || starts < 1) return -1;
  dev_state *s = state(ph);
  if (s->ctx) {
    if (sync_flags_to_host(ph)) return -8;
    spb_ctx_destroy(s->ctx);
    s->ctx = NULL;
  }
  s->starts = starts;
  s->flags_dev_bits = 0;
  release_model_images(ph);
  free_spare_model_images(ph);
  ph->model_iteration = ph->fmodel_iteration = ph->model_before_projection_iteration = -1;
  ph->old_model_iteration = ph->support_iteration = -1;
  return 0;
}

static int start_image(SpPhaser *ph, int start, Image *out, int which) {
  if (!out || sp_image_x(out) != ph->nx || sp_image_y(out) != ph->ny || sp_image_z(out) != ph->nz) return -1;
  if (ensure_ctx(ph)) return -8;
  if (spb_ctx_get_start_image(state(ph)->ctx, start, which, (float *)out->image->data))
    return dev_error("download start image");
  out->phased = 1;
  return 0;
}

int sp_phaser_start_model(SpPhaser *ph, int start, Image *out) { return start_image(ph, start, out, SPB_G1); }

int sp_phaser_start_model_before_projection(SpPhaser *ph, int start, Image *out) {
  return start_image(ph, start, out, SPB_GP);
}

int sp_phaser_start_fmodel(SpPhaser *ph, int start, Image *out) {
  if (sync_to_device(ph)) return -8;
  return start_image(ph, start, out, SPB_FMODEL);
}

int sp_phaser_start_support(SpPhaser *ph, int start, Image *out) {
  if (!out || sp_image_x(out) != ph->nx || sp_image_y(out) != ph->ny || sp_image_z(out) != ph->nz) return -1;
  if (sync_to_device(ph)) return -8;
  int *f = (int *)malloc(sizeof(int) * (size_t)ph->image_size);
  if (spb_ctx_get_start_flags(state(ph)->ctx, start, f)) {
    free(f);
    return dev_error("download start support");
  }
  for (int i = 0; i < ph->image_size; i++) out->image->data[i] = sp_cinit((f[i] & SpPixelInsideSupport) ? 1 : 0, 0);
  free(f);
  return 0;
}

int sp_phaser_starts_efourier(SpPhaser *ph, real *out, real *FcFo) {
  if (sync_to_device(ph)) return -8;
  const int nb = sp_phaser_starts(ph);
  double *s = (double *)malloc(sizeof(double) * 4 * (size_t)nb);
  if (spb_ctx_batch_efourier_sums(state(ph)->ctx, s)) {
    free(s);
    return dev_error("efourier");
  }
  for (int b = 0; b < nb; b++) {
    out[b] = (real)sqrt(s[4 * b] / s[4 * b + 1]);
    if (FcFo) FcFo[b] = (real)(s[4 * b + 2] / s[4 * b + 3]);
  }
  free(s);
  return 0;
}

int sp_phaser_starts_ereal(SpPhaser *ph, real *out) {
  if (ensure_ctx(ph)) return -8;
  const int nb = sp_phaser_starts(ph);
  double *s = (double *)malloc(sizeof(double) * 4 * (size_t)nb);
  if (spb_ctx_batch_ereal_sums(state(ph)->ctx, s)) {
    free(s);
    return dev_error("ereal");
  }
  for (int b = 0; b < nb; b++) out[b] = (real)sqrt(s[4 * b] / s[4 * b + 1]);
  free(s);
  return 0;
}

int sp_phaser_starts_support_fraction(SpPhaser *ph, real *out) {
  if (sync_to_device(ph)) return -8;
  const int nb = sp_phaser_starts(ph);
  long long *c = (long long *)malloc(sizeof(long long) * (size_t)nb);
  if (spb_ctx_batch_support_counts(state(ph)->ctx, c)) {
    free(c);
    return dev_error("support fraction");
  }
  for (int b = 0; b < nb; b++) out[b] = (real)c[b] / (real)ph->image_size;
  free(c);
  return 0;
}

/* phasing.c:727-778 */
int sp_phaser_init_support(SpPhaser *ph, const Image *support, int flags, real value) {
  if (support) {
    phaser_check_dimensions(ph, support);
    ensure_flags(ph);
    support_job job = {ph, support}; /* every pixel's support bit */
    spb_parallel_for(ph->image_size, support_span, &job);
    host_wrote_flags(ph, SpPixelInsideSupport);
    ph->support_iteration = -1;
    return 0;
  }
  if (flags & SpSupportFromPatterson) {
    ensure_flags(ph);
    if (sync_to_device(ph)) return -8;
    if (spb_ctx_support_patterson(state(ph)->ctx, value)) return dev_error("Patterson support");
    device_wrote_flags(ph, SpPixelInsideSupport);
    ph->support_iteration = -1;
    return 0;
  }
  return -1;
}

static void alg_desc(const SpPhaser *ph, spb_alg_desc *d, sp_smap **beta);

/* `k` phasing iterations of the current algorithm on the device */
static int run_phasing(SpPhaser *ph, int k) {
  if (k <= 0) return 0;
  spb_alg_desc d;
  sp_smap *beta = NULL;
  alg_desc(ph, &d, &beta);
  float *b = (float *)malloc(sizeof(float) * (size_t)k);
  for (int i = 0; i < k; i++) b[i] = beta ? sp_smap_interpolate(beta, ph->iteration + i) : 0.0f;
  const int rc = spb_ctx_iterate(state(ph)->ctx, &d, b, k, 1);
  free(b);
  if (rc) return dev_error("iterate");
  ph->iteration += k;
  return 0;
}

/* Not in the reference: launch shapes of this phaser's device passes chosen
 * by measurement for the current algorithm (spb_ctx_autotune), over calls of
 * one support period (or 16 iterations); the reconstruction is left where it
 * was.  Returns 0 or -8. */
int sp_phaser_autotune(SpPhaser *ph) {
  if (!ph || !ph->algorithm) return -2;
  if (sync_to_device(ph)) return -8;
  spb_alg_desc d;
  alg_desc(ph, &d, NULL);
  int its = ph->sup_algorithm ? ph->sup_algorithm->update_period - 1 : 16;
  if (its < 2) its = 2;
  if (its > 64) its = 64;
  if (spb_ctx_autotune(state(ph)->ctx, &d, its, 5, 0, NULL)) return dev_error("autotune");
  return 0;
}

/* the device descriptor of the current algorithm and its beta schedule */
static void alg_desc(const SpPhaser *ph, spb_alg_desc *dp, sp_smap **beta_out) {
  const SpPhasingAlgorithm *alg = ph->algorithm;
  spb_alg_desc d;
  memset(&d, 0, sizeof(d));
  d.algorithm = alg->type;
  d.objective = ph->phasing_objective;
  sp_smap *beta = NULL;
  if (alg->type == SpHIO || alg->type == SpRAAR) {
    const SpPhasingHIOParameters *p = (const SpPhasingHIOParameters *)alg->params;
    beta = p->beta;
    d.constraints = p->constraints;
  } else if (alg->type == SpDiffMap) {
    const SpPhasingDiffMapParameters *p = (const SpPhasingDiffMapParameters *)alg->params;
    beta = p->beta;
    d.constraints = p->constraints;
    d.gamma1 = p->gamma1;
    d.gamma2 = p->gamma2;
    d.objective = SpRecoverPhases; /* the reference's difference map always projects on amplitudes */
  } else {
    d.constraints = ((const SpPhasingERParameters *)alg->params)->constraints;
  }
  *dp = d;
  if (beta_out) *beta_out = beta;
}

/* phasing.c:895-1024 */
int sp_phaser_iterate(SpPhaser *ph, int iterations) {
  if (!ph) return -1;
  if (!ph->algorithm) return -2;
  if (!ph->model) return -3;
  if ((!ph->amplitudes && ph->phasing_objective == SpRecoverPhases) ||
      (!ph->phased_amplitudes && ph->phasing_objective == SpRecoverAmplitudes))
    return -4;
  if (!ph->pixel_flags) return -5;
  if (!ph->model_change) return -6;
  const int t = ph->algorithm->type;
  if (t != SpHIO && t != SpRAAR && t != SpDiffMap && t != SpER) return -7;
  if (ph->engine != SpEngineCUDA) return -8;
  if (sync_to_device(ph)) return -8;
  if (ph->sup_algorithm && ph->sup_algorithm->algorithms[0]->function) {
    while (iterations) {
      const int period = ph->sup_algorithm->update_period;
      int to_update = period - 1 - ph->iteration % period;
      const int to_iterate = (int)sp_min(iterations, to_update);
      if (run_phasing(ph, to_iterate)) return -8;
      iterations -= to_iterate;
      to_update -= to_iterate;
      if (to_update == 0 && iterations > 0) {
        if (sp_support_array_update(ph->sup_algorithm, ph) < 0) return -8;
        ph->iteration++;
        iterations -= 1;
      }
    }
  } else if (iterations) {
    if (run_phasing(ph, iterations)) return -8;
  }
  return 0;
}

/* ---------------------------------------------------------------- metrics */

/* phasing.c:803-832 (sums in double on the device) */
real sp_phaser_ereal(SpPhaser *ph) {
  if (sync_to_device(ph)) return -8; /* the support bits the host last set */
  double s[2];
  if (spb_ctx_ereal_sums(state(ph)->ctx, s)) return dev_error("ereal");
  return (real)sqrt(s[0] / s[1]);
}

/* phasing.c:852-891 */
real sp_phaser_efourier(SpPhaser *ph, real *FcFo) {
  if (sync_to_device(ph)) return -8;
  double s[4];
  if (spb_ctx_efourier_sums(state(ph)->ctx, s)) return dev_error("efourier");
  if (FcFo) *FcFo = (real)(s[2] / s[3]);
  return (real)sqrt(s[0] / s[1]);
}

/* phasing.c:834-850 */
real sp_phaser_support_fraction(SpPhaser *ph) {
  if (sync_to_device(ph)) return -8;
  long long c = 0;
  if (spb_ctx_support_count(state(ph)->ctx, &c)) return dev_error("support fraction");
  return (real)c / (real)ph->image_size;
}

int sp_phaser_set_cuda_stream(SpPhaser *ph, void *stream) {
  if (ensure_ctx(ph)) return -8;
  if (spb_ctx_set_stream(state(ph)->ctx, stream)) return dev_error("set stream");
  return 0;
}

void *sp_phaser_device_context(SpPhaser *ph) {
  if (!ph || ensure_ctx(ph)) return NULL;
  return state(ph)->ctx;
}

/* -------------------------------------------- hooks for support_update.c */

int spb_phaser_support_update(SpPhaser *ph, int type, real radius, real value) {
  if (sync_to_device(ph)) return -8;
  if (spb_ctx_support_update(state(ph)->ctx, type, radius, value)) return dev_error("support update");
  device_wrote_flags(ph, SpPixelInsideSupport);
  return 0;
}

int spb_phaser_support_close(SpPhaser *ph, int size) {
  if (sync_to_device(ph)) return -8;
  if (spb_ctx_support_close(state(ph)->ctx, size)) return dev_error("support close");
  device_wrote_flags(ph, SpPixelInsideSupport);
  return 0;
}

int spb_phaser_support_from_abs(SpPhaser *ph, const float *abs_values, real threshold) {
  if (sync_to_device(ph)) return -8;
  if (spb_ctx_support_from_abs(state(ph)->ctx, abs_values, threshold)) return dev_error("template support");
  device_wrote_flags(ph, SpPixelInsideSupport);
  return 0;
}

/* sp_pixel_flags_translate_mask (src/image_util.c:3587-3611): the support bit
 * moves by (dx,dy,dz) with wrap-around; the other bits stay in place */
static void translate_support(int *f, int *tmp, int nx, int ny, int nz, int dx, int dy, int dz) {
  while (dx < 0) dx += nx;
  while (dy < 0) dy += ny;
  while (dz < 0) dz += nz;
  for (int x = 0; x < nx; x++)
    for (int y = 0; y < ny; y++)
      for (int z = 0; z < nz; z++) {
        const int X = (x + dx) % nx, Y = (y + dy) % ny, Z = (z + dz) % nz;
        const int v1 = f[((long)z * ny + y) * nx + x];
        const long d = ((long)Z * ny + Y) * nx + X;
        tmp[d] = (v1 & SpPixelInsideSupport) ? (f[d] | SpPixelInsideSupport) : (f[d] & ~SpPixelInsideSupport);
      }
  memcpy(f, tmp, sizeof(int) * (size_t)nx * ny * nz);
}

/* sp_support_centre_image_cpu (src/support_update.c:305-389) on one start's
 * flags: translations that take the support off the borders of the shifted
 * layout, then the centre of mass (src/linear_alg.c:444-473: float sums in
 * pixel order, truncated to int) to the origin */
static void centre_support(int *f, int *tmp, int nx, int ny, int nz) {
#define IN(x, y, z) (f[((long)(z) * ny + (y)) * nx + (x)] & SpPixelInsideSupport)
  if (nz == 1) {
    for (int x = 0; x < nx; x++)
      if (IN(x, (ny - 1) / 2, 0)) {
        translate_support(f, tmp, nx, ny, nz, 0, (ny - 1) / 2, 0);
        break;
      }
    for (int y = 0; y < ny; y++)
      if (IN((nx - 1) / 2, y, 0)) {
        translate_support(f, tmp, nx, ny, nz, (nx - 1) / 2, 0, 0);
        break;
      }
  } else {
    /* as in the reference, each break leaves the inner loop only */
    for (int y = 0; y < ny; y++)
      for (int z = 0; z < nz; z++)
        if (IN((nx - 1) / 2, y, z)) {
          translate_support(f, tmp, nx, ny, nz, (nx - 1) / 2, 0, 0);
          break;
        }
    for (int x = 0; x < nx; x++)
      for (int z = 0; z < nz; z++)
        if (IN(x, (ny - 1) / 2, z)) {
          translate_support(f, tmp, nx, ny, nz, 0, (ny - 1) / 2, 0);
          break;
        }
    for (int x = 0; x < nx; x++)
      for (int y = 0; y < ny; y++)
        if (IN(x, y, (nz - 1) / 2)) {
          translate_support(f, tmp, nx, ny, nz, 0, 0, (nz - 1) / 2);
          break;
        }
  }
#undef IN
  float c[3] = {0.0f, 0.0f, 0.0f};
  int sum = 0;
  long i = 0;
  for (int z = 0; z < nz; z++)
    for (int y = 0; y < ny; y++)
      for (int x = 0; x < nx; x++, i++)
        if (f[i] & SpPixelInsideSupport) {
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
  translate_support(f, tmp, nx, ny, nz, (int)(0 - c[0]), (int)(0 - c[1]), (int)(0 - c[2]));
}

int spb_phaser_support_centre(SpPhaser *ph) {
  if (sync_to_device(ph)) return -8;
  spb_ctx *ctx = state(ph)->ctx;
  const size_t n = (size_t)ph->image_size;
  int *f = (int *)malloc(sizeof(int) * n), *tmp = (int *)calloc(n, sizeof(int));
  int rc = 0;
  for (int b = 0; b < sp_phaser_starts(ph) && !rc; b++) {
    if (spb_ctx_get_start_flags(ctx, b, f)) rc = dev_error("download support");
    if (!rc) {
      centre_support(f, tmp, ph->nx, ph->ny, ph->nz);
      if (spb_ctx_set_start_flags(ctx, b, f)) rc = dev_error("upload support");
    }
  }
  free(f);
  free(tmp);
  device_wrote_flags(ph, SpPixelInsideSupport);
  return rc;
}
