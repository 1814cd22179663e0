/*
 * Support-update algorithms (host C) over the device layer.  Allocation and
 * the support array follow src/support_update.c:7-122,458-494; the area and
 * threshold updates (src/support_update.c:136-179) run on the GPU: blur of
 * |model|, exact area quantile by radix select (or max * threshold), strict
 * '>' mask rebuild.  Schedules are evaluated with the same Bezier formula.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "spimage.h"
#include "spimage/spb_device.h"

int spb_phaser_support_update(SpPhaser *ph, int type, real radius, real value);
int spb_phaser_support_close(SpPhaser *ph, int size);
int spb_phaser_support_from_abs(SpPhaser *ph, const float *abs_values, real threshold);
int spb_phaser_support_centre(SpPhaser *ph);

SpSupportAlgorithm *sp_support_threshold_alloc(sp_smap *blur_radius, sp_smap *threshold) {
  SpSupportAlgorithm *ret = (SpSupportAlgorithm *)malloc(sizeof(SpSupportAlgorithm));
  SpSupportThresholdParameters *p = (SpSupportThresholdParameters *)malloc(sizeof(SpSupportThresholdParameters));
  ret->type = SpSupportThreshold;
  p->blur_radius_map = blur_radius;
  p->threshold = threshold;
  ret->params = p;
  ret->function = (void *)sp_support_threshold_update_support;
  return ret;
}

SpSupportAlgorithm *sp_support_area_alloc(sp_smap *blur_radius, sp_smap *area) {
  SpSupportAlgorithm *ret = (SpSupportAlgorithm *)malloc(sizeof(SpSupportAlgorithm));
  SpSupportAreaParameters *p = (SpSupportAreaParameters *)malloc(sizeof(SpSupportAreaParameters));
  ret->type = SpSupportArea;
  p->blur_radius_map = blur_radius;
  p->area = area;
  ret->params = p;
  ret->function = (void *)sp_support_area_update_support;
  return ret;
}

SpSupportAlgorithm *sp_support_static_alloc(void) {
  SpSupportAlgorithm *ret = (SpSupportAlgorithm *)malloc(sizeof(SpSupportAlgorithm));
  ret->type = SpSupportStatic;
  ret->params = calloc(1, sizeof(SpSupportStaticParameters));
  ret->function = (void *)sp_support_static_update_support;
  return ret;
}

/* support_update.c:44-49 */
SpSupportAlgorithm *sp_support_centre_image_alloc(void) {
  SpSupportAlgorithm *ret = (SpSupportAlgorithm *)malloc(sizeof(SpSupportAlgorithm));
  ret->type = SpSupportCentreImage;
  ret->params = calloc(1, sizeof(SpSupportCentreImageParameters));
  ret->function = (void *)sp_support_centre_image;
  return ret;
}

/* support_update.c:110-125 */
SpSupportAlgorithm *sp_support_close_alloc(int size) {
  SpSupportAlgorithm *ret = (SpSupportAlgorithm *)malloc(sizeof(SpSupportAlgorithm));
  SpSupportCloseParameters *p = (SpSupportCloseParameters *)malloc(sizeof(SpSupportCloseParameters));
  ret->type = SpSupportClose;
  p->size = size;
  ret->params = p;
  ret->function = (void *)sp_support_close_update_support;
  return ret;
}

static float cabs_ref(Complex a) { return (float)sqrt((double)(a.im * a.im + a.re * a.re)); }

static int desc_modulus(const void *pa, const void *pb) {
  const float a = cabs_ref(*(const Complex *)pa), b = cabs_ref(*(const Complex *)pb);
  return a < b ? 1 : (a == b ? 0 : -1);
}

/* support_update.c:51-84: the initial support blurred once (sp_gaussian_blur,
 * on the GPU), a copy sorted by descending modulus, and the fraction of the
 * pixels inside the initial support (accumulated in float) */
SpSupportAlgorithm *sp_support_template_alloc(Image *initial_support, real blur_radius, sp_smap *area) {
  SpSupportAlgorithm *ret = (SpSupportAlgorithm *)malloc(sizeof(SpSupportAlgorithm));
  SpSupportTemplateParameters *p = (SpSupportTemplateParameters *)malloc(sizeof(SpSupportTemplateParameters));
  ret->type = SpSupportTemplate;
  p->blured = sp_gaussian_blur(initial_support, blur_radius);
  p->area = area;
  p->original_area = 0.0f;
  const long long n = sp_image_size(initial_support);
  for (long long i = 0; i < n; i++)
    if (initial_support->image->data[i].re != 0.0f || initial_support->image->data[i].im != 0.0f)
      p->original_area += 1.0f;
  p->original_area /= (real)n;
  p->sorted = sp_image_duplicate(p->blured, SP_COPY_DATA);
  qsort(p->sorted->image->data, (size_t)n, sizeof(Complex), desc_modulus);
  ret->params = p;
  ret->function = (void *)sp_support_template_update_support;
  return ret;
}

/* support_update.c:193-205; the index is clamped to N-1 where the reference
 * would read past the end of the sorted values */
int sp_support_template_update_support(SpSupportAlgorithm *alg, SpPhaser *ph) {
  SpSupportTemplateParameters *p = (SpSupportTemplateParameters *)alg->params;
  const real area = sp_smap_interpolate(p->area, ph->iteration);
  const long long n = sp_image_size(p->sorted);
  long long k = (long long)(int)((real)n * area * p->original_area);
  if (k >= n) k = n - 1;
  if (k < 0) k = 0;
  const real t = cabs_ref(p->sorted->image->data[k]);
  float *absv = (float *)malloc(sizeof(float) * (size_t)n);
  for (long long i = 0; i < n; i++) absv[i] = cabs_ref(p->blured->image->data[i]);
  const int rc = spb_phaser_support_from_abs(ph, absv, t);
  free(absv);
  return rc;
}

/* support_update.c:225-290 */
int sp_support_close_update_support(SpSupportAlgorithm *alg, SpPhaser *ph) {
  return spb_phaser_support_close(ph, ((SpSupportCloseParameters *)alg->params)->size);
}

/* support_update.c:305-389 */
int sp_support_centre_image(SpSupportAlgorithm *alg, SpPhaser *ph) {
  (void)alg;
  return spb_phaser_support_centre(ph);
}

/* support_update.c:136-151 */
int sp_support_area_update_support(SpSupportAlgorithm *alg, SpPhaser *ph) {
  SpSupportAreaParameters *p = (SpSupportAreaParameters *)alg->params;
  const real radius = sp_smap_interpolate(p->blur_radius_map, ph->iteration);
  const real area = sp_smap_interpolate(p->area, ph->iteration);
  return spb_phaser_support_update(ph, SPB_SUPPORT_AREA, radius, area);
}

/* support_update.c:167-179 */
int sp_support_threshold_update_support(SpSupportAlgorithm *alg, SpPhaser *ph) {
  SpSupportThresholdParameters *p = (SpSupportThresholdParameters *)alg->params;
  const real radius = sp_smap_interpolate(p->blur_radius_map, ph->iteration);
  const real rel = sp_smap_interpolate(p->threshold, ph->iteration);
  return spb_phaser_support_update(ph, SPB_SUPPORT_THRESHOLD, radius, rel);
}

int sp_support_static_update_support(SpSupportAlgorithm *alg, SpPhaser *ph) {
  (void)alg;
  (void)ph;
  return 0;
}

SpSupportArray *sp_support_array_alloc(int size, int update_period) {
  SpSupportArray *a = (SpSupportArray *)malloc(sizeof(SpSupportArray));
  a->size = size;
  a->algorithms = (SpSupportAlgorithm **)calloc((size_t)(size > 0 ? size : 1), sizeof(SpSupportAlgorithm *));
  a->update_period = update_period;
  return a;
}

void sp_support_array_set(SpSupportArray *array, int i, SpSupportAlgorithm *algorithm) {
  array->algorithms[i] = algorithm;
}

SpSupportArray *sp_support_array_init(SpSupportAlgorithm *algorithm, int update_period) {
  SpSupportArray *a = sp_support_array_alloc(1, update_period);
  sp_support_array_set(a, 0, algorithm);
  return a;
}

void sp_support_array_append(SpSupportArray *array, SpSupportAlgorithm *algorithm) {
  SpSupportAlgorithm **algs =
      (SpSupportAlgorithm **)malloc(sizeof(SpSupportAlgorithm *) * (size_t)(array->size + 1));
  memcpy(algs, array->algorithms, sizeof(SpSupportAlgorithm *) * (size_t)array->size);
  algs[array->size] = algorithm;
  free(array->algorithms);
  array->algorithms = algs;
  array->size += 1;
}

/* support_update.c:489-494: every algorithm of the array, in order */
int sp_support_array_update(SpSupportArray *array, SpPhaser *ph) {
  for (int i = 0; i < array->size; i++) {
    int (*fn)(SpSupportAlgorithm *, SpPhaser *) =
        (int (*)(SpSupportAlgorithm *, SpPhaser *))array->algorithms[i]->function;
    if (fn && fn(array->algorithms[i], ph) < 0) return -8;
  }
  return 0;
}
