/*
 * Support-update algorithms (host C) over the device layer.  Allocation and
 * the support array follow src/support_update.c:7-122,458-494; the area and
 * threshold updates (src/support_update.c:136-179) run on the GPU: blur of
 * |model|, exact area quantile by radix select (or max * threshold), strict
 * '>' mask rebuild.  Schedules are evaluated with the same Bezier formula.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "spimage.h"
#include "spimage/spb_device.h"

int spb_phaser_support_update(SpPhaser *ph, int type, real radius, real value);

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
