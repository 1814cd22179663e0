/*
 * sp_smap: sorted {iteration -> value} schedule used for beta, blur radius,
 * support area and threshold (reference include/spimage/map.h:16-19,103-141).
 *
 * sp_smap_interpolate is the reference's piecewise cubic-Bezier schedule.  Its
 * closed form and its mixed float/double arithmetic are kept as in the
 * reference so that every schedule value (and so every iterate) matches the
 * reference engine bit for bit.
 */
#ifndef SPB_MAP_H
#define SPB_MAP_H 1
#include <math.h>
#include "list.h"
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  sp_list *keys;
  sp_list *values;
} sp_smap;

static inline sp_smap *sp_smap_alloc(unsigned int init_size) {
  sp_smap *m = (sp_smap *)malloc(sizeof(sp_smap));
  m->keys = sp_list_alloc(init_size);
  m->values = sp_list_alloc(init_size);
  return m;
}
static inline void sp_smap_free(sp_smap *m) {
  sp_list_free(m->keys);
  sp_list_free(m->values);
  free(m);
}
static inline sp_list *sp_smap_get_keys(sp_smap *m) { return m->keys; }
static inline sp_list *sp_smap_get_values(sp_smap *m) { return m->values; }
/* insert keeping keys ascending; equal keys go after existing ones */
static inline void sp_smap_insert(sp_smap *m, real key, real value) {
  unsigned int i = 0;
  while (i < sp_list_size(m->keys) && !(sp_list_get(m->keys, i) > key)) i++;
  sp_list_insert(m->keys, i, key);
  sp_list_insert(m->values, i, value);
}
static inline sp_smap *sp_smap_create_from_pair(real key, real value) {
  sp_smap *m = sp_smap_alloc(1);
  sp_smap_insert(m, key, value);
  return m;
}
static inline real sp_smap_max(sp_smap *m) {
  real r = sp_list_get(m->values, 0);
  for (unsigned int i = 1; i < sp_list_size(m->values); i++)
    if (sp_list_get(m->values, i) > r) r = sp_list_get(m->values, i);
  return r;
}
static inline real sp_smap_min(sp_smap *m) {
  real r = sp_list_get(m->values, 0);
  for (unsigned int i = 1; i < sp_list_size(m->values); i++)
    if (sp_list_get(m->values, i) < r) r = sp_list_get(m->values, i);
  return r;
}

/* Value of the schedule at x: first value before the first key, last value
 * after the last key, and between keys p0 and p3 the cubic Bezier with flat
 * tangents, inverted in closed form for t(x). */
static inline real sp_smap_interpolate(sp_smap *map, real x) {
  const sp_list *keys = map->keys, *values = map->values;
  unsigned int idx;
  for (idx = 0; idx < sp_list_size(keys); idx++)
    if (x < sp_list_get(keys, idx)) break;
  if (idx == 0) return sp_list_get(values, 0);
  if (idx == sp_list_size(keys)) return sp_list_get(values, sp_list_size(keys) - 1);
  const real p0y = sp_list_get(values, idx - 1), p0x = sp_list_get(keys, idx - 1);
  const real p3y = sp_list_get(values, idx), p3x = sp_list_get(keys, idx);
  const double root =
      pow((double)pow(p0x - p3x, 4) * (6 * p0x * p3x - 16 * p0x * x - 16 * p3x * x + 5 * pow(p0x, 2) +
                                       5 * pow(p3x, 2) + 16 * pow(x, 2)),
          0.5);
  const double cub = 8 * p0x * p3x * x - 2 * p3x * pow(p0x, 2) - 4 * x * pow(p0x, 2) + 2 * pow(p0x, 3) -
                     2 * p0x * pow(p3x, 2) - 4 * x * pow(p3x, 2) + 2 * pow(p3x, 3) + root;
  const real t = (2 - 2 * (p0x - p3x) * pow(cub, -0.3333333333333333) +
                  2 * pow(p0x - p3x, -1) * pow(cub, 0.3333333333333333)) /
                 4.;
  return 3 * p0y * t * pow(1 - t, 2) + p0y * pow(1 - t, 3) + 3 * p3y * (1 - t) * pow(t, 2) + p3y * pow(t, 3);
}

/* Not in the reference: exported forms of the static inline constructors
 * above, so that a foreign-function binding has symbols to call.
 * spb_smap_create inserts the n (key, value) pairs in order. */
sp_smap *spb_smap_create(int n, const real *keys, const real *values);
void spb_smap_free(sp_smap *m);
real spb_smap_interpolate(sp_smap *m, real x);

#ifdef __cplusplus
}
#endif
#endif
