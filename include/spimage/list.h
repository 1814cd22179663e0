/*
 * sp_list: growable array of real, the key/value storage of sp_smap.
 * Layout of the reference's include/spimage/list.h:12-16 ({data, used, size}).
 */
#ifndef SPB_LIST_H
#define SPB_LIST_H 1
#include <string.h>
#include "linear_alg.h"
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  real *data;
  unsigned int used;
  unsigned int size;
} sp_list;

static inline sp_list *sp_list_alloc(unsigned int init_size) {
  sp_list *l = (sp_list *)malloc(sizeof(sp_list));
  l->size = init_size ? init_size : 1;
  l->data = (real *)malloc(sizeof(real) * l->size);
  l->used = 0;
  return l;
}
static inline void sp_list_free(sp_list *l) { free(l->data); free(l); }
static inline unsigned int sp_list_size(const sp_list *l) { return l->used; }
static inline real sp_list_get(const sp_list *l, unsigned int i) { return l->data[i]; }
static inline void sp_list_set(sp_list *l, unsigned int i, real v) { l->data[i] = v; }
static inline void sp_list_clear(sp_list *l) { l->used = 0; }
static inline void sp_list_insert(sp_list *l, unsigned int i, real v) {
  if (l->used == l->size) {
    l->size = l->size < 4 ? 4 : 2 * l->size;
    l->data = (real *)realloc(l->data, sizeof(real) * l->size);
  }
  memmove(l->data + i + 1, l->data + i, sizeof(real) * (l->used - i));
  l->data[i] = v;
  l->used++;
}
static inline void sp_list_append(sp_list *l, real v) { sp_list_insert(l, l->used, v); }

#ifdef __cplusplus
}
#endif
#endif
