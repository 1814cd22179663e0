/*
 * Support-update algorithms (reference include/spimage/support_update.h:9-69).
 * Struct layouts are the reference's; area, threshold and static run on the
 * GPU (blur, exact area quantile by radix select, mask rebuild).
 */
#ifndef SPB_SUPPORT_UPDATE_H
#define SPB_SUPPORT_UPDATE_H 1
#include "image.h"
#include "map.h"
#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  SpSupportThreshold = 1,
  SpSupportArea,
  SpSupportCentreImage,
  SpSupportTemplate,
  SpSupportStatic,
  SpSupportClose
} SpSupportAlgorithmType;

typedef struct {
  sp_smap *blur_radius_map;
  sp_smap *threshold;
} SpSupportThresholdParameters;

typedef struct {
  sp_smap *blur_radius_map;
  sp_smap *area;
} SpSupportAreaParameters;

typedef struct {
  void *dummy;
} SpSupportCentreImageParameters;

typedef struct {
  Image *blured;       /* the initial support blurred once */
  Image *sorted;       /* the same values sorted by descending modulus */
  sp_smap *area;       /* fraction of the initial support's area, per iteration */
  real original_area;  /* fraction of the pixels inside the initial support */
} SpSupportTemplateParameters;

typedef struct {
  void *dummy;
} SpSupportStaticParameters;

typedef struct {
  int size;
} SpSupportCloseParameters;

typedef struct {
  SpSupportAlgorithmType type;
  void *params;
  void *function; /* int (*)(SpSupportAlgorithm *, SpPhaser *) */
} SpSupportAlgorithm;

typedef struct {
  int size;
  SpSupportAlgorithm **algorithms;
  int update_period;
} SpSupportArray;

/* support_update.c:7-23 */
SpSupportAlgorithm *sp_support_threshold_alloc(sp_smap *blur_radius, sp_smap *threshold);
/* support_update.c:25-42 */
SpSupportAlgorithm *sp_support_area_alloc(sp_smap *blur_radius, sp_smap *area);
/* support_update.c:95-108 */
SpSupportAlgorithm *sp_support_static_alloc(void);
/* support_update.c:51-84: blurs the initial support (on the GPU) and sorts it */
SpSupportAlgorithm *sp_support_template_alloc(Image *initial_support, real blur_radius, sp_smap *area);
/* support_update.c:110-125 */
SpSupportAlgorithm *sp_support_close_alloc(int size);
/* support_update.c:44-49 */
SpSupportAlgorithm *sp_support_centre_image_alloc(void);
/* support_update.c:458-463 */
SpSupportArray *sp_support_array_alloc(int size, int update_period);
/* support_update.c:471-477 */
SpSupportArray *sp_support_array_init(SpSupportAlgorithm *algorithm, int update_period);
/* support_update.c:466-468 */
void sp_support_array_set(SpSupportArray *array, int i, SpSupportAlgorithm *algorithm);
/* support_update.c:480-487 */
void sp_support_array_append(SpSupportArray *array, SpSupportAlgorithm *algorithm);

#ifdef __cplusplus
}
#endif
#endif
