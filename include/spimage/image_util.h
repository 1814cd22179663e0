/*
 * Image helpers used by callers of the phasing API (subset of the reference's
 * include/spimage/image_util.h: allocation :118-150, size accessors :290-310,
 * phase helpers :37-38,365-380, random numbers src/image_util.c:120-127).
 */
#ifndef SPB_IMAGE_UTIL_H
#define SPB_IMAGE_UTIL_H 1
#include "image.h"
#ifdef __cplusplus
extern "C" {
#endif

#define SP_ZERO_PHASE 1
#define SP_RANDOM_PHASE 2
#define SP_TO_TOP_LEFT 8
#define SP_COPY_DETECTOR 0
#define SP_COPY_DATA 1
#define SP_COPY_MASK 2
#define SP_COPY_ALL 3

/* include/spimage/image_util.h:75-83 of the reference */
typedef enum { SpFourierSpace = 1, SpRealSpace = 2 } SpSpace;
typedef enum { SpInPlace = 65536, SpOutOfPlace = 131072 } SpPlace;
typedef enum { SpEnantiomorph = 1, SpCorrectPhaseShift = 2 } SpSuperimposeFlags;

Image *_sp_image_alloc(int x, int y, int z, const char *file, int line);
#define sp_image_alloc(x, y, z) _sp_image_alloc(x, y, z, __FILE__, __LINE__)
Image *_sp_image_duplicate(const Image *in, int flags, const char *file, int line);
#define sp_image_duplicate(in, flags) _sp_image_duplicate(in, flags, __FILE__, __LINE__)
void _sp_image_free(Image *in, const char *file, int line);
#define sp_image_free(in) _sp_image_free(in, __FILE__, __LINE__)
void sp_image_memcpy(Image *dst, const Image *src);
void sp_image_fill(Image *a, Complex value);
void sp_image_scale(Image *img, real value);
void sp_image_dephase(Image *img);
void sp_image_rephase(Image *img, int type);
void sp_srand(int i);
real p_drand48(void);
/* Superimposes b on a with 1/precision-pixel precision (reference
 * src/image_util.c:3024-3066): b is translated (Fourier translation) to the
 * largest modulus of the cross-correlation of a and b computed on a grid
 * padded precision times (2-D images are not padded along z); with
 * SpEnantiomorph the reflected and conjugated b is taken when its
 * correlation peak is higher; with SpCorrectPhaseShift b's constant phase is
 * matched to a's at the peak.  On the GPU (spb_superimpose_fractional_host). */
void sp_image_superimpose_fractional(Image *a, Image *b, SpSuperimposeFlags flags, int precision);

static inline long long sp_image_size(const Image *a) {
  return (long long)a->image->x * a->image->y * a->image->z;
}
static inline int sp_image_x(const Image *a) { return (int)a->image->x; }
static inline int sp_image_y(const Image *a) { return (int)a->image->y; }
static inline int sp_image_z(const Image *a) { return (int)a->image->z; }
static inline Complex sp_image_get_by_index(const Image *a, long long i) { return a->image->data[i]; }

#ifdef __cplusplus
}
#endif
#endif
