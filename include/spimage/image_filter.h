/* Gaussian blur of the support update (reference src/image_filter.c:80-90):
 * Fourier-domain multiply by exp(-2 pi^2 (d/nx)^2 radius^2)/N, d the wrapped
 * distance to the origin.  Runs on the GPU. */
#ifndef SPB_IMAGE_FILTER_H
#define SPB_IMAGE_FILTER_H 1
#include "image.h"
#ifdef __cplusplus
extern "C" {
#endif
Image *sp_gaussian_blur(Image *in, real radius);
#ifdef __cplusplus
}
#endif
#endif
