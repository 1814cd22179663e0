/*
 * Image container of the phasing path, layout-compatible with the reference
 * (include/spimage/image.h:29-84): complex64 data (x fastest) plus an int mask.
 */
#ifndef SPB_IMAGE_H
#define SPB_IMAGE_H 1
#include <float.h>
#ifdef __cplusplus
extern "C" {
#endif

#define spimage_EXPORT

typedef enum { SP_1D = 1, SP_2D = 2, SP_3D = 3 } Dimensions;

#include "linear_alg.h"

typedef struct {
  real image_center[3];
  real pixel_size[3];
  real detector_distance;
  real wavelength;
  SpRotation *orientation;
} Detector;

typedef struct {
  int phased;
  int scaled;
  sp_c3matrix *image;
  sp_i3matrix *mask;
  Detector *detector;
  int shifted; /* 1 = FFT layout, zero frequency at index 0 */
  sp_3matrix *rec_coords;
  Dimensions num_dimensions;
} Image;

#ifdef __cplusplus
}
#endif
#endif
