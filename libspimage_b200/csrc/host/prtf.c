/*
 * PRTF and fractional superposition at the Image level (the reference's
 * src/prtf.c:6-78 and src/image_util.c:3024-3066), over the device entry
 * points spb_prtf_basic_host, spb_prtf_advanced_host and
 * spb_superimpose_fractional_host.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "spimage.h"
#include "spimage/spb_device.h"

static int same_size(Image **list, int n) {
  for (int i = 0; i < n; i++)
    if (sp_image_x(list[0]) != sp_image_x(list[i]) || sp_image_y(list[0]) != sp_image_y(list[i]) ||
        sp_image_z(list[0]) != sp_image_z(list[i]))
      return 0;
  return 1;
}

/* the n images' data side by side ([n][N] complex) */
static Complex *gather(Image **list, int n) {
  const long long N = sp_image_size(list[0]);
  Complex *buf = (Complex *)malloc(sizeof(Complex) * (size_t)(N * n));
  if (!buf) return NULL;
  for (int i = 0; i < n; i++) memcpy(buf + (size_t)i * N, list[i]->image->data, sizeof(Complex) * (size_t)N);
  return buf;
}

Image *sp_prtf_basic(Image **list, int n) {
  if (n < 1 || !same_size(list, n)) return NULL;
  Complex *buf = gather(list, n);
  if (!buf) return NULL;
  Image *ret = sp_image_duplicate(list[0], SP_COPY_ALL);
  if (spb_prtf_basic_host(sp_image_x(ret), sp_image_y(ret), sp_image_z(ret), n, (const float *)buf,
                          (float *)ret->image->data)) {
    fprintf(stderr, "sp_prtf_basic: %s\n", spb_error_string());
    sp_image_free(ret);
    ret = NULL;
  }
  free(buf);
  return ret;
}

Image *sp_prtf_advanced(Image **list, int n, int flags) {
  if ((flags & (SpInPlace | SpOutOfPlace)) == 0) return NULL;
  if (n < 1 || !same_size(list, n)) return NULL;
  int space;
  if (flags & SpRealSpace) {
    space = 2;
  } else if (flags & SpFourierSpace) {
    space = 1;
    for (int i = 0; i < n; i++)
      if (!list[i]->phased || !list[i]->shifted) {
        fprintf(stderr, "sp_prtf_advanced: Fourier-space image %d is not phased and shifted\n", i);
        return NULL;
      }
  } else {
    return NULL;
  }
  Complex *buf = gather(list, n);
  if (!buf) return NULL;
  /* the result of sp_prtf_basic on spectra made by sp_image_fft: shifted, phased */
  Image *ret = sp_image_alloc(sp_image_x(list[0]), sp_image_y(list[0]), sp_image_z(list[0]));
  ret->shifted = 1;
  ret->phased = 1;
  const int in_place = (flags & SpInPlace) != 0;
  if (spb_prtf_advanced_host(sp_image_x(ret), sp_image_y(ret), sp_image_z(ret), n, (float *)buf, space, in_place,
                             (float *)ret->image->data)) {
    fprintf(stderr, "sp_prtf_advanced: %s\n", spb_error_string());
    sp_image_free(ret);
    free(buf);
    return NULL;
  }
  if (in_place) {
    const long long N = sp_image_size(list[0]);
    for (int i = 0; i < n; i++) memcpy(list[i]->image->data, buf + (size_t)i * N, sizeof(Complex) * (size_t)N);
  }
  free(buf);
  return ret;
}

void sp_image_superimpose_fractional(Image *a, Image *b, SpSuperimposeFlags flags, int precision) {
  if (spb_superimpose_fractional_host(sp_image_x(a), sp_image_y(a), sp_image_z(a), (const float *)a->image->data,
                                      (float *)b->image->data, (int)flags, precision))
    fprintf(stderr, "sp_image_superimpose_fractional: %s\n", spb_error_string());
}
