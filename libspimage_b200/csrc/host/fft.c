/*
 * FFT and blur over Image (host C) on the GPU kernels of this library.
 * Semantics of the reference's src/fft.c:53-189 (allocating variants set the
 * phased/shifted flags; the backward one aborts on unphased or unshifted
 * input) and src/image_filter.c:80-90 (sp_gaussian_blur).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "spimage.h"
#include "spimage/spb_device.h"

static void device_fft(const Image *in, Image *out, int sign) {
  if (spb_fft_host(sp_image_x(in), sp_image_y(in), sp_image_z(in), sign, (const float *)in->image->data,
                   (float *)out->image->data)) {
    fprintf(stderr, "spimage-b200: device FFT failed: %s\n", spb_error_string());
    abort();
  }
}

Image *sp_image_fftw3(const Image *img) {
  Image *res = sp_image_duplicate(img, SP_COPY_DETECTOR);
  res->phased = 1;
  device_fft(img, res, -1);
  res->shifted = 1;
  res->detector->image_center[0] = sp_image_x(res) / 2.0;
  res->detector->image_center[1] = sp_image_y(res) / 2.0;
  res->detector->image_center[2] = sp_image_z(res) / 2.0;
  return res;
}

void sp_image_fftw3_fast(const Image *in, Image *out) { device_fft(in, out, -1); }

Image *sp_image_ifftw3(const Image *img) {
  if (!img->phased) {
    fprintf(stderr, "Error: Trying reverse fft an unphased image!\n");
    abort();
  }
  if (!img->shifted) {
    fprintf(stderr, "Error: Trying to rev_fft an unshifted image!\n");
    abort();
  }
  Image *res = sp_image_duplicate(img, SP_COPY_DETECTOR);
  device_fft(img, res, +1);
  res->shifted = 0;
  return res;
}

void sp_image_ifftw3_fast(const Image *in, Image *out) { device_fft(in, out, +1); }

int sp_init_fft(int nthreads) {
  (void)nthreads;
  return 0;
}

Image *sp_image_cuda_fft(const Image *img) { return sp_image_fftw3(img); }

Image *sp_image_cuda_ifft(const Image *img) {
  Image *res = sp_image_duplicate(img, SP_COPY_DETECTOR);
  device_fft(img, res, +1);
  res->shifted = 0;
  return res;
}

/* FFT, Gaussian multiply, backward FFT, all on the device */
Image *sp_gaussian_blur(Image *in, real radius) {
  Image *res = sp_image_duplicate(in, SP_COPY_DETECTOR);
  res->phased = 1;
  res->shifted = 0;
  if (spb_blur_host(sp_image_x(in), sp_image_y(in), sp_image_z(in), (const float *)in->image->data, radius,
                    (float *)res->image->data)) {
    fprintf(stderr, "spimage-b200: device blur failed: %s\n", spb_error_string());
    abort();
  }
  return res;
}
