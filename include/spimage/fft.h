/*
 * FFT entry points over Image (reference include/spimage/fft.h:25-34,87-131).
 * The public names are macros onto the exported sp_image_fftw3* symbols, as in
 * the reference, so existing callers link unchanged.  Here every transform
 * runs on the GPU (hand-written sm_100a kernels, no cuFFT/FFTW): forward is
 * exp(-2 pi i k x / n), unnormalised, x axis first; backward is unnormalised,
 * slowest axis first.
 */
#ifndef SPB_FFT_H
#define SPB_FFT_H 1
#include "image.h"
#ifdef __cplusplus
extern "C" {
#endif

#define sp_image_ifft(a) sp_image_ifftw3(a)
#define sp_image_fft(a) sp_image_fftw3(a)
#define sp_image_ifft_fast(a, b) sp_image_ifftw3_fast(a, b)
#define sp_image_fft_fast(a, b) sp_image_fftw3_fast(a, b)

/* src/fft.c:152-175: allocating forward FFT; result is phased and shifted */
Image *sp_image_fftw3(const Image *img);
/* src/fft.c:177-189: forward FFT of in into out (may alias) */
void sp_image_fftw3_fast(const Image *in, Image *out);
/* src/fft.c:53-85: allocating backward FFT; aborts on unphased or unshifted input */
Image *sp_image_ifftw3(const Image *img);
/* src/fft.c:87-99: backward FFT of in into out (may alias) */
void sp_image_ifftw3_fast(const Image *in, Image *out);
/* src/fft.c:34-49: thread count for the CPU FFT; the GPU path ignores it (returns 0) */
int sp_init_fft(int nthreads);
/* src/fft.cu:7-43: one-shot device FFTs (here identical to the above) */
Image *sp_image_cuda_fft(const Image *img);
Image *sp_image_cuda_ifft(const Image *img);

#ifdef __cplusplus
}
#endif
#endif
