/*
 * Phase-retrieval transfer function of many reconstructions (the reference's
 * include/spimage/prtf.h: sp_prtf_basic, sp_prtf_advanced; src/prtf.c:6-78).
 * Same signatures, argument meaning and results; the work runs on the GPU
 * (spb_prtf_basic_host, spb_prtf_advanced_host in spb_device.h).
 */
#ifndef SPB_PRTF_H
#define SPB_PRTF_H 1
#include "image.h"
#ifdef __cplusplus
extern "C" {
#endif

/* The complex sum of the n images divided by the sum of their moduli, per
 * pixel (left as the sum where every modulus is zero).  The images are taken
 * to be in Fourier space; no phase or centrosymmetry correction.  NULL for
 * n < 1 or images of different sizes (src/prtf.c:6-34). */
Image *sp_prtf_basic(Image **list, int n);
/* sp_prtf_basic after superimposing every image on the first with
 * sp_image_superimpose_fractional(SpCorrectPhaseShift | SpEnantiomorph, 4)
 * in real space.  flags: SpFourierSpace or SpRealSpace (what the inputs are),
 * SpInPlace (the inputs are overwritten with the superimposed images, in
 * their own space) or SpOutOfPlace.  NULL when a required flag is missing or
 * on a device error (src/prtf.c:38-78; the reference aborts on Fourier-space
 * inputs that are not phased and shifted, this returns NULL). */
Image *sp_prtf_advanced(Image **list, int n, int flags);

#ifdef __cplusplus
}
#endif
#endif
