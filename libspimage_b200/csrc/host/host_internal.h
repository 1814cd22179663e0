/*
 * Declarations shared by the library's host C sources (not part of the API).
 */
#ifndef SPB_HOST_INTERNAL_H
#define SPB_HOST_INTERNAL_H 1

/* phase[i] = p_drand48() * 2 pi rounded to float for n pixels: the phases
 * sp_image_rephase(SP_RANDOM_PHASE) draws, from the same rand() words in the
 * same pixel order, leaving the generator where n calls of rand() leave it
 * (image.c; drawn on all host threads). */
void spb_random_phases(float *phase, long long n);

#endif
