/*
 * Declarations shared by the library's host C sources (not part of the API).
 */
#ifndef SPB_HOST_INTERNAL_H
#define SPB_HOST_INTERNAL_H 1

#ifdef __cplusplus
extern "C" {
#endif

/* phase[i] = p_drand48() * 2 pi rounded to float for n pixels: the phases
 * sp_image_rephase(SP_RANDOM_PHASE) draws, from the same rand() words in the
 * same pixel order, leaving the generator where n calls of rand() leave it
 * (image.c; drawn on all host threads). */
void spb_random_phases(float *phase, long long n);

/* u[i] = p_drand48() for n consecutive draws, the same values and generator
 * state as n calls (drawn on all host threads) */
void spb_random_uniforms(float *u, long long n);

/* Runs fn(ctx, t, i0, i1) over [0, n) in contiguous spans on up to 8 host
 * threads (one span when n is small); span t covers [i0, i1).  Returns the
 * number of spans (at most SPB_PAR_MAX). */
#define SPB_PAR_MAX 8
typedef void (*spb_span_fn)(void *ctx, int t, long long i0, long long i1);
int spb_parallel_for(long long n, spb_span_fn fn, void *ctx);

/* Stores for host arrays that the GPU copies next.  A copy engine reads host
 * memory that several cores have just written (lines dirty in their private
 * caches) several times slower than memory one core wrote: 4 MiB written by
 * the host threads took 0.45-0.64 ms to upload against 0.09 ms clean.
 * Non-temporal stores put the values in memory directly, so the upload runs
 * at full speed.  A span that stores this way ends with spb_stream_fence()
 * (non-temporal stores are weakly ordered). */
#if defined(__SSE2__)
#include <emmintrin.h>
#include <string.h>
static inline void spb_stream_f32(float *p, float v) {
  int b;
  memcpy(&b, &v, sizeof b);
  _mm_stream_si32((int *)p, b);
}
static inline void spb_stream_u32(void *p, unsigned v) { _mm_stream_si32((int *)p, (int)v); }
static inline void spb_stream_fence(void) { _mm_sfence(); }
#else
static inline void spb_stream_f32(float *p, float v) { *p = v; }
static inline void spb_stream_u32(void *p, unsigned v) { *(unsigned *)p = v; }
static inline void spb_stream_fence(void) {}
#endif

#ifdef __cplusplus
}
#endif

#endif
