/*
 * Phase-retrieval API: drop-in for the reference's include/spimage/phasing.h.
 *
 * Enums, parameter structs and the SpPhaser field prefix up to gp keep the
 * reference's layout (phasing.h:14-91), because callers set ph->algorithm /
 * ph->sup_algorithm and read ph->model directly.  The private tail is one
 * opaque pointer to the device context.  Every iteration runs on the GPU
 * (SpEngineCUDA); there is no CPU engine in this library: SpEngineCPU makes
 * sp_phaser_init return -3 instead of silently running elsewhere.
 */
#ifndef SPB_PHASING_H
#define SPB_PHASING_H 1
#include "image.h"
#include "map.h"
#include "support_update.h"
#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  SpModelRandomPhases = 1,
  SpModelZeroPhases = 2,
  SpModelRandomValues = 4,
  SpModelMaskedOutZeroed = 256
} SpModelInitialization;
typedef enum { SpSupportFromPatterson = 1 } SpSupportInitialization;
typedef enum { SpHIO = 1, SpRAAR, SpDiffMap, SpER } SpPhasingAlgorithmType;
typedef enum {
  SpNoConstraints = 0,
  SpRealObject = 1,
  SpPositiveRealObject = 2,
  SpPositiveComplexObject = 4,
  SpPositivityFlipping = 8,
  SpCentrosymmetricObject = 16,
  SpAmplitudeErrorMargin = 32
} SpPhasingConstraints;
typedef enum { SpEngineAutomatic = 0, SpEngineCPU = 1, SpEngineCUDA = 2 } SpPhasingEngine;
typedef enum { SpPixelInsideSupport = 1, SpPixelMeasuredAmplitude = 2 } SpPhasingPixelFlags;
typedef enum { SpRecoverPhases = 0, SpRecoverAmplitudes = 1 } SpPhasingObjective;

typedef struct {
  sp_smap *beta;
  SpPhasingConstraints constraints;
} SpPhasingHIOParameters;
typedef struct {
  SpPhasingConstraints constraints;
} SpPhasingERParameters;
typedef SpPhasingHIOParameters SpPhasingRAARParameters;
typedef struct {
  sp_smap *beta;
  real gamma1;
  real gamma2;
  SpPhasingConstraints constraints;
} SpPhasingDiffMapParameters;
typedef struct {
  SpPhasingAlgorithmType type;
  void *params;
} SpPhasingAlgorithm;

typedef struct {
  sp_3matrix *amplitudes;
  sp_3matrix *amplitudes_min;
  sp_3matrix *amplitudes_max;
  sp_c3matrix *phased_amplitudes;
  sp_i3matrix *pixel_flags;
  SpPhasingObjective phasing_objective;
  SpPhasingAlgorithm *algorithm;
  SpSupportArray *sup_algorithm;
  int iteration;
  int image_size;
  int nx;
  int ny;
  int nz;
  Image *model;
  int model_iteration;
  Image *old_model;
  int old_model_iteration;
  Image *model_change;
  int model_change_iteration;
  Image *support;
  int support_iteration;
  Image *amplitudes_image;
  Image *fmodel;
  int fmodel_iteration;
  Image *model_before_projection;
  int model_before_projection_iteration;
  SpPhasingEngine engine;
  Image *g0; /* unused by the GPU engine (NULL), kept for layout */
  Image *g1;
  Image *gp;
  void *device; /* opaque spb_ctx */
} SpPhaser;

/* phasing.c:16-76 */
SpPhasingAlgorithm *sp_phasing_hio_alloc(sp_smap *beta, SpPhasingConstraints constraints);
SpPhasingAlgorithm *sp_phasing_raar_alloc(sp_smap *beta, SpPhasingConstraints constraints);
SpPhasingAlgorithm *sp_phasing_diff_map_alloc(sp_smap *beta, real gamma1, real gamma2,
                                              SpPhasingConstraints constraints);
SpPhasingAlgorithm *sp_phasing_er_alloc(SpPhasingConstraints constraints);

/* phasing.c:78-186 */
SpPhaser *sp_phaser_alloc(void);
void sp_phaser_free(SpPhaser *ph);

/* phasing.c:365-554: host copies cached per iteration */
const Image *sp_phaser_model(SpPhaser *ph);
const Image *sp_phaser_model_with_support(SpPhaser *ph);
const Image *sp_phaser_model_before_projection(SpPhaser *ph);
const Image *sp_phaser_old_model(SpPhaser *ph);
const Image *sp_phaser_fmodel(SpPhaser *ph);
const Image *sp_phaser_fmodel_with_mask(SpPhaser *ph);
Image *sp_phaser_model_change(SpPhaser *ph);
const Image *sp_phaser_support(SpPhaser *ph);
const Image *sp_phaser_amplitudes(SpPhaser *ph);

/* phasing.c:803-893 */
real sp_phaser_ereal(SpPhaser *ph);
real sp_phaser_efourier(SpPhaser *ph, real *FcFo);
real sp_phaser_support_fraction(SpPhaser *ph);

/* phasing.c:189-363 */
void sp_phaser_set_model(SpPhaser *ph, const Image *model);
void sp_phaser_set_support(SpPhaser *ph, const Image *support);
void sp_phaser_set_phased_amplitudes(SpPhaser *ph, const Image *phased_amplitudes);
void sp_phaser_set_amplitudes(SpPhaser *ph, const Image *amplitudes);
void sp_phaser_set_amplitudes_margins(SpPhaser *ph, const Image *amplitudes_min, const Image *amplitudes_max);

/* phasing.c:558-604 */
int sp_phaser_init(SpPhaser *ph, SpPhasingAlgorithm *alg, SpSupportArray *sup_alg, SpPhasingEngine engine);
int sp_phaser_set_phasing_algorithm(SpPhaser *ph, SpPhasingAlgorithm *alg);
int sp_phaser_set_support_algorithm(SpPhaser *ph, SpSupportArray *alg);
/* phasing.c:606-724 */
int sp_phaser_init_model(SpPhaser *ph, const Image *model, int flags);
/* phasing.c:727-778 */
int sp_phaser_init_support(SpPhaser *ph, const Image *support, int flags, real value);
/* phasing.c:895-1024 */
int sp_phaser_iterate(SpPhaser *ph, int iterations);
void sp_phaser_set_objective(SpPhaser *ph, SpPhasingObjective obj);

/* support updates, support_update.c:124-179 (GPU) */
int sp_support_area_update_support(SpSupportAlgorithm *alg, SpPhaser *ph);
int sp_support_threshold_update_support(SpSupportAlgorithm *alg, SpPhaser *ph);
int sp_support_static_update_support(SpSupportAlgorithm *alg, SpPhaser *ph);
/* support_update.c:193-205: mask where |blurred template| exceeds the
 * template's value at the scheduled area (mask rebuilt on the GPU) */
int sp_support_template_update_support(SpSupportAlgorithm *alg, SpPhaser *ph);
/* support_update.c:225-290: `size` dilations then `size` erosions of the
 * support over the 6-neighbourhood (on the GPU) */
int sp_support_close_update_support(SpSupportAlgorithm *alg, SpPhaser *ph);
/* support_update.c:305-389: moves the support away from the borders of the
 * shifted layout and its centre of mass to the origin.  The reference also
 * Fourier-translates the phaser's cached host copy of the model, which the
 * iterations do not read; here only the support moves.  Computed on the host
 * from each start's support (float accumulation in pixel order, as the
 * reference). */
int sp_support_centre_image(SpSupportAlgorithm *alg, SpPhaser *ph);
/* support_update.c:489-494 */
int sp_support_array_update(SpSupportArray *array, SpPhaser *ph);

/* Not in the reference: message of the last device error seen by this
 * library (the reference calls exit()/abort() on device errors instead). */
const char *sp_phaser_last_error(void);
/* Not in the reference: run this phaser's device work on the caller's
 * cudaStream_t (NULL = the phaser's own stream), so a host framework can
 * order and time it with its own events.  Returns 0 or -8. */
int sp_phaser_set_cuda_stream(SpPhaser *ph, void *stream);
/* Not in the reference: the phaser's device context (spb_ctx *, see
 * spimage/spb_device.h), created on first use; NULL before the dimensions
 * are known. */
void *sp_phaser_device_context(SpPhaser *ph);
/* Not in the reference: choose the launch shapes of this phaser's device
 * passes for its current algorithm by measurement (row lines per block,
 * dependent launch); the reconstruction is left where it was and the choice is
 * cached per process by shape, start count and algorithm.  Returns 0, -2
 * without an algorithm, -8 on a device error. */
int sp_phaser_autotune(SpPhaser *ph);

/* Not in the reference: batched random starts.  The reference's
 * Reconstructor.reconstruct_loop (src/_spimage_reconstructor.py:677-740) runs
 * one reconstruction after another from different random starts; here one
 * SpPhaser advances `starts` independent reconstructions of the same pattern
 * together.  Call sp_phaser_set_starts before sp_phaser_init_model (it drops
 * the device state and the model).  Afterwards every SpPhaser call applies to
 * all starts: the algorithm, schedules, support updates and host-side edits
 * of the support are shared, each start keeps its own model and support, and
 * the single-image accessors (sp_phaser_model, sp_phaser_support,
 * sp_phaser_efourier, ...) report start 0.  Start b's results are bit for
 * bit those of a one-start phaser given the same starting model.  Returns 0,
 * -1 for starts < 1, -8 on a device error. */
int sp_phaser_set_starts(SpPhaser *ph, int starts);
int sp_phaser_starts(const SpPhaser *ph);
/* Starting models drawn per start on the host exactly as sp_phaser_init_model
 * draws them after sp_srand(seeds[b]) (flags as there, user model not
 * allowed), so start b reproduces a one-start run seeded with seeds[b].  With
 * seeds NULL the starts are drawn one after another from the current rand()
 * stream, as nb consecutive sp_phaser_init_model calls would draw them. */
int sp_phaser_init_models(SpPhaser *ph, int flags, const int *seeds);
/* Random-phase starting models drawn on the device (Philox4x32-10 keyed by
 * seeds[b]); for throughput runs that do not need the reference's rand()
 * stream.  SpModelMaskedOutZeroed may be added to flags. */
int sp_phaser_init_models_device(SpPhaser *ph, int flags, const unsigned long long *seeds);
/* Start b's model, support (1 inside, 0 outside) or model before projection
 * copied into `out` (an image of the phaser's shape). */
int sp_phaser_start_model(SpPhaser *ph, int start, Image *out);
int sp_phaser_start_support(SpPhaser *ph, int start, Image *out);
int sp_phaser_start_model_before_projection(SpPhaser *ph, int start, Image *out);
/* Start b's Fourier-space model (FFT of its model), as sp_phaser_fmodel. */
int sp_phaser_start_fmodel(SpPhaser *ph, int start, Image *out);
/* Per-start metrics into out[starts] (FcFo may be NULL). */
int sp_phaser_starts_efourier(SpPhaser *ph, real *out, real *FcFo);
int sp_phaser_starts_ereal(SpPhaser *ph, real *out);
int sp_phaser_starts_support_fraction(SpPhaser *ph, real *out);

#ifdef __cplusplus
}
#endif
#endif
