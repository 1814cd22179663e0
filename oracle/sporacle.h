/*
 * sporacle -- CPU restatement of libspimage's phase-retrieval engine.
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker the CUDA path is compared
 * against.  Nothing in the product links or calls it.
 *
 * It restates the CPU engine of the reference (src/phasing.c,
 * src/support_update.c, src/image_filter.c:80-90, src/image_util.c helpers,
 * include/spimage/map.h:103-141) with the same floating-point types and
 * operation order, over the oracle FFT (oracle/cpufft).  Each function in
 * sporacle.c names the reference lines it follows.
 */
#ifndef SPORACLE_H
#define SPORACLE_H
#include "cpufft/spfft.h"

#ifdef __cplusplus
extern "C" {
#endif

enum { SPO_HIO = 1, SPO_RAAR = 2, SPO_DIFFMAP = 3, SPO_ER = 4 };
enum { SPO_SUP_THRESHOLD = 1, SPO_SUP_AREA = 2, SPO_SUP_CENTRE = 3, SPO_SUP_TEMPLATE = 4, SPO_SUP_STATIC = 5,
       SPO_SUP_CLOSE = 6 };
enum {
  SPO_REAL = 1, SPO_POS_REAL = 2, SPO_POS_COMPLEX = 4, SPO_FLIP = 8, SPO_CENTROSYM = 16,
  SPO_MARGIN = 32
};
enum { SPO_INSIDE = 1, SPO_MEASURED = 2 };
enum { SPO_RANDOM_PHASES = 1, SPO_ZERO_PHASES = 2, SPO_RANDOM_VALUES = 4, SPO_MASKED_OUT_ZEROED = 256 };

typedef struct spo_phaser spo_phaser;

void spo_srand(int seed);
float spo_bezier(int nkeys, const float *keys, const float *values, float x);

spo_phaser *spo_create(int nx, int ny, int nz);
void spo_destroy(spo_phaser *ph);
void spo_set_threads(spo_phaser *ph, int nthreads);
void spo_set_amplitudes(spo_phaser *ph, const float *amp, const int *mask);
void spo_set_amplitudes_margins(spo_phaser *ph, const float *amp_min, const float *amp_max);
void spo_set_phased_amplitudes(spo_phaser *ph, const spfft_cpx *pa, const int *mask);
void spo_set_objective(spo_phaser *ph, int objective);
void spo_set_support(spo_phaser *ph, const float *support_real);
void spo_init_support_patterson(spo_phaser *ph, float value);
void spo_set_algorithm(spo_phaser *ph, int type, int nbeta, const float *beta_keys, const float *beta_values,
                       float gamma1, float gamma2, int constraints);
void spo_clear_support_updates(spo_phaser *ph);
void spo_add_support_update(spo_phaser *ph, int type, int period, int nblur, const float *blur_keys,
                            const float *blur_values, int nsel, const float *sel_keys, const float *sel_values);
void spo_add_support_close(spo_phaser *ph, int period, int size);
void spo_add_support_centre(spo_phaser *ph, int period);
void spo_add_support_template(spo_phaser *ph, int period, const float *support_real, float blur_radius, int narea,
                              const float *area_keys, const float *area_values);
int spo_init_model(spo_phaser *ph, int flags, const spfft_cpx *user_model);
void spo_set_model(spo_phaser *ph, const spfft_cpx *model);
int spo_iterate(spo_phaser *ph, int iterations);
int spo_iteration(const spo_phaser *ph);
/* which: 0 = g0 (old model), 1 = g1 (model), 2 = gp (model before projection) */
void spo_get(const spo_phaser *ph, int which, spfft_cpx *out);
void spo_get_flags(const spo_phaser *ph, int *out);
float spo_efourier(spo_phaser *ph, float *FcFo);
float spo_ereal(spo_phaser *ph);
float spo_support_fraction(spo_phaser *ph);
float spo_dm_gamma(spo_phaser *ph, int which);

/* building blocks, exposed for element-level tests */
void spo_gaussian_blur(int nx, int ny, int nz, const spfft_cpx *in, float radius, spfft_cpx *out);
float spo_area_threshold(long n, const spfft_cpx *blur, float area);
void spo_module_projection(long n, spfft_cpx *G, const float *amp, const int *flags, int constraints);
void spo_fft(int nx, int ny, int nz, int sign, const spfft_cpx *in, spfft_cpx *out);

#ifdef __cplusplus
}
#endif
#endif
