/*
 * Small exported helpers compiled into oracle/_ref/libspref.so next to the
 * reference's own sources, so tests can drive the reference CPU engine through
 * ctypes: the reference's sp_smap constructors and sp_smap_interpolate are
 * static inline (include/spimage/map.h), and Image / SpPhaser fields are only
 * reachable through its headers.  Test infrastructure only.
 */
#include <spimage.h>

Image *ref_image_alloc(int nx, int ny, int nz) { return sp_image_alloc(nx, ny, nz); }
void ref_image_free(Image *img) { sp_image_free(img); }
Complex *ref_image_data(Image *img) { return img->image->data; }
int *ref_image_mask(Image *img) { return img->mask->data; }
void ref_image_set_flags(Image *img, int phased, int shifted) { img->phased = phased; img->shifted = shifted; }

sp_smap *ref_smap(int n, const float *keys, const float *values) {
  sp_smap *m = sp_smap_alloc(n > 0 ? n : 1);
  for (int i = 0; i < n; i++) sp_smap_insert(m, keys[i], values[i]);
  return m;
}
float ref_smap_interpolate(sp_smap *m, float x) { return sp_smap_interpolate(m, x); }

Complex *ref_phaser_g(SpPhaser *ph, int which) {
  Image *g = which == 0 ? ph->g0 : (which == 1 ? ph->g1 : ph->gp);
  return g ? g->image->data : NULL;
}
int *ref_phaser_flags(SpPhaser *ph) { return ph->pixel_flags ? ph->pixel_flags->data : NULL; }
int ref_phaser_iteration(SpPhaser *ph) { return ph->iteration; }
float ref_dm_gamma(SpPhasingAlgorithm *alg, int which) {
  SpPhasingDiffMapParameters *p = (SpPhasingDiffMapParameters *)alg->params;
  return which == 1 ? p->gamma1 : p->gamma2;
}
