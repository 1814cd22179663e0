// Internal device-layer declarations shared by the CUDA translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "spb_fft.cuh"

namespace spb {

// pixel flag bits kept per pixel on the device (uint8), same meaning as the
// reference's SpPhasingPixelFlags (include/spimage/phasing.h:19)
enum : uint8_t { FLAG_INSIDE = 1, FLAG_MEASURED = 2 };

enum Alg : int { ALG_HIO = 1, ALG_RAAR = 2, ALG_DM = 3, ALG_ER = 4 };

enum Constraint : int {
  C_REAL = 1, C_POS_REAL = 2, C_POS_COMPLEX = 4, C_FLIP = 8, C_CENTROSYM = 16, C_MARGIN = 32
};

// Row-pass modes (lines along x, contiguous)
enum RowMode : int {
  ROW_FWD = 0,          // X = fwd_x(src)
  ROW_FWD_DEPHASE = 1,  // X = fwd_x(|src| + 0i)
  ROW_INV = 2,          // out = inv_x(src)
  ROW_INV_SCALE = 3,    // out = inv_x(src) * (1/N) (complex multiply by (1/N, 0))
  ROW_INV_ABS = 4,      // absout = |inv_x(src)|
  ROW_ITER = 5,         // gp = inv_x(Y)/N; g1 = update(gp, g0); X = fwd_x(g1)
  ROW_DM_F1_FWD = 6,    // Xf = fwd_x(f1(g)) with f1 = inside ? g : -gamma1*g
  ROW_DM_ITER = 7,      // rho = inv_x(Y), f = inv_x(Yf); g1 = DM update; X = fwd_x(g1); Xf = fwd_x(f1(g1))
  ROW_FWD_F32 = 8,      // X = fwd_x(real32 + 0i)
  ROW_FWD_SQUARE_F32 = 9,  // X = fwd_x(real32^2 + 0i)
};

// Column-pass modes (lines along y or z, strided)
enum ColMode : int {
  COL_FWD = 0,
  COL_INV = 1,
  COL_PROJECT = 2,       // fwd, Fourier constraints + projection, inv
  COL_PROJECT_NOFC = 3,  // fwd, projection only (difference-map f1), inv
  COL_BLUR = 4,          // fwd, Gaussian multiplier, inv
  COL_INV_SQUARE_F32 = 5,  // inv of (real32^2 + 0i) input (Patterson)
};

struct PassArgs {
  // geometry
  int nx, ny, nz;
  long long n;  // nx*ny*nz
  // line addressing for column passes: addr = o*ostride + c + i*estride
  long long ostride, estride;
  int ncols, nouter;
  long long outer0;  // first outer line of this launch (grids are split at 65535)
  int line_axis;     // axis the column lines run along (1: y, outer = start*nz + z, column = x; 2: z, column = y*nx + x)
  // buffers
  const float2 *src;
  const float2 *src2;  // second input line (DM: Yf)
  const float2 *g0;    // previous iterate
  float2 *dst;         // main output (X or out)
  float2 *dst2;        // second output (DM: Xf)
  float2 *g1;          // new iterate
  float2 *gp;          // model before projection (optional)
  float *absout;
  const float *f32src;
  const float *amp, *amp_min, *amp_max;
  const float2 *phased_amp;
  const uint8_t *flags;
  // line-major copies for the projection pass (lines along the last axis):
  // amp_line[L*len + i] and measured bit i of line L in
  // meas_bits[L*meas_words + i/32]; null when not built
  const float *amp_line;
  const uint32_t *meas_bits;
  const int *amp_bad;  // nonzero: some amplitude of amp_line lies outside the branch-free quotient's domain
  int meas_words;
  // launch shape: lines per block of the row pass (0: the built-in choice)
  int row_lpb;
  int row_g0;  // g0 staging of the register row pass: 0 auto, 1 at the start, 2 between the transforms
  // 8 points per thread in the iteration's passes (spb_split.cu): 0 auto
  // (when the 16-point kernels would leave the SMs short of warps), 1 never,
  // 2 wherever a kernel exists
  int split;
  // columns per block of the projection pass (0: the built-in width); see col_width_ok
  int col_width;
  // projection pass column tiles by TMA (spb_fast.cu col_tma_kernel): 2 always where the
  // tile fits, 0 where it fits at the built-in width, 1 never
  int tma;
  int *err_flag;  // set by a kernel that could not do its work (device): 1 a bounded wait ran out, 2 a misaligned TMA tile
  // 1: launch the register pass kernels with programmatic dependent launch
  int pdl;
  // scalars
  int alg, constraints, objective;
  float beta, one_m2b, inv_n;
  // graph replays read beta from a device table: beta_tab[*beta_base + beta_idx]
  const float *beta_tab;
  const int *beta_base;
  int beta_idx;
  float gamma1, gamma2, one_p_g2, size_f;
  float inv_size_pow2;  // 1/size_f when the image size is a power of two (x/size_f == x*inv_size_pow2 then), else 0
  // pixels per start: the amplitude-side arrays (amp, amp_min, amp_max,
  // phased_amp) hold one start and are indexed modulo n_start
  long long n_start;
  // blur
  double blur_c0;   // -2*pow(pi,2) (host glibc)
  double blur_r2;   // pow(radius,2)
  const double *blur_r2_dev;  // when set, pow(radius,2) is read here (captured support updates)
  const float *blur_tab;      // when set, the blur factor of distances (dx, dy, dz): [dz][dy][dx], n/2+1 each
  float nx_f;       // (float)nx
  float n_f;        // (float)N
};

// Radix select state of one start: pass p (0..3) histograms the 8-bit digit
// of the keys that match pass_prefix[p] under pass_mask[p] into hist[p]; the
// digit picked from it narrows the prefix for pass p + 1 (pass_rank[p] is the
// rank sought among the keys matching pass p's prefix, 0-based, descending).
struct SelectState {
  unsigned long long rank;  // rank sought among all keys (pass 0)
  unsigned int hist[4][256];
  unsigned int pass_prefix[4], pass_mask[4];
  unsigned long long pass_rank[4];
  unsigned int reserved[1010];
  float result;  // the selected key (area rule) or the maximum (threshold rule)
  unsigned int maxbits;
};
static_assert(sizeof(SelectState) == 8216, "the selection state keeps its size");

// register-resident kernels (spb_fast.cu); cudaErrorNotSupported when the
// line length or mode has none
cudaError_t launch_row_fast(int mode, const LinePlan &px, const PassArgs &a, cudaStream_t st);
cudaError_t launch_col_fast(int mode, const LinePlan &pl, const PassArgs &a, cudaStream_t st);
// whether the projection pass has a kernel of w columns per block for lines of n points
bool col_width_ok(int n, int w);
// the same for the general kernels' compile-time-plan lengths (192, 384, 1000)
bool general_col_width_ok(int n, int w);
// all iterations of a call for every start of an N x N pattern (N = 32, 64,
// 128), one block per start with its spectrum resident (spb_fast.cu); a.dst
// holds X on entry and exit, g0/g1 are the two iterate buffers (start-major)
// the y and z passes of a 3-D volume with ny = nz = 64 or 128 in one launch
// (spb_fast.cu plane_kernel); cudaErrorNotSupported where it does not apply
bool plane_fits(int mode, const LinePlan &pl, const PassArgs &a);
cudaError_t launch_plane(int mode, const LinePlan &pl, const PassArgs &a, cudaStream_t st);
cudaError_t launch_persist(const LinePlan &px, const PassArgs &a, float2 *g0, float2 *g1, int cur0, int iters,
                           int keep_gp, int nb, cudaStream_t st);
// 8-point kernels of the iteration's two passes (spb_split.cu)
cudaError_t launch_row_split(int mode, const LinePlan &px, const PassArgs &a, cudaStream_t st);
cudaError_t launch_col_split(int mode, const LinePlan &pl, const PassArgs &a, cudaStream_t st);
cudaError_t launch_gauss_table(const PassArgs &a, float *tab, cudaStream_t st);
cudaError_t check_roundings(unsigned lo, unsigned hi, unsigned long long ndiv, unsigned long long seed,
                            unsigned a_stride, unsigned long long *d_bad);

// host-side launchers (spb_kernels.cu): register kernels where available,
// general kernels otherwise
cudaError_t launch_row(int mode, const LinePlan &px, const PassArgs &a, cudaStream_t st);
cudaError_t launch_col(int mode, const LinePlan &pl, int line_len, const PassArgs &a, cudaStream_t st);
// support selection and reductions; nb starts of n pixels each, start b at offset b*n
// k_dev / rel_dev: when set, the rank k / the relative threshold is read from
// device memory at run time instead of the value argument
// pdl: launch with programmatic dependent launch (each kernel waits for its
// predecessor's grid before touching memory)
cudaError_t launch_select_kth_desc(const float *absv, long long n, int nb, long long k, SelectState *state,
                                   cudaStream_t st, const unsigned long long *k_dev, bool pdl);
cudaError_t launch_max_abs(const float *absv, long long n, int nb, SelectState *state, cudaStream_t st, bool pdl);
cudaError_t launch_mask_from_abs(const float *absv, SelectState *state, float rel, int use_rel, uint8_t *flags,
                                 long long n, int nb, cudaStream_t st, const float *rel_dev, bool pdl);
// The selection and mask of every start in one launch over a thread-block
// cluster per start (area rule: use_rel 0, k-th largest at rank or *rank_dev;
// threshold rule: use_rel 1, maximum times rel or *rel_dev), where a start's
// keys fit the cluster's shared memory (select_cluster_fits); else
// cudaErrorNotSupported and nothing is launched.
bool select_cluster_fits(long long n);
cudaError_t launch_select_mask_cluster(const float *absv, long long n, int nb, int use_rel, unsigned long long rank,
                                       const unsigned long long *rank_dev, float rel, const float *rel_dev,
                                       SelectState *state, uint8_t *flags, cudaStream_t st, bool pdl);
// out[b*4 + k]; scratch of reduce_scratch_doubles(nb) doubles starting at out
int reduce_scratch_doubles(int nb);
cudaError_t launch_reduce_efourier(const float2 *F, const float *amp, const uint8_t *flags, long long n, int nb,
                                   double *out, cudaStream_t st);
cudaError_t launch_reduce_ereal(const float2 *gp, const uint8_t *flags, long long n, int nb, double *out,
                                cudaStream_t st);
cudaError_t launch_count_inside(const uint8_t *flags, long long n, int nb, double *out, cudaStream_t st);
cudaError_t launch_scale_cmul(float2 *a, long long n, float v, cudaStream_t st);

}  // namespace spb
