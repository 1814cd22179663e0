// Phasing pass kernels for sm_100a.
//
// A 2-D iteration is two launches:
//   column pass  Y = inv_y(P(fwd_y(X)))        (P = Fourier constraints + projection)
//   row pass     gp = inv_x(Y)/N;  g1 = update(gp, g0);  X = fwd_x(g1)
// so the row FFT of the new iterate is produced while it is still on chip and
// the next iteration starts from it.  3-D adds a forward and an inverse
// y-pass around a z-column projection pass.  Every pointwise step uses
// explicitly rounded float arithmetic in the reference engine's operation
// order (src/phasing.c:1026-1274), so results match the CPU engine bit for bit
// when the FFT does.
#include <math.h>

#include "spb_internal.h"

namespace spb {

__device__ __forceinline__ float2 scale_cmul_dev(float2 v, float s) {
  // sp_image_scale: complex multiply by (s, 0)
  return make_float2(fsub(fmul(v.x, s), fmul(v.y, 0.0f)), fadd(fmul(v.x, 0.0f), fmul(s, v.y)));
}

__device__ __forceinline__ float2 apply_constraints(float2 g, uint8_t f, int c) {
  if (f & FLAG_INSIDE) {
    if (c & C_REAL) {
      g.y = 0.0f;
    } else if (c & C_POS_REAL) {
      if (g.x < 0) g.x = (c & C_FLIP) ? fabsf(g.x) : 0.0f;
      g.y = 0.0f;
    } else if (c & C_POS_COMPLEX) {
      if (g.x < 0) g.x = (c & C_FLIP) ? fabsf(g.x) : 0.0f;
      if (g.y < 0) g.y = (c & C_FLIP) ? fabsf(g.y) : 0.0f;
    }
  }
  return g;
}

// Fourier-space projection at pixel idx (src/phasing.c:1061-1109)
__device__ __forceinline__ float2 project(float2 G, long long idx, const PassArgs &a, bool fourier_constraints) {
  const uint8_t f = a.flags[idx];
  if (fourier_constraints && (a.constraints & C_CENTROSYM)) G.y = 0.0f;
  if (a.objective == 0) {
    if (f & FLAG_MEASURED) {
      float m = 1.0f;
      const float amp = a.amp[idx];
      if (!(a.constraints & C_MARGIN)) {
        m = __fdiv_rn(amp, cabs_ref(G));
      } else {
        const float av = cabs_ref(G);
        const float lo = a.amp_min[idx], hi = a.amp_max[idx];
        if (av < lo) m = __fdiv_rn(lo, av);
        else if (av > hi) m = __fdiv_rn(hi, av);
      }
      if (isfinite(m)) G = make_float2(fmul(G.x, m), fmul(G.y, m));
      else G = make_float2(amp, 0.0f);
    }
  } else {
    if (f & FLAG_MEASURED) G = a.phased_amp[idx];
  }
  return G;
}

// Fourier-domain Gaussian of sp_gaussian_blur (src/image_filter.c:80-90)
__device__ __forceinline__ float2 gauss_mult(float2 F, long long idx, const PassArgs &a) {
  const long long nxy = (long long)a.nx * a.ny;
  const float z = (float)(idx / nxy);
  const float y = (float)((idx % nxy) / a.nx);
  const float x = (float)(idx % a.nx);
  const float fx = (float)a.nx, fy = (float)a.ny, fz = (float)a.nz;
  const float dx = (__fsub_rn(fx, x) < x) ? __fsub_rn(fx, x) : x;
  const float dy = (__fsub_rn(fy, y) < y) ? __fsub_rn(fy, y) : y;
  const float dz = (__fsub_rn(fz, z) < z) ? __fsub_rn(fz, z) : z;
  const double s = __dadd_rn(__dadd_rn(__dmul_rn((double)dx, (double)dx), __dmul_rn((double)dy, (double)dy)),
                             __dmul_rn((double)dz, (double)dz));
  const float dist = __double2float_rn(__dsqrt_rn(s));
  const float cr = __fdiv_rn(dist, a.nx_f);
  const double arg = __dmul_rn(__dmul_rn(a.blur_c0, __dmul_rn((double)cr, (double)cr)), a.blur_r2);
  const float m = __double2float_rn(__ddiv_rn(exp(arg), (double)a.n_f));
  return scale_cmul_dev(F, m);
}

// ---------------------------------------------------------------- row pass
template <int MODE>
__global__ void __launch_bounds__(256) row_pass_kernel(LinePlan px, PassArgs a, int tpr, int rpb, long long nrows) {
  extern __shared__ float2 smem[];
  const int n = px.n;
  const int lr = threadIdx.x / tpr, t = threadIdx.x % tpr;
  const long long row = (long long)blockIdx.x * rpb + lr;
  const bool valid = row < nrows;
  const long long base = row * n;
  const size_t slab = (size_t)rpb * n;
  float2 *A = smem + (size_t)lr * n;
  float2 *B = A + slab;
  float2 *Cb = A + 2 * slab;
  float2 *D = A + 3 * slab;

  for (int i = t; i < n; i += tpr) {
    float2 v = make_float2(0.0f, 0.0f), w = make_float2(0.0f, 0.0f);
    if (valid) {
      if constexpr (MODE == ROW_FWD_DEPHASE) {
        v = make_float2(cabs_ref(a.src[base + i]), 0.0f);
      } else if constexpr (MODE == ROW_FWD_F32) {
        v = make_float2(a.f32src[base + i], 0.0f);
      } else if constexpr (MODE == ROW_FWD_SQUARE_F32) {
        const float s = a.f32src[base + i];
        v = make_float2(fmul(s, s), 0.0f);
      } else if constexpr (MODE == ROW_DM_F1_FWD) {
        v = a.src[base + i];
        if (!(a.flags[base + i] & FLAG_INSIDE)) v = make_float2(fmul(-a.gamma1, v.x), fmul(-a.gamma1, v.y));
      } else {
        v = a.src[base + i];
        if constexpr (MODE == ROW_DM_ITER) w = a.src2[base + i];
      }
    }
    A[i] = v;
    if constexpr (MODE == ROW_DM_ITER) Cb[i] = w;
  }
  __syncthreads();

  if constexpr (MODE == ROW_FWD || MODE == ROW_FWD_DEPHASE || MODE == ROW_FWD_F32 || MODE == ROW_FWD_SQUARE_F32 ||
                MODE == ROW_DM_F1_FWD) {
    float2 *r = line_fft<false>(A, B, px, 1, t, tpr);
    if (valid)
      for (int i = t; i < n; i += tpr) a.dst[base + i] = r[i];
  } else if constexpr (MODE == ROW_INV || MODE == ROW_INV_SCALE || MODE == ROW_INV_ABS) {
    float2 *r = line_fft<true>(A, B, px, 1, t, tpr);
    if (valid) {
      for (int i = t; i < n; i += tpr) {
        if constexpr (MODE == ROW_INV) a.dst[base + i] = r[i];
        else if constexpr (MODE == ROW_INV_SCALE) a.dst[base + i] = scale_cmul_dev(r[i], a.inv_n);
        else a.absout[base + i] = cabs_ref(r[i]);
      }
    }
  } else if constexpr (MODE == ROW_ITER) {
    float2 *r = line_fft<true>(A, B, px, 1, t, tpr);
    for (int i = t; i < n; i += tpr) {
      float2 g = make_float2(0.0f, 0.0f);
      if (valid) {
        const long long idx = base + i;
        const float2 gp = scale_cmul_dev(r[i], a.inv_n);
        if (a.gp) a.gp[idx] = gp;
        const uint8_t f = a.flags[idx];
        if (f & FLAG_INSIDE) {
          g = gp;
        } else if (a.alg == ALG_HIO) {
          const float2 g0 = a.g0[idx];
          g = make_float2(fsub(g0.x, fmul(gp.x, a.beta)), fsub(g0.y, fmul(gp.y, a.beta)));
        } else if (a.alg == ALG_RAAR) {
          const float2 g0 = a.g0[idx];
          g = make_float2(fadd(fmul(gp.x, a.one_m2b), fmul(g0.x, a.beta)),
                          fadd(fmul(gp.y, a.one_m2b), fmul(g0.y, a.beta)));
        }
        g = apply_constraints(g, f, a.constraints);
        a.g1[idx] = g;
      }
      r[i] = g;
    }
    __syncthreads();
    float2 *o = (r == A) ? B : A;
    float2 *x = line_fft<false>(r, o, px, 1, t, tpr);
    if (valid)
      for (int i = t; i < n; i += tpr) a.dst[base + i] = x[i];
  } else if constexpr (MODE == ROW_DM_ITER) {
    float2 *rho = line_fft<true>(A, B, px, 1, t, tpr);
    float2 *fr = line_fft<true>(Cb, D, px, 1, t, tpr);
    for (int i = t; i < n; i += tpr) {
      float2 g = make_float2(0.0f, 0.0f), f1 = g;
      if (valid) {
        const long long idx = base + i;
        const float2 rv = rho[i], fv = fr[i], g0 = a.g0[idx];
        if (a.gp) a.gp[idx] = rv;
        const uint8_t f = a.flags[idx];
        if (f & FLAG_INSIDE) {
          g.x = fadd(g0.x, fmul(a.beta, fsub(__fdiv_rn(fmul(a.one_p_g2, rv.x), a.size_f), fmul(a.gamma2, g0.x))));
          g.y = fadd(g0.y, fmul(a.beta, fsub(__fdiv_rn(fmul(a.one_p_g2, rv.y), a.size_f), fmul(a.gamma2, g0.y))));
        } else {
          g = g0;
        }
        g.x = fsub(g.x, __fdiv_rn(fmul(a.beta, fv.x), a.size_f));
        g.y = fsub(g.y, __fdiv_rn(fmul(a.beta, fv.y), a.size_f));
        g = apply_constraints(g, f, a.constraints);
        a.g1[idx] = g;
        f1 = (f & FLAG_INSIDE) ? g : make_float2(fmul(-a.gamma1, g.x), fmul(-a.gamma1, g.y));
      }
      rho[i] = g;
      fr[i] = f1;
    }
    __syncthreads();
    float2 *o1 = (rho == A) ? B : A;
    float2 *x = line_fft<false>(rho, o1, px, 1, t, tpr);
    float2 *o2 = (fr == Cb) ? D : Cb;
    float2 *xf = line_fft<false>(fr, o2, px, 1, t, tpr);
    if (valid)
      for (int i = t; i < n; i += tpr) {
        a.dst[base + i] = x[i];
        a.dst2[base + i] = xf[i];
      }
  }
}

// ------------------------------------------------------------- column pass
template <int MODE>
__global__ void __launch_bounds__(1024) col_pass_kernel(LinePlan pl, PassArgs a, int ct, int tpc) {
  extern __shared__ float2 smem[];
  const int n = pl.n;
  const int cc = threadIdx.x % ct, t = threadIdx.x / ct;
  const long long o = blockIdx.y;
  const int c = blockIdx.x * ct + cc;
  const bool valid = c < a.ncols;
  float2 *A = smem + cc;
  float2 *B = smem + (size_t)n * ct + cc;
  const long long lbase = o * a.ostride + c;

  for (int i = t; i < n; i += tpc) {
    float2 v = make_float2(0.0f, 0.0f);
    if (valid) {
      if constexpr (MODE == COL_INV_SQUARE_F32) {
        const float s = a.f32src[lbase + i * a.estride];
        v = make_float2(fmul(s, s), 0.0f);
      } else {
        v = a.src[lbase + i * a.estride];
      }
    }
    A[(size_t)i * ct] = v;
  }
  __syncthreads();

  float2 *r;
  if constexpr (MODE == COL_FWD) {
    r = line_fft<false>(A, B, pl, ct, t, tpc);
  } else if constexpr (MODE == COL_INV || MODE == COL_INV_SQUARE_F32) {
    r = line_fft<true>(A, B, pl, ct, t, tpc);
  } else {
    float2 *f = line_fft<false>(A, B, pl, ct, t, tpc);
    if (valid) {
      for (int i = t; i < n; i += tpc) {
        const long long idx = lbase + i * a.estride;
        float2 G = f[(size_t)i * ct];
        if constexpr (MODE == COL_PROJECT) G = project(G, idx, a, true);
        else if constexpr (MODE == COL_PROJECT_NOFC) G = project(G, idx, a, false);
        else G = gauss_mult(G, idx, a);
        f[(size_t)i * ct] = G;
      }
    }
    __syncthreads();
    float2 *o2 = (f == A) ? B : A;
    r = line_fft<true>(f, o2, pl, ct, t, tpc);
  }
  if (valid)
    for (int i = t; i < n; i += tpc) a.dst[lbase + i * a.estride] = r[(size_t)i * ct];
}

// ---------------------------------------------------------------- launchers
static int pow2_at_least(int v) {
  int p = 1;
  while (p < v) p <<= 1;
  return p;
}

template <int MODE>
static cudaError_t row_launch(const LinePlan &px, const PassArgs &a, cudaStream_t st) {
  const int n = px.n;
  int tpr = pow2_at_least((n + 15) / 16);
  if (tpr > 256) tpr = 256;
  if (tpr < 1) tpr = 1;
  const int rpb = 256 / tpr;
  const long long nrows = a.n / n;
  const int nbuf = (MODE == ROW_DM_ITER) ? 4 : 2;
  const size_t smem = (size_t)nbuf * rpb * n * sizeof(float2);
  auto k = row_pass_kernel<MODE>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const long long grid = (nrows + rpb - 1) / rpb;
  k<<<(unsigned)grid, rpb * tpr, smem, st>>>(px, a, tpr, rpb, nrows);
  return cudaGetLastError();
}

cudaError_t launch_row(int mode, const LinePlan &px, const PassArgs &a, cudaStream_t st) {
  switch (mode) {
    case ROW_FWD: return row_launch<ROW_FWD>(px, a, st);
    case ROW_FWD_DEPHASE: return row_launch<ROW_FWD_DEPHASE>(px, a, st);
    case ROW_INV: return row_launch<ROW_INV>(px, a, st);
    case ROW_INV_SCALE: return row_launch<ROW_INV_SCALE>(px, a, st);
    case ROW_INV_ABS: return row_launch<ROW_INV_ABS>(px, a, st);
    case ROW_ITER: return row_launch<ROW_ITER>(px, a, st);
    case ROW_DM_F1_FWD: return row_launch<ROW_DM_F1_FWD>(px, a, st);
    case ROW_DM_ITER: return row_launch<ROW_DM_ITER>(px, a, st);
    case ROW_FWD_F32: return row_launch<ROW_FWD_F32>(px, a, st);
    case ROW_FWD_SQUARE_F32: return row_launch<ROW_FWD_SQUARE_F32>(px, a, st);
  }
  return cudaErrorInvalidValue;
}

template <int MODE>
static cudaError_t col_launch(const LinePlan &pl, const PassArgs &a, cudaStream_t st) {
  const int n = pl.n;
  int ct = 4096 / (n > 0 ? n : 1);
  if (ct > 16) ct = 16;
  if (ct < 1) ct = 1;
  int tpc = pow2_at_least((n + 15) / 16);
  if (tpc * ct > 1024) tpc = 1024 / ct;
  if (tpc * ct < 32) tpc = 32 / ct;
  const size_t smem = (size_t)2 * n * ct * sizeof(float2);
  auto k = col_pass_kernel<MODE>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((a.ncols + ct - 1) / ct, a.nouter);
  k<<<grid, ct * tpc, smem, st>>>(pl, a, ct, tpc);
  return cudaGetLastError();
}

cudaError_t launch_col(int mode, const LinePlan &pl, int line_len, const PassArgs &a, cudaStream_t st) {
  (void)line_len;
  switch (mode) {
    case COL_FWD: return col_launch<COL_FWD>(pl, a, st);
    case COL_INV: return col_launch<COL_INV>(pl, a, st);
    case COL_PROJECT: return col_launch<COL_PROJECT>(pl, a, st);
    case COL_PROJECT_NOFC: return col_launch<COL_PROJECT_NOFC>(pl, a, st);
    case COL_BLUR: return col_launch<COL_BLUR>(pl, a, st);
    case COL_INV_SQUARE_F32: return col_launch<COL_INV_SQUARE_F32>(pl, a, st);
  }
  return cudaErrorInvalidValue;
}

// ------------------------------------------------- support selection kernels
// Keys are the bit patterns of non-negative floats, which order like the floats.
__global__ void select_hist_kernel(const float *__restrict__ v, long long n, SelectState *s, int shift, int bits) {
  __shared__ unsigned int h[2048];
  const int nb = 1 << bits;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) h[i] = 0;
  __syncthreads();
  const unsigned int prefix = s->prefix, pmask = s->prefix_mask;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const unsigned int key = __float_as_uint(v[i]);
    if ((key & pmask) == prefix) atomicAdd(&h[(key >> shift) & (nb - 1)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nb; i += blockDim.x)
    if (h[i]) atomicAdd(&s->hist[i], h[i]);
}

// one block: find the digit holding the rank-th largest key, narrow the prefix
__global__ void select_pick_kernel(SelectState *s, int shift, int bits, int last) {
  __shared__ unsigned long long csum[2048];
  const int nb = 1 << bits;
  // inclusive suffix sums (counts of digits >= d), computed per thread by a simple loop
  for (int d = threadIdx.x; d < nb; d += blockDim.x) csum[d] = s->hist[d];
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long cum = 0;
    const unsigned long long rank = s->rank;
    int pick = 0;
    for (int d = nb - 1; d >= 0; d--) {
      const unsigned long long c = csum[d];
      if (cum + c > rank) { pick = d; s->rank = rank - cum; break; }
      cum += c;
    }
    s->prefix |= ((unsigned int)pick) << shift;
    s->prefix_mask |= ((unsigned int)(nb - 1)) << shift;
    if (last) s->result = __uint_as_float(s->prefix);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < nb; d += blockDim.x) s->hist[d] = 0;
}

__global__ void select_init_kernel(SelectState *s, unsigned long long rank) {
  for (int d = threadIdx.x; d < 2048; d += blockDim.x) s->hist[d] = 0;
  if (threadIdx.x == 0) {
    s->prefix = 0;
    s->prefix_mask = 0;
    s->rank = rank;
    s->maxbits = 0;
  }
}

cudaError_t launch_select_kth_desc(const float *absv, long long n, long long k, SelectState *state,
                                   cudaStream_t st) {
  select_init_kernel<<<1, 256, 0, st>>>(state, (unsigned long long)k);
  const int shifts[3] = {21, 10, 0}, widths[3] = {11, 11, 10};
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  for (int p = 0; p < 3; p++) {
    select_hist_kernel<<<(unsigned)blocks, 256, 0, st>>>(absv, n, state, shifts[p], widths[p]);
    select_pick_kernel<<<1, 256, 0, st>>>(state, shifts[p], widths[p], p == 2);
  }
  return cudaGetLastError();
}

__global__ void max_abs_kernel(const float *__restrict__ v, long long n, SelectState *s) {
  unsigned int m = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float x = v[i];
    if (!isnan(x)) m = max(m, __float_as_uint(x));
  }
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(&s->maxbits, m);
}

__global__ void max_finish_kernel(SelectState *s) { s->result = __uint_as_float(s->maxbits); }

cudaError_t launch_max_abs(const float *absv, long long n, SelectState *state, cudaStream_t st) {
  select_init_kernel<<<1, 256, 0, st>>>(state, 0);
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  max_abs_kernel<<<(unsigned)blocks, 256, 0, st>>>(absv, n, state);
  max_finish_kernel<<<1, 1, 0, st>>>(state);
  return cudaGetLastError();
}

// support_from_absolute_threshold (src/support_update.c:392-400): strict '>'
__global__ void mask_kernel(const float *__restrict__ v, const SelectState *s, float rel, int use_rel,
                            uint8_t *flags, long long n) {
  const float t = use_rel ? __fmul_rn(s->result, rel) : s->result;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const uint8_t f = flags[i];
    flags[i] = (v[i] > t) ? (uint8_t)(f | FLAG_INSIDE) : (uint8_t)(f & ~FLAG_INSIDE);
  }
}

cudaError_t launch_mask_from_abs(const float *absv, const float *thr_dev, float rel, int use_rel, uint8_t *flags,
                                 long long n, cudaStream_t st) {
  (void)thr_dev;
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  mask_kernel<<<(unsigned)blocks, 256, 0, st>>>(absv, reinterpret_cast<const SelectState *>(thr_dev), rel, use_rel,
                                                flags, n);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- reductions
#define RED_BLOCKS 592

// efourier terms (src/phasing.c:852-891): nom, den, FcFo numerator, denominator
__global__ void efourier_partial_kernel(const float2 *__restrict__ F, const float *__restrict__ amp,
                                        const uint8_t *__restrict__ flags, long long n, double *part) {
  double s[4] = {0, 0, 0, 0};
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float fa = cabs_ref(F[i]);
    if (flags[i] & FLAG_MEASURED) {
      const float aa = fabsf(amp[i]);
      const double d = (double)__fsub_rn(fa, aa);
      s[0] += d * d;
      s[1] += (double)aa * (double)aa;
      s[2] += aa;
      s[3] += fa;
    } else {
      s[1] += (double)fa * (double)fa;
    }
  }
  __shared__ double sh[4][256];
  for (int k = 0; k < 4; k++) sh[k][threadIdx.x] = s[k];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      for (int k = 0; k < 4; k++) sh[k][threadIdx.x] += sh[k][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 4; k++) part[blockIdx.x * 4 + k] = sh[k][0];
}

__global__ void ereal_partial_kernel(const float2 *__restrict__ gp, const uint8_t *__restrict__ flags, long long n,
                                     double *part) {
  double s[4] = {0, 0, 0, 0};
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double a = (double)cabs_ref(gp[i]);
    if (!(flags[i] & FLAG_INSIDE)) s[0] += a * a;
    s[1] += a * a;
  }
  __shared__ double sh[4][256];
  for (int k = 0; k < 4; k++) sh[k][threadIdx.x] = s[k];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      for (int k = 0; k < 4; k++) sh[k][threadIdx.x] += sh[k][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 4; k++) part[blockIdx.x * 4 + k] = sh[k][0];
}

__global__ void finish4_kernel(const double *part, int nparts, double *out4) {
  __shared__ double sh[4][256];
  double s[4] = {0, 0, 0, 0};
  for (int i = threadIdx.x; i < nparts; i += blockDim.x)
    for (int k = 0; k < 4; k++) s[k] += part[i * 4 + k];
  for (int k = 0; k < 4; k++) sh[k][threadIdx.x] = s[k];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      for (int k = 0; k < 4; k++) sh[k][threadIdx.x] += sh[k][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 4; k++) out4[k] = sh[k][0];
}

cudaError_t launch_reduce_efourier(const float2 *F, const float *amp, const uint8_t *flags, long long n,
                                   double *out4, cudaStream_t st) {
  double *part = out4 + 4;
  efourier_partial_kernel<<<RED_BLOCKS, 256, 0, st>>>(F, amp, flags, n, part);
  finish4_kernel<<<1, 256, 0, st>>>(part, RED_BLOCKS, out4);
  return cudaGetLastError();
}

cudaError_t launch_reduce_ereal(const float2 *gp, const uint8_t *flags, long long n, double *out4,
                                cudaStream_t st) {
  double *part = out4 + 4;
  ereal_partial_kernel<<<RED_BLOCKS, 256, 0, st>>>(gp, flags, n, part);
  finish4_kernel<<<1, 256, 0, st>>>(part, RED_BLOCKS, out4);
  return cudaGetLastError();
}

__global__ void count_inside_kernel(const uint8_t *flags, long long n, unsigned long long *out) {
  unsigned long long c = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    c += (flags[i] & FLAG_INSIDE) ? 1 : 0;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, c);
}

cudaError_t launch_count_inside(const uint8_t *flags, long long n, unsigned long long *out, cudaStream_t st) {
  cudaMemsetAsync(out, 0, sizeof(unsigned long long), st);
  count_inside_kernel<<<RED_BLOCKS, 256, 0, st>>>(flags, n, out);
  return cudaGetLastError();
}

__global__ void flags_from_int_kernel(const int *src, uint8_t *dst, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] = (uint8_t)(src[i] & 3);
}
__global__ void flags_to_int_kernel(const uint8_t *src, int *dst, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] = (int)src[i];
}
cudaError_t launch_flags_from_int(const int *src, uint8_t *dst, long long n, cudaStream_t st) {
  flags_from_int_kernel<<<RED_BLOCKS, 256, 0, st>>>(src, dst, n);
  return cudaGetLastError();
}
cudaError_t launch_flags_to_int(const uint8_t *src, int *dst, long long n, cudaStream_t st) {
  flags_to_int_kernel<<<RED_BLOCKS, 256, 0, st>>>(src, dst, n);
  return cudaGetLastError();
}

__global__ void scale_cmul_kernel(float2 *a, long long n, float v) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    a[i] = scale_cmul_dev(a[i], v);
}
cudaError_t launch_scale_cmul(float2 *a, long long n, float v, cudaStream_t st) {
  scale_cmul_kernel<<<RED_BLOCKS, 256, 0, st>>>(a, n, v);
  return cudaGetLastError();
}

}  // namespace spb
