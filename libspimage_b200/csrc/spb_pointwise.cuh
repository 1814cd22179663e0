// Pointwise steps of the phasing passes, shared by the general and the
// register-resident kernels.  Each follows the reference engine's float
// operation order with explicitly rounded intrinsics.
#pragma once
#include "spb_internal.h"

namespace spb {

__device__ __forceinline__ float2 scale_cmul_dev(float2 v, float s) {
  // sp_image_scale: complex multiply by (s, 0)
  return make_float2(fsub(fmul(v.x, s), fmul(v.y, 0.0f)), fadd(fmul(v.x, 0.0f), fmul(s, v.y)));
}

// beta of this iteration: kernel argument, or the device table during graph replays
__device__ __forceinline__ float iter_beta(const PassArgs &a) {
  return a.beta_tab ? a.beta_tab[*a.beta_base + a.beta_idx] : a.beta;
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

// ---------------------------------------------------------------------------
// Branch-free correctly rounded square root, reciprocal and quotient of floats
// (the bits of __fsqrt_rn, __frcp_rn and __fdiv_rn), from Newton-Raphson steps
// with fused multiply-adds after P. Markstein, "Computation of elementary
// functions on the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1),
// 1990, and "IA-64 and Elementary Functions" (2000), ch. 8:
//  * square root: seed t ~ 1/sqrt(x) (PTX rsqrt.approx.f32, relative error
//    <= 2^-22.9); g = x t, h = t/2; one coupled Newton step on (g, h) from the
//    residual 1/2 - g h; then the final rounding g + (x - g^2) h, whose
//    residual x - g^2 the fused multiply-add forms exactly;
//  * reciprocal: seed y0 ~ 1/b (PTX rcp.approx.f32, <= 1 ulp); y = y0 + y0 (1 - b y0);
//  * quotient: q0 = a y, one Newton correction q1 = q0 + (a - b q0) y, then
//    Markstein's final rounding q1 + (a - b q1) y (exact residuals).
// The square root and the reciprocal are checked bit for bit against the
// intrinsics on every float of their domains, the quotient on every pair of
// significands (spb_check_roundings; scaling by powers of two is exact inside
// the domains).  Domains: x in [2^-96, 2^126] (below 2^-102 the residual
// x - g^2 leaves the normal range and the square root misrounds); b in
// [2^-63, 2^63]; a zero or with |a| in [2^-60, 2^60] (quotient and residuals
// stay normal).  Outside them the callers use the intrinsics.
__device__ __forceinline__ float rsqrt_seed(float x) {
  float t;
  asm("rsqrt.approx.f32 %0, %1;" : "=f"(t) : "f"(x));
  return t;
}
__device__ __forceinline__ float rcp_seed(float x) {
  float t;
  asm("rcp.approx.f32 %0, %1;" : "=f"(t) : "f"(x));
  return t;
}
__device__ __forceinline__ bool sqrt_rn_nb_domain(float x) { return x >= 0x1p-96f && x <= 0x1p126f; }
__device__ __forceinline__ bool div_rn_nb_domain(float a) {
  const float m = fabsf(a);
  return m == 0.0f || (m >= 0x1p-60f && m <= 0x1p60f);
}
__device__ __forceinline__ float sqrt_rn_nb(float x) {
  const float t = rsqrt_seed(x);
  float g = __fmul_rn(x, t);
  float h = __fmul_rn(0.5f, t);
  const float r = __fmaf_rn(-g, h, 0.5f);
  g = __fmaf_rn(g, r, g);
  h = __fmaf_rn(h, r, h);
  const float d = __fmaf_rn(-g, g, x);
  return __fmaf_rn(d, h, g);
}
// 1/b for b in [2^-63, 2^63]
__device__ __forceinline__ float rcp_rn_nb(float b) {
  const float y0 = rcp_seed(b);
  return __fmaf_rn(__fmaf_rn(-b, y0, 1.0f), y0, y0);
}
// a / b for b in [2^-63, 2^63] and a in div_rn_nb_domain
__device__ __forceinline__ float div_rn_nb(float a, float b) {
  const float y = rcp_rn_nb(b);
  const float q0 = __fmul_rn(a, y);
  const float q1 = __fmaf_rn(__fmaf_rn(-b, q0, a), y, q0);
  return __fmaf_rn(__fmaf_rn(-b, q1, a), y, q1);
}

// Fourier-space projection (src/phasing.c:1061-1109) of G with the pixel's
// flags f and amplitude amp (ai: its index within a start)
__device__ __forceinline__ float2 project_vals(float2 G, uint8_t f, float amp, long long ai, const PassArgs &a,
                                               bool fourier_constraints) {
  if (fourier_constraints && (a.constraints & C_CENTROSYM)) G.y = 0.0f;
  if (a.objective == 0) {
    if (f & FLAG_MEASURED) {
      float m = 1.0f;
      if (!(a.constraints & C_MARGIN)) {
        // amp / |G|, |G| = sqrt(im*im + re*re) rounded once (cabs_ref)
        const float s2 = fadd(fmul(G.y, G.y), fmul(G.x, G.x));
        m = (sqrt_rn_nb_domain(s2) && div_rn_nb_domain(amp)) ? div_rn_nb(amp, sqrt_rn_nb(s2))
                                                             : __fdiv_rn(amp, __fsqrt_rn(s2));
      } else {
        const float av = cabs_ref(G);
        const float lo = a.amp_min[ai], hi = a.amp_max[ai];
        if (av < lo) m = __fdiv_rn(lo, av);
        else if (av > hi) m = __fdiv_rn(hi, av);
      }
      if (isfinite(m)) G = make_float2(fmul(G.x, m), fmul(G.y, m));
      else G = make_float2(amp, 0.0f);
    }
  } else {
    if (f & FLAG_MEASURED) G = a.phased_amp[ai];
  }
  return G;
}

// the same at pixel idx, operands read from global memory
__device__ __forceinline__ float2 project(float2 G, long long idx, const PassArgs &a, bool fourier_constraints) {
  const long long ai = idx % a.n_start;  // amplitude-side arrays hold one start
  return project_vals(G, a.flags[idx], a.amp[ai], ai, a, fourier_constraints);
}

// Fourier-domain Gaussian of sp_gaussian_blur (src/image_filter.c:80-90):
// the factor at distances (dx, dy, dz) of a pixel from the zero frequency
// (each the smaller of x and n - x, an integer held in a float)
__device__ __forceinline__ float gauss_factor(float dx, float dy, float dz, const PassArgs &a) {
  const double s = __dadd_rn(__dadd_rn(__dmul_rn((double)dx, (double)dx), __dmul_rn((double)dy, (double)dy)),
                             __dmul_rn((double)dz, (double)dz));
  const float dist = __double2float_rn(__dsqrt_rn(s));
  const float cr = __fdiv_rn(dist, a.nx_f);
  const double r2 = a.blur_r2_dev ? *a.blur_r2_dev : a.blur_r2;
  const double arg = __dmul_rn(__dmul_rn(a.blur_c0, __dmul_rn((double)cr, (double)cr)), r2);
  return __double2float_rn(__ddiv_rn(exp(arg), (double)a.n_f));
}

__device__ __forceinline__ float2 gauss_mult(float2 F, long long gidx, const PassArgs &a) {
  const long long idx = gidx % a.n_start;  // position within its start
  const long long nxy = (long long)a.nx * a.ny;
  const int z = (int)(idx / nxy), y = (int)((idx % nxy) / a.nx), x = (int)(idx % a.nx);
  const int dx = min(a.nx - x, x), dy = min(a.ny - y, y), dz = min(a.nz - z, z);
  // the factor table of this blur (gauss_table_kernel) holds the same floats
  const float m = a.blur_tab ? a.blur_tab[((long long)dz * (a.ny / 2 + 1) + dy) * (a.nx / 2 + 1) + dx]
                             : gauss_factor((float)dx, (float)dy, (float)dz, a);
  return scale_cmul_dev(F, m);
}

}  // namespace spb
