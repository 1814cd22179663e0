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
// Branch-free correctly rounded square root and quotient of floats.
//
// Method: evaluate the result in double precision to within one double ulp
// (relative error < 2^-52), then round once to float.  A float square root or
// quotient is never a float midpoint, and its distance from the nearest
// midpoint is at least 2^-51 (square root) or 2^-49 (quotient) relative: the
// midpoint M*2^e has an odd 25-bit M, so x - m^2 (resp. a - m*b) is a nonzero
// multiple of the finer of the two grids.  A faithful double therefore lies on
// the same side of every midpoint as the exact value and rounds to the
// correctly rounded float (the double-rounding bound of S. Figueroa, "When is
// double rounding innocuous?", SIGNUM Newsletter 30(3), 1995: p' >= 2p + 2).
// The seeds are the hardware approximations of PTX rsqrt.approx.f32 (relative
// error <= 2^-22.9) and rcp.approx.f32 (<= 1 ulp), refined by one Taylor step
// in double:
//   sqrt(x) = g (1 - r)^(-1/2) = g (1 + r/2 + 3r^2/8 + O(r^3)),  g = x t,  r = 1 - x t^2
//   1/b     = t (1 - e)^(-1)   = t (1 + e + e^2 + O(e^3)),        e = 1 - b t
// with |r|, |e| < 2^-21, so the truncation (< 2^-62) and the roundings of the
// small terms are far below the last rounding.  Domain: x in [2^-126, 2^126]
// (normal, with a normal reciprocal square root); b in [2^-63, 2^63]; a any
// float (an infinite or NaN a propagates; an overflowing quotient rounds to
// infinity as the IEEE quotient does).  Outside the domain the callers use
// the IEEE intrinsics.
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
__device__ __forceinline__ bool sqrt_rn_nb_domain(float x) { return x >= 0x1p-126f && x <= 0x1p126f; }
__device__ __forceinline__ float sqrt_rn_nb(float x) {
  const double X = (double)x, T = (double)rsqrt_seed(x);
  const double G = X * T;                 // exact: 24 x 24 bits
  const double R = fma(-G, T, 1.0);       // 1 - x t^2
  const double H = R * fma(0.375, R, 0.5);
  return __double2float_rn(fma(G, H, G));
}
// a / b for b in [2^-63, 2^63]
__device__ __forceinline__ float div_rn_nb(float a, float b) {
  const double B = (double)b, T = (double)rcp_seed(b);
  const double E = fma(-B, T, 1.0);       // 1 - b t, exact (Sterbenz)
  const double Y = fma(T, fma(E, E, E), T);
  return __double2float_rn((double)a * Y);
}

// Fourier-space projection at pixel idx (src/phasing.c:1061-1109)
__device__ __forceinline__ float2 project(float2 G, long long idx, const PassArgs &a, bool fourier_constraints) {
  const uint8_t f = a.flags[idx];
  const long long ai = idx % a.n_start;  // amplitude-side arrays hold one start
  if (fourier_constraints && (a.constraints & C_CENTROSYM)) G.y = 0.0f;
  if (a.objective == 0) {
    if (f & FLAG_MEASURED) {
      float m = 1.0f;
      const float amp = a.amp[ai];
      if (!(a.constraints & C_MARGIN)) {
        m = __fdiv_rn(amp, cabs_ref(G));
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
