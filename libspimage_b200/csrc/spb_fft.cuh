// Device FFT building blocks for the phasing passes (sm_100a).
//
// One 1-D complex-float transform of length n is a mixed-radix Stockham
// autosort: radices from spb_radix_plan() (host), stage s with radix r and
// Ns = product of the earlier radices computes, for every butterfly b in
// [0, n/r):  k = b % Ns;  a[m] = x[b + m*n/r];  a[m] *= W_n^(m*k*n/(Ns*r))
// when m*k != 0;  a = DFT_r(a);  y[(b/Ns)*Ns*r + k + m*Ns] = a[m].
// Twiddles come from a per-length table W_n^i = (cos 2pi i/n, -sin 2pi i/n)
// computed in double on the host and rounded to float (conjugated for the
// backward direction).  Every multiply and add is an explicitly rounded
// intrinsic, so no fused multiply-add changes the rounding: the transform is
// reproducible bit for bit by any implementation of the same recipe.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define SPB_MAX_STAGES 24

namespace spb {

struct LinePlan {
  int n;
  int nstages;
  int radix[SPB_MAX_STAGES];
  const float2 *tw;   // n forward twiddles W_n^i (device)
  const float2 *stw;  // the same values per stage: [stage][m-1][k] = W_n^(m*k*n/(Ns*R)) (device)
};

__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }

// Complex add and subtract as one packed f32x2 add (sm_100): each lane is
// rounded exactly as __fadd_rn, and a - b is a + (-b) by IEEE definition, so
// the bits equal the scalar recipe's while the instruction count halves.
// Multiplies stay scalar: a packed product feeding a packed add is not kept
// apart from it (measured: one-ulp differences), a scalar __fmul_rn is.
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
// (a.re*w.re - a.im*w.im, a.re*w.im + a.im*w.re), each product rounded
__device__ __forceinline__ float2 cmulw(float2 a, float wr, float wi) {
  const float t1 = fmul(a.x, wr), t2 = fmul(a.y, wi), t3 = fmul(a.x, wi), t4 = fmul(a.y, wr);
  return make_float2(fsub(t1, t2), fadd(t3, t4));
}
// |a| as the reference computes it: sqrt(im*im + re*re) rounded once
__device__ __forceinline__ float cabs_ref(float2 a) { return __fsqrt_rn(fadd(fmul(a.y, a.y), fmul(a.x, a.x))); }

#define SPB_C8 0.70710678118654752440f
#define SPB_C16 0.92387953251128675613f
#define SPB_S16 0.38268343236508977173f
#define SPB_S3 0.86602540378443864676f
#define SPB_C51 0.30901699437494742410f
#define SPB_C52 (-0.80901699437494742410f)
#define SPB_S51 0.95105651629515357212f
#define SPB_S52 0.58778525229247312917f

template <bool INV>
__device__ __forceinline__ float2 mul_w4(float2 a) {
  return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}
template <bool INV>
__device__ __forceinline__ float2 mul_w8_1(float2 a) {
  return INV ? make_float2(fmul(fsub(a.x, a.y), SPB_C8), fmul(fadd(a.x, a.y), SPB_C8))
             : make_float2(fmul(fadd(a.x, a.y), SPB_C8), fmul(fsub(a.y, a.x), SPB_C8));
}
template <bool INV>
__device__ __forceinline__ float2 mul_w8_3(float2 a) {
  return INV ? make_float2(-fmul(fadd(a.x, a.y), SPB_C8), fmul(fsub(a.x, a.y), SPB_C8))
             : make_float2(fmul(fsub(a.y, a.x), SPB_C8), -fmul(fadd(a.x, a.y), SPB_C8));
}

template <bool INV>
__device__ __forceinline__ void bf2(float2 &a0, float2 &a1) {
  const float2 t = a0;
  a0 = cadd(t, a1);
  a1 = csub(t, a1);
}

template <bool INV>
__device__ __forceinline__ void bf4(float2 &a0, float2 &a1, float2 &a2, float2 &a3) {
  const float2 t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3), d = csub(a1, a3);
  const float2 t3 = mul_w4<INV>(d);
  a0 = cadd(t0, t2);
  a1 = cadd(t1, t3);
  a2 = csub(t0, t2);
  a3 = csub(t1, t3);
}

template <bool INV>
__device__ __forceinline__ void bf8(float2 *a) {
  bf4<INV>(a[0], a[2], a[4], a[6]);
  bf4<INV>(a[1], a[3], a[5], a[7]);
  a[3] = mul_w8_1<INV>(a[3]);
  a[5] = mul_w4<INV>(a[5]);
  a[7] = mul_w8_3<INV>(a[7]);
  float2 t[8];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    t[k] = cadd(a[2 * k], a[2 * k + 1]);
    t[k + 4] = csub(a[2 * k], a[2 * k + 1]);
  }
#pragma unroll
  for (int k = 0; k < 8; k++) a[k] = t[k];
}

template <bool INV>
__device__ __forceinline__ void bf16(float2 *a) {
  const float s = INV ? -1.0f : 1.0f;
#pragma unroll
  for (int q2 = 0; q2 < 4; q2++) bf4<INV>(a[q2], a[q2 + 4], a[q2 + 8], a[q2 + 12]);
  a[1 + 4 * 1] = cmulw(a[1 + 4 * 1], SPB_C16, -SPB_S16 * s);
  a[1 + 4 * 2] = mul_w8_1<INV>(a[1 + 4 * 2]);
  a[1 + 4 * 3] = cmulw(a[1 + 4 * 3], SPB_S16, -SPB_C16 * s);
  a[2 + 4 * 1] = mul_w8_1<INV>(a[2 + 4 * 1]);
  a[2 + 4 * 2] = mul_w4<INV>(a[2 + 4 * 2]);
  a[2 + 4 * 3] = mul_w8_3<INV>(a[2 + 4 * 3]);
  a[3 + 4 * 1] = cmulw(a[3 + 4 * 1], SPB_S16, -SPB_C16 * s);
  a[3 + 4 * 2] = mul_w8_3<INV>(a[3 + 4 * 2]);
  a[3 + 4 * 3] = cmulw(a[3 + 4 * 3], -SPB_C16, SPB_S16 * s);
#pragma unroll
  for (int k1 = 0; k1 < 4; k1++) bf4<INV>(a[4 * k1], a[4 * k1 + 1], a[4 * k1 + 2], a[4 * k1 + 3]);
  float2 t[16];
#pragma unroll
  for (int k1 = 0; k1 < 4; k1++)
#pragma unroll
    for (int k2 = 0; k2 < 4; k2++) t[k1 + 4 * k2] = a[4 * k1 + k2];
#pragma unroll
  for (int k = 0; k < 16; k++) a[k] = t[k];
}

template <bool INV>
__device__ __forceinline__ void bf3(float2 *a) {
  const float2 t1 = cadd(a[1], a[2]), d = csub(a[1], a[2]);
  const float2 m = make_float2(fsub(a[0].x, fmul(t1.x, 0.5f)), fsub(a[0].y, fmul(t1.y, 0.5f)));
  const float2 t3 = INV ? make_float2(-fmul(d.y, SPB_S3), fmul(d.x, SPB_S3))
                        : make_float2(fmul(d.y, SPB_S3), -fmul(d.x, SPB_S3));
  a[0] = cadd(a[0], t1);
  a[1] = cadd(m, t3);
  a[2] = csub(m, t3);
}

template <bool INV>
__device__ __forceinline__ void bf5(float2 *a) {
  const float2 b1 = cadd(a[1], a[4]), b2 = cadd(a[2], a[3]);
  const float2 d1 = csub(a[1], a[4]), d2 = csub(a[2], a[3]);
  const float2 y0 = cadd(cadd(a[0], b1), b2);
  const float2 m1 = make_float2(fadd(fadd(a[0].x, fmul(b1.x, SPB_C51)), fmul(b2.x, SPB_C52)),
                                fadd(fadd(a[0].y, fmul(b1.y, SPB_C51)), fmul(b2.y, SPB_C52)));
  const float2 m2 = make_float2(fadd(fadd(a[0].x, fmul(b1.x, SPB_C52)), fmul(b2.x, SPB_C51)),
                                fadd(fadd(a[0].y, fmul(b1.y, SPB_C52)), fmul(b2.y, SPB_C51)));
  const float2 n1 = make_float2(fadd(fmul(d1.x, SPB_S51), fmul(d2.x, SPB_S52)),
                                fadd(fmul(d1.y, SPB_S51), fmul(d2.y, SPB_S52)));
  const float2 n2 = make_float2(fsub(fmul(d1.x, SPB_S52), fmul(d2.x, SPB_S51)),
                                fsub(fmul(d1.y, SPB_S52), fmul(d2.y, SPB_S51)));
  a[0] = y0;
  if (!INV) {
    a[1] = make_float2(fadd(m1.x, n1.y), fsub(m1.y, n1.x));
    a[4] = make_float2(fsub(m1.x, n1.y), fadd(m1.y, n1.x));
    a[2] = make_float2(fadd(m2.x, n2.y), fsub(m2.y, n2.x));
    a[3] = make_float2(fsub(m2.x, n2.y), fadd(m2.y, n2.x));
  } else {
    a[1] = make_float2(fsub(m1.x, n1.y), fadd(m1.y, n1.x));
    a[4] = make_float2(fadd(m1.x, n1.y), fsub(m1.y, n1.x));
    a[2] = make_float2(fsub(m2.x, n2.y), fadd(m2.y, n2.x));
    a[3] = make_float2(fadd(m2.x, n2.y), fsub(m2.y, n2.x));
  }
}

template <int R, bool INV>
__device__ __forceinline__ void bfly(float2 *a) {
  if constexpr (R == 2) bf2<INV>(a[0], a[1]);
  else if constexpr (R == 3) bf3<INV>(a);
  else if constexpr (R == 4) bf4<INV>(a[0], a[1], a[2], a[3]);
  else if constexpr (R == 5) bf5<INV>(a);
  else if constexpr (R == 8) bf8<INV>(a);
  else if constexpr (R == 16) bf16<INV>(a);
}

__device__ __forceinline__ float2 twiddle(const float2 *tw, int idx, bool inv) {
  const float2 w = __ldg(tw + idx);
  return make_float2(w.x, inv ? -w.y : w.y);
}

// Element i of a line lives at x[i * es] (es = element stride in the staging
// buffer).  The butterflies of one stage are shared out as b = t0, t0+tn, ...
template <int R, bool INV>
__device__ __forceinline__ void stage_fixed(const float2 *__restrict__ x, float2 *__restrict__ y, const LinePlan &p,
                                            int ns, int es, int t0, int tn) {
  const int n = p.n, nb = n / R, tstep = n / (ns * R);
  for (int b = t0; b < nb; b += tn) {
    const int k = b % ns;
    float2 a[R];
#pragma unroll
    for (int m = 0; m < R; m++) a[m] = x[(b + m * nb) * es];
    if (k) {
#pragma unroll
      for (int m = 1; m < R; m++) {
        const float2 w = twiddle(p.tw, m * k * tstep, INV);
        a[m] = cmulw(a[m], w.x, w.y);
      }
    }
    bfly<R, INV>(a);
    const int base = (b / ns) * ns * R + k;
#pragma unroll
    for (int m = 0; m < R; m++) y[(base + m * ns) * es] = a[m];
  }
}

// Prime radix without a dedicated butterfly: y_m = a_0 + sum_q a_q W_r^(mq mod r),
// accumulated left to right on the twiddled inputs (recomputed per output; the
// recomputation is deterministic, so every output sees identical a_q).
template <bool INV>
__device__ void stage_generic(const float2 *__restrict__ x, float2 *__restrict__ y, const LinePlan &p, int R, int ns,
                              int es, int t0, int tn) {
  const int n = p.n, nb = n / R, tstep = n / (ns * R), rstep = n / R;
  for (int b = t0; b < nb; b += tn) {
    const int k = b % ns;
    const int base = (b / ns) * ns * R + k;
    for (int m = 0; m < R; m++) {
      float2 acc = x[b * es];
      for (int q = 1; q < R; q++) {
        float2 aq = x[(b + q * nb) * es];
        if (k) {
          const float2 w = twiddle(p.tw, q * k * tstep, INV);
          aq = cmulw(aq, w.x, w.y);
        }
        if (m == 0) {
          acc = cadd(acc, aq);
        } else {
          const int e = (int)(((long long)m * q) % R);
          const float2 w = twiddle(p.tw, e * rstep, INV);
          acc = cadd(acc, cmulw(aq, w.x, w.y));
        }
      }
      y[(base + m * ns) * es] = acc;
    }
  }
}

// ------------------------------------------- compile-time plans (2,3,4,5,8,16)
// The canonical radix plan of a length known at compile time: 16s first, then
// one 8/4/2 (a trailing 2 after a 16 turns that 16 into 8*4), then 3s and 5s;
// -1 when another prime remains.
__host__ __device__ constexpr int ct_plan(int n, int *r) {
  int k = 0, m = n, n16 = 0;
  while (m % 16 == 0) { r[k++] = 16; m /= 16; n16++; }
  if (m % 8 == 0) { r[k++] = 8; m /= 8; }
  else if (m % 4 == 0) { r[k++] = 4; m /= 4; }
  else if (m % 2 == 0) {
    if (n16 > 0) { r[k - 1] = 8; r[k++] = 4; }
    else r[k++] = 2;
    m /= 2;
  }
  while (m % 3 == 0) { r[k++] = 3; m /= 3; }
  while (m % 5 == 0) { r[k++] = 5; m /= 5; }
  return m > 1 ? -1 : k;
}
__host__ __device__ constexpr int ct_plan_len(int n) {
  int r[32] = {};
  return ct_plan(n, r);
}
__host__ __device__ constexpr int ct_plan_radix(int n, int s) {
  int r[32] = {};
  ct_plan(n, r);
  return r[s];
}

// the largest number of butterflies of any stage: threads per line that give
// every thread at most one butterfly per stage
__host__ __device__ constexpr int ct_max_butterflies(int n) {
  int r[32] = {};
  const int k = ct_plan(n, r);
  int m = 0;
  for (int s = 0; s < k; s++) m = (n / r[s] > m) ? n / r[s] : m;
  return m;
}

// The stages of stage_fixed with the plan, the strides and the divisions known
// at compile time; twiddles from the per-stage table ([stage][m-1][k], the
// same float values as tw[m*k*tstep]; N - 1 entries in all), read from
// shared memory where the kernel staged it, else from global memory, so the
// arithmetic is unchanged.
template <int N, int S, int NS, bool INV>
struct CtStages {
  static __device__ float2 *run(float2 *x, float2 *y, const float2 *__restrict__ stw, int es, int t0, int tn) {
    constexpr int R = ct_plan_radix(N, S);
    constexpr int NB = N / R;
    for (int b = t0; b < NB; b += tn) {
      const int k = b % NS;
      float2 a[R];
#pragma unroll
      for (int m = 0; m < R; m++) a[m] = x[(b + m * NB) * es];
      if (NS > 1 && k) {
#pragma unroll
        for (int m = 1; m < R; m++) {
          float2 w = stw[(m - 1) * NS + k];  // shared-memory or global table
          if (INV) w.y = -w.y;
          a[m] = cmulw(a[m], w.x, w.y);
        }
      }
      bfly<R, INV>(a);
      const int base = (b / NS) * NS * R + k;
#pragma unroll
      for (int m = 0; m < R; m++) y[(base + m * NS) * es] = a[m];
    }
    __syncthreads();
    if constexpr (S + 1 < ct_plan_len(N)) return CtStages<N, S + 1, NS * R, INV>::run(y, x, stw + (R - 1) * NS, es, t0, tn);
    else return y;
  }
};

// Runs every stage of a line transform between two staging buffers.  All
// threads of the block must call it (it synchronises the block between
// stages).  Returns the buffer holding the result.
template <bool INV>
__device__ float2 *line_fft(float2 *bufA, float2 *bufB, const LinePlan &p, int es, int t0, int tn) {
  float2 *x = bufA, *y = bufB;
  int ns = 1;
  for (int s = 0; s < p.nstages; s++) {
    const int r = p.radix[s];
    switch (r) {
      case 2: stage_fixed<2, INV>(x, y, p, ns, es, t0, tn); break;
      case 3: stage_fixed<3, INV>(x, y, p, ns, es, t0, tn); break;
      case 4: stage_fixed<4, INV>(x, y, p, ns, es, t0, tn); break;
      case 5: stage_fixed<5, INV>(x, y, p, ns, es, t0, tn); break;
      case 8: stage_fixed<8, INV>(x, y, p, ns, es, t0, tn); break;
      case 16: stage_fixed<16, INV>(x, y, p, ns, es, t0, tn); break;
      default: stage_generic<INV>(x, y, p, r, ns, es, t0, tn); break;
    }
    ns *= r;
    float2 *t = x;
    x = y;
    y = t;
    __syncthreads();
  }
  return x;
}

}  // namespace spb

namespace spb {
// line_fft with the plan fixed at compile time when NC > 0 (stage table `stw`:
// p.stw or a shared-memory copy of it)
template <bool INV, int NC>
__device__ __forceinline__ float2 *line_fft_sel(float2 *bufA, float2 *bufB, const LinePlan &p, int es, int t0, int tn,
                                               const float2 *stw) {
  if constexpr (NC > 0) return CtStages<NC, 0, 1, INV>::run(bufA, bufB, stw, es, t0, tn);
  else return line_fft<INV>(bufA, bufB, p, es, t0, tn);
}
}  // namespace spb
