// Register-resident pass kernels with 8 points per thread, for patterns whose
// lines are too few to fill the GPU with the 16-point kernels of spb_fast.cu
// (a single 256x256 pattern has 256 lines per pass: 16 threads a line at 16
// points each give less than one warp per SM, and the passes wait on
// latency).  Here a line of N points is held by 2T threads (T = N/16 thread
// pairs), so twice the warps share the same work, for some 20 % more
// instructions (the selects and shuffles of the split butterflies).
//
// The transform is the same one, operation for operation: the canonical
// radix plan, the butterflies of spb_fft.cuh and the same twiddle values, so
// the bits do not change.  The two threads of a pair (lanes l and l ^ 16 of
// one warp) split each 16-point register set of the 16-point kernels:
// thread (t, h) holds the points of line index t + T*m for
//     m in M_h = {2h, 2h+1, 2h+4, 2h+5, 2h+8, 2h+9, 2h+12, 2h+13},
// register i holding m_i = 2h + (i & 1) + 4*(i >> 1).
//  * radix 16 (16 = 4 x 4): the first four-point layer needs a[q2 + 4*q1]
//    for fixed q2 = 2h + e, which thread h holds; the internal twiddles of
//    the rows q2 = 2h + e are applied without divergence (the constants are
//    selected per thread, and the identity rows of h = 0 select their input
//    back); the second layer, over q2 for fixed k1, takes k1 = 2h, 2h+1 on
//    thread h after the pair swaps four values by warp shuffle.  Its outputs
//    X[k1 + 4*k2] are again the positions M_h.
//  * radix 8 (two butterflies j = 0, 1 per 16-point set): thread h holds
//    the even (h = 0) or odd (h = 1) inputs of both; each runs its
//    four-point butterflies and the odd twiddles, then the pair swaps four
//    values so that thread h finishes butterfly j = h.
//  * radix 4 (four butterflies j per 16-point set): thread h holds the whole
//    butterflies j = 2h, 2h+1.
// Between stages the outputs go through the padded shared-memory line as in
// spb_fast.cu.  Supported: N = 256, 512, 1024, 4096 (plans 16.16, 16.8.4,
// 16.16.4, 16.16.16), whose last stage leaves the outputs at M_h.
//
// Kernels: the row iteration pass (ROW_ITER: inverse x, update, forward x)
// and the column projection pass (COL_PROJECT / COL_PROJECT_NOFC with the
// line-major amplitudes and measured bits) -- the two passes of every
// HIO/RAAR/ER iteration; the other passes keep the 16-point kernels.
#include <math.h>

#include "spb_internal.h"
#include "spb_passes.cuh"
#include "spb_pointwise.cuh"

namespace spb {
namespace split {

__host__ __device__ constexpr int plan_radix(int n, int s) {
  int r[16] = {0};
  int k = 0, m = n, n16 = 0;
  while (m % 16 == 0) { r[k++] = 16; m /= 16; n16++; }
  if (m % 8 == 0) { r[k++] = 8; m /= 8; }
  else if (m % 4 == 0) { r[k++] = 4; m /= 4; }
  else if (m % 2 == 0) {
    if (n16 > 0) { r[k - 1] = 8; r[k++] = 4; }
    else r[k++] = 2;
    m /= 2;
  }
  return r[s];
}
__host__ __device__ constexpr int plan_len(int n) {
  int k = 0;
  while (k < 16 && plan_radix(n, k) != 0) k++;
  return k;
}
// the lengths whose every stage is radix 16, 8 or 4 and whose last stage is 16 or 4
__host__ __device__ constexpr bool supported(int n) {
  return n == 256 || n == 512 || n == 1024 || n == 4096;
}

// m offset of register i without the 2h part
__host__ __device__ constexpr int mi0(int i) { return (i & 1) + 4 * (i >> 1); }

__device__ __forceinline__ int pad(int i) { return i + (i >> 4); }

__device__ __forceinline__ float2 sel(bool c, float2 a, float2 b) { return c ? a : b; }
__device__ __forceinline__ float2 shfl16(float2 v) {
  return make_float2(__shfl_xor_sync(0xffffffffu, v.x, 16), __shfl_xor_sync(0xffffffffu, v.y, 16));
}

// W8^1 (h = 0) or W8^3 (h = 1) from shared products: the roundings of
// mul_w8_1 / mul_w8_3 exactly (negation is exact)
template <bool INV>
__device__ __forceinline__ float2 mul_w8_13(float2 a, bool h) {
  const float p = fmul(fadd(a.x, a.y), SPB_C8);
  if (!INV) {
    const float q = fmul(fsub(a.y, a.x), SPB_C8);
    return h ? make_float2(q, -p) : make_float2(p, q);
  } else {
    const float q = fmul(fsub(a.x, a.y), SPB_C8);
    return h ? make_float2(-p, q) : make_float2(q, p);
  }
}

// Radix-16 butterfly split over the pair (see the file comment); in and out
// at the positions M_h.
template <bool INV>
__device__ __forceinline__ void bf16_half(float2 (&a)[8], bool h) {
  const float s = INV ? -1.0f : 1.0f;
  // first layer: DFT4 over q1 for q2 = 2h + e (registers e + 2*q1)
  bf4<INV>(a[0], a[2], a[4], a[6]);
  bf4<INV>(a[1], a[3], a[5], a[7]);
  // internal twiddles W16^(q2*k1) of the rows q2 = 2h + e, register e + 2*k1
  // e = 1: q2 = 1 (W^1, W^2, W^3) or q2 = 3 (W^3, W^6, W^9)
  a[3] = cmulw(a[3], h ? SPB_S16 : SPB_C16, h ? -SPB_C16 * s : -SPB_S16 * s);
  a[5] = mul_w8_13<INV>(a[5], h);
  a[7] = cmulw(a[7], h ? -SPB_C16 : SPB_S16, h ? SPB_S16 * s : -SPB_C16 * s);
  // e = 0: q2 = 0 (identity) or q2 = 2 (W^2, W^4, W^6)
  a[2] = sel(h, mul_w8_1<INV>(a[2]), a[2]);
  a[4] = sel(h, mul_w4<INV>(a[4]), a[4]);
  a[6] = sel(h, mul_w8_3<INV>(a[6]), a[6]);
  // second layer: DFT4 over q2 for k1 = 2h + f; (e, k1) sits in register
  // e + 2*k1 of b (the outputs overwrite a)
  float2 b[8];
#pragma unroll
  for (int i = 0; i < 8; i++) b[i] = a[i];
#pragma unroll
  for (int f = 0; f < 2; f++) {
    float2 in[4];
#pragma unroll
    for (int e = 0; e < 2; e++) {
      const float2 lo = b[e + 2 * f], hi = b[e + 4 + 2 * f];  // k1 = f, k1 = 2 + f
      const float2 r = shfl16(sel(h, lo, hi));                 // the partner's q2 = 2(1-h) + e at my k1
      in[e] = sel(h, r, lo);
      in[2 + e] = sel(h, hi, r);
    }
    bf4<INV>(in[0], in[1], in[2], in[3]);
    // X[k1 + 4*k2] with k1 = 2h + f: register f + 2*k2
#pragma unroll
    for (int k2 = 0; k2 < 4; k2++) a[f + 2 * k2] = in[k2];
  }
}

// Radix-8 stage part: register e + 2k holds input m = h + 2k of butterfly
// j = e.  Returns in o[m] the eight outputs of butterfly j = h.
template <bool INV>
__device__ __forceinline__ void bf8_half(const float2 (&a_in)[8], float2 (&o)[8], bool h) {
  float2 a[8];
#pragma unroll
  for (int i = 0; i < 8; i++) a[i] = a_in[i];
  // DFT4 over the even (h = 0) or odd (h = 1) inputs of both butterflies
  bf4<INV>(a[0], a[2], a[4], a[6]);
  bf4<INV>(a[1], a[3], a[5], a[7]);
  // odd outputs o_1, o_2, o_3 times W8^1, W4^1, W8^3 (h = 1 only)
#pragma unroll
  for (int e = 0; e < 2; e++) {
    a[e + 2] = sel(h, mul_w8_1<INV>(a[e + 2]), a[e + 2]);
    a[e + 4] = sel(h, mul_w4<INV>(a[e + 4]), a[e + 4]);
    a[e + 6] = sel(h, mul_w8_3<INV>(a[e + 6]), a[e + 6]);
  }
  // thread h keeps butterfly j = h: swap the other butterfly's values
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const float2 j0 = a[2 * k], j1 = a[1 + 2 * k];
    const float2 r = shfl16(sel(h, j0, j1));
    const float2 ev = sel(h, r, j0), od = sel(h, j1, r);  // e_k, o_k of butterfly j = h
    o[k] = cadd(ev, od);
    o[k + 4] = csub(ev, od);
  }
}

template <int N, int S, int NS, bool INV>
struct Stages {
  static __device__ __forceinline__ void run(float2 (&v)[8], float2 *line, int t, bool h, const float2 *stw) {
    constexpr int R = plan_radix(N, S);
    constexpr int T = N / 16;
    constexpr bool LAST = (S == plan_len(N) - 1);
    static_assert(R == 16 || R == 8 || R == 4, "radix");
    static_assert(!LAST || R != 8, "a radix-8 last stage leaves the outputs off M_h");
    const int hh = h ? 1 : 0;
    if constexpr (R == 16) {
      const int b = t;
      const int k = b & (NS - 1);
      if constexpr (NS > 1) {
#pragma unroll
        for (int i = 0; i < 8; i++) {
          const int m = 2 * hh + mi0(i);
          if (i == 0) {  // m = 0 (h = 0) takes no twiddle
            float2 w = stw[(m > 0 ? m - 1 : 0) * NS + k];
            if (INV) w.y = -w.y;
            const float2 p = cmulw(v[i], w.x, w.y);
            v[i] = (k && m) ? p : v[i];
          } else {
            float2 w = stw[(m - 1) * NS + k];
            if (INV) w.y = -w.y;
            const float2 p = cmulw(v[i], w.x, w.y);
            v[i] = k ? p : v[i];
          }
        }
      }
      bf16_half<INV>(v, h);
      if constexpr (!LAST) {
        if constexpr (NS == 1) {
          float2 *p = line + b * 17 + 2 * hh;  // pad(16b + m) = 17b + m for m < 16
#pragma unroll
          for (int i = 0; i < 8; i++) p[mi0(i)] = v[i];
        } else {
          static_assert(NS % 16 == 0, "stride");
          constexpr int PS = NS + NS / 16;
          float2 *p = line + pad((b / NS) * NS * 16 + k) + 2 * hh * PS;
#pragma unroll
          for (int i = 0; i < 8; i++) p[mi0(i) * PS] = v[i];
        }
      }
    } else if constexpr (R == 8) {
      static_assert(NS % 16 == 0, "a radix-8 stage follows a radix-16 stage here");
      // register e + 2k: butterfly j = e (b = t + T*e), input m = h + 2k
#pragma unroll
      for (int i = 0; i < 8; i++) {
        const int e = i & 1, m = hh + 2 * (i >> 1);
        const int b = t + T * e;
        const int k = b & (NS - 1);
        float2 w = stw[(m > 0 ? m - 1 : 0) * NS + k];
        if (INV) w.y = -w.y;
        const float2 p = cmulw(v[i], w.x, w.y);
        v[i] = (k && m) ? p : v[i];
      }
      float2 o[8];
      bf8_half<INV>(v, o, h);
      const int b = t + T * hh;
      const int k = b & (NS - 1);
      constexpr int PS = NS + NS / 16;
      float2 *p = line + pad((b / NS) * NS * 8 + k);
#pragma unroll
      for (int m = 0; m < 8; m++) p[m * PS] = o[m];
    } else {  // R == 4: register e + 2m holds input m of butterfly j = 2h + e
#pragma unroll
      for (int e = 0; e < 2; e++) {
        const int b = t + T * (2 * hh + e);
        const int k = b & (NS - 1);
        if constexpr (NS > 1) {
#pragma unroll
          for (int m = 1; m < 4; m++) {
            float2 w = stw[(m - 1) * NS + k];
            if (INV) w.y = -w.y;
            const float2 p = cmulw(v[e + 2 * m], w.x, w.y);
            v[e + 2 * m] = k ? p : v[e + 2 * m];
          }
        }
        bf4<INV>(v[e], v[e + 2], v[e + 4], v[e + 6]);
        if constexpr (!LAST) {
          const int base = (b / NS) * NS * 4 + k;
#pragma unroll
          for (int m = 0; m < 4; m++) line[pad(base + m * NS)] = v[e + 2 * m];
        }
      }
    }
    if constexpr (!LAST) {
      __syncthreads();
      constexpr int PT = T + T / 16;
      static_assert(T % 16 == 0, "T");
      const float2 *p = line + pad(t) + 2 * hh * PT;
#pragma unroll
      for (int i = 0; i < 8; i++) v[i] = p[mi0(i) * PT];
      __syncthreads();
      Stages<N, S + 1, NS * R, INV>::run(v, line, t, h, stw + (R - 1) * NS);
    }
  }
};

template <int N, bool INV>
__device__ __forceinline__ void fft(float2 (&v)[8], float2 *line, int t, bool h, const float2 *stw) {
  Stages<N, 0, 1, INV>::run(v, line, t, h, stw);
}

}  // namespace split

// Projection of a thread's 8 points (line index t + T*m_i) with the line's
// amplitudes and measured bits in shared memory: branch-free when every
// measured point is inside the domains of the branch-free square root and
// quotient, else with the IEEE intrinsics -- the bits of project_with.
template <int T, bool FC>
__device__ __forceinline__ void project8(float2 (&v)[8], const float *amp_l, const uint32_t *meas_l, int t, int hh,
                                         size_t lbase, size_t qstride, const PassArgs &a) {
  if (FC && (a.constraints & C_CENTROSYM))
#pragma unroll
    for (int q = 0; q < 8; q++) v[q].y = 0.0f;
  bool fast = a.objective == 0 && !(a.constraints & C_MARGIN) && a.amp_bad && !*a.amp_bad;
  float s2[8];
  unsigned mm = 0;
#pragma unroll
  for (int q = 0; q < 8; q++) {
    const int i = t + T * (2 * hh + split::mi0(q));
    const unsigned meas = (meas_l[i >> 5] >> (i & 31)) & 1u;
    mm |= meas << q;
    s2[q] = fadd(fmul(v[q].y, v[q].y), fmul(v[q].x, v[q].x));
    fast = fast && (!meas || sqrt_rn_nb_domain(s2[q]));
  }
  if (fast) {
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const float amp = amp_l[t + T * (2 * hh + split::mi0(q))];
      const float m = div_rn_nb(amp, sqrt_rn_nb(s2[q]));
      const float2 p = isfinite(m) ? make_float2(fmul(v[q].x, m), fmul(v[q].y, m)) : make_float2(amp, 0.0f);
      if ((mm >> q) & 1u) v[q] = p;
    }
  } else {
#pragma unroll
    for (int q = 0; q < 8; q++)
      v[q] = project_with(v[q], amp_l[t + T * (2 * hh + split::mi0(q))], (mm >> q) & 1u,
                          lbase + split::mi0(q) * qstride, a, false);
  }
}

// ------------------------------------------------------------ row kernel
// Block: LPB lines of 2T threads.  Within a line, warp w and lane l give
// h = bit 4 of l and t = (l & 15) + 16*w.  Shared memory as the 16-point row
// kernel: [twiddles N][LPB exchange lines][LPB rows of g0 unless G0LATE]
// [LPB rows of flags].
template <int N, bool G0LATE>
__global__ void __launch_bounds__(512) row_split_kernel(PassArgs a, const float2 *__restrict__ stw, int nrows) {
  constexpr int T = N / 16;
  constexpr int TL = 2 * T;  // threads per line
  constexpr int S = N + N / 16;
  extern __shared__ __align__(16) float2 sm[];
  const int lpb = blockDim.x / TL;
  const int lr = threadIdx.x / TL, u = threadIdx.x % TL;
  const int lane = u & 31;
  const int hh = (lane >> 4) & 1;
  const bool h = hh != 0;
  const int t = (lane & 15) + 16 * (u >> 5);
  const int row0 = blockIdx.x * lpb;
  const int row = row0 + lr;
  const bool valid = row < nrows;
  float2 *tw_s = sm;
  float2 *line = sm + N + lr * S;
  const size_t base = (size_t)row * N + t + (size_t)(2 * hh) * T;  // point of register i: base + T*mi0(i)
  stage_twiddles<N>(tw_s, stw);
  float2 *g0_s = sm + ((N + lpb * S + 1) & ~1);
  uint8_t *fl_s = reinterpret_cast<uint8_t *>(g0_s + (G0LATE ? 0 : lpb * N));
  const int vrows = min(lpb, nrows - row0);
  if constexpr (!G0LATE) {
    const float2 *g0src = a.g0 + (size_t)row0 * N;
    const int nchunk = vrows * N / 2;
    for (int c = threadIdx.x; c < nchunk; c += blockDim.x) cp_async16(g0_s + 2 * c, g0src + 2 * c);
  }
  {
    const uint8_t *fsrc = a.flags + (size_t)row0 * N;
    const int fchunk = vrows * N / 16;
    for (int c = threadIdx.x; c < fchunk; c += blockDim.x) cp_async16(fl_s + 16 * c, fsrc + 16 * c);
  }
  pdl_wait();
  float2 v[8];
#pragma unroll
  for (int i = 0; i < 8; i++) v[i] = valid ? a.src[base + T * split::mi0(i)] : make_float2(0.0f, 0.0f);
  cp_async_wait_all();
  __syncthreads();
  const float beta = iter_beta(a);
  const float one_m2b = fsub(1.0f, fmul(2.0f, beta));  // 1 - 2*beta in float, as the reference
  split::fft<N, true>(v, line, t, h, tw_s);
  if constexpr (G0LATE) {
    // g0 of the block's rows into their exchange lines: the transform's last
    // stage uses registers only, and a barrier followed its last exchange
    const float2 *g0src = a.g0 + (size_t)row0 * N;
    if constexpr (S % 2 == 0) {
      for (int c = threadIdx.x; c < vrows * (N / 2); c += blockDim.x) {
        const int r = c / (N / 2), j = c % (N / 2);
        cp_async16(sm + N + r * S + 2 * j, g0src + (size_t)r * N + 2 * j);
      }
    } else {
      for (int c = threadIdx.x; c < vrows * N; c += blockDim.x) {
        const int r = c / N, j = c % N;
        cp_async8(sm + N + r * S + j, g0src + (size_t)r * N + j);
      }
    }
    cp_async_wait_all();
    __syncthreads();
  }
  const int lo = t + 2 * hh * T;  // line index of register 0
  const float2 *g0r = G0LATE ? line + lo : g0_s + lr * N + lo;
  const uint8_t *flr = fl_s + lr * N + lo;
  float2 *gp = a.gp;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const int off = T * split::mi0(i);
    float2 g = make_float2(0.0f, 0.0f);
    if (valid) {
      const float2 gpv = scale_cmul_dev(v[i], a.inv_n);
      if (gp) gp[base + off] = gpv;
      const uint8_t f = flr[off];
      if (f & FLAG_INSIDE) {
        g = gpv;
      } else if (a.alg == ALG_HIO) {
        const float2 g0 = g0r[off];
        g = make_float2(fsub(g0.x, fmul(gpv.x, beta)), fsub(g0.y, fmul(gpv.y, beta)));
      } else if (a.alg == ALG_RAAR) {
        const float2 g0 = g0r[off];
        g = make_float2(fadd(fmul(gpv.x, one_m2b), fmul(g0.x, beta)), fadd(fmul(gpv.y, one_m2b), fmul(g0.y, beta)));
      }
      g = apply_constraints(g, f, a.constraints);
      a.g1[base + off] = g;
    }
    v[i] = g;
  }
  if constexpr (G0LATE) __syncthreads();  // every g0 read done before the forward transform writes the lines
  split::fft<N, false>(v, line, t, h, tw_s);
  pdl_release();
  if (valid)
#pragma unroll
    for (int i = 0; i < 8; i++) a.dst[base + T * split::mi0(i)] = v[i];
}

// --------------------------------------------------------- column kernel
// Block: C columns x 2T threads; lane l = c + C*tl + 16*h (C divides 16), so a
// warp loads C adjacent columns of 16/C rows for each half; t = tl + (16/C)*w.
template <int N, int MODE, int C>
__global__ void __launch_bounds__(512) col_split_kernel(PassArgs a, const float2 *__restrict__ stw) {
  constexpr int T = N / 16;
  constexpr int S = N + N / 16 + (C > 1 ? 16 / C : 0);
  constexpr int TPW = 16 / C;  // t values per warp half
  extern __shared__ __align__(16) float2 sm[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int c = lane % C;
  const int hh = (lane >> 4) & 1;
  const bool h = hh != 0;
  const int t = (lane & 15) / C + TPW * w;
  const int col0 = blockIdx.x * C;
  const int col = col0 + c;
  const bool valid = col < a.ncols;
  float2 *tw_s = sm;
  float2 *line = sm + N + c * S;
  constexpr int W = proj_words(N);
  constexpr int SA = amp_stride<N, C>();
  constexpr int SW = bits_stride<N, C>();
  float *amp_s = reinterpret_cast<float *>(sm + N + C * S);
  uint32_t *meas_s = reinterpret_cast<uint32_t *>(amp_s + C * SA);
  stage_twiddles<N>(tw_s, stw);
  {
    const int vl = min(C, a.ncols - col0);
    const float *asrc = a.amp_line + (size_t)col0 * N;
    for (int k = threadIdx.x; k < vl * (N / 4); k += blockDim.x) {
      const int l = k / (N / 4), j = k % (N / 4);
      cp_async16(amp_s + l * SA + 4 * j, asrc + (size_t)l * N + 4 * j);
    }
    const uint32_t *msrc = a.meas_bits + (size_t)col0 * W;
    for (int k = threadIdx.x; k < vl * (W / 4); k += blockDim.x) {
      const int l = k / (W / 4), j = k % (W / 4);
      cp_async16(meas_s + l * SW + 4 * j, msrc + (size_t)l * W + 4 * j);
    }
  }
  const size_t qstride = (size_t)T * a.estride;
  const size_t lbase = (size_t)(a.outer0 + blockIdx.y) * a.ostride + col + (size_t)(t + 2 * hh * T) * a.estride;
  pdl_wait();
  float2 v[8];
#pragma unroll
  for (int i = 0; i < 8; i++) v[i] = valid ? a.src[lbase + split::mi0(i) * qstride] : make_float2(0.0f, 0.0f);
  cp_async_wait_all();
  __syncthreads();
  split::fft<N, false>(v, line, t, h, tw_s);
  if (valid) project8<T, MODE == COL_PROJECT>(v, amp_s + c * SA, meas_s + c * SW, t, hh, lbase, qstride, a);
  split::fft<N, true>(v, line, t, h, tw_s);
  pdl_release();
  if (valid)
#pragma unroll
    for (int i = 0; i < 8; i++) a.dst[lbase + split::mi0(i) * qstride] = v[i];
}

// ---------------------------------------------------------------- launch
template <int N>
static cudaError_t row_split_launch(const LinePlan &px, const PassArgs &a, cudaStream_t st) {
  constexpr int TL = N / 8;
  constexpr int LPB = (256 / TL) > 0 ? (256 / TL) : 1;
  const long long nrows = a.n / N;
  const long long grid = (nrows + LPB - 1) / LPB;
  const size_t smem0 = (size_t)((N + LPB * (N + N / 16) + 1) & ~1) * sizeof(float2);
  // g0 staged up front (the latency-bound grids these kernels serve), or
  // between the transforms when SPB_TUNE_ROW_G0 asks for it
  if (a.row_g0 == 2) {
    const size_t smem = smem0 + (size_t)LPB * N;
    cudaError_t e = ensure_smem<row_split_kernel<N, true>>(smem);
    if (e != cudaSuccess) return e;
    return launch_maybe_pdl(row_split_kernel<N, true>, dim3((unsigned)grid), dim3(LPB * TL), smem, st, a.pdl != 0, a,
                            px.stw, (int)nrows);
  }
  const size_t smem = smem0 + (size_t)LPB * N * (sizeof(float2) + 1);
  cudaError_t e = ensure_smem<row_split_kernel<N, false>>(smem);
  if (e != cudaSuccess) return e;
  return launch_maybe_pdl(row_split_kernel<N, false>, dim3((unsigned)grid), dim3(LPB * TL), smem, st, a.pdl != 0, a,
                          px.stw, (int)nrows);
}

template <int N, int MODE>
static cudaError_t col_split_launch(const LinePlan &pl, const PassArgs &a, cudaStream_t st) {
  constexpr int C = N >= 4096 ? 1 : (N >= 1024 ? 4 : 8);
  constexpr int TL = N / 8;
  static_assert(C * TL <= 512, "block size");
  if (!(a.amp_line && a.meas_bits && a.meas_words == proj_words(N))) return cudaErrorNotSupported;
  const size_t smem = (size_t)(N + C * (N + N / 16 + (C > 1 ? 16 / C : 0))) * sizeof(float2) +
                      (size_t)C * amp_stride<N, C>() * sizeof(float) + (size_t)C * bits_stride<N, C>() * sizeof(uint32_t);
  cudaError_t e = ensure_smem<col_split_kernel<N, MODE, C>>(smem);
  if (e != cudaSuccess) return e;
  dim3 grid((a.ncols + C - 1) / C, a.nouter);
  return launch_maybe_pdl(col_split_kernel<N, MODE, C>, grid, dim3(C * TL), smem, st, a.pdl != 0, a, pl.stw);
}

// The 8-point kernels for the iteration's two passes: cudaErrorNotSupported
// for other line lengths and modes (the caller then takes the 16-point ones).
cudaError_t launch_row_split(int mode, const LinePlan &px, const PassArgs &a, cudaStream_t st) {
  if (!px.stw || mode != ROW_ITER) return cudaErrorNotSupported;
  switch (px.n) {
    case 256: return row_split_launch<256>(px, a, st);
    case 512: return row_split_launch<512>(px, a, st);
    case 1024: return row_split_launch<1024>(px, a, st);
    case 4096: return row_split_launch<4096>(px, a, st);
  }
  return cudaErrorNotSupported;
}

cudaError_t launch_col_split(int mode, const LinePlan &pl, const PassArgs &a, cudaStream_t st) {
  if (!pl.stw || (mode != COL_PROJECT && mode != COL_PROJECT_NOFC)) return cudaErrorNotSupported;
  const bool fc = mode == COL_PROJECT;
  switch (pl.n) {
    case 256: return fc ? col_split_launch<256, COL_PROJECT>(pl, a, st) : col_split_launch<256, COL_PROJECT_NOFC>(pl, a, st);
    case 512: return fc ? col_split_launch<512, COL_PROJECT>(pl, a, st) : col_split_launch<512, COL_PROJECT_NOFC>(pl, a, st);
    case 1024: return fc ? col_split_launch<1024, COL_PROJECT>(pl, a, st) : col_split_launch<1024, COL_PROJECT_NOFC>(pl, a, st);
    case 4096: return fc ? col_split_launch<4096, COL_PROJECT>(pl, a, st) : col_split_launch<4096, COL_PROJECT_NOFC>(pl, a, st);
  }
  return cudaErrorNotSupported;
}

}  // namespace spb
