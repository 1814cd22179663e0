// Register-resident pass kernels for power-of-two line lengths 16..4096.
//
// Same transform as spb_fft.cuh (canonical radix plan, same butterflies and
// twiddle values, explicitly rounded arithmetic), organised for throughput:
// a line of N points is held by T = N/16 threads, 16 points each, in the
// "natural" layout v[q] = x[t + T*q].  In that layout the inputs of every
// butterfly of every stage are already in the thread's registers
// (a[m] = v[j + m*16/R]), so a stage only scatters its outputs to shared
// memory and reads the natural layout back: nstages-1 shared-memory
// exchanges per transform, none after the last stage.  Shared memory is
// padded (index i -> i + i/16, plus a per-line skew in the column kernels) so
// that every exchange is free of bank conflicts.  Twiddles are read from a
// per-stage table laid out [stage][m-1][k] (consecutive k for consecutive
// threads), holding the very same float values as the per-length table.
//
// Row kernels: forward/inverse/|.| transforms, the HIO/RAAR/ER iteration
// (inverse x, update, forward x) and the difference map's iteration (two
// lines per row: inverse x of Y and Yf, the update, forward x of g and f1).
// Column kernels: transforms, the Fourier projection with line-major
// amplitudes and measured bits, the blur multiplier.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <math.h>

#include "spb_internal.h"
#include "spb_passes.cuh"
#include "spb_pointwise.cuh"

namespace spb {
namespace reg {

// number of stages of the canonical plan of a power of two (a trailing 2
// after 16s turns one 16 into 8*4: still one extra stage)
__host__ __device__ constexpr int plan_len(int n) {
  int k = 0, m = n;
  while (m % 16 == 0) { k++; m /= 16; }
  if (m > 1) k++;
  return k;
}

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

__device__ __forceinline__ int pad(int i) { return i + (i >> 4); }

template <int N, int S, int NS, bool INV>
struct Stages {
  static __device__ __forceinline__ void run(float2 (&v)[16], float2 *line, int t, const float2 *stw) {
    constexpr int R = plan_radix(N, S);
    constexpr int T = N / 16;
    constexpr int J = 16 / R;
    constexpr bool LAST = (S == plan_len(N) - 1);
#pragma unroll
    for (int j = 0; j < J; j++) {
      float2 a[R];
#pragma unroll
      for (int m = 0; m < R; m++) a[m] = v[j + m * J];
      const int b = t + T * j;
      const int k = b & (NS - 1);
      if constexpr (NS > 1) {
#pragma unroll
        for (int m = 1; m < R; m++) {
          float2 w = stw[(m - 1) * NS + k];  // shared-memory stage table
          if (INV) w.y = -w.y;
          const float2 p = cmulw(a[m], w.x, w.y);
          a[m] = k ? p : a[m];
        }
      }
      bfly<R, INV>(a);
      if constexpr (LAST) {
#pragma unroll
        for (int m = 0; m < R; m++) v[j + m * J] = a[m];
      } else if constexpr (NS % 16 == 0) {
        // m*NS leaves the low 4 bits of base alone: pad(base + m*NS) = pad(base) + m*(NS + NS/16)
        float2 *p = line + pad((b / NS) * NS * R + k);
#pragma unroll
        for (int m = 0; m < R; m++) p[m * (NS + NS / 16)] = a[m];
      } else if constexpr (NS == 1) {
        // R divides 16 and m < R: pad(b*R + m) = pad(b*R) + m
        float2 *p = line + pad(b * R);
#pragma unroll
        for (int m = 0; m < R; m++) p[m] = a[m];
      } else {
        const int base = (b / NS) * NS * R + k;
#pragma unroll
        for (int m = 0; m < R; m++) line[pad(base + m * NS)] = a[m];
      }
    }
    if constexpr (!LAST) {
      __syncthreads();
      if constexpr (T % 16 == 0) {
        const float2 *p = line + pad(t);
#pragma unroll
        for (int q = 0; q < 16; q++) v[q] = p[q * (T + T / 16)];
      } else {
#pragma unroll
        for (int q = 0; q < 16; q++) v[q] = line[pad(t + T * q)];
      }
      __syncthreads();
      Stages<N, S + 1, NS * R, INV>::run(v, line, t, stw + (R - 1) * NS);
    }
  }
};

template <int N, bool INV>
__device__ __forceinline__ void fft(float2 (&v)[16], float2 *line, int t, const float2 *stw) {
  Stages<N, 0, 1, INV>::run(v, line, t, stw);
}

}  // namespace reg


// |v[q]| of 16 values as cabs_ref computes them: without a branch per value
// when every |v|^2 is zero or in the domain of the branch-free square root,
// else with the IEEE intrinsic for all 16 (the same bits either way)
__device__ __forceinline__ void cabs16(const float2 (&v)[16], float (&r)[16]) {
  bool fast = true;
#pragma unroll
  for (int q = 0; q < 16; q++) {
    r[q] = fadd(fmul(v[q].y, v[q].y), fmul(v[q].x, v[q].x));
    fast = fast && (r[q] == 0.0f || sqrt_rn_nb_domain(r[q]));
  }
  if (fast) {
#pragma unroll
    for (int q = 0; q < 16; q++) r[q] = r[q] == 0.0f ? r[q] : sqrt_rn_nb(r[q]);
  } else {
#pragma unroll
    for (int q = 0; q < 16; q++) r[q] = __fsqrt_rn(r[q]);
  }
}

// Blur factor of a thread's 16 points of a column line (line index t + T*q),
// from the line's coordinates instead of per-point index arithmetic: the
// same factors as gauss_mult.
template <int T>
__device__ __forceinline__ void blur16(float2 (&v)[16], int col, long long o, int t, const PassArgs &a) {
  int x, y, z;  // coordinates of point q = 0; the line runs along y (axis 1) or z (axis 2)
  if (a.line_axis == 2) {
    x = col % a.nx;
    y = col / a.nx;
    z = t;
  } else {
    x = col;
    y = t;
    z = (int)(o % a.nz);
  }
  const int hx = a.nx / 2 + 1, hy = a.ny / 2 + 1;
#pragma unroll
  for (int q = 0; q < 16; q++) {
    const int yy = a.line_axis == 2 ? y : y + T * q, zz = a.line_axis == 2 ? z + T * q : z;
    const int dx = min(a.nx - x, x), dy = min(a.ny - yy, yy), dz = min(a.nz - zz, zz);
    const float m = a.blur_tab ? a.blur_tab[((long long)dz * hy + dy) * hx + dx]
                               : gauss_factor((float)dx, (float)dy, (float)dz, a);
    v[q] = scale_cmul_dev(v[q], m);
  }
}

// Projection of a thread's 16 points (line index i = t + T*q) with the
// line's amplitudes and measured bits in shared memory.  When every measured
// point's |G|^2 lies in the domain of the branch-free square root and every
// amplitude in the quotient's (the common case) the 16 projections contain no
// branch, so the compiler interleaves them; otherwise the thread projects all
// 16 with the IEEE intrinsics.  Both give the bits of project_with.
template <int T, bool FC>
__device__ __forceinline__ void project16(float2 (&v)[16], const float *amp_l, const uint32_t *meas_l, int t,
                                          size_t lbase, size_t qstride, const PassArgs &a) {
  if (FC && (a.constraints & C_CENTROSYM))
#pragma unroll
    for (int q = 0; q < 16; q++) v[q].y = 0.0f;
  // amp_bad: some amplitude lies outside the quotient's domain (set when the lines are built)
  bool fast = a.objective == 0 && !(a.constraints & C_MARGIN) && a.amp_bad && !*a.amp_bad;
  float s2[16];
  unsigned mm = 0;
#pragma unroll
  for (int q = 0; q < 16; q++) {
    const int i = t + T * q;
    const unsigned meas = (meas_l[i >> 5] >> (i & 31)) & 1u;
    mm |= meas << q;
    s2[q] = fadd(fmul(v[q].y, v[q].y), fmul(v[q].x, v[q].x));
    fast = fast && (!meas || sqrt_rn_nb_domain(s2[q]));
  }
  if (fast) {
#pragma unroll
    for (int q = 0; q < 16; q++) {
      const float amp = amp_l[t + T * q];
      const float m = div_rn_nb(amp, sqrt_rn_nb(s2[q]));
      const float2 p = isfinite(m) ? make_float2(fmul(v[q].x, m), fmul(v[q].y, m)) : make_float2(amp, 0.0f);
      if ((mm >> q) & 1u) v[q] = p;
    }
  } else {
#pragma unroll
    for (int q = 0; q < 16; q++)
      v[q] = project_with(v[q], amp_l[t + T * q], (mm >> q) & 1u, lbase + q * qstride, a, false);
  }
}


// ------------------------------------------------------------ row kernels
// Shared memory: [twiddles N][LPB exchange lines of N+N/16]
//                (ROW_ITER) [LPB rows of g0, unless G0LATE][LPB rows of flags]
// ROW_ITER copies g0 either at the start, to overlap its load with the
// inverse transform (latency-bound grids), or with G0LATE into each row's
// exchange line between the two transforms (the line is free then): less
// shared memory per block, so more blocks share an SM (throughput-bound grids).
template <int N, int MODE, bool G0LATE>
__global__ void __launch_bounds__(256) row_fast_kernel(PassArgs a, const float2 *__restrict__ stw, int nrows) {
  constexpr int T = N / 16;
  constexpr int S = N + N / 16;
  extern __shared__ __align__(16) float2 sm[];
  const int lpb = blockDim.x / T;
  const int lr = threadIdx.x / T, t = threadIdx.x % T;
  const int row0 = blockIdx.x * lpb;
  const int row = row0 + lr;
  const bool valid = row < nrows;
  float2 *tw_s = sm;
  float2 *line = sm + N + lr * S;
  const size_t base = (size_t)row * N + t;
  stage_twiddles<N>(tw_s, stw);
  // g0 rows start on a 16-byte boundary (an even float2 offset) for the 16-byte copies
  float2 *g0_s = sm + ((N + lpb * S + 1) & ~1);
  uint8_t *fl_s = reinterpret_cast<uint8_t *>(g0_s + (G0LATE ? 0 : lpb * N));
  const int vrows = min(lpb, nrows - row0);
  if constexpr (MODE == ROW_ITER || MODE == ROW_DM_ITER) {
    // g0 (unless G0LATE) and flags of this block's rows: contiguous, copied in 16-byte chunks
    if constexpr (!G0LATE) {
      const float2 *g0src = a.g0 + (size_t)row0 * N;
      const int nchunk = vrows * N / 2;
      for (int c = threadIdx.x; c < nchunk; c += blockDim.x) cp_async16(g0_s + 2 * c, g0src + 2 * c);
    }
    const uint8_t *fsrc = a.flags + (size_t)row0 * N;
    const int fchunk = vrows * N / 16;
    for (int c = threadIdx.x; c < fchunk; c += blockDim.x) cp_async16(fl_s + 16 * c, fsrc + 16 * c);
  }
  pdl_wait();
  float2 v[16];
  float2 w[MODE == ROW_DM_ITER ? 16 : 1];  // the difference map's second line (Yf)
#pragma unroll
  for (int q = 0; q < 16; q++) {
    float2 x = make_float2(0.0f, 0.0f);
    if constexpr (MODE == ROW_DM_ITER) w[q] = valid ? a.src2[base + T * q] : x;
    if (valid) {
      const size_t idx = base + T * q;
      if constexpr (MODE == ROW_FWD_F32) x = make_float2(a.f32src[idx], 0.0f);
      else if constexpr (MODE == ROW_FWD_SQUARE_F32) {
        const float s = a.f32src[idx];
        x = make_float2(fmul(s, s), 0.0f);
      } else x = a.src[idx];
    }
    v[q] = x;
  }
  if constexpr (MODE == ROW_FWD_DEPHASE) {
    float r[16];
    cabs16(v, r);
#pragma unroll
    for (int q = 0; q < 16; q++) v[q] = make_float2(r[q], 0.0f);
  }
  cp_async_wait_all();
  __syncthreads();
  if constexpr (MODE == ROW_FWD || MODE == ROW_FWD_DEPHASE || MODE == ROW_FWD_F32 || MODE == ROW_FWD_SQUARE_F32) {
    reg::fft<N, false>(v, line, t, tw_s);
    pdl_release();
    if (valid)
#pragma unroll
      for (int q = 0; q < 16; q++) a.dst[base + T * q] = v[q];
  } else if constexpr (MODE == ROW_INV || MODE == ROW_INV_SCALE || MODE == ROW_INV_ABS) {
    reg::fft<N, true>(v, line, t, tw_s);
    float r[16];
    if constexpr (MODE == ROW_INV_ABS) cabs16(v, r);
    pdl_release();
    if (valid)
#pragma unroll
      for (int q = 0; q < 16; q++) {
        if constexpr (MODE == ROW_INV) a.dst[base + T * q] = v[q];
        else if constexpr (MODE == ROW_INV_SCALE) a.dst[base + T * q] = scale_cmul_dev(v[q], a.inv_n);
        else a.absout[base + T * q] = r[q];
      }
  } else if constexpr (MODE == ROW_ITER) {
    const float beta = iter_beta(a);
    const float one_m2b = fsub(1.0f, fmul(2.0f, beta));  // 1 - 2*beta in float, as the reference
    reg::fft<N, true>(v, line, t, tw_s);
    // G0LATE: g0 of the block's rows into their exchange lines; the
    // transform's last stage uses registers only, and a barrier followed its
    // last exchange
    if constexpr (G0LATE) {
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
    const float2 *g0r = G0LATE ? line + t : g0_s + lr * N + t;
    const uint8_t *flr = fl_s + lr * N + t;
    float2 *gp = a.gp;
#pragma unroll
    for (int q = 0; q < 16; q++) {
      float2 g = make_float2(0.0f, 0.0f);
      if (valid) {
        const float2 gpv = scale_cmul_dev(v[q], a.inv_n);
        if (gp) gp[base + T * q] = gpv;
        const uint8_t f = flr[T * q];
        if (f & FLAG_INSIDE) {
          g = gpv;
        } else if (a.alg == ALG_HIO) {
          const float2 g0 = g0r[T * q];
          g = make_float2(fsub(g0.x, fmul(gpv.x, beta)), fsub(g0.y, fmul(gpv.y, beta)));
        } else if (a.alg == ALG_RAAR) {
          const float2 g0 = g0r[T * q];
          g = make_float2(fadd(fmul(gpv.x, one_m2b), fmul(g0.x, beta)),
                          fadd(fmul(gpv.y, one_m2b), fmul(g0.y, beta)));
        }
        g = apply_constraints(g, f, a.constraints);
        a.g1[base + T * q] = g;
      }
      v[q] = g;
    }
    if constexpr (G0LATE) __syncthreads();  // every g0 read done before the forward transform writes the lines
    reg::fft<N, false>(v, line, t, tw_s);
    pdl_release();
    if (valid)
#pragma unroll
      for (int q = 0; q < 16; q++) a.dst[base + T * q] = v[q];
  } else if constexpr (MODE == ROW_DM_ITER) {
    // difference map (src/phasing.c:1111-1168 as restated by the general row
    // pass): inverse x of Y and Yf, the update of g and f1, forward x of both
    const float beta = iter_beta(a);
    reg::fft<N, true>(v, line, t, tw_s);
    reg::fft<N, true>(w, line, t, tw_s);
    if constexpr (G0LATE) {
      const float2 *g0src = a.g0 + (size_t)row0 * N;
      for (int c = threadIdx.x; c < vrows * (N / 2); c += blockDim.x) {
        const int r = c / (N / 2), j = c % (N / 2);
        if constexpr (S % 2 == 0) cp_async16(sm + N + r * S + 2 * j, g0src + (size_t)r * N + 2 * j);
        else {
          cp_async8(sm + N + r * S + 2 * j, g0src + (size_t)r * N + 2 * j);
          cp_async8(sm + N + r * S + 2 * j + 1, g0src + (size_t)r * N + 2 * j + 1);
        }
      }
      cp_async_wait_all();
      __syncthreads();
    }
    const float2 *g0r = G0LATE ? line + t : g0_s + lr * N + t;
    const uint8_t *flr = fl_s + lr * N + t;
    // x / size as the reference divides; a multiply by the exact reciprocal when the size is a power of two
    auto div_size = [&](float x) { return a.inv_size_pow2 != 0.0f ? fmul(x, a.inv_size_pow2) : __fdiv_rn(x, a.size_f); };
#pragma unroll
    for (int q = 0; q < 16; q++) {
      float2 g = make_float2(0.0f, 0.0f), f1 = g;
      if (valid) {
        const float2 rv = v[q], fv = w[q], g0 = g0r[T * q];
        if (a.gp) a.gp[base + T * q] = rv;
        const uint8_t f = flr[T * q];
        if (f & FLAG_INSIDE) {
          g.x = fadd(g0.x, fmul(beta, fsub(div_size(fmul(a.one_p_g2, rv.x)), fmul(a.gamma2, g0.x))));
          g.y = fadd(g0.y, fmul(beta, fsub(div_size(fmul(a.one_p_g2, rv.y)), fmul(a.gamma2, g0.y))));
        } else {
          g = g0;
        }
        g.x = fsub(g.x, div_size(fmul(beta, fv.x)));
        g.y = fsub(g.y, div_size(fmul(beta, fv.y)));
        g = apply_constraints(g, f, a.constraints);
        a.g1[base + T * q] = g;
        f1 = (f & FLAG_INSIDE) ? g : make_float2(fmul(-a.gamma1, g.x), fmul(-a.gamma1, g.y));
      }
      v[q] = g;
      w[q] = f1;
    }
    if constexpr (G0LATE) __syncthreads();  // every g0 read done before the forward transforms write the lines
    reg::fft<N, false>(v, line, t, tw_s);
    reg::fft<N, false>(w, line, t, tw_s);
    pdl_release();
    if (valid)
#pragma unroll
      for (int q = 0; q < 16; q++) {
        a.dst[base + T * q] = v[q];
        a.dst2[base + T * q] = w[q];
      }
  }
}

// --------------------------------------------------------- column kernels
// Shared memory: [twiddles N][C exchange lines of S]
//                (projection with line-major operands) [C lines of amp][C lines of measured bits]
template <int N, int MODE, int C, bool PREFETCH>
__global__ void __launch_bounds__(256) col_fast_kernel(PassArgs a, const float2 *__restrict__ stw) {
  constexpr int T = N / 16;
  constexpr int S = N + N / 16 + (C > 1 ? 16 / C : 0);
  extern __shared__ __align__(16) float2 sm[];
  const int c = threadIdx.x % C, t = threadIdx.x / C;
  const int col0 = blockIdx.x * C;
  const int col = col0 + c;
  const bool valid = col < a.ncols;
  float2 *tw_s = sm;
  float2 *line = sm + N + c * S;
  // staged operand lines: strides skewed so the C lines of a warp fall in
  // different banks (multiples of 4 words keep the 16-byte copies aligned)
  constexpr int W = proj_words(N);
  constexpr int SA = amp_stride<N, C>();
  constexpr int SW = bits_stride<N, C>();
  float *amp_s = reinterpret_cast<float *>(sm + N + C * S);
  uint32_t *meas_s = reinterpret_cast<uint32_t *>(amp_s + C * SA);
  stage_twiddles<N>(tw_s, stw);
  if constexpr (PREFETCH) {
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
  const size_t lbase = (size_t)(a.outer0 + blockIdx.y) * a.ostride + col + (size_t)t * a.estride;
  const size_t qstride = (size_t)T * a.estride;
  pdl_wait();
  float2 v[16];
#pragma unroll
  for (int q = 0; q < 16; q++) {
    float2 x = make_float2(0.0f, 0.0f);
    if (valid) {
      const size_t idx = lbase + q * qstride;
      if constexpr (MODE == COL_INV_SQUARE_F32) {
        const float s = a.f32src[idx];
        x = make_float2(fmul(s, s), 0.0f);
      } else {
        x = a.src[idx];
      }
    }
    v[q] = x;
  }
  cp_async_wait_all();
  __syncthreads();
  if constexpr (MODE == COL_FWD) {
    reg::fft<N, false>(v, line, t, tw_s);
  } else if constexpr (MODE == COL_INV || MODE == COL_INV_SQUARE_F32) {
    reg::fft<N, true>(v, line, t, tw_s);
  } else {
    reg::fft<N, false>(v, line, t, tw_s);
    if (valid) {
      if constexpr (PREFETCH) {
        project16<T, MODE == COL_PROJECT>(v, amp_s + c * SA, meas_s + c * SW, t, lbase, qstride, a);
      } else {
#pragma unroll
        for (int q = 0; q < 16; q++) {
          const size_t idx = lbase + q * qstride;
          if constexpr (MODE == COL_PROJECT) v[q] = project(v[q], idx, a, true);
          else if constexpr (MODE == COL_PROJECT_NOFC) v[q] = project(v[q], idx, a, false);
        }
        if constexpr (MODE == COL_BLUR) blur16<T>(v, col, a.outer0 + blockIdx.y, t, a);
      }
    }
    reg::fft<N, true>(v, line, t, tw_s);
  }
  pdl_release();
  if (valid)
#pragma unroll
    for (int q = 0; q < 16; q++) a.dst[lbase + q * qstride] = v[q];
}

// --------------------------------------- projection pass staged by TMA
// The column projection pass with its column tile moved by the tensor memory
// accelerator: one thread issues cp.async.bulk.tensor loads of the block's C
// columns (N rows, boxes of up to 256 rows) into shared memory under an
// mbarrier, the threads read their natural-layout points from the dense tile,
// and after the inverse transform the tile is written back to shared memory
// and stored by cp.async.bulk.tensor.  The tile lives in the exchange lines'
// space, which is free before the first stage and after the last.  The
// tensor maps cover only this GPU's memory (the iterate buffers of the
// context) and no load uses cluster multicast.  Transforms, projection and
// bits are those of col_fast_kernel.
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
          smem_u32(dst)),
      "l"((unsigned long long)map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_store_2d(const CUtensorMap *map, int x, int y, const void *src) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];\n" ::"l"(
                   (unsigned long long)map),
               "r"(x), "r"(y), "r"(smem_u32(src))
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// polls of the tile's mbarrier before the block gives up (each try_wait may
// suspend the thread for a while; a stuck copy ends the block within seconds)
constexpr long long kTmaWaitPolls = 1LL << 22;

// Waits for phase `parity` of the mbarrier with a bounded number of polls.
// The answer is the block's (a barrier): false on every thread if any gave
// up, so the block leaves together and no thread is left at a later barrier.
__device__ __forceinline__ bool mbar_wait_block(uint64_t *bar, unsigned parity) {
  bool ok = false;
  for (long long i = 0; i < kTmaWaitPolls && !ok; i++) ok = mbar_try_wait(bar, parity);
  return !__syncthreads_or(!ok);
}

// 1-D bulk copy of `bytes` (a multiple of 16; both addresses 16-byte aligned)
// from global to shared memory, completing on the mbarrier's byte count
__device__ __forceinline__ void bulk_load(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_u32(dst)),
               "l"((unsigned long long)src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// shared-memory alignment of the bulk tensor copies' boxes (bytes)
constexpr unsigned kTmaSmemAlign = 128;

template <int N, int MODE, int C>
__global__ void __launch_bounds__(256) col_tma_kernel(PassArgs a, const float2 *__restrict__ stw,
                                                      const __grid_constant__ CUtensorMap tin,
                                                      const __grid_constant__ CUtensorMap tout) {
  constexpr int T = N / 16;
  constexpr int S = N + N / 16 + (C > 1 ? 16 / C : 0);
  constexpr int BOX = N < 256 ? N : 256;
  static_assert(C * S >= C * N, "the tile fits the exchange lines");
  static_assert((N * sizeof(float2)) % kTmaSmemAlign == 0 && (BOX * C * sizeof(float2)) % kTmaSmemAlign == 0,
                "every box of the tile starts on the bulk tensor copies' shared-memory alignment");
  // The dynamic shared memory of a kernel starts where the file's first
  // declaration of an extern shared array says, not where a later one asks
  // for; the block rounds its base up to the copies' alignment itself (the
  // launch adds kTmaSmemAlign bytes for it).
  extern __shared__ unsigned char tma_smem_raw[];
  __shared__ __align__(8) uint64_t bar;
  float2 *sm = reinterpret_cast<float2 *>(
      tma_smem_raw + ((kTmaSmemAlign - (smem_u32(tma_smem_raw) & (kTmaSmemAlign - 1))) & (kTmaSmemAlign - 1)));
  constexpr bool PROJ = MODE == COL_PROJECT || MODE == COL_PROJECT_NOFC;  // else the blur pass
  const int c = threadIdx.x % C, t = threadIdx.x / C;
  const int col0 = blockIdx.x * C;
  // self-check before any copy is issued (uniform over the block): a tile
  // that is not aligned, or a first column whose byte offset is not a
  // multiple of 16, is reported through the error flag and nothing is copied
  if ((smem_u32(sm + N) & (kTmaSmemAlign - 1)) || ((col0 * (int)sizeof(float2)) & 15)) {
    if (threadIdx.x == 0 && a.err_flag) atomicExch(a.err_flag, 2);
    return;
  }
  float2 *tw_s = sm;
  float2 *tile = sm + N;  // [N][C] dense, in the exchange lines' space
  float2 *line = sm + N + c * S;
  constexpr int W = proj_words(N);
  constexpr int SA = amp_stride<N, C>();
  constexpr int SW = bits_stride<N, C>();
  float *amp_s = reinterpret_cast<float *>(sm + N + C * S);
  uint32_t *meas_s = reinterpret_cast<uint32_t *>(amp_s + C * SA);
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_init_fence();
  }
  stage_twiddles<N>(tw_s, stw);
  if constexpr (PROJ) {
    const float *asrc = a.amp_line + (size_t)col0 * N;
    for (int k = threadIdx.x; k < C * (N / 4); k += blockDim.x) {
      const int l = k / (N / 4), j = k % (N / 4);
      cp_async16(amp_s + l * SA + 4 * j, asrc + (size_t)l * N + 4 * j);
    }
    const uint32_t *msrc = a.meas_bits + (size_t)col0 * W;
    for (int k = threadIdx.x; k < C * (W / 4); k += blockDim.x) {
      const int l = k / (W / 4), j = k % (W / 4);
      cp_async16(meas_s + l * SW + 4 * j, msrc + (size_t)l * W + 4 * j);
    }
  }
  __syncthreads();  // the barrier's initialisation before any wait on it
  const long long o = a.outer0 + blockIdx.y;
  const size_t qstride = (size_t)T * a.estride;
  const size_t lbase = (size_t)o * a.ostride + col0 + c + (size_t)t * a.estride;
  pdl_wait();
  if (threadIdx.x == 0) {
    mbar_expect_tx(&bar, (unsigned)(N * C * sizeof(float2)));
#pragma unroll
    for (int k = 0; k < N / BOX; k++) tma_load_2d(tile + k * BOX * C, &tin, col0, (int)(o * N + k * BOX), &bar);
  }
  if (!mbar_wait_block(&bar, 0)) {  // the tile never arrived: flag it and leave (nothing of this block is written)
    if (threadIdx.x == 0 && a.err_flag) atomicExch(a.err_flag, 1);
    return;
  }
  float2 v[16];
#pragma unroll
  for (int q = 0; q < 16; q++) v[q] = tile[(t + T * q) * C + c];
  cp_async_wait_all();
  __syncthreads();  // every tile read (and the operand lines in) before the exchanges reuse the space
  reg::fft<N, false>(v, line, t, tw_s);
  if constexpr (PROJ) project16<T, MODE == COL_PROJECT>(v, amp_s + c * SA, meas_s + c * SW, t, lbase, qstride, a);
  else blur16<T>(v, col0 + c, o, t, a);
  reg::fft<N, true>(v, line, t, tw_s);
  __syncthreads();  // the exchange lines are free again
#pragma unroll
  for (int q = 0; q < 16; q++) tile[(t + T * q) * C + c] = v[q];
  fence_proxy_async_smem();  // the tile's writes visible to the tensor copies
  __syncthreads();
  pdl_release();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < N / BOX; k++) tma_store_2d(&tout, col0, (int)(o * N + k * BOX), tile + k * BOX * C);
    bulk_commit();
    bulk_wait_read0();  // the shared-memory tile stays until the copies have read it
  }
}

// cuTensorMapEncodeTiled from the driver (no link-time dependency on libcuda)
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  return fn;
}

// a 2-D view of a buffer of float2: rows of `inner` elements (the column
// stride), `rows` rows; boxes of C elements by `box_rows` rows
static bool make_tile_map(CUtensorMap *m, const void *base, long long inner, long long rows, int C, int box_rows) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)inner * sizeof(float2)};
  const cuuint32_t box[2] = {(cuuint32_t)C, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT64, 2, const_cast<void *>(base), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Whether the TMA form serves this projection launch: 16-byte-aligned tile
// columns (C >= 2 columns of 8 bytes, an even column stride), whole tiles
// (ncols a multiple of C), lines of the tile's length, 16-byte-aligned bases.
template <int N, int C>
static bool tma_tile_fits(const PassArgs &a) {
  if (C < 2 || a.ncols % C != 0 || (a.estride & 1) || a.ostride != (long long)N * a.estride) return false;
  return !((uintptr_t)a.src & 15) && !((uintptr_t)a.dst & 15);
}
template <int N, int C>
static bool tma_fits(const PassArgs &a) {
  return tma_tile_fits<N, C>(a) && a.amp_line && a.meas_bits && a.meas_words == proj_words(N);
}

template <int N, int MODE, int C>
static cudaError_t col_tma_launch(const LinePlan &pl, const PassArgs &a, cudaStream_t st) {
  constexpr int T = N / 16;
  constexpr bool PROJ = MODE == COL_PROJECT || MODE == COL_PROJECT_NOFC;
  const size_t smem = (size_t)(N + C * (N + N / 16 + (C > 1 ? 16 / C : 0))) * sizeof(float2) +
                      (PROJ ? (size_t)C * amp_stride<N, C>() * sizeof(float) +
                                  (size_t)C * bits_stride<N, C>() * sizeof(uint32_t)
                            : 0) +
                      kTmaSmemAlign;  // room to round the block's base up to the copies' alignment
  CUtensorMap tin, tout;
  const long long rows = (a.outer0 + a.nouter) * (long long)N;
  constexpr int BOX = N < 256 ? N : 256;
  if (!make_tile_map(&tin, a.src, a.estride, rows, C, BOX) || !make_tile_map(&tout, a.dst, a.estride, rows, C, BOX))
    return cudaErrorNotSupported;
  cudaError_t e = ensure_smem<col_tma_kernel<N, MODE, C>>(smem);
  if (e != cudaSuccess) return e;
  dim3 grid((a.ncols + C - 1) / C, a.nouter);
  return launch_maybe_pdl(col_tma_kernel<N, MODE, C>, grid, dim3(C * T), smem, st, a.pdl != 0, a, pl.stw, tin, tout);
}

// --------------------------------------- iteration row pass staged by TMA
// The row pass of an HIO/RAAR/ER iteration (row_fast_kernel<N, ROW_ITER,
// G0LATE>) with its inputs moved by 1-D bulk copies: one thread arms an
// mbarrier with the block's byte count and copies each row's flags (and,
// unless G0LATE, its previous iterate) before the dependent-launch wait --
// they were written two or more kernels earlier -- and each row of Y after
// it, dense into the row's exchange line, which is free before the first
// stage.  With G0LATE the previous iterate's rows are copied into the
// exchange lines between the two transforms under a second mbarrier.  The
// transforms, the update and the outputs are those of row_fast_kernel, so
// the bits are too.  Rows of N >= 64 points: every row, line and flag row
// starts on a 16-byte boundary and is a multiple of 16 bytes long.
template <int N, bool G0LATE>
__global__ void __launch_bounds__(256) row_tma_kernel(PassArgs a, const float2 *__restrict__ stw, int nrows) {
  constexpr int T = N / 16;
  constexpr int S = N + N / 16;
  static_assert(N >= 64 && (S * sizeof(float2)) % 16 == 0 && N % 16 == 0, "rows and lines of whole 16-byte chunks");
  extern __shared__ __align__(16) float2 sm[];
  __shared__ __align__(8) uint64_t bar[2];
  const int lpb = blockDim.x / T;
  const int lr = threadIdx.x / T, t = threadIdx.x % T;
  const int row0 = blockIdx.x * lpb;
  const int row = row0 + lr;
  const bool valid = row < nrows;
  float2 *tw_s = sm;
  float2 *line = sm + N + lr * S;
  const size_t base = (size_t)row * N + t;
  float2 *g0_s = sm + N + lpb * S;  // an even float2 offset: 16-byte aligned
  uint8_t *fl_s = reinterpret_cast<uint8_t *>(g0_s + (G0LATE ? 0 : lpb * N));
  const int vrows = min(lpb, nrows - row0);
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init_fence();
  }
  stage_twiddles<N>(tw_s, stw);
  __syncthreads();  // the barriers' initialisation before any copy or wait
  if (threadIdx.x == 0) {
    const unsigned per_row = N * (unsigned)(sizeof(float2) + 1 + (G0LATE ? 0 : sizeof(float2)));
    mbar_expect_tx(&bar[0], per_row * (unsigned)vrows);
    for (int r = 0; r < vrows; r++) bulk_load(fl_s + r * N, a.flags + (size_t)(row0 + r) * N, N, &bar[0]);
    if constexpr (!G0LATE)
      for (int r = 0; r < vrows; r++)
        bulk_load(g0_s + r * N, a.g0 + (size_t)(row0 + r) * N, N * (unsigned)sizeof(float2), &bar[0]);
  }
  pdl_wait();
  if (threadIdx.x == 0)
    for (int r = 0; r < vrows; r++)
      bulk_load(sm + N + r * S, a.src + (size_t)(row0 + r) * N, N * (unsigned)sizeof(float2), &bar[0]);
  if (!mbar_wait_block(&bar[0], 0)) {  // the rows never arrived: flag it and leave (nothing is written)
    if (threadIdx.x == 0 && a.err_flag) atomicExch(a.err_flag, 1);
    return;
  }
  float2 v[16];
#pragma unroll
  for (int q = 0; q < 16; q++) v[q] = valid ? line[t + T * q] : make_float2(0.0f, 0.0f);
  cp_async_wait_all();  // twiddles
  __syncthreads();      // every row read before the exchanges reuse the lines
  const float beta = iter_beta(a);
  const float one_m2b = fsub(1.0f, fmul(2.0f, beta));  // 1 - 2*beta in float, as the reference
  reg::fft<N, true>(v, line, t, tw_s);
  if constexpr (G0LATE) {
    // the transform's last stage uses registers only and a barrier followed
    // its last exchange: the lines are free for the previous iterate
    if (threadIdx.x == 0) {
      fence_proxy_async_smem();
      mbar_expect_tx(&bar[1], (unsigned)vrows * N * (unsigned)sizeof(float2));
      for (int r = 0; r < vrows; r++)
        bulk_load(sm + N + r * S, a.g0 + (size_t)(row0 + r) * N, N * (unsigned)sizeof(float2), &bar[1]);
    }
    if (!mbar_wait_block(&bar[1], 0)) {
      if (threadIdx.x == 0 && a.err_flag) atomicExch(a.err_flag, 1);
      return;
    }
  }
  const float2 *g0r = G0LATE ? line + t : g0_s + lr * N + t;
  const uint8_t *flr = fl_s + lr * N + t;
  float2 *gp = a.gp;
#pragma unroll
  for (int q = 0; q < 16; q++) {
    float2 g = make_float2(0.0f, 0.0f);
    if (valid) {
      const float2 gpv = scale_cmul_dev(v[q], a.inv_n);
      if (gp) gp[base + T * q] = gpv;
      const uint8_t f = flr[T * q];
      if (f & FLAG_INSIDE) {
        g = gpv;
      } else if (a.alg == ALG_HIO) {
        const float2 g0 = g0r[T * q];
        g = make_float2(fsub(g0.x, fmul(gpv.x, beta)), fsub(g0.y, fmul(gpv.y, beta)));
      } else if (a.alg == ALG_RAAR) {
        const float2 g0 = g0r[T * q];
        g = make_float2(fadd(fmul(gpv.x, one_m2b), fmul(g0.x, beta)), fadd(fmul(gpv.y, one_m2b), fmul(g0.y, beta)));
      }
      g = apply_constraints(g, f, a.constraints);
      a.g1[base + T * q] = g;
    }
    v[q] = g;
  }
  if constexpr (G0LATE) __syncthreads();  // every g0 read done before the forward transform writes the lines
  reg::fft<N, false>(v, line, t, tw_s);
  pdl_release();
  if (valid)
#pragma unroll
    for (int q = 0; q < 16; q++) a.dst[base + T * q] = v[q];
}

// Whether the TMA row pass serves this launch: rows of 64..4096 points whose
// buffers start on 16-byte boundaries (every row then does too).  It runs
// only when asked for (SPB_TUNE_TMA = 2): measured on one B200 (graph-
// replayed calls, us per slot, plain / TMA rows) RAAR 1024^2 19.1-19.3 /
// 20.1-20.2, HIO 256^2 9.84 / 9.83, 512 starts of 512^2 1531-1547 /
// 1546-1548, HIO 128^3 40.2 / 40.9 -- the plain rows are coalesced 256-byte
// warp loads already, and the block waits for all of its rows either way.
template <int N>
static bool row_tma_fits(const PassArgs &a) {
  if (N < 64) return false;
  return !(((uintptr_t)a.src | (uintptr_t)a.g0 | (uintptr_t)a.flags) & 15);
}

// ------------------------------------------------ persistent small patterns
// One block per start of an N x N pattern (N = 32, 64, 128) runs every
// iteration of a call with the start's spectrum resident in shared memory:
// X (the row transform of the model) stays in the block between iterations,
// and each iteration is the column pass (forward y, projection, inverse y)
// and the row pass (inverse x, update, forward x) of the two-pass kernels,
// separated by block barriers instead of kernel boundaries.  The previous
// iterate, the flags and the amplitude lines are read from global memory
// (L2); the new iterate is written there.  Same transforms and pointwise
// steps, so the bits are those of the two-pass kernels.
//
// Shared memory: [twiddles N][N rows of pitch P = N + N/16].  Element (row i,
// column x) of X sits at i*P + x; a row's exchanges use the padded positions
// of its own P slots, a column's exchanges use its own elements (stride P).
namespace reg {
template <int N, int S, int NS, bool INV, int STRIDE>
struct PStages {
  // storage address of line index i: padded within a row (STRIDE 0) or down a column
  static __device__ __forceinline__ int at(int i) { return STRIDE == 0 ? pad(i) : i * STRIDE; }
  static __device__ __forceinline__ void run(float2 (&v)[16], float2 *line, int t, const float2 *stw) {
    constexpr int R = plan_radix(N, S);
    constexpr int T = N / 16;
    constexpr int J = 16 / R;
    constexpr bool LAST = (S == plan_len(N) - 1);
#pragma unroll
    for (int j = 0; j < J; j++) {
      float2 a[R];
#pragma unroll
      for (int m = 0; m < R; m++) a[m] = v[j + m * J];
      const int b = t + T * j;
      const int k = b & (NS - 1);
      if constexpr (NS > 1) {
#pragma unroll
        for (int m = 1; m < R; m++) {
          float2 w = stw[(m - 1) * NS + k];
          if (INV) w.y = -w.y;
          const float2 p = cmulw(a[m], w.x, w.y);
          a[m] = k ? p : a[m];
        }
      }
      bfly<R, INV>(a);
      if constexpr (LAST) {
#pragma unroll
        for (int m = 0; m < R; m++) v[j + m * J] = a[m];
      } else {
        const int base = (b / NS) * NS * R + k;
#pragma unroll
        for (int m = 0; m < R; m++) line[at(base + m * NS)] = a[m];
      }
    }
    if constexpr (!LAST) {
      __syncthreads();
#pragma unroll
      for (int q = 0; q < 16; q++) v[q] = line[at(t + T * q)];
      __syncthreads();
      PStages<N, S + 1, NS * R, INV, STRIDE>::run(v, line, t, stw + (R - 1) * NS);
    }
  }
};
}  // namespace reg

// blocks per SM the register budget is sized for (64 registers a thread)
template <int N>
__host__ __device__ constexpr int persist_min_blocks() {
  return N >= 128 ? 1 : (N == 64 ? 4 : 16);
}

template <int N>
__global__ void __launch_bounds__(N * N / 16, persist_min_blocks<N>())
    persist_kernel(PassArgs a, const float2 *__restrict__ stw, float2 *gbuf0, float2 *gbuf1, int cur0, int iters,
                   int keep_gp) {
  constexpr int T = N / 16;
  constexpr int P = N + N / 16;
  constexpr int W = proj_words(N);
  extern __shared__ __align__(16) float2 sm[];
  float2 *tw_s = sm;
  float2 *Xs = sm + N;
  const size_t off = (size_t)blockIdx.x * N * N;
  const uint8_t *flags = a.flags + off;
  float2 *Xg = a.dst + off;
  stage_twiddles<N>(tw_s, stw);
  for (int i = threadIdx.x; i < N * N; i += blockDim.x) Xs[(i / N) * P + (i % N)] = Xg[i];
  cp_async_wait_all();
  __syncthreads();
  int cur = cur0;
  for (int it = 0; it < iters; it++) {
    cur ^= 1;
    const float2 *g0 = (cur ? gbuf0 : gbuf1) + off;  // the previous model
    float2 *g1 = (cur ? gbuf1 : gbuf0) + off;        // the new one
    const float beta = a.alg == ALG_ER ? 0.0f : (a.beta_tab ? a.beta_tab[*a.beta_base + it] : a.beta);
    const float one_m2b = fsub(1.0f, fmul(2.0f, beta));
    {  // column pass: column c, thread t of its T
      const int c = threadIdx.x % N, t = threadIdx.x / N;
      float2 v[16];
#pragma unroll
      for (int q = 0; q < 16; q++) v[q] = Xs[(t + T * q) * P + c];
      __syncthreads();  // every column read before its elements serve as exchange space
      reg::PStages<N, 0, 1, false, P>::run(v, Xs + c, t, tw_s);
      project16<T, true>(v, a.amp_line + (size_t)c * N, a.meas_bits + (size_t)c * W, t, (size_t)t * N + c,
                         (size_t)T * N, a);
      reg::PStages<N, 0, 1, true, P>::run(v, Xs + c, t, tw_s);
#pragma unroll
      for (int q = 0; q < 16; q++) Xs[(t + T * q) * P + c] = v[q];
      __syncthreads();
    }
    {  // row pass: row r, thread t of its T
      const int r = threadIdx.x / T, t = threadIdx.x % T;
      float2 v[16];
#pragma unroll
      for (int q = 0; q < 16; q++) v[q] = Xs[r * P + t + T * q];
      __syncthreads();  // every row read before its slots serve as exchange space
      reg::PStages<N, 0, 1, true, 0>::run(v, Xs + r * P, t, tw_s);
      const bool last = keep_gp && it == iters - 1;
#pragma unroll
      for (int q = 0; q < 16; q++) {
        const int idx = r * N + t + T * q;
        const float2 gpv = scale_cmul_dev(v[q], a.inv_n);
        if (last) a.gp[off + idx] = gpv;
        const uint8_t f = flags[idx];
        float2 g = make_float2(0.0f, 0.0f);
        if (f & FLAG_INSIDE) {
          g = gpv;
        } else if (a.alg == ALG_HIO) {
          const float2 o = g0[idx];
          g = make_float2(fsub(o.x, fmul(gpv.x, beta)), fsub(o.y, fmul(gpv.y, beta)));
        } else if (a.alg == ALG_RAAR) {
          const float2 o = g0[idx];
          g = make_float2(fadd(fmul(gpv.x, one_m2b), fmul(o.x, beta)), fadd(fmul(gpv.y, one_m2b), fmul(o.y, beta)));
        }
        g = apply_constraints(g, f, a.constraints);
        g1[idx] = g;
        v[q] = g;
      }
      reg::PStages<N, 0, 1, false, 0>::run(v, Xs + r * P, t, tw_s);
#pragma unroll
      for (int q = 0; q < 16; q++) Xs[r * P + t + T * q] = v[q];
      __syncthreads();
    }
  }
  for (int i = threadIdx.x; i < N * N; i += blockDim.x) Xg[i] = Xs[(i / N) * P + (i % N)];
}

template <int N>
static cudaError_t persist_launch(const LinePlan &px, const PassArgs &a, float2 *g0, float2 *g1, int cur0, int iters,
                                  int keep_gp, int nb, cudaStream_t st) {
  const size_t smem = (size_t)(N + N * (N + N / 16)) * sizeof(float2);
  cudaError_t e = ensure_smem<persist_kernel<N>>(smem);
  if (e != cudaSuccess) return e;
  persist_kernel<N><<<nb, N * N / 16, smem, st>>>(a, px.stw, g0, g1, cur0, iters, keep_gp);
  return cudaGetLastError();
}

cudaError_t launch_persist(const LinePlan &px, const PassArgs &a, float2 *g0, float2 *g1, int cur0, int iters,
                           int keep_gp, int nb, cudaStream_t st) {
  if (!px.stw || a.meas_words != proj_words(px.n)) return cudaErrorNotSupported;
  switch (px.n) {
    case 32: return persist_launch<32>(px, a, g0, g1, cur0, iters, keep_gp, nb, st);
    case 64: return persist_launch<64>(px, a, g0, g1, cur0, iters, keep_gp, nb, st);
    case 128: return persist_launch<128>(px, a, g0, g1, cur0, iters, keep_gp, nb, st);
  }
  return cudaErrorNotSupported;
}

// ------------------------------------------------- 3-D plane pass (ny = nz)
// The y and z passes of a 3-D iteration in one launch: one block per x-plane
// of a start holds the plane's N x N points (rows along y, one per z) in
// shared memory and runs the forward y transforms (rows), then per column
// (one per y) the forward z transform, the projection and the inverse z
// transform, then the inverse y transforms (rows).  That is the work of the
// forward y, z projection and inverse y column passes, with one read and one
// write of the volume instead of three of each.  Same transforms, projection
// and order, so the bits are those of the three passes.
//
// Shared memory: [twiddles N][N rows of pitch P = N + N/16] as in the
// persistent form: point (z, y) of the plane at z*P + y; a row's exchanges
// use the padded positions of its own P slots, a column's use its own
// elements (stride P).  Plane loads and stores are 8-byte accesses at stride
// nx points; the neighbouring planes' blocks run at the same time and share
// the sectors in L2.
template <int N, int MODE>
__global__ void __launch_bounds__(N * N / 16, 1) plane_kernel(PassArgs a, const float2 *__restrict__ stw) {
  constexpr int T = N / 16;
  constexpr int P = N + N / 16;
  constexpr int W = proj_words(N);
  extern __shared__ __align__(16) float2 sm[];
  float2 *tw_s = sm;
  float2 *Ps = sm + N;
  const int x = blockIdx.x;
  const long long b = a.outer0 + blockIdx.y;
  const long long nxy = (long long)a.nx * N;  // points per z-slice (ny = N)
  const long long off = b * a.n_start + x;     // point (z, y) of the plane at off + z*nxy + y*nx
  stage_twiddles<N>(tw_s, stw);
  pdl_wait();
  {  // forward y: row r (z = r), thread t of its T, straight from global memory
    const int r = threadIdx.x / T, t = threadIdx.x % T;
    const float2 *src = a.src + off + (long long)r * nxy + (long long)t * a.nx;
    float2 v[16];
#pragma unroll
    for (int q = 0; q < 16; q++) v[q] = src[(long long)(T * q) * a.nx];
    cp_async_wait_all();
    __syncthreads();  // twiddles in
    reg::PStages<N, 0, 1, false, 0>::run(v, Ps + r * P, t, tw_s);
#pragma unroll
    for (int q = 0; q < 16; q++) Ps[r * P + t + T * q] = v[q];
    __syncthreads();
  }
  {  // column c (y = c), thread t of its T: forward z, projection, inverse z
    const int c = threadIdx.x % N, t = threadIdx.x / N;
    float2 v[16];
#pragma unroll
    for (int q = 0; q < 16; q++) v[q] = Ps[(t + T * q) * P + c];
    __syncthreads();  // every column read before its elements serve as exchange space
    reg::PStages<N, 0, 1, false, P>::run(v, Ps + c, t, tw_s);
    const long long line = (long long)c * a.nx + x;  // z-line index y*nx + x
    project16<T, MODE == COL_PROJECT>(v, a.amp_line + line * N, a.meas_bits + line * W, t,
                                      (size_t)(off + (long long)c * a.nx + (long long)t * nxy), (size_t)T * nxy, a);
    reg::PStages<N, 0, 1, true, P>::run(v, Ps + c, t, tw_s);
#pragma unroll
    for (int q = 0; q < 16; q++) Ps[(t + T * q) * P + c] = v[q];
    __syncthreads();
  }
  {  // inverse y: row r, thread t
    const int r = threadIdx.x / T, t = threadIdx.x % T;
    float2 v[16];
#pragma unroll
    for (int q = 0; q < 16; q++) v[q] = Ps[r * P + t + T * q];
    __syncthreads();  // every row read before its slots serve as exchange space
    reg::PStages<N, 0, 1, true, 0>::run(v, Ps + r * P, t, tw_s);
    pdl_release();
    float2 *dst = a.dst + off + (long long)r * nxy + (long long)t * a.nx;
#pragma unroll
    for (int q = 0; q < 16; q++) dst[(long long)(T * q) * a.nx] = v[q];
  }
}

template <int N, int MODE>
static cudaError_t plane_launch_n(const LinePlan &pl, const PassArgs &a, cudaStream_t st) {
  const size_t smem = (size_t)(N + N * (N + N / 16)) * sizeof(float2);
  cudaError_t e = ensure_smem<plane_kernel<N, MODE>>(smem);
  if (e != cudaSuccess) return e;
  return launch_maybe_pdl(plane_kernel<N, MODE>, dim3(a.nx, a.nouter), dim3(N * N / 16), smem, st, a.pdl != 0, a,
                          pl.stw);
}

// Whether the plane pass serves this projection: a 3-D volume with ny = nz =
// 64 or 128, a projection mode, the line-major amplitudes and measured bits.
bool plane_fits(int mode, const LinePlan &pl, const PassArgs &a) {
  if (mode != COL_PROJECT && mode != COL_PROJECT_NOFC) return false;
  if (a.nz == 1 || pl.n != a.ny || a.ny != a.nz || (pl.n != 64 && pl.n != 128)) return false;
  return pl.stw && a.amp_line && a.meas_bits && a.meas_words == proj_words(pl.n);
}

// The plane pass (cudaErrorNotSupported where plane_fits says no); a.nouter
// starts from a.outer0 (at most 65535 per launch).
cudaError_t launch_plane(int mode, const LinePlan &pl, const PassArgs &a, cudaStream_t st) {
  if (!plane_fits(mode, pl, a)) return cudaErrorNotSupported;
  switch (pl.n) {
    case 64:
      return mode == COL_PROJECT ? plane_launch_n<64, COL_PROJECT>(pl, a, st) : plane_launch_n<64, COL_PROJECT_NOFC>(pl, a, st);
    case 128:
      return mode == COL_PROJECT ? plane_launch_n<128, COL_PROJECT>(pl, a, st)
                                 : plane_launch_n<128, COL_PROJECT_NOFC>(pl, a, st);
  }
  return cudaErrorNotSupported;
}

// ------------------------------------------- self-check of the roundings
// Bit-for-bit comparisons of the branch-free forms with the IEEE intrinsics,
// counting differences: every float x with bit pattern in [lo, hi) inside the
// square-root domain (square root) and inside [2^-63, 2^63] (reciprocal);
// n pseudo-random quotients a/b with a and b drawn over their domains; and the
// quotients of significand pairs a in [1, 2) (every a_stride-th significand)
// and b in [1, 2) (every significand; for divisor significand mb the
// dividend's run over (mb * 2654435761 + seed) mod a_stride + k * a_stride, so
// the calls with seed = 0 .. a_stride-1 cover every pair once).
__global__ void check_sqrt_rcp_kernel(unsigned lo, unsigned hi, unsigned long long *bad) {
  unsigned long long nsq = 0, nrc = 0;
  for (unsigned long long u = lo + (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; u < hi;
       u += (unsigned long long)gridDim.x * blockDim.x) {
    const float x = __uint_as_float((unsigned)u);
    if (sqrt_rn_nb_domain(x)) nsq += __float_as_uint(sqrt_rn_nb(x)) != __float_as_uint(__fsqrt_rn(x));
    if (x >= 0x1p-63f && x <= 0x1p63f) nrc += __float_as_uint(rcp_rn_nb(x)) != __float_as_uint(__frcp_rn(x));
  }
  if (nsq) atomicAdd(bad, nsq);
  if (nrc) atomicAdd(bad + 1, nrc);
}

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;  // splitmix64 finaliser
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__global__ void check_div_kernel(unsigned long long n, unsigned long long seed, unsigned long long *bad) {
  unsigned long long nbad = 0;
  for (unsigned long long k = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long r = mix64(seed ^ mix64(k));
    // a: random sign and significand, exponent in [-60, 60) (one in 64 draws: zero)
    const unsigned ea = 67u + (unsigned)((r >> 24) % 120u);
    const float a = ((r >> 58) == 0) ? 0.0f : __uint_as_float(((unsigned)r & 0x807FFFFFu) | (ea << 23));
    // b: exponent in [-63, 63), random significand
    const unsigned eb = 64u + (unsigned)((r >> 32) % 126u);
    const float b = __uint_as_float((eb << 23) | ((unsigned)(r >> 40) & 0x7FFFFFu));
    nbad += __float_as_uint(div_rn_nb(a, b)) != __float_as_uint(__fdiv_rn(a, b));
  }
  if (nbad) atomicAdd(bad, nbad);
}

__global__ void check_div_significands_kernel(unsigned a_stride, unsigned phase, unsigned long long *bad) {
  unsigned long long nbad = 0;
  for (unsigned mb = blockIdx.x * blockDim.x + threadIdx.x; mb < (1u << 23); mb += gridDim.x * blockDim.x) {
    const float b = __uint_as_float(0x3F800000u | mb);
    for (unsigned ma = (mb * 2654435761u + phase) % a_stride; ma < (1u << 23); ma += a_stride) {
      const float a = __uint_as_float(0x3F800000u | ma);
      nbad += __float_as_uint(div_rn_nb(a, b)) != __float_as_uint(__fdiv_rn(a, b));
    }
  }
  if (nbad) atomicAdd(bad, nbad);
}

cudaError_t check_roundings(unsigned lo, unsigned hi, unsigned long long ndiv, unsigned long long seed,
                            unsigned a_stride, unsigned long long *d_bad) {
  if (hi > lo) check_sqrt_rcp_kernel<<<148 * 8, 256>>>(lo, hi, d_bad);
  if (ndiv) check_div_kernel<<<148 * 8, 256>>>(ndiv, seed, d_bad + 2);
  if (a_stride) check_div_significands_kernel<<<148 * 8, 256>>>(a_stride, (unsigned)(seed % a_stride), d_bad + 3);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- launch
template <typename K>
static cudaError_t set_smem(K k, size_t smem, bool &done) {
  if (done) return cudaSuccess;
  const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) done = true;
  return e;
}


template <int N, int MODE>
static cudaError_t row_fast_launch(const LinePlan &px, const PassArgs &a, cudaStream_t st) {
  constexpr int T = N / 16;
  constexpr int LPB_MAX = (256 / T) > 0 ? (256 / T) : 1;  // 256 threads per block at most
  const long long nrows = a.n / N;
  static int nsm = 0;
  if (!nsm && cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, 0) != cudaSuccess) return cudaGetLastError();
  // a few short difference-map rows per SM: the general row pass (one
  // butterfly per thread, more threads per row) is faster
  if (MODE == ROW_DM_ITER && N < 256 && nrows < 4LL * nsm) return cudaErrorNotSupported;
  int LPB = (a.row_lpb > 0 && a.row_lpb < LPB_MAX) ? a.row_lpb : LPB_MAX;
  if (a.row_lpb <= 0) {
    // built-in choice: 256 threads per block, fewer (down to one warp) while
    // the grid would leave SMs without a block
    while (LPB > 1 && LPB * T > 32 && (nrows + LPB - 1) / LPB < nsm) LPB >>= 1;
  }
  const long long grid = (nrows + LPB - 1) / LPB;
  const size_t smem0 = (size_t)((N + LPB * (N + N / 16) + 1) & ~1) * sizeof(float2);
  if constexpr (MODE == ROW_ITER || MODE == ROW_DM_ITER) {
    // g0 staging: SPB_TUNE_ROW_G0 1 = at the start, 2 = between the
    // transforms; 0 = between the transforms when the grid is larger than the
    // blocks that fit on the device at once with the larger staging
    const size_t smem_early = smem0 + (size_t)LPB * N * (sizeof(float2) + 1), smem_late = smem0 + (size_t)LPB * N;
    bool late = a.row_g0 == 2;
    if (a.row_g0 == 0) {
      int per_sm = 0;
      cudaError_t e = ensure_smem<row_fast_kernel<N, MODE, false>>(smem_early);
      if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, row_fast_kernel<N, MODE, false>, LPB * T, smem_early);
      if (e != cudaSuccess) return e;
      late = grid > (long long)per_sm * nsm;
    }
    if constexpr (MODE == ROW_ITER && N >= 64) {
      // the rows staged by TMA (knob 2; same shared memory as the plain form)
      if (a.tma == 2 && row_tma_fits<N>(a)) {
        if (late) {
          cudaError_t e = ensure_smem<row_tma_kernel<N, true>>(smem_late);
          if (e != cudaSuccess) return e;
          return launch_maybe_pdl(row_tma_kernel<N, true>, dim3((unsigned)grid), dim3(LPB * T), smem_late, st,
                                  a.pdl != 0, a, px.stw, (int)nrows);
        }
        cudaError_t e = ensure_smem<row_tma_kernel<N, false>>(smem_early);
        if (e != cudaSuccess) return e;
        return launch_maybe_pdl(row_tma_kernel<N, false>, dim3((unsigned)grid), dim3(LPB * T), smem_early, st,
                                a.pdl != 0, a, px.stw, (int)nrows);
      }
    }
    if (late) {
      cudaError_t e = ensure_smem<row_fast_kernel<N, MODE, true>>(smem_late);
      if (e != cudaSuccess) return e;
      return launch_maybe_pdl(row_fast_kernel<N, MODE, true>, dim3((unsigned)grid), dim3(LPB * T), smem_late, st,
                              a.pdl != 0, a, px.stw, (int)nrows);
    }
    cudaError_t e = ensure_smem<row_fast_kernel<N, MODE, false>>(smem_early);
    if (e != cudaSuccess) return e;
    return launch_maybe_pdl(row_fast_kernel<N, MODE, false>, dim3((unsigned)grid), dim3(LPB * T), smem_early, st,
                            a.pdl != 0, a, px.stw, (int)nrows);
  }
  cudaError_t e = ensure_smem<row_fast_kernel<N, MODE, false>>(smem0);
  if (e != cudaSuccess) return e;
  return launch_maybe_pdl(row_fast_kernel<N, MODE, false>, dim3((unsigned)grid), dim3(LPB * T), smem0, st,
                          a.pdl != 0, a, px.stw, (int)nrows);
}

template <int N>
__host__ __device__ static constexpr int col_width() {
  return N >= 2048 ? (4096 / N) : (N >= 512 ? 4 : (N >= 256 ? 8 : 16));
}

template <int N, int MODE, bool PREFETCH, int C = col_width<N>()>
static cudaError_t col_fast_launch_p(const LinePlan &pl, const PassArgs &a, cudaStream_t st) {
  constexpr int T = N / 16;
  size_t smem = (size_t)(N + C * (N + N / 16 + (C > 1 ? 16 / C : 0))) * sizeof(float2);
  if (PREFETCH) {
    if (a.meas_words != proj_words(N)) return cudaErrorInvalidValue;
    smem += (size_t)C * amp_stride<N, C>() * sizeof(float) + (size_t)C * bits_stride<N, C>() * sizeof(uint32_t);
  }
  auto k = col_fast_kernel<N, MODE, C, PREFETCH>;
  static bool done = false;
  static size_t done_smem = 0;
  if (smem > done_smem) done = false;
  cudaError_t e = set_smem(k, smem, done);
  if (e != cudaSuccess) return e;
  if (smem > done_smem) done_smem = smem;
  dim3 grid((a.ncols + C - 1) / C, a.nouter);
  return launch_maybe_pdl(k, grid, dim3(C * T), smem, st, a.pdl != 0, a, pl.stw);
}

// Columns per block the projection pass offers besides the built-in width:
// lines of 256, 512 and 1024 points, C a power of two with C*N/16 <= 256
// threads and C <= 16 (the shared-memory skew is 16/C words); and the
// lengths the general kernels run with compile-time plans (general_col_width_ok).
bool col_width_ok(int n, int w) {
  if (w < 1 || w > 16 || (w & (w - 1))) return false;
  if (n != 256 && n != 512 && n != 1024) return general_col_width_ok(n, w);
  return w * (n / 16) <= 256;
}

template <int N, int MODE>
static cudaError_t col_fast_launch(const LinePlan &pl, const PassArgs &a, cudaStream_t st) {
  constexpr bool PROJ = (MODE == COL_PROJECT || MODE == COL_PROJECT_NOFC);
  // projection passes run along the last axis; every start (outer index)
  // shares the line-major amplitude and measured-bit lines of its column
  if (PROJ && a.amp_line && a.meas_bits && (a.meas_words % 4) == 0) {
    if constexpr (PROJ && N >= 64) {
      // the tile staged by the tensor memory accelerator at the built-in
      // width: by default (knob 0) unless another width is asked for, always
      // with knob 2, never with knob 1
      constexpr int C = col_width<N>();
      const bool want = a.tma == 2 || (a.tma == 0 && (a.col_width == 0 || a.col_width == C));
      if (want && tma_fits<N, C>(a)) {
        const cudaError_t te = col_tma_launch<N, MODE, C>(pl, a, st);
        if (te != cudaErrorNotSupported) return te;
      }
    }
    if constexpr (PROJ && (N == 256 || N == 512 || N == 1024)) {
      // a launch-shape knob: another number of columns per block
      switch (a.col_width) {
        case 1: return col_fast_launch_p<N, MODE, true, 1>(pl, a, st);
        case 2: return col_fast_launch_p<N, MODE, true, 2>(pl, a, st);
        case 4: return col_fast_launch_p<N, MODE, true, 4>(pl, a, st);
        case 8: if constexpr (8 * (N / 16) <= 256) return col_fast_launch_p<N, MODE, true, 8>(pl, a, st); break;
        case 16: if constexpr (16 * (N / 16) <= 256) return col_fast_launch_p<N, MODE, true, 16>(pl, a, st); break;
        default: break;
      }
    }
    return col_fast_launch_p<N, MODE, PROJ>(pl, a, st);
  }
  if constexpr (MODE == COL_BLUR && N >= 64) {
    // the blur pass's column tiles by the tensor memory accelerator too
    // (knob 1: plain loads), at the built-in width
    constexpr int C = col_width<N>();
    if (a.tma != 1 && tma_tile_fits<N, C>(a)) {
      const cudaError_t te = col_tma_launch<N, MODE, C>(pl, a, st);
      if (te != cudaErrorNotSupported) return te;
    }
  }
  return col_fast_launch_p<N, MODE, false>(pl, a, st);
}

template <int N>
static cudaError_t row_fast_mode(int mode, const LinePlan &px, const PassArgs &a, cudaStream_t st) {
  switch (mode) {
    case ROW_FWD: return row_fast_launch<N, ROW_FWD>(px, a, st);
    case ROW_FWD_DEPHASE: return row_fast_launch<N, ROW_FWD_DEPHASE>(px, a, st);
    case ROW_INV: return row_fast_launch<N, ROW_INV>(px, a, st);
    case ROW_INV_SCALE: return row_fast_launch<N, ROW_INV_SCALE>(px, a, st);
    case ROW_INV_ABS: return row_fast_launch<N, ROW_INV_ABS>(px, a, st);
    case ROW_ITER: return row_fast_launch<N, ROW_ITER>(px, a, st);
    case ROW_DM_ITER: return row_fast_launch<N, ROW_DM_ITER>(px, a, st);
    case ROW_FWD_F32: return row_fast_launch<N, ROW_FWD_F32>(px, a, st);
    case ROW_FWD_SQUARE_F32: return row_fast_launch<N, ROW_FWD_SQUARE_F32>(px, a, st);
  }
  return cudaErrorNotSupported;
}

template <int N>
static cudaError_t col_fast_mode(int mode, const LinePlan &pl, const PassArgs &a, cudaStream_t st) {
  switch (mode) {
    case COL_FWD: return col_fast_launch<N, COL_FWD>(pl, a, st);
    case COL_INV: return col_fast_launch<N, COL_INV>(pl, a, st);
    case COL_PROJECT: return col_fast_launch<N, COL_PROJECT>(pl, a, st);
    case COL_PROJECT_NOFC: return col_fast_launch<N, COL_PROJECT_NOFC>(pl, a, st);
    case COL_BLUR: return col_fast_launch<N, COL_BLUR>(pl, a, st);
    case COL_INV_SQUARE_F32: return col_fast_launch<N, COL_INV_SQUARE_F32>(pl, a, st);
  }
  return cudaErrorNotSupported;
}

// Returns cudaErrorNotSupported when no register kernel exists for the line
// length or mode; the caller then uses the general kernels.
cudaError_t launch_row_fast(int mode, const LinePlan &px, const PassArgs &a, cudaStream_t st) {
  if (!px.stw) return cudaErrorNotSupported;
  switch (px.n) {
    case 16: return row_fast_mode<16>(mode, px, a, st);
    case 32: return row_fast_mode<32>(mode, px, a, st);
    case 64: return row_fast_mode<64>(mode, px, a, st);
    case 128: return row_fast_mode<128>(mode, px, a, st);
    case 256: return row_fast_mode<256>(mode, px, a, st);
    case 512: return row_fast_mode<512>(mode, px, a, st);
    case 1024: return row_fast_mode<1024>(mode, px, a, st);
    case 2048: return row_fast_mode<2048>(mode, px, a, st);
    case 4096: return row_fast_mode<4096>(mode, px, a, st);
  }
  return cudaErrorNotSupported;
}

cudaError_t launch_col_fast(int mode, const LinePlan &pl, const PassArgs &a, cudaStream_t st) {
  if (!pl.stw) return cudaErrorNotSupported;
  switch (pl.n) {
    case 16: return col_fast_mode<16>(mode, pl, a, st);
    case 32: return col_fast_mode<32>(mode, pl, a, st);
    case 64: return col_fast_mode<64>(mode, pl, a, st);
    case 128: return col_fast_mode<128>(mode, pl, a, st);
    case 256: return col_fast_mode<256>(mode, pl, a, st);
    case 512: return col_fast_mode<512>(mode, pl, a, st);
    case 1024: return col_fast_mode<1024>(mode, pl, a, st);
    case 2048: return col_fast_mode<2048>(mode, pl, a, st);
    case 4096: return col_fast_mode<4096>(mode, pl, a, st);
  }
  return cudaErrorNotSupported;
}

}  // namespace spb
