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

#include <cooperative_groups.h>

#include "spb_internal.h"
#include "spb_passes.cuh"
#include "spb_pointwise.cuh"

namespace spb {

// ---------------------------------------------------------------- row pass
template <int MODE, int NC>
__device__ __forceinline__ void row_pass_body(const LinePlan &px, const PassArgs &a, int tpr, int rpb,
                                              long long nrows) {
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
  // the update's operands, loaded with the line: g0 after the transform
  // buffers, then the flags (bytes)
  constexpr bool UPD = (MODE == ROW_ITER || MODE == ROW_DM_ITER);
  constexpr int NBUF = (MODE == ROW_DM_ITER) ? 4 : 2;
  float2 *G0S = smem + (size_t)NBUF * slab + (size_t)lr * n;
  uint8_t *FLS = reinterpret_cast<uint8_t *>(smem + (size_t)(NBUF + 1) * slab) + (size_t)lr * n;

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
    if constexpr (UPD) {
      if (valid) {
        G0S[i] = a.g0[base + i];
        FLS[i] = a.flags[base + i];
      }
    }
  }
  __syncthreads();

  if constexpr (MODE == ROW_FWD || MODE == ROW_FWD_DEPHASE || MODE == ROW_FWD_F32 || MODE == ROW_FWD_SQUARE_F32 ||
                MODE == ROW_DM_F1_FWD) {
    float2 *r = line_fft_sel<false, NC>(A, B, px, 1, t, tpr, px.stw);
    if (valid)
      for (int i = t; i < n; i += tpr) a.dst[base + i] = r[i];
  } else if constexpr (MODE == ROW_INV || MODE == ROW_INV_SCALE || MODE == ROW_INV_ABS) {
    float2 *r = line_fft_sel<true, NC>(A, B, px, 1, t, tpr, px.stw);
    if (valid) {
      for (int i = t; i < n; i += tpr) {
        if constexpr (MODE == ROW_INV) a.dst[base + i] = r[i];
        else if constexpr (MODE == ROW_INV_SCALE) a.dst[base + i] = scale_cmul_dev(r[i], a.inv_n);
        else a.absout[base + i] = cabs_ref(r[i]);
      }
    }
  } else if constexpr (MODE == ROW_ITER) {
    const float beta = iter_beta(a);
    const float one_m2b = fsub(1.0f, fmul(2.0f, beta));  // 1 - 2*beta in float, as the reference
    float2 *r = line_fft_sel<true, NC>(A, B, px, 1, t, tpr, px.stw);
    for (int i = t; i < n; i += tpr) {
      float2 g = make_float2(0.0f, 0.0f);
      if (valid) {
        const long long idx = base + i;
        const float2 gp = scale_cmul_dev(r[i], a.inv_n);
        if (a.gp) a.gp[idx] = gp;
        const uint8_t f = FLS[i];
        if (f & FLAG_INSIDE) {
          g = gp;
        } else if (a.alg == ALG_HIO) {
          const float2 g0 = G0S[i];
          g = make_float2(fsub(g0.x, fmul(gp.x, beta)), fsub(g0.y, fmul(gp.y, beta)));
        } else if (a.alg == ALG_RAAR) {
          const float2 g0 = G0S[i];
          g = make_float2(fadd(fmul(gp.x, one_m2b), fmul(g0.x, beta)),
                          fadd(fmul(gp.y, one_m2b), fmul(g0.y, beta)));
        }
        g = apply_constraints(g, f, a.constraints);
        a.g1[idx] = g;
      }
      r[i] = g;
    }
    __syncthreads();
    float2 *o = (r == A) ? B : A;
    float2 *x = line_fft_sel<false, NC>(r, o, px, 1, t, tpr, px.stw);
    if (valid)
      for (int i = t; i < n; i += tpr) a.dst[base + i] = x[i];
  } else if constexpr (MODE == ROW_DM_ITER) {
    const float beta = iter_beta(a);
    float2 *rho = line_fft_sel<true, NC>(A, B, px, 1, t, tpr, px.stw);
    float2 *fr = line_fft_sel<true, NC>(Cb, D, px, 1, t, tpr, px.stw);
    for (int i = t; i < n; i += tpr) {
      float2 g = make_float2(0.0f, 0.0f), f1 = g;
      if (valid) {
        const long long idx = base + i;
        const float2 rv = rho[i], fv = fr[i], g0 = G0S[i];
        if (a.gp) a.gp[idx] = rv;
        const uint8_t f = FLS[i];
        if (f & FLAG_INSIDE) {
          g.x = fadd(g0.x, fmul(beta, fsub(__fdiv_rn(fmul(a.one_p_g2, rv.x), a.size_f), fmul(a.gamma2, g0.x))));
          g.y = fadd(g0.y, fmul(beta, fsub(__fdiv_rn(fmul(a.one_p_g2, rv.y), a.size_f), fmul(a.gamma2, g0.y))));
        } else {
          g = g0;
        }
        g.x = fsub(g.x, __fdiv_rn(fmul(beta, fv.x), a.size_f));
        g.y = fsub(g.y, __fdiv_rn(fmul(beta, fv.y), a.size_f));
        g = apply_constraints(g, f, a.constraints);
        a.g1[idx] = g;
        f1 = (f & FLAG_INSIDE) ? g : make_float2(fmul(-a.gamma1, g.x), fmul(-a.gamma1, g.y));
      }
      rho[i] = g;
      fr[i] = f1;
    }
    __syncthreads();
    float2 *o1 = (rho == A) ? B : A;
    float2 *x = line_fft_sel<false, NC>(rho, o1, px, 1, t, tpr, px.stw);
    float2 *o2 = (fr == Cb) ? D : Cb;
    float2 *xf = line_fft_sel<false, NC>(fr, o2, px, 1, t, tpr, px.stw);
    if (valid)
      for (int i = t; i < n; i += tpr) {
        a.dst[base + i] = x[i];
        a.dst2[base + i] = xf[i];
      }
  }
}

template <int MODE, int NC>
__global__ void __launch_bounds__(256) row_pass_kernel(LinePlan px, PassArgs a, int tpr, int rpb, long long nrows) {
  row_pass_body<MODE, NC>(px, a, tpr, rpb, nrows);
}

// 1000-point rows (the mixed batches' largest non-power-of-two length) run
// as one row of 200 threads per block with at most 32 registers, so that nine
// blocks share an SM and a 1000-row pattern takes one wave (the difference
// map's iteration keeps the general kernel).  Measured on one B200, HIO
// 1000x1000 per slot: 43.2 us with the general budget (42 registers), 43.6
// with 40, 39.9 with 32 (a few bytes of spills, more blocks in flight).
template <int MODE>
__global__ void __maxnreg__(32)
    row_pass_kernel_1000(LinePlan px, PassArgs a, int tpr, int rpb, long long nrows) {
  row_pass_body<MODE, 1000>(px, a, tpr, rpb, nrows);
}

// ------------------------------------------------------------- column pass
// byte offset of the stage table behind a column block's buffers (16-byte aligned)
__host__ __device__ constexpr size_t col_tw_offset(int n, int ct, bool proj) {
  return ((size_t)2 * n * ct * 8 + (proj ? (size_t)n * ct * 5 : 0) + 15) / 16 * 16;
}

// compile-time plans read their stage table from shared memory
template <int MODE, int NC>
__device__ __forceinline__ void col_pass_body(const LinePlan &pl, const PassArgs &a, int ct, int tpc) {
  extern __shared__ float2 smem[];
  const int n = pl.n;
  const int cc = threadIdx.x % ct, t = threadIdx.x / ct;
  const long long o = a.outer0 + blockIdx.y;
  const int c = blockIdx.x * ct + cc;
  const bool valid = c < a.ncols;
  float2 *A = smem + cc;
  float2 *B = smem + (size_t)n * ct + cc;
  const long long lbase = o * a.ostride + c;
  // projection operands, loaded with the line: amplitudes after the two
  // transform buffers, then the flags (bytes); ai0 = amplitude index of element 0
  constexpr bool PROJ = (MODE == COL_PROJECT || MODE == COL_PROJECT_NOFC);
  float *AMc = reinterpret_cast<float *>(smem + (size_t)2 * n * ct) + cc;
  uint8_t *FLc = reinterpret_cast<uint8_t *>(reinterpret_cast<float *>(smem + (size_t)2 * n * ct) + (size_t)n * ct) + cc;
  const long long ai0 = PROJ ? lbase % a.n_start : 0;
  float2 *TW = reinterpret_cast<float2 *>(reinterpret_cast<unsigned char *>(smem) + col_tw_offset(n, ct, PROJ));
  if constexpr (NC > 0)
    for (int i = threadIdx.x; i < NC - 1; i += blockDim.x) TW[i] = pl.stw[i];

  for (int i = t; i < n; i += tpc) {
    float2 v = make_float2(0.0f, 0.0f);
    if (valid) {
      if constexpr (MODE == COL_INV_SQUARE_F32) {
        const float s = a.f32src[lbase + i * a.estride];
        v = make_float2(fmul(s, s), 0.0f);
      } else {
        v = a.src[lbase + i * a.estride];
      }
      if constexpr (PROJ) {
        AMc[(size_t)i * ct] = a.amp[ai0 + i * a.estride];
        FLc[(size_t)i * ct] = a.flags[lbase + i * a.estride];
      }
    }
    A[(size_t)i * ct] = v;
  }
  __syncthreads();

  float2 *r;
  if constexpr (MODE == COL_FWD) {
    r = line_fft_sel<false, NC>(A, B, pl, ct, t, tpc, TW);
  } else if constexpr (MODE == COL_INV || MODE == COL_INV_SQUARE_F32) {
    r = line_fft_sel<true, NC>(A, B, pl, ct, t, tpc, TW);
  } else {
    float2 *f = line_fft_sel<false, NC>(A, B, pl, ct, t, tpc, TW);
    if (valid) {
      for (int i = t; i < n; i += tpc) {
        const long long idx = lbase + i * a.estride;
        float2 G = f[(size_t)i * ct];
        if constexpr (PROJ)
          G = project_vals(G, FLc[(size_t)i * ct], AMc[(size_t)i * ct], ai0 + i * a.estride, a, MODE == COL_PROJECT);
        else G = gauss_mult(G, idx, a);
        f[(size_t)i * ct] = G;
      }
    }
    __syncthreads();
    float2 *o2 = (f == A) ? B : A;
    r = line_fft_sel<true, NC>(f, o2, pl, ct, t, tpc, TW);
  }
  if (valid)
    for (int i = t; i < n; i += tpc) a.dst[lbase + i * a.estride] = r[(size_t)i * ct];
}

template <int MODE, int NC>
__global__ void __launch_bounds__(1024) col_pass_kernel(LinePlan pl, PassArgs a, int ct, int tpc) {
  col_pass_body<MODE, NC>(pl, a, ct, tpc);
}

// 1000-point columns run as four columns of 200 threads per block with at
// most 32 registers, so that two blocks share an SM (a 1000-column pattern:
// 250 blocks, one wave)
template <int MODE>
__global__ void __maxnreg__(32) col_pass_kernel_1000(LinePlan pl, PassArgs a, int ct, int tpc) {
  col_pass_body<MODE, 1000>(pl, a, ct, tpc);
}

// ---------------------------------------------------------------- launchers
static int pow2_at_least(int v) {
  int p = 1;
  while (p < v) p <<= 1;
  return p;
}

// dynamic shared memory attribute, set once per kernel and size
template <typename K>
static cudaError_t smem_attr(K k, size_t smem, size_t &done) {
  if (smem <= done) return cudaSuccess;
  const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) done = smem;
  return e;
}

// lengths with a compile-time plan in the general kernels (the non-power-of-two
// sizes of the mixed batches); others use the run-time plan
#define SPB_CT_LENGTHS(X) X(192) X(384) X(1000)
// the difference map's row passes also take compile-time plans at powers of
// two: grids of a few short rows per SM run here rather than in the register
// kernel (spb_fast.cu), and so does the f1 transform (ROW_DM_F1_FWD)
#define SPB_CT_LENGTHS_DM(X) X(64) X(128) X(256) X(512) X(1024) X(2048)

template <int MODE, int NC>
static cudaError_t row_launch_n(const LinePlan &px, const PassArgs &a, cudaStream_t st) {
  const int n = px.n;
  // compile-time plans: one butterfly per thread, at least two warps per row
  int tpr = NC > 0 ? (ct_max_butterflies(NC) > 64 ? ct_max_butterflies(NC) : 64) : pow2_at_least((n + 15) / 16);
  if (tpr > 256) tpr = 256;
  if (tpr < 1) tpr = 1;
  const long long nrows = a.n / n;
  int rpb = 256 / tpr;
  if (NC > 0) {  // no fewer blocks than two per SM when the rows allow it
    const long long cap = nrows / 296;
    if (cap < rpb) rpb = cap > 0 ? (int)cap : 1;
  }
  const int nbuf = (MODE == ROW_DM_ITER) ? 4 : 2;
  constexpr bool UPD = (MODE == ROW_ITER || MODE == ROW_DM_ITER);
  // transform buffers, then (UPD) a slab of g0 and rpb*n bytes of flags
  const size_t smem = (size_t)(nbuf + (UPD ? 1 : 0)) * rpb * n * sizeof(float2) + (UPD ? (size_t)rpb * n : 0);
  auto k = row_pass_kernel<MODE, NC>;
  if constexpr (NC == 1000 && MODE != ROW_DM_ITER) k = row_pass_kernel_1000<MODE>;
  static size_t done = 0;
  cudaError_t e = smem_attr(k, smem, done);
  if (e != cudaSuccess) return e;
  const long long grid = (nrows + rpb - 1) / rpb;
  k<<<(unsigned)grid, rpb * tpr, smem, st>>>(px, a, tpr, rpb, nrows);
  return cudaGetLastError();
}

template <int MODE>
static cudaError_t row_launch(const LinePlan &px, const PassArgs &a, cudaStream_t st) {
  if (px.stw) {
    switch (px.n) {
#define SPB_CASE(n) \
  case n: return row_launch_n<MODE, n>(px, a, st);
      SPB_CT_LENGTHS(SPB_CASE)
#undef SPB_CASE
    }
    if constexpr (MODE == ROW_DM_ITER || MODE == ROW_DM_F1_FWD) {
      switch (px.n) {
#define SPB_CASE(n) \
  case n: return row_launch_n<MODE, n>(px, a, st);
        SPB_CT_LENGTHS_DM(SPB_CASE)
#undef SPB_CASE
      }
    }
  }
  return row_launch_n<MODE, 0>(px, a, st);
}

// The 8-point kernels for a pass of `nlines` lines of length n: asked for
// (knob 2), or chosen when the 16-point kernels' n/16 threads per line would
// give the SMs fewer than 8 warps (256 threads) each.  Measured on one B200,
// iterations per second of one pattern, 16 -> 8 points per thread: 256x256
// 80.1k -> 96.9k (0.9 warps per SM with 16 points), 512x512 69.4k -> 72.3k
// (3.5), 1024x1024 47.8k -> 44.3k (13.8: the extra selects and shuffles
// outweigh the added warps once the passes are near issue-bound).
static bool want_split(const PassArgs &a, int n, long long nlines) {
  if (a.split == 1) return false;
  if (a.split == 2) return true;
  static int nsm = 0;
  if (!nsm && cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, 0) != cudaSuccess) nsm = 148;
  return nlines * (n / 16) < 256LL * nsm;
}

cudaError_t launch_row(int mode, const LinePlan &px, const PassArgs &a, cudaStream_t st) {
  if (mode == ROW_ITER && px.n > 0 && want_split(a, px.n, a.n / px.n)) {
    const cudaError_t se = launch_row_split(mode, px, a, st);
    if (se != cudaErrorNotSupported) return se;
  }
  const cudaError_t fe = launch_row_fast(mode, px, a, st);
  if (fe != cudaErrorNotSupported) return fe;
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

// Columns per block SPB_TUNE_COL_WIDTH may ask of the general projection pass
// for the compile-time-plan lengths: a power of two up to 16 that keeps one
// butterfly per thread within 1024 threads.
bool general_col_width_ok(int n, int w) {
  if (w < 1 || w > 16 || (w & (w - 1))) return false;
  switch (n) {
#define SPB_CASE(len) \
  case len: return w * ct_max_butterflies(len) <= 1024;
    SPB_CT_LENGTHS(SPB_CASE)
#undef SPB_CASE
  }
  return false;
}

template <int MODE, int NC>
static cudaError_t col_launch_n(const LinePlan &pl, const PassArgs &a, cudaStream_t st) {
  const int n = pl.n;
  constexpr bool PROJ = (MODE == COL_PROJECT || MODE == COL_PROJECT_NOFC);
  int ct = 4096 / (n > 0 ? n : 1);
  if (ct > 16) ct = 16;
  if (ct < 1) ct = 1;
  int tpc = NC > 0 ? ct_max_butterflies(NC) : pow2_at_least((n + 15) / 16);
  if (NC > 0 && tpc * ct > 1024) ct = 1024 / tpc > 0 ? 1024 / tpc : 1;  // keep one butterfly per thread
  // projection with a compile-time plan: four columns per block (a full
  // 32-byte sector per row, and more blocks than the wider default gives a
  // single pattern).  Measured on one B200, HIO per slot at 16/8/4/2/1 columns:
  // 192^2 13.6/12.2/11.6/11.9/12.6 us, 384^2 -/16.4/14.9/15.9/17.8 us, 1000^2
  // (four by default) 39.2, 49.2 at 2, 57.7 at 1.  A launch-shape knob may
  // ask for another number of columns per block.
  if (NC > 0 && PROJ) {
    if (ct > 4) ct = 4;
    if (a.col_width > 0 && general_col_width_ok(NC, a.col_width)) ct = a.col_width;
  }
  if (tpc * ct > 1024) tpc = 1024 / ct;
  if (tpc * ct < 32) tpc = 32 / ct;
  // two transform buffers, then (projection) n*ct amplitudes and n*ct flag
  // bytes, then (compile-time plans) the n - 1 entries of the stage table
  const size_t smem = NC > 0 ? col_tw_offset(n, ct, PROJ) + (size_t)(NC - 1) * sizeof(float2)
                             : (size_t)2 * n * ct * sizeof(float2) + (PROJ ? (size_t)n * ct * (sizeof(float) + 1) : 0);
  auto k = col_pass_kernel<MODE, NC>;
  if constexpr (NC == 1000) k = col_pass_kernel_1000<MODE>;
  static size_t done = 0;
  cudaError_t e = smem_attr(k, smem, done);
  if (e != cudaSuccess) return e;
  dim3 grid((a.ncols + ct - 1) / ct, a.nouter);
  k<<<grid, ct * tpc, smem, st>>>(pl, a, ct, tpc);
  return cudaGetLastError();
}

template <int MODE>
static cudaError_t col_launch(const LinePlan &pl, const PassArgs &a, cudaStream_t st) {
  if (pl.stw) {
    switch (pl.n) {
#define SPB_CASE(n) \
  case n: return col_launch_n<MODE, n>(pl, a, st);
      SPB_CT_LENGTHS(SPB_CASE)
#undef SPB_CASE
    }
  }
  return col_launch_n<MODE, 0>(pl, a, st);
}

cudaError_t launch_col(int mode, const LinePlan &pl, int line_len, const PassArgs &a, cudaStream_t st) {
  if ((mode == COL_PROJECT || mode == COL_PROJECT_NOFC) && pl.n > 0 &&
      want_split(a, pl.n, (long long)a.ncols * a.nouter)) {
    const cudaError_t se = launch_col_split(mode, pl, a, st);
    if (se != cudaErrorNotSupported) return se;
  }
  (void)line_len;
  const cudaError_t fe = launch_col_fast(mode, pl, a, st);
  if (fe != cudaErrorNotSupported) return fe;
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

// --------------------------------------------------------- blur factor table
// The Gaussian factor of every distance triple (dx, dy, dz) from the zero
// frequency, dx in [0, nx/2] etc.: the blur's column pass looks the factor
// up instead of evaluating it per pixel, and every start of a batch shares
// the table.  Same function, same floats.
__global__ void gauss_table_kernel(PassArgs a, float *__restrict__ tab) {
  pdl_wait();
  pdl_release();  // the table is read by the blur pass, which waits for this grid
  const int hx = a.nx / 2 + 1, hy = a.ny / 2 + 1;
  const long long total = (long long)hx * hy * (a.nz / 2 + 1);
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int dx = (int)(t % hx), dy = (int)((t / hx) % hy), dz = (int)(t / ((long long)hx * hy));
    tab[t] = gauss_factor((float)dx, (float)dy, (float)dz, a);
  }
}

cudaError_t launch_gauss_table(const PassArgs &a, float *tab, cudaStream_t st) {
  const long long total = (long long)(a.nx / 2 + 1) * (a.ny / 2 + 1) * (a.nz / 2 + 1);
  long long blocks = (total + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  return launch_maybe_pdl(gauss_table_kernel, dim3((unsigned)blocks), dim3(256), 0, st, a.pdl != 0, a, tab);
}

// ------------------------------------------------- support selection kernels
// Exact k-th largest value per start by most-significant-digit radix select
// over the float bit patterns (non-negative floats order like their bits):
// four passes of 8 bits, each a histogram of the keys that match the digits
// fixed so far.  Histograms are kept per warp in shared memory and lanes
// holding the same digit are combined with a match before the atomic,
// because the leading digits of |blur| concentrate in a few bins.  Start b
// owns v[b*n .. (b+1)*n) and state s[b]; the grid's y dimension runs over
// starts.  The digit a pass picks is found at the start of the next pass
// (and of the mask kernel, after the last) by warp 0 of every block from the
// previous pass's histogram, so the selection takes one launch per pass.
#define SEL_BITS 8
#define SEL_BINS 256
// Each thread loads SEL_UNROLL keys (independent loads in flight) before it
// bins them; a warp skips the match when none of its keys carries the prefix.
#define SEL_UNROLL 8
// VEC forms (batches, where each thread streams many keys): four keys a
// 16-byte load, SEL_UNROLL4 loads in flight per thread
#define SEL_UNROLL4 4

// Warp 0 of a block: the digit of histogram `hist` (digits at `shift` of the
// keys matching prefix/mask) that holds the rank-th largest of those keys,
// and the narrowed prefix, mask and rank.  Lane l owns digits [8l, 8l+8);
// the keys with a larger digit are counted from the higher lanes.  Results in
// out[0..1] (prefix, mask) and *orank, shared by the block.
__device__ void select_pick_warp(const unsigned int *hist, unsigned long long rank, unsigned int prefix,
                                 unsigned int mask, int shift, unsigned int *out, unsigned long long *orank) {
  const int lane = threadIdx.x & 31;
  unsigned long long own = 0;
  unsigned int c[8];
#pragma unroll
  for (int j = 0; j < 8; j++) {
    c[j] = hist[lane * 8 + j];
    own += c[j];
  }
  // keys with a larger digit than lane's: the suffix sum over the higher lanes
  unsigned long long suf = own;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long x = __shfl_down_sync(0xffffffffu, suf, o);
    if (lane + o < 32) suf += x;
  }
  const unsigned long long above = suf - own;
  if (lane == 0) {  // unchanged unless a lane finds the digit (it always does: rank < the count)
    out[0] = prefix;
    out[1] = mask;
    *orank = rank;
  }
  __syncwarp();
  unsigned long long cum = above;
#pragma unroll
  for (int j = 7; j >= 0; j--) {
    if (cum <= rank && cum + c[j] > rank) {
      out[0] = prefix | ((unsigned int)(lane * 8 + j) << shift);
      out[1] = mask | ((unsigned int)(SEL_BINS - 1) << shift);
      *orank = rank - cum;
    }
    cum += c[j];
  }
}

template <bool VEC>
__global__ void __launch_bounds__(256) select_hist_kernel(const float *__restrict__ v, long long n, SelectState *s,
                                                          int pass) {
  __shared__ unsigned int h[8][SEL_BINS];
  __shared__ unsigned int pm[2];
  __shared__ unsigned long long pr;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int b = blockIdx.y;
  v += (long long)b * n;
  s += b;
  for (int i = threadIdx.x; i < 8 * SEL_BINS; i += blockDim.x) (&h[0][0])[i] = 0;
  pdl_wait();
  if (pass == 0) {
    if (threadIdx.x == 0) {
      pm[0] = s->pass_prefix[0];
      pm[1] = s->pass_mask[0];
    }
  } else if (warp == 0) {
    // the digit the previous pass picks: narrows the prefix for this pass
    const int q = pass - 1;
    select_pick_warp(s->hist[q], s->pass_rank[q], s->pass_prefix[q], s->pass_mask[q], 24 - SEL_BITS * q, pm, &pr);
    __syncwarp();
    if (lane == 0 && blockIdx.x == 0) {
      s->pass_prefix[pass] = pm[0];
      s->pass_mask[pass] = pm[1];
      s->pass_rank[pass] = pr;
    }
  }
  __syncthreads();
  const int shift = 24 - SEL_BITS * pass;
  const unsigned int prefix = pm[0], pmask = pm[1];
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long start = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if constexpr (VEC) {
    // a warp's keys binned with one atomic per distinct digit; every lane
    // reaches each call (the loops are uniform over the block)
    auto bin = [&](unsigned int key, bool in) {
      const int digit = (in && (key & pmask) == prefix) ? (int)((key >> shift) & (SEL_BINS - 1)) : -1;
      if (__ballot_sync(0xffffffffu, digit >= 0) == 0u) return;  // warp-uniform
      const unsigned int peers = __match_any_sync(0xffffffffu, digit);
      if (digit >= 0 && lane == __ffs(peers) - 1) atomicAdd(&h[warp][digit], (unsigned)__popc(peers));
    };
    const float4 *v4 = reinterpret_cast<const float4 *>(v);
    const long long n4 = n >> 2;
    const long long rounds4 = (n4 + stride * SEL_UNROLL4 - 1) / (stride * SEL_UNROLL4);
    for (long long r = 0; r < rounds4; r++) {
      float4 q[SEL_UNROLL4];
      bool in[SEL_UNROLL4];
#pragma unroll
      for (int u = 0; u < SEL_UNROLL4; u++) {
        const long long i = start + (r * SEL_UNROLL4 + u) * stride;
        in[u] = i < n4;
        q[u] = in[u] ? v4[i] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      }
#pragma unroll
      for (int u = 0; u < SEL_UNROLL4; u++) {
        bin(__float_as_uint(q[u].x), in[u]);
        bin(__float_as_uint(q[u].y), in[u]);
        bin(__float_as_uint(q[u].z), in[u]);
        bin(__float_as_uint(q[u].w), in[u]);
      }
    }
  }
  const long long rounds = VEC ? 0 : (n + stride * SEL_UNROLL - 1) / (stride * SEL_UNROLL);
  for (long long r = 0; r < rounds; r++) {
    unsigned int key[SEL_UNROLL];
    bool in[SEL_UNROLL];
#pragma unroll
    for (int u = 0; u < SEL_UNROLL; u++) {
      const long long i = start + (r * SEL_UNROLL + u) * stride;
      in[u] = i < n;
      key[u] = in[u] ? __float_as_uint(v[i]) : 0u;
    }
#pragma unroll
    for (int u = 0; u < SEL_UNROLL; u++) {
      const int digit = (in[u] && (key[u] & pmask) == prefix) ? (int)((key[u] >> shift) & (SEL_BINS - 1)) : -1;
      if (__ballot_sync(0xffffffffu, digit >= 0) == 0u) continue;  // warp-uniform
      const unsigned int peers = __match_any_sync(0xffffffffu, digit);
      if (digit >= 0 && lane == __ffs(peers) - 1) atomicAdd(&h[warp][digit], (unsigned)__popc(peers));
    }
  }
  __syncthreads();
  pdl_release();
  for (int d = threadIdx.x; d < SEL_BINS; d += blockDim.x) {
    unsigned int c = 0;
    for (int w = 0; w < 8; w++) c += h[w][d];
    if (c) atomicAdd(&s->hist[pass][d], c);
  }
}

__global__ void select_init_kernel(SelectState *states, unsigned long long rank, const unsigned long long *rank_dev) {
  pdl_wait();
  pdl_release();
  SelectState *s = states + blockIdx.x;
  for (int d = threadIdx.x; d < 4 * SEL_BINS; d += blockDim.x) (&s->hist[0][0])[d] = 0;
  if (threadIdx.x == 0) {
    s->rank = rank_dev ? *rank_dev : rank;
    s->pass_prefix[0] = 0;
    s->pass_mask[0] = 0;
    s->pass_rank[0] = s->rank;
    s->maxbits = 0;
  }
}

// The VEC forms of the histogram and mask launches: where every start's keys
// (and flags) start on 16-byte (4-byte) boundaries and each thread streams at
// least 32 keys a pass (batches).  Measured: the 512-start batch of 512^2
// 1456 -> 1440 and 1532 -> 1518 us per slot on two boxes; latency-bound
// single patterns keep the scalar forms (seven keys a thread at 1024^2).
static bool select_vec(const float *v, const uint8_t *flags, long long n, unsigned blocks) {
  return (n & 3) == 0 && ((uintptr_t)v & 15) == 0 && ((uintptr_t)flags & 3) == 0 && n >= 32LL * blocks * 256;
}

static unsigned blocks_per_start(long long n, int nb) {
  long long b = (n + 255) / 256;
  long long cap = 148 * 4 / nb;
  if (cap < 2) cap = 2;
  if (b > cap) b = cap;
  return (unsigned)(b > 0 ? b : 1);
}

// the four histogram passes; the last pick happens in the mask kernel
cudaError_t launch_select_kth_desc(const float *absv, long long n, int nb, long long k, SelectState *state,
                                   cudaStream_t st, const unsigned long long *k_dev, bool pdl) {
  cudaError_t e = launch_maybe_pdl(select_init_kernel, dim3(nb), dim3(256), 0, st, pdl, state, (unsigned long long)k, k_dev);
  const dim3 grid(blocks_per_start(n, nb), nb);
  const bool vec = select_vec(absv, nullptr, n, grid.x);
  for (int p = 0; p < 4 && e == cudaSuccess; p++)
    e = vec ? launch_maybe_pdl(select_hist_kernel<true>, grid, dim3(256), 0, st, pdl, absv, n, state, p)
            : launch_maybe_pdl(select_hist_kernel<false>, grid, dim3(256), 0, st, pdl, absv, n, state, p);
  return e;
}

__global__ void max_abs_kernel(const float *__restrict__ v, long long n, SelectState *states) {
  pdl_wait();
  pdl_release();
  SelectState *s = states + blockIdx.y;
  v += (long long)blockIdx.y * n;
  unsigned int m = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float x = v[i];
    if (!isnan(x)) m = max(m, __float_as_uint(x));
  }
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(&s->maxbits, m);
}

__global__ void max_finish_kernel(SelectState *states) {
  pdl_wait();
  pdl_release();
  SelectState *s = states + blockIdx.x;
  s->result = __uint_as_float(s->maxbits);
}

cudaError_t launch_max_abs(const float *absv, long long n, int nb, SelectState *state, cudaStream_t st, bool pdl) {
  cudaError_t e = launch_maybe_pdl(select_init_kernel, dim3(nb), dim3(256), 0, st, pdl, state, 0ULL,
                                   (const unsigned long long *)nullptr);
  if (e == cudaSuccess)
    e = launch_maybe_pdl(max_abs_kernel, dim3(blocks_per_start(n, nb), nb), dim3(256), 0, st, pdl, absv, n, state);
  if (e == cudaSuccess) e = launch_maybe_pdl(max_finish_kernel, dim3(nb), dim3(1), 0, st, pdl, state);
  return e;
}

// support_from_absolute_threshold (src/support_update.c:392-400): strict '>'.
// Threshold: the maximum times rel (use_rel), or the key the radix select's
// last pass picks (found here by warp 0 of every block; block 0 records it).
template <bool VEC>
__global__ void mask_kernel(const float *__restrict__ v, SelectState *states, float rel, int use_rel,
                            uint8_t *flags, long long n, const float *rel_dev) {
  __shared__ unsigned int pm[2];
  __shared__ unsigned long long pr;
  const int b = blockIdx.y;
  SelectState *s = states + b;
  pdl_wait();
  float t;
  if (use_rel) {
    t = __fmul_rn(s->result, rel_dev ? *rel_dev : rel);
  } else {
    if (threadIdx.x < 32) {
      select_pick_warp(s->hist[3], s->pass_rank[3], s->pass_prefix[3], s->pass_mask[3], 0, pm, &pr);
      __syncwarp();
      if (threadIdx.x == 0 && blockIdx.x == 0) s->result = __uint_as_float(pm[0]);
    }
    __syncthreads();
    t = __uint_as_float(pm[0]);
  }
  pdl_release();
  v += (long long)b * n;
  flags += (long long)b * n;
  const long long stride = (long long)gridDim.x * blockDim.x;
  if constexpr (VEC) {
    // four consecutive pixels a thread: one 16-byte load of |blur|, one 4-byte
    // load and store of their flags
    const float4 *v4 = reinterpret_cast<const float4 *>(v);
    uchar4 *f4 = reinterpret_cast<uchar4 *>(flags);
    const long long n4 = n >> 2;
    for (long long i0 = (long long)blockIdx.x * blockDim.x + threadIdx.x; i0 < n4; i0 += 2 * stride) {
      float4 x[2];
      uchar4 f[2];
#pragma unroll
      for (int u = 0; u < 2; u++) {
        const long long i = i0 + u * stride;
        if (i < n4) {
          x[u] = v4[i];
          f[u] = f4[i];
        }
      }
#pragma unroll
      for (int u = 0; u < 2; u++) {
        const long long i = i0 + u * stride;
        if (i < n4) {
          const uint8_t in = FLAG_INSIDE, out = (uint8_t)~FLAG_INSIDE;
          f4[i] = make_uchar4(x[u].x > t ? (uint8_t)(f[u].x | in) : (uint8_t)(f[u].x & out),
                              x[u].y > t ? (uint8_t)(f[u].y | in) : (uint8_t)(f[u].y & out),
                              x[u].z > t ? (uint8_t)(f[u].z | in) : (uint8_t)(f[u].z & out),
                              x[u].w > t ? (uint8_t)(f[u].w | in) : (uint8_t)(f[u].w & out));
        }
      }
    }
    return;
  }
  // four elements per thread and round, their loads in flight together
  for (long long i0 = (long long)blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += 4 * stride) {
    float x[4];
    uint8_t f[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const long long i = i0 + u * stride;
      x[u] = i < n ? v[i] : 0.0f;
      f[u] = i < n ? flags[i] : (uint8_t)0;
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const long long i = i0 + u * stride;
      if (i < n) flags[i] = (x[u] > t) ? (uint8_t)(f[u] | FLAG_INSIDE) : (uint8_t)(f[u] & ~FLAG_INSIDE);
    }
  }
}

cudaError_t launch_mask_from_abs(const float *absv, SelectState *state, float rel, int use_rel, uint8_t *flags,
                                 long long n, int nb, cudaStream_t st, const float *rel_dev, bool pdl) {
  const dim3 grid(blocks_per_start(n, nb), nb);
  if (select_vec(absv, flags, n, grid.x))
    return launch_maybe_pdl(mask_kernel<true>, grid, dim3(256), 0, st, pdl, absv, state, rel, use_rel, flags, n,
                            rel_dev);
  return launch_maybe_pdl(mask_kernel<false>, grid, dim3(256), 0, st, pdl, absv, state, rel, use_rel, flags, n,
                          rel_dev);
}

// ------------------------------------- one-launch selection over a cluster
// The support selection and mask of a start whose |blur| fits in the shared
// memory of one thread-block cluster: the SEL_CLUSTER blocks of the cluster
// each load a contiguous slice of the start's keys once, then
//   area rule: four radix passes, each a histogram of the block's slice that
//   the cluster's blocks read from one another's shared memory (distributed
//   shared memory) after a cluster barrier; every block sums them in the same
//   order and picks the same digit (select_pick_warp, as the launch-per-pass
//   path), so all blocks hold the same k-th largest key after the fourth;
//   threshold rule: each block's maximum (NaN skipped, as max_abs_kernel),
//   exchanged the same way, times rel;
// and each block writes the inside bit of its slice (strict '>', as
// mask_kernel).  The same key is found as by the launch-per-pass path (the
// k-th largest key is one value), so the same flags.  One launch replaces
// six (area) or four (threshold), and the keys are read from memory once
// instead of five times.  Every block runs the same cluster barriers
// (no early exit); the last keeps each block's shared memory alive until no
// block reads it any more.  The grid's y dimension runs over starts.
#define SEL_CLUSTER 8
#define SEL_CLUSTER_THREADS 1024
#define SEL_CLUSTER_MAX_SLICE 40960  // keys per block: 160 KiB of shared memory

namespace cg = cooperative_groups;

static size_t sel_cluster_smem(long long slice) {
  return sizeof(unsigned int) * ((size_t)slice + 8 * SEL_BINS + 2 * SEL_BINS + SEL_BINS);
}

__global__ void __launch_bounds__(SEL_CLUSTER_THREADS) select_mask_cluster_kernel(
    const float *__restrict__ v, long long n, long long slice, SelectState *states, uint8_t *flags, int use_rel,
    float rel, const float *rel_dev, unsigned long long rank, const unsigned long long *rank_dev) {
  extern __shared__ unsigned int sel_smem[];
  unsigned int *keys = sel_smem;                       // [slice]
  unsigned int *sub = keys + slice;                    // [8][SEL_BINS] partial histograms
  unsigned int *hout = sub + 8 * SEL_BINS;             // [2][SEL_BINS] the block's histogram, read by the cluster
  unsigned int *hsum = hout + 2 * SEL_BINS;            // [SEL_BINS] the cluster's histogram
  __shared__ unsigned int pm[2];
  __shared__ unsigned long long pr;
  cg::cluster_group cluster = cg::this_cluster();
  const unsigned int crank = cluster.block_rank();
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int b = blockIdx.y;
  SelectState *s = states + b;
  const long long i0 = (long long)crank * slice;
  const long long cnt = i0 >= n ? 0 : (n - i0 < slice ? n - i0 : slice);
  v += (long long)b * n + i0;
  flags += (long long)b * n + i0;

  pdl_wait();
  pdl_release();
  for (long long i = tid; i < cnt; i += SEL_CLUSTER_THREADS) keys[i] = __float_as_uint(v[i]);
  const long long rounds = (cnt + SEL_CLUSTER_THREADS - 1) / SEL_CLUSTER_THREADS;

  float t;
  if (use_rel) {
    unsigned int m = 0;
    __syncthreads();
    for (long long i = tid; i < cnt; i += SEL_CLUSTER_THREADS)
      if (!isnan(__uint_as_float(keys[i]))) m = max(m, keys[i]);
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (tid == 0) hout[0] = 0;
    __syncthreads();
    if (lane == 0) atomicMax(&hout[0], m);
    cluster.sync();  // every block's maximum is in its hout[0]
    if (tid == 0) {
      unsigned int mx = 0;
      for (unsigned int r = 0; r < SEL_CLUSTER; r++) mx = max(mx, *cluster.map_shared_rank(&hout[0], r));
      pm[0] = mx;
      if (crank == 0) s->result = __uint_as_float(mx);
    }
    __syncthreads();
    t = __fmul_rn(__uint_as_float(pm[0]), rel_dev ? *rel_dev : rel);
  } else {
    if (tid == 0) {
      pm[0] = 0;  // prefix
      pm[1] = 0;  // mask
      pr = rank_dev ? *rank_dev : rank;
    }
    for (int pass = 0; pass < 4; pass++) {
      for (int i = tid; i < 8 * SEL_BINS; i += SEL_CLUSTER_THREADS) sub[i] = 0;
      __syncthreads();  // keys loaded, partial histograms clear, prefix of this pass set
      const int shift = 24 - SEL_BITS * pass;
      const unsigned int prefix = pm[0], pmask = pm[1];
      unsigned int *h = sub + (warp & 7) * SEL_BINS;
      for (long long r = 0; r < rounds; r++) {
        const long long i = r * SEL_CLUSTER_THREADS + tid;
        const unsigned int key = i < cnt ? keys[i] : 0u;
        const int digit = (i < cnt && (key & pmask) == prefix) ? (int)((key >> shift) & (SEL_BINS - 1)) : -1;
        if (__ballot_sync(0xffffffffu, digit >= 0) == 0u) continue;  // warp-uniform
        const unsigned int peers = __match_any_sync(0xffffffffu, digit);
        if (digit >= 0 && lane == __ffs(peers) - 1) atomicAdd(&h[digit], (unsigned)__popc(peers));
      }
      __syncthreads();
      unsigned int *ho = hout + (pass & 1) * SEL_BINS;
      for (int d = tid; d < SEL_BINS; d += SEL_CLUSTER_THREADS) {
        unsigned int c = 0;
        for (int w = 0; w < 8; w++) c += sub[w * SEL_BINS + d];
        ho[d] = c;
      }
      // hout[pass & 1] of every block is complete; the buffer of the pass
      // before was last read before this barrier, so the next pass may reuse it
      cluster.sync();
      for (int d = tid; d < SEL_BINS; d += SEL_CLUSTER_THREADS) {
        unsigned int c[SEL_CLUSTER];
#pragma unroll
        for (unsigned int r = 0; r < SEL_CLUSTER; r++) c[r] = *cluster.map_shared_rank(&ho[d], r);  // all in flight
        unsigned int t = 0;
#pragma unroll
        for (unsigned int r = 0; r < SEL_CLUSTER; r++) t += c[r];
        hsum[d] = t;
      }
      __syncthreads();
      // the narrowed prefix, mask and rank for the next pass (its arguments are
      // copies, so it may write them in place; the other warps read them after
      // the barrier)
      if (warp == 0) select_pick_warp(hsum, pr, prefix, pmask, shift, pm, &pr);
      __syncthreads();
    }
    t = __uint_as_float(pm[0]);
    if (tid == 0 && crank == 0) s->result = t;
  }
  for (long long i = tid; i < cnt; i += SEL_CLUSTER_THREADS) {
    const uint8_t f = flags[i];
    flags[i] = (__uint_as_float(keys[i]) > t) ? (uint8_t)(f | FLAG_INSIDE) : (uint8_t)(f & ~FLAG_INSIDE);
  }
  cluster.sync();  // no block exits while another may still read its histograms
}

bool select_cluster_fits(long long n) { return n > 0 && (n + SEL_CLUSTER - 1) / SEL_CLUSTER <= SEL_CLUSTER_MAX_SLICE; }

cudaError_t launch_select_mask_cluster(const float *absv, long long n, int nb, int use_rel, unsigned long long rank,
                                       const unsigned long long *rank_dev, float rel, const float *rel_dev,
                                       SelectState *state, uint8_t *flags, cudaStream_t st, bool pdl) {
  if (!select_cluster_fits(n) || nb < 1 || nb > 65535) return cudaErrorNotSupported;
  static bool attr_set[64] = {};  // per device
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorNotSupported;
  const long long slice = (n + SEL_CLUSTER - 1) / SEL_CLUSTER;
  const size_t smem = sel_cluster_smem(slice);
  if (!attr_set[dev]) {
    e = cudaFuncSetAttribute(select_mask_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sel_cluster_smem(SEL_CLUSTER_MAX_SLICE));
    if (e != cudaSuccess) return e;
    attr_set[dev] = true;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(SEL_CLUSTER, nb);
  cfg.blockDim = dim3(SEL_CLUSTER_THREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[2];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = SEL_CLUSTER;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl ? 2 : 1;
  return cudaLaunchKernelEx(&cfg, select_mask_cluster_kernel, absv, n, slice, state, flags, use_rel, rel, rel_dev,
                            rank, rank_dev);
}

// ---------------------------------------------------------------- reductions
// Per start b: partial sums of blocks_per_start blocks into part[b][blk][4],
// then one block per start adds them in a fixed order (deterministic).
static __device__ void block_sum4(double s[4], double *out) {
  __shared__ double sh[4][256];
  for (int k = 0; k < 4; k++) sh[k][threadIdx.x] = s[k];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      for (int k = 0; k < 4; k++) sh[k][threadIdx.x] += sh[k][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 4; k++) out[k] = sh[k][0];
}

// efourier terms (src/phasing.c:852-891): nom, den, FcFo numerator, denominator
__global__ void efourier_partial_kernel(const float2 *__restrict__ F, const float *__restrict__ amp,
                                        const uint8_t *__restrict__ flags, long long n, double *part) {
  const int b = blockIdx.y;
  F += (long long)b * n;
  flags += (long long)b * n;
  double s[4] = {0, 0, 0, 0};
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float fa = cabs_ref(F[i]);
    if (flags[i] & FLAG_MEASURED) {
      const float aa = cabs_ref(make_float2(amp[i], 0.0f));
      const double d = (double)__fsub_rn(fa, aa);
      s[0] += d * d;
      s[1] += (double)aa * (double)aa;
      s[2] += aa;
      s[3] += fa;
    } else {
      s[1] += (double)fa * (double)fa;
    }
  }
  block_sum4(s, part + ((size_t)b * gridDim.x + blockIdx.x) * 4);
}

__global__ void ereal_partial_kernel(const float2 *__restrict__ gp, const uint8_t *__restrict__ flags, long long n,
                                     double *part) {
  const int b = blockIdx.y;
  gp += (long long)b * n;
  flags += (long long)b * n;
  double s[4] = {0, 0, 0, 0};
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double a = (double)cabs_ref(gp[i]);
    if (!(flags[i] & FLAG_INSIDE)) s[0] += a * a;
    s[1] += a * a;
  }
  block_sum4(s, part + ((size_t)b * gridDim.x + blockIdx.x) * 4);
}

__global__ void count_inside_partial_kernel(const uint8_t *__restrict__ flags, long long n, double *part) {
  const int b = blockIdx.y;
  flags += (long long)b * n;
  double s[4] = {0, 0, 0, 0};
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    s[0] += (flags[i] & FLAG_INSIDE) ? 1.0 : 0.0;
  block_sum4(s, part + ((size_t)b * gridDim.x + blockIdx.x) * 4);
}

__global__ void finish4_kernel(const double *part, int nparts, double *out) {
  const int b = blockIdx.x;
  double s[4] = {0, 0, 0, 0};
  for (int i = threadIdx.x; i < nparts; i += blockDim.x)
    for (int k = 0; k < 4; k++) s[k] += part[((size_t)b * nparts + i) * 4 + k];
  block_sum4(s, out + (size_t)b * 4);
}

int reduce_scratch_doubles(int nb) { return nb * 4 + nb * 4 * (int)blocks_per_start(1LL << 40, nb); }

cudaError_t launch_reduce_efourier(const float2 *F, const float *amp, const uint8_t *flags, long long n, int nb,
                                   double *out, cudaStream_t st) {
  const unsigned bl = blocks_per_start(1LL << 40, nb);
  double *part = out + (size_t)nb * 4;
  efourier_partial_kernel<<<dim3(bl, nb), 256, 0, st>>>(F, amp, flags, n, part);
  finish4_kernel<<<nb, 256, 0, st>>>(part, bl, out);
  return cudaGetLastError();
}

cudaError_t launch_reduce_ereal(const float2 *gp, const uint8_t *flags, long long n, int nb, double *out,
                                cudaStream_t st) {
  const unsigned bl = blocks_per_start(1LL << 40, nb);
  double *part = out + (size_t)nb * 4;
  ereal_partial_kernel<<<dim3(bl, nb), 256, 0, st>>>(gp, flags, n, part);
  finish4_kernel<<<nb, 256, 0, st>>>(part, bl, out);
  return cudaGetLastError();
}

cudaError_t launch_count_inside(const uint8_t *flags, long long n, int nb, double *out, cudaStream_t st) {
  const unsigned bl = blocks_per_start(1LL << 40, nb);
  double *part = out + (size_t)nb * 4;
  count_inside_partial_kernel<<<dim3(bl, nb), 256, 0, st>>>(flags, n, part);
  finish4_kernel<<<nb, 256, 0, st>>>(part, bl, out);
  return cudaGetLastError();
}

__global__ void scale_cmul_kernel(float2 *a, long long n, float v) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    a[i] = scale_cmul_dev(a[i], v);
}
cudaError_t launch_scale_cmul(float2 *a, long long n, float v, cudaStream_t st) {
  scale_cmul_kernel<<<592, 256, 0, st>>>(a, n, v);
  return cudaGetLastError();
}

}  // namespace spb
