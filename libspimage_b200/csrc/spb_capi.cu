// C-ABI device layer of the phasing path (include/spimage/spb_device.h).
//
// A context owns the device buffers of one phasing problem:
//   amp[N] f32, flags[N] u8 (bit0 inside support, bit1 measured),
//   g[2][N] c64 ping-pong iterates (g1 = model, g0 = old model),
//   X[N] c64 = row FFT of g1 (kept valid between iterations),
//   Y[N] c64 scratch of the column passes, gp[N] c64 (last model before
//   projection), T[N] c64 and absb[N] f32 scratch of the support update,
//   Xf/Yf[N] c64 for the difference map's second transform pair.
// All work is enqueued on one non-blocking stream per context.
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "spb_internal.h"
#include "spimage/spb_device.h"

using namespace spb;

static thread_local char g_err[512];

static int fail(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return -1;
}

#define CK(call)                                                                      \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess) return fail("%s: %s", #call, cudaGetErrorString(e_));      \
  } while (0)

extern "C" const char *spb_error_string(void) { return g_err; }

extern "C" int spb_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n;
}

namespace {

// Canonical radix sequence: 16s first, then one 8/4/2 (a trailing 2 after a
// 16 becomes 8*4), then 3s, 5s, then the remaining primes ascending.
int radix_plan(int n, int *radix) {
  int k = 0, m = n, n16 = 0;
  if (n <= 1) return 0;
  while (m % 16 == 0) { radix[k++] = 16; m /= 16; n16++; }
  if (m % 8 == 0) { radix[k++] = 8; m /= 8; }
  else if (m % 4 == 0) { radix[k++] = 4; m /= 4; }
  else if (m % 2 == 0) {
    if (n16 > 0) { radix[k - 1] = 8; radix[k++] = 4; }
    else radix[k++] = 2;
    m /= 2;
  }
  while (m % 3 == 0) { radix[k++] = 3; m /= 3; }
  while (m % 5 == 0) { radix[k++] = 5; m /= 5; }
  for (int p = 7; p * p <= m; p += 2)
    while (m % p == 0) { radix[k++] = p; m /= p; }
  if (m > 1) radix[k++] = m;
  return k;
}

struct Axis {
  LinePlan lp{};
  float2 *tw = nullptr;
};

int make_axis(Axis &ax, int n) {
  int radix[64];
  const int ns = radix_plan(n, radix);
  if (ns > SPB_MAX_STAGES) return fail("axis length %d has too many radix stages", n);
  ax.lp.n = n;
  ax.lp.nstages = ns;
  for (int s = 0; s < ns; s++) ax.lp.radix[s] = radix[s];
  std::vector<float2> h((size_t)n);
  for (int i = 0; i < n; i++) {
    const double ang = (2.0 * 3.14159265358979323846 * (double)i) / (double)n;
    h[i] = make_float2((float)cos(ang), (float)(-sin(ang)));
  }
  CK(cudaMalloc(&ax.tw, sizeof(float2) * (size_t)n));
  CK(cudaMemcpy(ax.tw, h.data(), sizeof(float2) * (size_t)n, cudaMemcpyHostToDevice));
  ax.lp.tw = ax.tw;
  return 0;
}

// Largest line the staging buffers hold: two n-point complex lines per row in
// shared memory (row pass) or per column tile of two columns (column pass).
const int kMaxAxis = 8192;

}  // namespace

struct spb_ctx {
  int nx = 0, ny = 0, nz = 0;
  long long n = 0;
  cudaStream_t st = nullptr;
  Axis ax, ay, az;
  float *amp = nullptr, *amin = nullptr, *amax = nullptr;
  float2 *pamp = nullptr;
  uint8_t *flags = nullptr;
  float2 *g[2] = {nullptr, nullptr};
  int cur = 0;
  float2 *X = nullptr, *Y = nullptr, *Xf = nullptr, *Yf = nullptr, *gp = nullptr, *T = nullptr;
  float *absb = nullptr;
  SelectState *sel = nullptr;
  double *red = nullptr;
  unsigned long long *cnt = nullptr;
  int x_valid = 0, xf_valid = 0;
  float xf_gamma1 = 0.0f;
};

namespace {

PassArgs base_args(const spb_ctx *c) {
  PassArgs a;
  memset(&a, 0, sizeof(a));
  a.nx = c->nx;
  a.ny = c->ny;
  a.nz = c->nz;
  a.n = c->n;
  a.amp = c->amp;
  a.amp_min = c->amin;
  a.amp_max = c->amax;
  a.phased_amp = c->pamp;
  a.flags = c->flags;
  a.inv_n = (float)(1.0 / (double)c->n);
  a.nx_f = (float)c->nx;
  a.n_f = (float)c->n;
  return a;
}

// Column-line geometry: axis 1 = y lines (per z slab), 2 = z lines, 0 = lines
// of length 1 over every pixel (pointwise pass for 1-D problems).
void col_geometry(const spb_ctx *c, int axis, PassArgs &a, const LinePlan **pl) {
  if (axis == 1) {
    a.estride = c->nx;
    a.ostride = (long long)c->nx * c->ny;
    a.ncols = c->nx;
    a.nouter = c->nz;
    *pl = &c->ay.lp;
  } else if (axis == 2) {
    a.estride = (long long)c->nx * c->ny;
    a.ostride = 0;
    a.ncols = c->nx * c->ny;
    a.nouter = 1;
    *pl = &c->az.lp;
  } else {
    a.estride = 1;
    a.ostride = 0;
    a.ncols = (int)c->n;
    a.nouter = 1;
    *pl = nullptr;
  }
}

LinePlan unit_plan() {
  LinePlan p;
  memset(&p, 0, sizeof(p));
  p.n = 1;
  p.nstages = 0;
  return p;
}

int col(spb_ctx *c, int axis, int mode, const float2 *src, float2 *dst, PassArgs a) {
  const LinePlan *pl = nullptr;
  col_geometry(c, axis, a, &pl);
  a.src = src;
  a.dst = dst;
  LinePlan unit = unit_plan();
  CK(launch_col(mode, pl ? *pl : unit, pl ? pl->n : 1, a, c->st));
  return 0;
}

int row(spb_ctx *c, int mode, PassArgs a) {
  CK(launch_row(mode, c->ax.lp, a, c->st));
  return 0;
}

// Non-x axes in transform order (forward: y then z).
int other_axes(const spb_ctx *c, int *axes) {
  int k = 0;
  if (c->ny > 1) axes[k++] = 1;
  if (c->nz > 1) axes[k++] = 2;
  return k;
}

// dst = B(M(F(src))) over the non-x axes, M applied in the last axis pass
// (or pointwise if there is no other axis).  src may equal dst.
int middle(spb_ctx *c, int mid_mode, const float2 *src, float2 *dst, PassArgs a) {
  int axes[2];
  const int k = other_axes(c, axes);
  if (k == 0) return col(c, 0, mid_mode, src, dst, a);
  const float2 *s = src;
  for (int i = 0; i < k - 1; i++) {
    if (col(c, axes[i], COL_FWD, s, dst, a)) return -1;
    s = dst;
  }
  if (col(c, axes[k - 1], mid_mode, s, dst, a)) return -1;
  for (int i = k - 2; i >= 0; i--)
    if (col(c, axes[i], COL_INV, dst, dst, a)) return -1;
  return 0;
}

// dst = forward FFT of the x-transformed src over the remaining axes
int forward_rest(spb_ctx *c, const float2 *src, float2 *dst) {
  int axes[2];
  const int k = other_axes(c, axes);
  PassArgs a = base_args(c);
  if (k == 0) {
    if (src != dst) CK(cudaMemcpyAsync(dst, src, sizeof(float2) * c->n, cudaMemcpyDeviceToDevice, c->st));
    return 0;
  }
  const float2 *s = src;
  for (int i = 0; i < k; i++) {
    if (col(c, axes[i], COL_FWD, s, dst, a)) return -1;
    s = dst;
  }
  return 0;
}

// dst = backward FFT of src over the non-x axes (slowest first)
int backward_rest(spb_ctx *c, const float2 *src, float2 *dst) {
  int axes[2];
  const int k = other_axes(c, axes);
  PassArgs a = base_args(c);
  if (k == 0) {
    if (src != dst) CK(cudaMemcpyAsync(dst, src, sizeof(float2) * c->n, cudaMemcpyDeviceToDevice, c->st));
    return 0;
  }
  const float2 *s = src;
  for (int i = k - 1; i >= 0; i--) {
    if (col(c, axes[i], COL_INV, s, dst, a)) return -1;
    s = dst;
  }
  return 0;
}

int ensure_x(spb_ctx *c) {
  if (c->x_valid) return 0;
  PassArgs a = base_args(c);
  a.src = c->g[c->cur];
  a.dst = c->X;
  if (row(c, ROW_FWD, a)) return -1;
  c->x_valid = 1;
  return 0;
}

int ensure_xf(spb_ctx *c, float gamma1) {
  if (c->xf_valid && c->xf_gamma1 == gamma1) return 0;
  PassArgs a = base_args(c);
  a.src = c->g[c->cur];
  a.dst = c->Xf;
  a.gamma1 = gamma1;
  if (row(c, ROW_DM_F1_FWD, a)) return -1;
  c->xf_valid = 1;
  c->xf_gamma1 = gamma1;
  return 0;
}

int check_dims(int nx, int ny, int nz) {
  if (nx < 1 || ny < 1 || nz < 1) return fail("invalid dimensions %d x %d x %d", nx, ny, nz);
  if (nx > kMaxAxis || ny > kMaxAxis || nz > kMaxAxis)
    return fail("axis longer than %d is not supported (%d x %d x %d)", kMaxAxis, nx, ny, nz);
  return 0;
}

}  // namespace

extern "C" int spb_ctx_create(spb_ctx **out, int nx, int ny, int nz) {
  *out = nullptr;
  if (check_dims(nx, ny, nz)) return -1;
  spb_ctx *c = new spb_ctx();
  c->nx = nx;
  c->ny = ny;
  c->nz = nz;
  c->n = (long long)nx * ny * nz;
  const size_t nc = sizeof(float2) * (size_t)c->n, nf = sizeof(float) * (size_t)c->n;
  int rc = 0;
  auto alloc = [&](void **p, size_t bytes) {
    if (rc) return;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) rc = fail("cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
  };
  cudaError_t e = cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    return fail("cudaStreamCreate: %s", cudaGetErrorString(e));
  }
  alloc((void **)&c->amp, nf);
  alloc((void **)&c->flags, (size_t)c->n);
  alloc((void **)&c->g[0], nc);
  alloc((void **)&c->g[1], nc);
  alloc((void **)&c->X, nc);
  alloc((void **)&c->Y, nc);
  alloc((void **)&c->gp, nc);
  alloc((void **)&c->T, nc);
  alloc((void **)&c->absb, nf);
  alloc((void **)&c->sel, sizeof(SelectState));
  alloc((void **)&c->red, sizeof(double) * (4 + 4 * 592));
  alloc((void **)&c->cnt, sizeof(unsigned long long));
  if (!rc && make_axis(c->ax, nx)) rc = -1;
  if (!rc && make_axis(c->ay, ny)) rc = -1;
  if (!rc && make_axis(c->az, nz)) rc = -1;
  if (!rc) {
    cudaMemsetAsync(c->amp, 0, nf, c->st);
    cudaMemsetAsync(c->flags, 0, (size_t)c->n, c->st);
    cudaMemsetAsync(c->g[0], 0, nc, c->st);
    cudaMemsetAsync(c->g[1], 0, nc, c->st);
    cudaMemsetAsync(c->gp, 0, nc, c->st);
    e = cudaStreamSynchronize(c->st);
    if (e != cudaSuccess) rc = fail("context init: %s", cudaGetErrorString(e));
  }
  if (rc) {
    spb_ctx_destroy(c);
    return rc;
  }
  *out = c;
  return 0;
}

extern "C" void spb_ctx_destroy(spb_ctx *c) {
  if (!c) return;
  if (c->st) cudaStreamSynchronize(c->st);
  void *ptrs[] = {c->amp, c->amin, c->amax, c->pamp, c->flags, c->g[0], c->g[1], c->X, c->Y, c->Xf, c->Yf,
                  c->gp, c->T, c->absb, c->sel, c->red, c->cnt, c->ax.tw, c->ay.tw, c->az.tw};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
}

extern "C" int spb_ctx_synchronize(spb_ctx *c) {
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

static int upload(spb_ctx *c, void *dst, const void *src, size_t bytes) {
  CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

static int download(spb_ctx *c, void *dst, const void *src, size_t bytes) {
  CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

extern "C" int spb_ctx_set_amplitudes(spb_ctx *c, const float *amp) {
  return upload(c, c->amp, amp, sizeof(float) * (size_t)c->n);
}

extern "C" int spb_ctx_set_margins(spb_ctx *c, const float *amp_min, const float *amp_max) {
  const size_t nf = sizeof(float) * (size_t)c->n;
  if (!c->amin) CK(cudaMalloc(&c->amin, nf));
  if (!c->amax) CK(cudaMalloc(&c->amax, nf));
  if (upload(c, c->amin, amp_min, nf)) return -1;
  return upload(c, c->amax, amp_max, nf);
}

extern "C" int spb_ctx_set_phased_amplitudes(spb_ctx *c, const float *pa) {
  const size_t nc = sizeof(float2) * (size_t)c->n;
  if (!c->pamp) CK(cudaMalloc(&c->pamp, nc));
  return upload(c, c->pamp, pa, nc);
}

extern "C" int spb_ctx_set_flags(spb_ctx *c, const int *flags) {
  std::vector<uint8_t> h((size_t)c->n);
  for (long long i = 0; i < c->n; i++) h[i] = (uint8_t)(flags[i] & 3);
  if (upload(c, c->flags, h.data(), (size_t)c->n)) return -1;
  c->xf_valid = 0;
  return 0;
}

extern "C" int spb_ctx_get_flags(spb_ctx *c, int *flags) {
  std::vector<uint8_t> h((size_t)c->n);
  if (download(c, h.data(), c->flags, (size_t)c->n)) return -1;
  for (long long i = 0; i < c->n; i++) flags[i] = h[i];
  return 0;
}

static int reset_iterates(spb_ctx *c) {
  const size_t nc = sizeof(float2) * (size_t)c->n;
  CK(cudaMemsetAsync(c->g[c->cur ^ 1], 0, nc, c->st));
  CK(cudaMemsetAsync(c->gp, 0, nc, c->st));
  return 0;
}

extern "C" int spb_ctx_set_model(spb_ctx *c, const float *model, int reset_others) {
  if (upload(c, c->g[c->cur], model, sizeof(float2) * (size_t)c->n)) return -1;
  c->x_valid = c->xf_valid = 0;
  if (reset_others && reset_iterates(c)) return -1;
  return 0;
}

// g1 = backward FFT(T) * (1/N)
static int inverse_scaled_into_model(spb_ctx *c) {
  if (backward_rest(c, c->T, c->T)) return -1;
  PassArgs a = base_args(c);
  a.src = c->T;
  a.dst = c->g[c->cur];
  if (row(c, ROW_INV_SCALE, a)) return -1;
  c->x_valid = c->xf_valid = 0;
  return 0;
}

extern "C" int spb_ctx_model_from_fourier(spb_ctx *c, const float *fourier, int reset_others) {
  CK(cudaMemcpyAsync(c->T, fourier, sizeof(float2) * (size_t)c->n, cudaMemcpyHostToDevice, c->st));
  if (inverse_scaled_into_model(c)) return -1;
  if (reset_others && reset_iterates(c)) return -1;
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

namespace spb {
__global__ void zero_unmeasured_kernel(float2 *F, const uint8_t *flags, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    if (!(flags[i] & FLAG_MEASURED)) F[i] = make_float2(0.0f, 0.0f);
}
}  // namespace spb

extern "C" int spb_ctx_mask_out_unmeasured(spb_ctx *c) {
  PassArgs a = base_args(c);
  a.src = c->g[c->cur];
  a.dst = c->T;
  if (row(c, ROW_FWD, a)) return -1;
  if (forward_rest(c, c->T, c->T)) return -1;
  zero_unmeasured_kernel<<<592, 256, 0, c->st>>>(c->T, c->flags, c->n);
  CK(cudaGetLastError());
  if (inverse_scaled_into_model(c)) return -1;
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

extern "C" int spb_ctx_iterate(spb_ctx *c, const spb_alg_desc *alg, const float *beta, int iterations,
                               int keep_gp) {
  if (iterations <= 0) return 0;
  const int A = alg->algorithm;
  if (A < 1 || A > 4) return fail("unknown algorithm %d", A);
  if (alg->objective == 0 && !c->amp) return fail("amplitudes not set");
  if (alg->objective == 1 && !c->pamp) return fail("phased amplitudes not set");
  if ((alg->constraints & C_MARGIN) && (!c->amin || !c->amax)) return fail("amplitude margins not set");
  const size_t nc = sizeof(float2) * (size_t)c->n;
  if (A == ALG_DM) {
    if (!c->Xf) CK(cudaMalloc(&c->Xf, nc));
    if (!c->Yf) CK(cudaMalloc(&c->Yf, nc));
  }
  if (ensure_x(c)) return -1;
  if (A == ALG_DM && ensure_xf(c, alg->gamma1)) return -1;
  PassArgs a = base_args(c);
  a.alg = A;
  a.constraints = alg->constraints;
  a.objective = alg->objective;
  a.gamma1 = alg->gamma1;
  a.gamma2 = alg->gamma2;
  a.one_p_g2 = 1 + alg->gamma2;
  a.size_f = (float)(int)c->n;
  for (int it = 0; it < iterations; it++) {
    const float b = (A == ALG_ER) ? 0.0f : beta[it];
    a.beta = b;
    a.one_m2b = 1 - 2 * b;
    c->cur ^= 1;
    a.g0 = c->g[c->cur ^ 1];
    a.g1 = c->g[c->cur];
    a.gp = (keep_gp && it == iterations - 1) ? c->gp : nullptr;
    if (middle(c, COL_PROJECT, c->X, c->Y, a)) return -1;
    if (A == ALG_DM) {
      if (middle(c, COL_PROJECT_NOFC, c->Xf, c->Yf, a)) return -1;
      a.src = c->Y;
      a.src2 = c->Yf;
      a.dst = c->X;
      a.dst2 = c->Xf;
      if (row(c, ROW_DM_ITER, a)) return -1;
    } else {
      a.src = c->Y;
      a.dst = c->X;
      if (row(c, ROW_ITER, a)) return -1;
    }
  }
  if (A != ALG_DM) c->xf_valid = 0;
  return 0;
}

// blur |g1| (or |img| when img != nullptr) into c->absb
static int blur_abs(spb_ctx *c, const float2 *img, float radius) {
  PassArgs a = base_args(c);
  a.src = img ? img : c->g[c->cur];
  a.dst = c->T;
  if (row(c, ROW_FWD_DEPHASE, a)) return -1;
  a.blur_c0 = -2. * pow(3.14159265358979323846, 2);
  a.blur_r2 = pow((double)radius, 2);
  if (middle(c, COL_BLUR, c->T, c->T, a)) return -1;
  a.src = c->T;
  a.absout = c->absb;
  if (row(c, ROW_INV_ABS, a)) return -1;
  return 0;
}

// Area rule: threshold = k-th largest |blur| with k = (int)(N * area) (float
// product, as the reference indexes its descending sort); k is clamped to
// N-1 where the reference would read past the end.  Threshold rule: max|blur|
// times value.  Then inside = |blur| > threshold.
static int select_and_mask_on(cudaStream_t st, SelectState *sel, const float *absv, long long n, int type,
                              float value, uint8_t *flags) {
  if (type == SPB_SUPPORT_AREA) {
    long long k = (long long)(int)((float)n * value);
    if (k >= n) k = n - 1;
    if (k < 0) k = 0;
    CK(launch_select_kth_desc(absv, n, k, sel, st));
    CK(launch_mask_from_abs(absv, (const float *)sel, 0.0f, 0, flags, n, st));
  } else if (type == SPB_SUPPORT_THRESHOLD) {
    CK(launch_max_abs(absv, n, sel, st));
    CK(launch_mask_from_abs(absv, (const float *)sel, value, 1, flags, n, st));
  } else {
    return fail("unknown support update type %d", type);
  }
  return 0;
}

static int select_and_mask(spb_ctx *c, const float *absv, long long n, int type, float value, uint8_t *flags) {
  return select_and_mask_on(c->st, c->sel, absv, n, type, value, flags);
}

extern "C" int spb_ctx_support_update(spb_ctx *c, int type, float radius, float value) {
  if (blur_abs(c, nullptr, radius)) return -1;
  if (select_and_mask(c, c->absb, c->n, type, value, c->flags)) return -1;
  c->xf_valid = 0;
  return 0;
}

extern "C" int spb_ctx_support_patterson(spb_ctx *c, float value) {
  int axes[2];
  const int k = other_axes(c, axes);
  PassArgs a = base_args(c);
  a.f32src = c->amp;
  if (k == 0) {
    if (col(c, 0, COL_INV_SQUARE_F32, nullptr, c->T, a)) return -1;
  } else {
    if (col(c, axes[k - 1], COL_INV_SQUARE_F32, nullptr, c->T, a)) return -1;
    for (int i = k - 2; i >= 0; i--)
      if (col(c, axes[i], COL_INV, c->T, c->T, a)) return -1;
  }
  a.src = c->T;
  a.absout = c->absb;
  if (row(c, ROW_INV_ABS, a)) return -1;
  if (select_and_mask(c, c->absb, c->n, SPB_SUPPORT_THRESHOLD, value, c->flags)) return -1;
  c->xf_valid = 0;
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

static int fmodel_into_T(spb_ctx *c) {
  if (ensure_x(c)) return -1;
  return forward_rest(c, c->X, c->T);
}

extern "C" int spb_ctx_get_image(spb_ctx *c, int which, float *out) {
  const size_t nc = sizeof(float2) * (size_t)c->n;
  const float2 *src = nullptr;
  switch (which) {
    case SPB_G0: src = c->g[c->cur ^ 1]; break;
    case SPB_G1: src = c->g[c->cur]; break;
    case SPB_GP: src = c->gp; break;
    case SPB_FMODEL:
      if (fmodel_into_T(c)) return -1;
      src = c->T;
      break;
    default: return fail("unknown image %d", which);
  }
  return download(c, out, src, nc);
}

extern "C" int spb_ctx_efourier_sums(spb_ctx *c, double sums[4]) {
  if (fmodel_into_T(c)) return -1;
  CK(launch_reduce_efourier(c->T, c->amp, c->flags, c->n, c->red, c->st));
  return download(c, sums, c->red, sizeof(double) * 4);
}

extern "C" int spb_ctx_ereal_sums(spb_ctx *c, double sums[2]) {
  CK(launch_reduce_ereal(c->gp, c->flags, c->n, c->red, c->st));
  return download(c, sums, c->red, sizeof(double) * 2);
}

extern "C" int spb_ctx_support_count(spb_ctx *c, long long *count) {
  CK(launch_count_inside(c->flags, c->n, c->cnt, c->st));
  unsigned long long v = 0;
  if (download(c, &v, c->cnt, sizeof(v))) return -1;
  *count = (long long)v;
  return 0;
}

// ------------------------------------------------------------ one-shot API
extern "C" int spb_fft_host(int nx, int ny, int nz, int sign, const float *in, float *out) {
  spb_ctx *c = nullptr;
  if (spb_ctx_create(&c, nx, ny, nz)) return -1;
  const size_t nc = sizeof(float2) * (size_t)c->n;
  int rc = 0;
  if (upload(c, c->T, in, nc)) rc = -1;
  PassArgs a = base_args(c);
  if (!rc && sign < 0) {
    a.src = c->T;
    a.dst = c->Y;
    if (row(c, ROW_FWD, a) || forward_rest(c, c->Y, c->Y)) rc = -1;
  } else if (!rc) {
    if (backward_rest(c, c->T, c->T)) rc = -1;
    a.src = c->T;
    a.dst = c->Y;
    if (!rc && row(c, ROW_INV, a)) rc = -1;
  }
  if (!rc) rc = download(c, out, c->Y, nc);
  spb_ctx_destroy(c);
  return rc;
}

extern "C" int spb_blur_host(int nx, int ny, int nz, const float *in, float radius, float *out) {
  spb_ctx *c = nullptr;
  if (spb_ctx_create(&c, nx, ny, nz)) return -1;
  const size_t nc = sizeof(float2) * (size_t)c->n;
  int rc = upload(c, c->Y, in, nc);
  if (!rc) {
    // full complex blur (no dephasing): forward x, middle blur, backward x
    PassArgs a = base_args(c);
    a.src = c->Y;
    a.dst = c->T;
    if (row(c, ROW_FWD, a)) rc = -1;
    a.blur_c0 = -2. * pow(3.14159265358979323846, 2);
    a.blur_r2 = pow((double)radius, 2);
    if (!rc && middle(c, COL_BLUR, c->T, c->T, a)) rc = -1;
    a.src = c->T;
    a.dst = c->Y;
    if (!rc && row(c, ROW_INV, a)) rc = -1;
  }
  if (!rc) rc = download(c, out, c->Y, nc);
  spb_ctx_destroy(c);
  return rc;
}

namespace spb {
__global__ void abs_kernel(const float2 *in, float *out, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = cabs_ref(in[i]);
}
}  // namespace spb

static int support_from_blur_impl(long long n, const float *blur, int type, float value, int *flags,
                                  cudaStream_t st, float2 *dblur, float *dabs, uint8_t *dflags, SelectState *sel) {
  std::vector<uint8_t> h((size_t)n);
  for (long long i = 0; i < n; i++) h[i] = (uint8_t)(flags[i] & 3);
  CK(cudaMemcpyAsync(dblur, blur, sizeof(float2) * (size_t)n, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dflags, h.data(), (size_t)n, cudaMemcpyHostToDevice, st));
  abs_kernel<<<592, 256, 0, st>>>(dblur, dabs, n);
  CK(cudaGetLastError());
  if (select_and_mask_on(st, sel, dabs, n, type, value, dflags)) return -1;
  CK(cudaMemcpyAsync(h.data(), dflags, (size_t)n, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  for (long long i = 0; i < n; i++) flags[i] = h[i];
  return 0;
}

extern "C" int spb_support_from_blur_host(long long n, const float *blur, int type, float value, int *flags) {
  if (n < 1 || n > (1LL << 31)) return fail("invalid size %lld", n);
  cudaStream_t st = nullptr;
  float2 *dblur = nullptr;
  float *dabs = nullptr;
  uint8_t *dflags = nullptr;
  SelectState *sel = nullptr;
  int rc = 0;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&dblur, sizeof(float2) * (size_t)n) != cudaSuccess ||
      cudaMalloc(&dabs, sizeof(float) * (size_t)n) != cudaSuccess || cudaMalloc(&dflags, (size_t)n) != cudaSuccess ||
      cudaMalloc(&sel, sizeof(SelectState)) != cudaSuccess)
    rc = fail("allocation for %lld pixels failed", n);
  if (!rc) rc = support_from_blur_impl(n, blur, type, value, flags, st, dblur, dabs, dflags, sel);
  if (st) cudaStreamSynchronize(st);
  cudaFree(dblur);
  cudaFree(dabs);
  cudaFree(dflags);
  cudaFree(sel);
  if (st) cudaStreamDestroy(st);
  return rc;
}
