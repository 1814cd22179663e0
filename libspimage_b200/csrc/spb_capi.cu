// C-ABI device layer of the phasing path (include/spimage/spb_device.h).
//
// A context holds nb independent starts ("batch") of one nx*ny*nz problem;
// a single phaser is nb = 1.  Per-start buffers are stacked start-major
// (start b at offset b*N):
//   flags[nb*N] u8 (bit0 inside support, bit1 measured),
//   g[2][nb*N] c64 ping-pong iterates (g1 = model, g0 = old model),
//   X[nb*N] c64 = row FFT of g1 (kept valid between iterations),
//   Y[nb*N] c64 projection-pass output, gp[nb*N] c64 (last model before
//   projection), T[nb*N] c64 and absb[nb*N] f32 support-update scratch,
//   Xf/Yf[nb*N] c64 for the difference map's second transform pair.
// Shared by all starts (one pattern): amp[N], amp_line[N], meas_bits,
// amp_min/amp_max/phased_amp[N].
// Rows of all starts form one tall row pass; column passes treat the start
// index as one more outer dimension.  All work is enqueued on one stream.
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <map>
#include <mutex>
#include <vector>

#include "host/host_internal.h"
#include "spb_internal.h"
#include "spb_pointwise.cuh"
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

extern "C" int spb_check_roundings(unsigned lo, unsigned hi, unsigned long long ndiv, unsigned long long seed,
                                   unsigned a_stride, unsigned long long *bad) {
  unsigned long long *d = nullptr, h[4] = {0, 0, 0, 0};
  if (cudaMalloc(&d, sizeof h) != cudaSuccess) return fail("cudaMalloc failed");
  cudaError_t e = cudaMemset(d, 0, sizeof h);
  if (e == cudaSuccess) e = check_roundings(lo, hi, ndiv, seed, a_stride, d);
  if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof h, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return fail("rounding self-check: %s", cudaGetErrorString(e));
  for (int k = 0; k < 4; k++) bad[k] = h[k];
  return 0;
}

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
  // per-stage copy of the twiddles used by stage s: [m-1][k] = W_n^(m*k*n/(Ns*R))
  std::vector<float2> st;
  int ns_ = 1;
  for (int s = 0; s < ns; s++) {
    const int r = radix[s], tstep = n / (ns_ * r);
    for (int m = 1; m < r; m++)
      for (int k = 0; k < ns_; k++) st.push_back(h[(size_t)m * k * tstep]);
    ns_ *= r;
  }
  if (st.empty()) st.push_back(make_float2(1.0f, 0.0f));
  CK(cudaMalloc(&ax.tw, sizeof(float2) * ((size_t)n + st.size())));
  CK(cudaMemcpy(ax.tw, h.data(), sizeof(float2) * (size_t)n, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(ax.tw + n, st.data(), sizeof(float2) * st.size(), cudaMemcpyHostToDevice));
  ax.lp.tw = ax.tw;
  ax.lp.stw = ax.tw + n;
  return 0;
}

// Largest line the staging buffers hold: two n-point complex lines per row in
// shared memory (row pass) or per column tile (column pass).
const int kMaxAxis = 8192;
// iterations per captured graph (even: the iterate buffers return to their roles)
const int kGraphIters = 16;
const int kMaxGraphs = 24;
// calls of at most this many iterations run as one captured graph each
const int kWholeGraphMax = 64;
// iterations whose beta values one call can stage on the device
const int kBetaCap = 1 << 16;
// Pinned staging of the host->device parameter copies: the host reuses a
// segment only after its copy has run, so it can run this many calls ahead of
// the device before it waits.  Beta uploads of at most kSmallBeta values use
// the small segments, longer ones the two large ones.
const int kParamRing = 64;
const int kSmallBeta = 256;
const int kLargeRing = 2;
// grid y-dimension limit of the column passes
const int kMaxGridY = 65535;

}  // namespace

struct GraphEntry {
  bool used = false;
  int alg = 0, constraints = 0, objective = 0;
  float gamma1 = 0.0f, gamma2 = 0.0f;
  int parity = 0;
  // 0: a replayable chunk of kGraphIters iterations reading beta at
  // *beta_base + i; n > 0: a whole call of n iterations reading beta[i]
  int n = 0, keep_gp = 0;
  long long nodes = 0;  // kernel launches per replay
  cudaGraphExec_t exec = nullptr;
};

// Parameters of a captured support update, read by its kernels at run time.
struct SupportParams {
  double r2;                // pow(blur radius, 2)
  unsigned long long rank;  // area rule: index of the threshold in descending order
  float rel;                // threshold rule: fraction of the maximum
  int pad;
};

struct SupportGraph {
  cudaGraphExec_t exec = nullptr;
  long long nodes = 0;
};

struct KernelProfile {
  bool on = false;
  std::vector<cudaEvent_t> ev;  // pairs (start, stop) per launch
  std::vector<int> kind;
  size_t used = 0;
  long long launches[SPB_KERNEL_KINDS] = {};
  double ms[SPB_KERNEL_KINDS] = {};
};

struct spb_ctx {
  int nx = 0, ny = 0, nz = 0;
  long long n = 0;     // pixels per start
  int nb = 1;          // starts
  long long ntot = 0;  // nb * n
  cudaStream_t st = nullptr;      // active stream
  cudaStream_t own_st = nullptr;  // the context's own stream
  KernelProfile prof;
  long long launches = 0;  // kernels enqueued by this context (graph replays count their nodes)
  Axis ax, ay, az;
  float *amp = nullptr, *amin = nullptr, *amax = nullptr;
  float2 *pamp = nullptr;
  uint8_t *flags = nullptr;
  float2 *g[2] = {nullptr, nullptr};
  int cur = 0;
  float2 *X = nullptr, *Y = nullptr, *Xf = nullptr, *Yf = nullptr, *gp = nullptr, *T = nullptr;
  float *absb = nullptr;
  float *gtab = nullptr;  // blur factor table, (nx/2+1)(ny/2+1)(nz/2+1)
  // line-major operands of the projection pass (lines along the last axis)
  float *amp_line = nullptr;
  int *amp_bad = nullptr;  // set when an amplitude lies outside the branch-free quotient's domain
  uint32_t *meas_bits = nullptr;
  int proj_len = 0, meas_words = 0;
  long long proj_lines = 0, proj_estride = 0;
  // CUDA graphs of iteration chunks
  GraphEntry graphs[kMaxGraphs];
  int graph_evict = 0;
  bool use_graphs = true;
  int warm_alg[5] = {0, 0, 0, 0, 0};
  float *beta_dev = nullptr;
  float *beta_pinned = nullptr;  // kLargeRing x kBetaCap, then kParamRing x kSmallBeta
  int beta_cap = 0;
  int *beta_base = nullptr;
  cudaEvent_t beta_ev[kLargeRing + kParamRing] = {};
  int beta_seg_large = 0, beta_seg_small = 0;
  std::vector<float> beta_shadow;  // values of the last upload (the table's content in stream order)
  int *beta_zero = nullptr;        // device 0: base of whole-call graphs
  // captured support updates [type 1 threshold, 2 area][parity], their parameters
  SupportGraph sup_graph[3][2];
  int warm_sup[3] = {0, 0, 0};
  SupportParams *spar = nullptr, *spar_pinned = nullptr;  // pinned: kParamRing entries
  cudaEvent_t spar_ev[kParamRing] = {};
  int spar_seg = 0;
  bool spar_valid = false;
  SupportParams spar_shadow{};
  SelectState *sel = nullptr;  // one per start
  double *red = nullptr;       // reduce_scratch_doubles(nb)
  unsigned *nonfinite = nullptr;  // sticky flag of spb_ctx_nonfinite_async
  int *err_flag = nullptr;        // set by a kernel that gave up (bounded wait, misaligned TMA tile)
  long long *hard = nullptr;      // random starts: elements the host evaluates (spb_ctx_models_from_phases)
  unsigned *hard_n = nullptr;
  unsigned long long *seeds = nullptr;  // per-start generator keys (device starts)
  void *hstage = nullptr;               // pinned host staging buffer (spb_ctx_host_stage)
  size_t hstage_bytes = 0;
  int x_valid = 0, xf_valid = 0;
  float xf_gamma1 = 0.0f;
  int tune[SPB_TUNE_KNOBS] = {};  // launch-shape choices (0: built-in)
};

namespace {

PassArgs base_args(const spb_ctx *c) {
  PassArgs a;
  memset(&a, 0, sizeof(a));
  a.nx = c->nx;
  a.ny = c->ny;
  a.nz = c->nz;
  a.n = c->ntot;
  a.n_start = c->n;
  a.amp = c->amp;
  a.amp_min = c->amin;
  a.amp_max = c->amax;
  a.phased_amp = c->pamp;
  a.flags = c->flags;
  a.amp_line = c->amp_line;
  a.amp_bad = c->amp_bad;
  a.meas_bits = c->meas_bits;
  a.meas_words = c->meas_words;
  a.row_lpb = c->tune[SPB_TUNE_ROW_LINES];
  a.row_g0 = c->tune[SPB_TUNE_ROW_G0];
  a.pdl = c->tune[SPB_TUNE_NO_PDL] ? 0 : 1;
  a.split = c->tune[SPB_TUNE_SPLIT];
  a.col_width = c->tune[SPB_TUNE_COL_WIDTH];
  a.tma = c->tune[SPB_TUNE_TMA];
  a.err_flag = c->err_flag;
  a.inv_n = (float)(1.0 / (double)c->n);
  a.nx_f = (float)c->nx;
  a.n_f = (float)c->n;
  return a;
}

// Column-line geometry: axis 1 = y lines (one set per z slab of every start),
// 2 = z lines (one set per start), 0 = lines of length 1 over every pixel
// (pointwise pass for 1-D problems).
void col_geometry(const spb_ctx *c, int axis, PassArgs &a, const LinePlan **pl) {
  a.line_axis = axis;
  if (axis == 1) {
    a.estride = c->nx;
    a.ostride = (long long)c->nx * c->ny;
    a.ncols = c->nx;
    a.nouter = c->nb * c->nz;
    *pl = &c->ay.lp;
  } else if (axis == 2) {
    a.estride = (long long)c->nx * c->ny;
    a.ostride = c->n;
    a.ncols = c->nx * c->ny;
    a.nouter = c->nb;
    *pl = &c->az.lp;
  } else {
    a.estride = 1;
    a.ostride = 0;
    a.ncols = (int)c->ntot;
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

// ---- optional per-launch event timing
const int kProfPairs = 4096;

int prof_flush(spb_ctx *c) {
  KernelProfile &p = c->prof;
  if (!p.used) return 0;
  CK(cudaEventSynchronize(p.ev[p.used - 1]));
  for (size_t i = 0; i < p.used; i += 2) {
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, p.ev[i], p.ev[i + 1]));
    const int k = p.kind[i / 2];
    p.ms[k] += ms;
    p.launches[k] += 1;
  }
  p.used = 0;
  return 0;
}

int prof_begin(spb_ctx *c) {
  KernelProfile &p = c->prof;
  if (!p.on) return 0;
  if (p.used + 2 > p.ev.size() && prof_flush(c)) return -1;
  CK(cudaEventRecord(p.ev[p.used], c->st));
  return 0;
}

int prof_end(spb_ctx *c, int kind) {
  KernelProfile &p = c->prof;
  if (!p.on) return 0;
  CK(cudaEventRecord(p.ev[p.used + 1], c->st));
  p.kind[p.used / 2] = kind;
  p.used += 2;
  return 0;
}

int col(spb_ctx *c, int axis, int mode, const float2 *src, float2 *dst, PassArgs a) {
  const LinePlan *pl = nullptr;
  col_geometry(c, axis, a, &pl);
  a.src = src;
  a.dst = dst;
  LinePlan unit = unit_plan();
  const int nouter = a.nouter;
  if (prof_begin(c)) return -1;
  for (int o0 = 0; o0 < nouter; o0 += kMaxGridY) {
    a.outer0 = o0;
    a.nouter = nouter - o0 < kMaxGridY ? nouter - o0 : kMaxGridY;
    CK(launch_col(mode, pl ? *pl : unit, pl ? pl->n : 1, a, c->st));
    c->launches++;
  }
  return prof_end(c, 10 + mode);
}

int row(spb_ctx *c, int mode, PassArgs a) {
  if (prof_begin(c)) return -1;
  CK(launch_row(mode, c->ax.lp, a, c->st));
  c->launches++;
  return prof_end(c, mode);
}

// Non-x axes in transform order (forward: y then z).
int other_axes(const spb_ctx *c, int *axes) {
  int k = 0;
  if (c->ny > 1) axes[k++] = 1;
  if (c->nz > 1) axes[k++] = 2;
  return k;
}

// The projection of a 3-D volume with ny = nz = 64 or 128 as one plane pass
// (spb_fast.cu plane_kernel) instead of three column passes, when
// SPB_TUNE_PLANE is 2.  Not the built-in choice: measured on one B200, HIO
// 128^3 per slot, three column passes / plane pass: 38.9 / 63.6 us for one
// start, 266 / 441 us for 8 starts -- a 140 KB plane per block leaves one
// block of 32 warps per SM for four transforms, while the column passes
// spread the same transforms over many small blocks.  Returns 1 when it ran,
// 0 when it does not apply (the column passes run), -1 on error.
static int plane_pass(spb_ctx *c, int mode, const float2 *src, float2 *dst, PassArgs a) {
  if (c->tune[SPB_TUNE_PLANE] != 2 || !plane_fits(mode, c->az.lp, a)) return 0;
  a.src = src;
  a.dst = dst;
  a.line_axis = 2;
  if (prof_begin(c)) return -1;
  for (int o0 = 0; o0 < c->nb; o0 += kMaxGridY) {
    a.outer0 = o0;
    a.nouter = c->nb - o0 < kMaxGridY ? c->nb - o0 : kMaxGridY;
    CK(launch_plane(mode, c->az.lp, a, c->st));
    c->launches++;
  }
  return prof_end(c, 10 + mode) ? -1 : 1;
}

// dst = B(M(F(src))) over the non-x axes, M applied in the last axis pass
// (or pointwise if there is no other axis).  src may equal dst.
int middle(spb_ctx *c, int mid_mode, const float2 *src, float2 *dst, PassArgs a) {
  int axes[2];
  const int k = other_axes(c, axes);
  if (k == 0) return col(c, 0, mid_mode, src, dst, a);
  if (k == 2) {
    const int pr = plane_pass(c, mid_mode, src, dst, a);
    if (pr) return pr < 0 ? -1 : 0;
  }
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
    if (src != dst) CK(cudaMemcpyAsync(dst, src, sizeof(float2) * c->ntot, cudaMemcpyDeviceToDevice, c->st));
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
    if (src != dst) CK(cudaMemcpyAsync(dst, src, sizeof(float2) * c->ntot, cudaMemcpyDeviceToDevice, c->st));
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

int check_dims(int nx, int ny, int nz, int nb) {
  if (nx < 1 || ny < 1 || nz < 1 || nb < 1) return fail("invalid dimensions %d x %d x %d x %d", nx, ny, nz, nb);
  if (nx > kMaxAxis || ny > kMaxAxis || nz > kMaxAxis)
    return fail("axis longer than %d is not supported (%d x %d x %d)", kMaxAxis, nx, ny, nz);
  if ((long long)nx * ny * nz * nb >= (1LL << 31)) return fail("more than 2^31 pixels in one context");
  return 0;
}

long long gauss_table_len(int nx, int ny, int nz) { return (long long)(nx / 2 + 1) * (ny / 2 + 1) * (nz / 2 + 1); }

int check_start(const spb_ctx *c, int start) {
  if (start < 0 || start >= c->nb) return fail("start %d out of range [0, %d)", start, c->nb);
  return 0;
}

}  // namespace

extern "C" void spb_ctx_destroy(spb_ctx *c);

extern "C" int spb_ctx_create_batch(spb_ctx **out, int nx, int ny, int nz, int nb) {
  *out = nullptr;
  if (check_dims(nx, ny, nz, nb)) return -1;
  spb_ctx *c = new spb_ctx();
  c->nx = nx;
  c->ny = ny;
  c->nz = nz;
  c->n = (long long)nx * ny * nz;
  c->nb = nb;
  c->ntot = c->n * nb;
  const size_t nc = sizeof(float2) * (size_t)c->ntot, nf = sizeof(float) * (size_t)c->ntot;
  const size_t nf1 = sizeof(float) * (size_t)c->n;
  int rc = 0;
  auto alloc = [&](void **p, size_t bytes) {
    if (rc) return;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) rc = fail("cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
  };
  cudaError_t e = cudaStreamCreateWithFlags(&c->own_st, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    return fail("cudaStreamCreate: %s", cudaGetErrorString(e));
  }
  c->st = c->own_st;
  alloc((void **)&c->amp, nf1);
  alloc((void **)&c->flags, (size_t)c->ntot);
  alloc((void **)&c->g[0], nc);
  alloc((void **)&c->g[1], nc);
  alloc((void **)&c->X, nc);
  alloc((void **)&c->Y, nc);
  alloc((void **)&c->gp, nc);
  alloc((void **)&c->T, nc);
  alloc((void **)&c->absb, nf);
  alloc((void **)&c->gtab, sizeof(float) * (size_t)gauss_table_len(nx, ny, nz));
  alloc((void **)&c->sel, sizeof(SelectState) * (size_t)nb);
  alloc((void **)&c->red, sizeof(double) * (size_t)reduce_scratch_doubles(nb));
  alloc((void **)&c->nonfinite, sizeof(unsigned));
  alloc((void **)&c->err_flag, sizeof(int));
  if (!rc && cudaMemsetAsync(c->err_flag, 0, sizeof(int), c->st) != cudaSuccess) rc = fail("cudaMemsetAsync");
  alloc((void **)&c->seeds, sizeof(unsigned long long) * (size_t)nb);
  alloc((void **)&c->beta_zero, sizeof(int));
  alloc((void **)&c->spar, sizeof(SupportParams));
  if (!rc && cudaMallocHost(&c->spar_pinned, sizeof(SupportParams) * kParamRing) != cudaSuccess)
    rc = fail("cudaMallocHost");
  for (int k = 0; k < kParamRing && !rc; k++) {
    if (cudaEventCreateWithFlags(&c->spar_ev[k], cudaEventDisableTiming) != cudaSuccess) rc = fail("cudaEventCreate");
    else if (cudaEventRecord(c->spar_ev[k], c->st) != cudaSuccess) rc = fail("cudaEventRecord");
  }
  if (!rc) cudaMemsetAsync(c->beta_zero, 0, sizeof(int), c->st);
  alloc((void **)&c->beta_base, sizeof(int));
  alloc((void **)&c->beta_dev, sizeof(float) * kBetaCap);
  if (!rc && cudaMallocHost(&c->beta_pinned, sizeof(float) * ((size_t)kBetaCap * kLargeRing +
                                                                (size_t)kSmallBeta * kParamRing)) != cudaSuccess)
    rc = fail("cudaMallocHost");
  c->beta_cap = kBetaCap;
  for (int k = 0; k < kLargeRing + kParamRing && !rc; k++) {
    if (cudaEventCreateWithFlags(&c->beta_ev[k], cudaEventDisableTiming) != cudaSuccess) rc = fail("cudaEventCreate");
    else if (cudaEventRecord(c->beta_ev[k], c->st) != cudaSuccess) rc = fail("cudaEventRecord");
  }
  if (!rc && make_axis(c->ax, nx)) rc = -1;
  if (!rc && make_axis(c->ay, ny)) rc = -1;
  if (!rc && make_axis(c->az, nz)) rc = -1;
  if (!rc) {
    cudaMemsetAsync(c->amp, 0, nf1, c->st);
    cudaMemsetAsync(c->flags, 0, (size_t)c->ntot, c->st);
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

extern "C" int spb_ctx_create(spb_ctx **out, int nx, int ny, int nz) {
  return spb_ctx_create_batch(out, nx, ny, nz, 1);
}

extern "C" int spb_ctx_starts(spb_ctx *c) { return c->nb; }

// Captured graphs hold launch shapes and parity-dependent pointers: a change
// of launch shape drops them, and the next call of each kind runs directly.
static void drop_graphs(spb_ctx *c) {
  cudaStreamSynchronize(c->st);
  for (auto &g : c->graphs) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g = GraphEntry();
  }
  for (auto &row : c->sup_graph)
    for (auto &g : row) {
      if (g.exec) cudaGraphExecDestroy(g.exec);
      g = SupportGraph();
    }
  for (auto &w : c->warm_alg) w = 0;
  for (auto &w : c->warm_sup) w = 0;
}

extern "C" int spb_ctx_set_tuning(spb_ctx *c, int knob, int value) {
  if (knob < 0 || knob >= SPB_TUNE_KNOBS) return fail("unknown tuning knob %d", knob);
  if (knob == SPB_TUNE_COL_WIDTH && value != 0 && !col_width_ok(c->nz > 1 ? c->nz : c->ny, value))
    return fail("no projection pass of %d columns per block for lines of %d points", value,
                c->nz > 1 ? c->nz : c->ny);
  if (value < 0) return fail("negative tuning value %d", value);
  if (c->tune[knob] != value) {
    c->tune[knob] = value;
    drop_graphs(c);
  }
  return 0;
}

extern "C" int spb_ctx_get_tuning(spb_ctx *c, int knob) {
  return (knob >= 0 && knob < SPB_TUNE_KNOBS) ? c->tune[knob] : -1;
}

// Bytes spb_ctx_create_batch and the first uses of a context allocate
// (margins and phased amplitudes, allocated only when set, not included).
extern "C" long long spb_ctx_footprint(int nx, int ny, int nz, int nb, int dm) {
  if (check_dims(nx, ny, nz, nb)) return -1;
  const long long n = (long long)nx * ny * nz, ntot = n * nb;
  long long b = 0;
  b += 4 * n;                                   // amp
  b += ntot;                                    // flags
  b += 6 * 8 * ntot;                            // g[2], X, Y, gp, T
  b += 4 * ntot;                                // absb
  b += 4 * gauss_table_len(nx, ny, nz);         // gtab
  b += (long long)sizeof(SelectState) * nb;     // sel
  b += 8LL * reduce_scratch_doubles(nb);        // red
  b += 256;                                     // non-finite flag (one allocation)
  b += 8LL * nb + 4 + 4LL * kBetaCap;           // seeds, beta_base, beta table
  b += 4 * n + n / 8 + 4096;                    // amp_line, meas_bits (upper bound)
  b += 8LL * 2 * (nx + ny + nz) + 8LL * 3 * 65536;  // twiddles and stage tables (upper bound)
  if (dm) b += 2 * 8 * ntot;                    // Xf, Yf
  return b;
}

extern "C" void spb_ctx_destroy(spb_ctx *c) {
  if (!c) return;
  if (c->st) cudaStreamSynchronize(c->st);
  void *ptrs[] = {c->amp, c->amin, c->amax, c->pamp, c->flags, c->g[0], c->g[1], c->X, c->Y, c->Xf, c->Yf,
                  c->gp, c->T, c->absb, c->gtab, c->sel, c->red, c->nonfinite, c->err_flag, c->ax.tw, c->ay.tw,
                  c->az.tw,
                  c->amp_line, c->amp_bad, c->meas_bits, c->beta_dev, c->beta_base, c->seeds, c->beta_zero, c->spar,
                  c->hard, c->hard_n};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  for (auto &e : c->prof.ev) cudaEventDestroy(e);
  for (auto &g : c->graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  if (c->beta_pinned) cudaFreeHost(c->beta_pinned);
  for (auto &e : c->beta_ev)
    if (e) cudaEventDestroy(e);
  for (auto &e : c->spar_ev)
    if (e) cudaEventDestroy(e);
  if (c->spar_pinned) cudaFreeHost(c->spar_pinned);
  if (c->hstage) cudaFreeHost(c->hstage);
  for (auto &row : c->sup_graph)
    for (auto &g : row)
      if (g.exec) cudaGraphExecDestroy(g.exec);
  if (c->own_st) cudaStreamDestroy(c->own_st);
  delete c;
}

static int check_err_flag(spb_ctx *c);
extern "C" int spb_ctx_synchronize(spb_ctx *c) {
  CK(cudaStreamSynchronize(c->st));
  return check_err_flag(c);
}

static const char *kKernelNames[SPB_KERNEL_KINDS] = {
    "row_fwd",        "row_fwd_dephase", "row_inv",     "row_inv_scale", "row_inv_abs",
    "row_iter",       "row_dm_f1_fwd",   "row_dm_iter", "row_fwd_f32",   "row_fwd_square_f32",
    "col_fwd",        "col_inv",         "col_project", "col_project_nofc", "col_blur",
    "col_inv_square", "select_area",     "select_max",  "unused18",      "unused19"};

extern "C" const char *spb_kernel_name(int kind) {
  return (kind >= 0 && kind < SPB_KERNEL_KINDS) ? kKernelNames[kind] : "";
}

extern "C" int spb_ctx_profile(spb_ctx *c, int enable) {
  KernelProfile &p = c->prof;
  if (enable && p.ev.empty()) {
    p.ev.resize(2 * kProfPairs);
    p.kind.resize(kProfPairs);
    for (auto &e : p.ev) CK(cudaEventCreate(&e));
  }
  if (!enable && prof_flush(c)) return -1;
  p.on = enable != 0;
  if (enable) {
    for (int k = 0; k < SPB_KERNEL_KINDS; k++) {
      p.launches[k] = 0;
      p.ms[k] = 0;
    }
  }
  return 0;
}

extern "C" int spb_ctx_profile_read(spb_ctx *c, int kind, long long *launches, double *total_ms) {
  if (kind < 0 || kind >= SPB_KERNEL_KINDS) return fail("bad kernel kind %d", kind);
  if (prof_flush(c)) return -1;
  *launches = c->prof.launches[kind];
  *total_ms = c->prof.ms[kind];
  return 0;
}

extern "C" long long spb_ctx_launch_count(spb_ctx *c) { return c->launches; }

extern "C" int spb_ctx_set_stream(spb_ctx *c, void *stream) {
  if (prof_flush(c)) return -1;
  CK(cudaStreamSynchronize(c->st));
  c->st = stream ? (cudaStream_t)stream : c->own_st;
  return 0;
}

// Pinned host buffer of at least `bytes`, owned by the context: host data
// written here crosses to the device by DMA at full speed instead of through
// the driver's pageable staging.  Valid until the next call with a larger
// size; the caller's copies from it complete before it is handed out again
// (every upload through it synchronizes the stream).
extern "C" void *spb_ctx_host_stage(spb_ctx *c, size_t bytes) {
  if (bytes <= c->hstage_bytes) return c->hstage;
  if (c->hstage) {
    if (cudaStreamSynchronize(c->st) != cudaSuccess) return nullptr;
    cudaFreeHost(c->hstage);
    c->hstage = nullptr;
    c->hstage_bytes = 0;
  }
  const size_t cap = (bytes + 0xFFFFF) & ~(size_t)0xFFFFF;  // whole MiB
  if (cudaMallocHost(&c->hstage, cap) != cudaSuccess) {
    cudaGetLastError();
    c->hstage = nullptr;
    fail("cudaMallocHost of a %zu-byte staging buffer", cap);
    return nullptr;
  }
  c->hstage_bytes = cap;
  return c->hstage;
}

// Page-locks a host range the library owns and reuses (amplitudes, the model
// image), so its copies run by DMA; 0 on success.  A range that cannot be
// locked still works through pageable copies.
extern "C" int spb_host_register(void *p, size_t bytes) {
  if (!p || !bytes) return -1;
  if (cudaHostRegister(p, bytes, cudaHostRegisterPortable) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  return 0;
}

extern "C" void spb_host_unregister(void *p) {
  if (p && cudaHostUnregister(p) != cudaSuccess) cudaGetLastError();
}

static int upload(spb_ctx *c, void *dst, const void *src, size_t bytes) {
  CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

// after the context's stream has drained: a TMA pass kernel whose bounded
// wait ran out (a tile or row that never arrived: 1) or whose tile was
// misaligned (2) has set the error flag; it stays set (the results are not
// to be trusted again)
static int check_err_flag(spb_ctx *c) {
  if (c->tune[SPB_TUNE_TMA] == 1) return 0;  // no TMA pass runs
  int h = 0;
  CK(cudaMemcpyAsync(&h, c->err_flag, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (h == 2) return fail("a TMA pass kernel found its shared-memory tile or first column misaligned and copied nothing: results are invalid");
  if (h) return fail("a TMA pass kernel gave up waiting for its tile or rows (bounded mbarrier wait): results are invalid");
  return 0;
}

static int download(spb_ctx *c, void *dst, const void *src, size_t bytes) {
  CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return check_err_flag(c);
}

namespace spb {
// amp_line[L*len + i] = amp[i*estride + L]; *bad = 1 if some amplitude is
// neither zero nor of magnitude in [2^-60, 2^60] (the branch-free quotient's domain)
__global__ void build_amp_line_kernel(const float *amp, float *amp_line, int len, long long estride,
                                      long long nlines, int *bad) {
  const long long total = nlines * len;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (long long)gridDim.x * blockDim.x) {
    const long long L = k / len, i = k % len;
    const float v = amp[i * estride + L];
    amp_line[k] = v;
    if (!div_rn_nb_domain(v)) *bad = 1;
  }
}
// bit i of line L = measured flag of pixel i*estride + L (of start 0)
__global__ void build_meas_bits_kernel(const uint8_t *flags, uint32_t *bits, int len, int W, long long estride,
                                       long long nlines) {
  const long long total = nlines * W;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (long long)gridDim.x * blockDim.x) {
    const long long L = k / W;
    const int w = (int)(k % W);
    uint32_t word = 0;
    for (int b = 0; b < 32; b++) {
      const int i = w * 32 + b;
      if (i < len && (flags[i * estride + L] & FLAG_MEASURED)) word |= 1u << b;
    }
    bits[k] = word;
  }
}
// every start's flag bits in `mask` from the n bytes at src, the other bits kept
__global__ void merge_flags_kernel(uint8_t *flags, const uint8_t *__restrict__ src, long long n, int nb, uint8_t mask) {
  const long long total = n * nb;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (long long)gridDim.x * blockDim.x)
    flags[k] = (uint8_t)((flags[k] & ~mask) | (src[k % n] & mask));
}
// every start's flags = start 0's (bits in `mask`), keeping the other bits
__global__ void broadcast_flags_kernel(uint8_t *flags, long long n, int nb, uint8_t mask) {
  const long long total = n * (nb - 1);
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (long long)gridDim.x * blockDim.x) {
    const long long i = k % n;
    uint8_t *f = flags + n + k;
    *f = (uint8_t)((*f & ~mask) | (flags[i] & mask));
  }
}
}  // namespace spb

// Projection-pass operands in line-major order; only for 2-D/3-D problems
// whose last axis has a register kernel (power-of-two length).
static int proj_geometry(spb_ctx *c) {
  if (c->proj_len) return 1;
  int len = 0;
  long long estride = 0;
  if (c->nz > 1) {
    len = c->nz;
    estride = (long long)c->nx * c->ny;
  } else if (c->ny > 1) {
    len = c->ny;
    estride = c->nx;
  } else {
    return 0;
  }
  if (len < 16 || len > 4096 || (len & (len - 1))) return 0;
  c->proj_len = len;
  c->proj_estride = estride;
  c->proj_lines = estride;
  c->meas_words = ((len + 127) / 128) * 4;
  return 1;
}

static int build_amp_line(spb_ctx *c) {
  if (!proj_geometry(c)) return 0;
  if (!c->amp_line) CK(cudaMalloc(&c->amp_line, sizeof(float) * (size_t)c->n));
  if (!c->amp_bad) CK(cudaMalloc(&c->amp_bad, sizeof(int)));
  CK(cudaMemsetAsync(c->amp_bad, 0, sizeof(int), c->st));
  build_amp_line_kernel<<<592, 256, 0, c->st>>>(c->amp, c->amp_line, c->proj_len, c->proj_estride, c->proj_lines,
                                                c->amp_bad);
  CK(cudaGetLastError());
  return 0;
}

static int build_meas_bits(spb_ctx *c) {
  if (!proj_geometry(c)) return 0;
  const size_t words = (size_t)c->proj_lines * c->meas_words;
  if (!c->meas_bits) CK(cudaMalloc(&c->meas_bits, sizeof(uint32_t) * words));
  build_meas_bits_kernel<<<592, 256, 0, c->st>>>(c->flags, c->meas_bits, c->proj_len, c->meas_words,
                                                 c->proj_estride, c->proj_lines);
  CK(cudaGetLastError());
  return 0;
}

extern "C" int spb_ctx_set_amplitudes(spb_ctx *c, const float *amp) {
  if (upload(c, c->amp, amp, sizeof(float) * (size_t)c->n)) return -1;
  if (build_amp_line(c)) return -1;
  CK(cudaStreamSynchronize(c->st));
  return 0;
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

// host int flags <-> device byte flags, converted on the host threads
struct FlagsCopy {
  const int *in32;
  uint8_t *out8;
  const uint8_t *in8;
  int *out32;
  int bits;  // bytes_to_flags: 0 = whole value, else only these bits (the others kept)
};
static void flags_to_bytes(void *ctx, int, long long i0, long long i1) {
  const FlagsCopy *j = (const FlagsCopy *)ctx;
  const int *in = j->in32;
  uint8_t *out = j->out8;
  long long i = i0;
#if defined(__SSE2__)  // x86: little-endian
  for (; i < i1 && (i & 3); i++) out[i] = (uint8_t)(in[i] & 3);
  // four bytes a store, straight to memory (uploaded next; the stage is page-aligned)
  for (; i + 4 <= i1; i += 4)
    spb_stream_u32(out + i, (unsigned)(in[i] & 3) | (unsigned)(in[i + 1] & 3) << 8 | (unsigned)(in[i + 2] & 3) << 16 |
                                (unsigned)(in[i + 3] & 3) << 24);
#endif
  for (; i < i1; i++) out[i] = (uint8_t)(in[i] & 3);
  spb_stream_fence();
}
static void bytes_to_flags(void *ctx, int, long long i0, long long i1) {
  const FlagsCopy *j = (const FlagsCopy *)ctx;
  if (!j->bits) {
    for (long long i = i0; i < i1; i++) j->out32[i] = j->in8[i];
  } else {
    const int keep = ~j->bits;
    for (long long i = i0; i < i1; i++) j->out32[i] = (j->out32[i] & keep) | (j->in8[i] & j->bits);
  }
}

static int put_flags(spb_ctx *c, int start, const int *flags) {
  uint8_t *h = (uint8_t *)spb_ctx_host_stage(c, (size_t)c->n);
  if (!h) return -1;
  FlagsCopy job = {flags, h, nullptr, nullptr, 0};
  spb_parallel_for(c->n, flags_to_bytes, &job);
  return upload(c, c->flags + (size_t)start * c->n, h, (size_t)c->n);
}

// every start gets these flags; measured bits feed the shared bitmap
extern "C" int spb_ctx_set_flags(spb_ctx *c, const int *flags) {
  if (put_flags(c, 0, flags)) return -1;
  if (c->nb > 1) {
    broadcast_flags_kernel<<<592, 256, 0, c->st>>>(c->flags, c->n, c->nb, 3);
    CK(cudaGetLastError());
  }
  if (build_meas_bits(c)) return -1;
  CK(cudaStreamSynchronize(c->st));
  c->xf_valid = 0;
  return 0;
}

// Only the flag bits in `bits` from the host (every start), the others kept
// as the device has them: the host edited those bits alone, and the device
// may hold newer values of the others (support updates).
extern "C" int spb_ctx_set_flags_bits(spb_ctx *c, const int *flags, int bits) {
  bits &= FLAG_INSIDE | FLAG_MEASURED;
  if (bits == (FLAG_INSIDE | FLAG_MEASURED)) return spb_ctx_set_flags(c, flags);
  if (!bits) return 0;
  uint8_t *scratch = (uint8_t *)c->absb;  // n bytes of the support-update scratch, free between calls
  uint8_t *h = (uint8_t *)spb_ctx_host_stage(c, (size_t)c->n);
  if (!h) return -1;
  FlagsCopy job = {flags, h, nullptr, nullptr, 0};
  spb_parallel_for(c->n, flags_to_bytes, &job);
  if (upload(c, scratch, h, (size_t)c->n)) return -1;
  merge_flags_kernel<<<592, 256, 0, c->st>>>(c->flags, scratch, c->n, c->nb, (uint8_t)bits);
  CK(cudaGetLastError());
  if ((bits & FLAG_MEASURED) && build_meas_bits(c)) return -1;
  CK(cudaStreamSynchronize(c->st));
  c->xf_valid = 0;
  return 0;
}

// one start's flags; its measured bits must equal start 0's (one pattern)
extern "C" int spb_ctx_set_start_flags(spb_ctx *c, int start, const int *flags) {
  if (check_start(c, start)) return -1;
  if (put_flags(c, start, flags)) return -1;
  if (start == 0 && build_meas_bits(c)) return -1;
  CK(cudaStreamSynchronize(c->st));
  c->xf_valid = 0;
  return 0;
}

static int get_flags(spb_ctx *c, int start, int *flags, int bits) {
  if (check_start(c, start)) return -1;
  uint8_t *h = (uint8_t *)spb_ctx_host_stage(c, (size_t)c->n);
  if (!h) return -1;
  if (download(c, h, c->flags + (size_t)start * c->n, (size_t)c->n)) return -1;
  FlagsCopy job = {nullptr, nullptr, h, flags, bits};
  spb_parallel_for(c->n, bytes_to_flags, &job);
  return 0;
}

extern "C" int spb_ctx_get_start_flags(spb_ctx *c, int start, int *flags) { return get_flags(c, start, flags, 0); }

extern "C" int spb_ctx_get_flags(spb_ctx *c, int *flags) { return get_flags(c, 0, flags, 0); }

extern "C" int spb_ctx_get_flags_bits(spb_ctx *c, int *flags, int bits) {
  bits &= FLAG_INSIDE | FLAG_MEASURED;
  return bits ? get_flags(c, 0, flags, bits) : 0;
}

static int reset_iterates(spb_ctx *c) {
  const size_t nc = sizeof(float2) * (size_t)c->ntot;
  CK(cudaMemsetAsync(c->g[c->cur ^ 1], 0, nc, c->st));
  CK(cudaMemsetAsync(c->gp, 0, nc, c->st));
  return 0;
}

extern "C" int spb_ctx_set_start_model(spb_ctx *c, int start, const float *model, int reset_others) {
  if (check_start(c, start)) return -1;
  if (upload(c, c->g[c->cur] + (size_t)start * c->n, model, sizeof(float2) * (size_t)c->n)) return -1;
  c->x_valid = c->xf_valid = 0;
  if (reset_others && reset_iterates(c)) return -1;
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

// the same model for every start
extern "C" int spb_ctx_set_model(spb_ctx *c, const float *model, int reset_others) {
  for (int b = 0; b < c->nb; b++)
    if (spb_ctx_set_start_model(c, b, model, reset_others && b == 0)) return -1;
  return 0;
}

// g1 = backward FFT(T) * (1/N), every start
static int inverse_scaled_into_model(spb_ctx *c) {
  if (backward_rest(c, c->T, c->T)) return -1;
  PassArgs a = base_args(c);
  a.src = c->T;
  a.dst = c->g[c->cur];
  if (row(c, ROW_INV_SCALE, a)) return -1;
  c->x_valid = c->xf_valid = 0;
  return 0;
}

// fourier holds nb spectra (start-major), or one spectrum when `one` is set
static int models_from_fourier(spb_ctx *c, const float *fourier, int one, int reset_others) {
  const size_t ns = sizeof(float2) * (size_t)c->n;
  for (int b = 0; b < c->nb; b++)
    CK(cudaMemcpyAsync(c->T + (size_t)b * c->n, fourier + (one ? 0 : 2 * (size_t)b * c->n), ns,
                       cudaMemcpyHostToDevice, c->st));
  if (inverse_scaled_into_model(c)) return -1;
  if (reset_others && reset_iterates(c)) return -1;
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

extern "C" int spb_ctx_model_from_fourier(spb_ctx *c, const float *fourier, int reset_others) {
  return models_from_fourier(c, fourier, 1, reset_others);
}

namespace spb {
// Whether the float rounding of the double p could differ from that of a
// double within 16 ulps of it: a rounding midpoint between two floats lies
// that close (or p is too close to the ends of the float range to tell).
__device__ __forceinline__ bool near_float_midpoint(double p) {
  const double ap = fabs(p);
  if (ap == 0.0) return false;
  if (ap < 1e-30 || ap > 1e38) return true;
  const float f = __double2float_rn(p);
  const double up = 0.5 * ((double)f + (double)nextafterf(f, INFINITY));  // exact: two neighbouring floats
  const double dn = 0.5 * ((double)f + (double)nextafterf(f, -INFINITY));
  int e;
  frexp(ap, &e);  // ap = m 2^e, m in [1/2, 1): one ulp is 2^(e-53)
  return fmin(fabs(p - up), fabs(p - dn)) <= ldexp(16.0, e - 53);
}

// T[k] (k = b*n + i) = the random-phase start of pixel i from its phase, as
// the reference's sp_image_rephase computes it (src/image_util.c:1035-1067):
// (cos(phase) |amp|, sin(phase) |amp|) in double, rounded to float, |amp| as
// sp_cabs of (amp, 0).  CUDA's double sincos is within 2 ulps of the exact
// values and the C library's cos and sin within 1, so the two can round to
// different floats only where a product lies within a few ulps of a float
// rounding midpoint: such elements are listed in hard[] (up to cap) for the
// host to evaluate with the C library.  phase holds one start (one) or nb.
__global__ void phases_to_spectra_kernel(float2 *T, const float *amp, const float *phase, long long n, int nb, int one,
                                         unsigned *hard_n, long long *hard, unsigned cap) {
  const long long total = n * nb;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (long long)gridDim.x * blockDim.x) {
    const long long i = k % n;
    const float ph = phase[one ? i : k];
    const float a = cabs_ref(make_float2(amp[i], 0.0f));
    double sn, cs;
    sincos((double)ph, &sn, &cs);
    const double pr = cs * (double)a, pi = sn * (double)a;
    T[k] = make_float2(__double2float_rn(pr), __double2float_rn(pi));
    if (near_float_midpoint(pr) || near_float_midpoint(pi)) {
      const unsigned slot = atomicAdd(hard_n, 1u);
      if (slot < cap) hard[slot] = k;
    }
  }
}
}  // namespace spb

// elements of a random start the host may have to evaluate (typically none)
constexpr unsigned kHardCap = 4096;

extern "C" int spb_ctx_models_from_phases(spb_ctx *c, const float *phases, const float *amp, int one,
                                          int reset_others) {
  const long long count = (long long)c->n * (one ? 1 : c->nb);
  if (!c->hard) CK(cudaMalloc(&c->hard, sizeof(long long) * kHardCap));
  if (!c->hard_n) CK(cudaMalloc(&c->hard_n, sizeof(unsigned)));
  CK(cudaMemcpyAsync(c->absb, phases, sizeof(float) * (size_t)count, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemsetAsync(c->hard_n, 0, sizeof(unsigned), c->st));
  phases_to_spectra_kernel<<<1184, 256, 0, c->st>>>(c->T, c->amp, c->absb, c->n, c->nb, one, c->hard_n, c->hard,
                                                     kHardCap);
  CK(cudaGetLastError());
  c->launches++;
  unsigned nh = 0;
  CK(cudaMemcpyAsync(&nh, c->hard_n, sizeof(unsigned), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (nh > kHardCap) return fail("random start: %u elements near a float rounding midpoint (more than %u)", nh, kHardCap);
  if (nh) {
    std::vector<long long> ks(nh);
    CK(cudaMemcpy(ks.data(), c->hard, sizeof(long long) * nh, cudaMemcpyDeviceToHost));
    std::vector<float2> v(nh);
    for (unsigned j = 0; j < nh; j++) {
      const long long k = ks[j], i = k % c->n;
      const float ph = phases[one ? i : k];
      const float s2 = 0.0f * 0.0f + amp[i] * amp[i];  // sp_cabs of (amp, 0)
      const float a = (float)sqrt((double)s2);
      v[j] = make_float2((float)(cos((double)ph) * (double)a), (float)(sin((double)ph) * (double)a));
    }
    for (unsigned j = 0; j < nh; j++)
      CK(cudaMemcpyAsync(c->T + ks[j], &v[j], sizeof(float2), cudaMemcpyHostToDevice, c->st));
  }
  if (inverse_scaled_into_model(c)) return -1;
  if (reset_others && reset_iterates(c)) return -1;
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

extern "C" int spb_ctx_models_from_fourier(spb_ctx *c, const float *fourier, int reset_others) {
  return models_from_fourier(c, fourier, 0, reset_others);
}

namespace spb {
// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror and Shaw, "Parallel
// random numbers: as easy as 1, 2, 3", SC 2011): 10 rounds of two 32x32->64
// multiplies, key bumped by the Weyl constants between rounds.
__device__ __forceinline__ uint4 philox4x32_10(uint4 ctr, uint2 key) {
  for (int r = 0; r < 10; r++) {
    const unsigned lo0 = 0xD2511F53u * ctr.x, hi0 = __umulhi(0xD2511F53u, ctr.x);
    const unsigned lo1 = 0xCD9E8D57u * ctr.z, hi1 = __umulhi(0xCD9E8D57u, ctr.z);
    ctr = make_uint4(hi1 ^ ctr.y ^ key.x, lo1, hi0 ^ ctr.w ^ key.y, lo0);
    key.x += 0x9E3779B9u;
    key.y += 0xBB67AE85u;
  }
  return ctr;
}

// T[b][i] = amp[i] * exp(2 pi i u), u uniform in [0,1) from (seed_b, i)
__global__ void random_phase_spectra_kernel(float2 *T, const float *amp, const unsigned long long *seeds, long long n,
                                            int nb) {
  const long long total = n * nb;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(k / n);
    const long long i = k % n;
    const unsigned long long s = seeds[b];
    const uint4 r = philox4x32_10(make_uint4((unsigned)i, (unsigned)(i >> 32), 0u, 0u),
                                  make_uint2((unsigned)s, (unsigned)(s >> 32)));
    const float u = (float)(r.x >> 8) * (1.0f / 16777216.0f);
    float sn, cs;
    sincospif(2.0f * u, &sn, &cs);
    const float a = amp[i];
    T[k] = make_float2(a * cs, a * sn);
  }
}
}  // namespace spb

// Random-phase starts drawn on the device (throughput runs; the host API's
// SpModelRandomPhases path reproduces the reference's rand() sequence instead)
extern "C" int spb_ctx_random_phase_models(spb_ctx *c, const unsigned long long *seeds, int reset_others) {
  if (upload(c, c->seeds, seeds, sizeof(unsigned long long) * (size_t)c->nb)) return -1;
  random_phase_spectra_kernel<<<1184, 256, 0, c->st>>>(c->T, c->amp, c->seeds, c->n, c->nb);
  CK(cudaGetLastError());
  c->launches++;
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
  zero_unmeasured_kernel<<<592, 256, 0, c->st>>>(c->T, c->flags, c->ntot);
  CK(cudaGetLastError());
  if (inverse_scaled_into_model(c)) return -1;
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

// whether the persistent form applies to this context and algorithm
static bool persist_wanted_shape(const spb_ctx *c, const spb_alg_desc *alg) {
  if (c->nz != 1 || c->nx != c->ny || (c->nx != 32 && c->nx != 64 && c->nx != 128)) return false;
  if (alg->algorithm == ALG_DM || alg->objective != 0 || (alg->constraints & C_MARGIN)) return false;
  return c->amp_line && c->meas_bits;
}

// The built-in choice between the persistent and the two-pass forms of a
// supported pattern: persistent for 32x32 and 64x64 patterns with at least
// one start per SM.  Measured on one B200 (HIO, calls of 20 iterations and an
// area update between them), start-iterations/s persistent / two-pass:
// 32x32 x 148 and 592 starts 1.46 and 1.30; 64x64 x 148, 296, 592 starts
// 1.11, 1.12, 1.27 but x 1 and 8 starts 0.84, 0.89 (one SM per start);
// 128x128 x 148 and 296 starts 0.99 (both forms at the same issue-bound
// pixel rate) and x 1, 8 starts 0.39, 0.40.
static bool persist_auto(const spb_ctx *c) {
  static int nsm = 0;
  if (!nsm && cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, 0) != cudaSuccess) nsm = 148;
  return c->nx <= 64 && c->nb >= nsm;
}

// One iteration of every start: g0 <- g1 (buffer roles swap), X -> Y
// (projection pass) -> row pass writing g1 and the next X.  `a` carries the
// algorithm scalars.
static int one_iteration(spb_ctx *c, PassArgs a, float2 *gp_out) {
  c->cur ^= 1;
  a.g0 = c->g[c->cur ^ 1];
  a.g1 = c->g[c->cur];
  a.gp = gp_out;
  if (middle(c, COL_PROJECT, c->X, c->Y, a)) return -1;
  if (a.alg == ALG_DM) {
    if (middle(c, COL_PROJECT_NOFC, c->Xf, c->Yf, a)) return -1;
    a.src = c->Y;
    a.src2 = c->Yf;
    a.dst = c->X;
    a.dst2 = c->Xf;
    return row(c, ROW_DM_ITER, a);
  }
  a.src = c->Y;
  a.dst = c->X;
  return row(c, ROW_ITER, a);
}

namespace spb {
__global__ void add_int_kernel(int *p, int v, int set) {
  if (set) *p = v;
  else *p += v;
}
}  // namespace spb

static bool same_alg(const GraphEntry &g, const spb_alg_desc *d) {
  return g.alg == d->algorithm && g.constraints == d->constraints && g.objective == d->objective &&
         g.gamma1 == d->gamma1 && g.gamma2 == d->gamma2;
}

// Graph of kGraphIters iterations reading beta from the device table at
// *beta_base + i, followed by beta_base += kGraphIters.  kGraphIters is even,
// so the iterate buffers return to their roles and the graph can be replayed.
// whole_n > 0: a graph of one whole call of whole_n iterations reading
// beta[i] (base pointer at a device 0), the last storing gp when keep_gp.
static int capture_graph(spb_ctx *c, const PassArgs &tmpl, GraphEntry &g, int whole_n = 0, int keep_gp = 0) {
  cudaGraph_t graph = nullptr;
  CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
  int rc = 0;
  const int cur0 = c->cur;
  const long long l0 = c->launches;
  const int n = whole_n > 0 ? whole_n : kGraphIters;
  for (int i = 0; i < n && !rc; i++) {
    PassArgs a = tmpl;
    a.beta_tab = c->beta_dev;
    a.beta_base = whole_n > 0 ? c->beta_zero : c->beta_base;
    a.beta_idx = i;
    rc = one_iteration(c, a, (keep_gp && i == n - 1) ? c->gp : nullptr);
  }
  if (!rc && whole_n == 0) {
    add_int_kernel<<<1, 1, 0, c->st>>>(c->beta_base, kGraphIters, 0);
    if (cudaGetLastError() != cudaSuccess) rc = fail("graph capture: kernel launch failed");
    c->launches++;
  }
  const cudaError_t ee = cudaStreamEndCapture(c->st, &graph);
  c->cur = cur0;
  g.nodes = c->launches - l0;
  g.n = whole_n;
  g.keep_gp = keep_gp;
  c->launches = l0;
  if (rc) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (ee != cudaSuccess) return fail("cudaStreamEndCapture: %s", cudaGetErrorString(ee));
  const cudaError_t ie = cudaGraphInstantiate(&g.exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ie != cudaSuccess) return fail("cudaGraphInstantiate: %s", cudaGetErrorString(ie));
  return 0;
}

static GraphEntry *find_graph(spb_ctx *c, const spb_alg_desc *d, int whole_n = 0, int keep_gp = 0) {
  for (auto &g : c->graphs)
    if (g.used && same_alg(g, d) && g.parity == c->cur && g.n == whole_n && (whole_n == 0 || g.keep_gp == keep_gp))
      return &g;
  return nullptr;
}

static GraphEntry *new_graph_slot(spb_ctx *c, const spb_alg_desc *d) {
  GraphEntry *slot = nullptr;
  for (auto &g : c->graphs)
    if (!g.used) {
      slot = &g;
      break;
    }
  if (!slot) {
    slot = &c->graphs[c->graph_evict];
    c->graph_evict = (c->graph_evict + 1) % kMaxGraphs;
    if (slot->exec) cudaGraphExecDestroy(slot->exec);
  }
  *slot = GraphEntry();
  slot->used = true;
  slot->alg = d->algorithm;
  slot->constraints = d->constraints;
  slot->objective = d->objective;
  slot->gamma1 = d->gamma1;
  slot->gamma2 = d->gamma2;
  slot->parity = c->cur;
  return slot;
}

// beta values of this call into the device table (pinned staging, reused
// only after the previous upload has completed).  The table has a fixed
// capacity (kBetaCap) allocated with the context: captured graphs hold its
// address.
static int upload_betas(spb_ctx *c, const float *beta, int n) {
  if (n > c->beta_cap) return fail("beta table holds %d iterations, %d requested", c->beta_cap, n);
  // the table already holds these values (in stream order): nothing to copy
  if (n <= (int)c->beta_shadow.size() && memcmp(beta, c->beta_shadow.data(), sizeof(float) * (size_t)n) == 0)
    return 0;
  int ev;
  float *stage;
  if (n <= kSmallBeta) {
    const int seg = c->beta_seg_small;
    c->beta_seg_small = (seg + 1) % kParamRing;
    ev = kLargeRing + seg;
    stage = c->beta_pinned + (size_t)kBetaCap * kLargeRing + (size_t)seg * kSmallBeta;
  } else {
    const int seg = c->beta_seg_large;
    c->beta_seg_large = (seg + 1) % kLargeRing;
    ev = seg;
    stage = c->beta_pinned + (size_t)seg * kBetaCap;
  }
  CK(cudaEventSynchronize(c->beta_ev[ev]));
  memcpy(stage, beta, sizeof(float) * (size_t)n);
  CK(cudaMemcpyAsync(c->beta_dev, stage, sizeof(float) * (size_t)n, cudaMemcpyHostToDevice, c->st));
  CK(cudaEventRecord(c->beta_ev[ev], c->st));
  c->beta_shadow.assign(beta, beta + n);
  return 0;
}

// The persistent form for this call: asked for (knob 2) or the built-in
// choice, on a 32x32, 64x64 or 128x128 pattern with HIO, RAAR or ER and the
// plain modulus projection (line-major operands built); never while per-kernel
// profiling is on.
static bool persist_wanted(const spb_ctx *c, const spb_alg_desc *alg) {
  const int k = c->tune[SPB_TUNE_PERSIST];
  if (k == 1 || c->prof.on || !persist_wanted_shape(c, alg)) return false;
  return k == 2 ? true : persist_auto(c);
}

extern "C" int spb_ctx_iterate(spb_ctx *c, const spb_alg_desc *alg, const float *beta, int iterations,
                               int keep_gp) {
  if (iterations <= 0) return 0;
  if (iterations > c->beta_cap) {
    // longer runs go through in table-sized pieces; gp only at the very end
    for (int off = 0; off < iterations; off += c->beta_cap) {
      const int k = iterations - off < c->beta_cap ? iterations - off : c->beta_cap;
      if (spb_ctx_iterate(c, alg, beta + off, k, keep_gp && off + k == iterations)) return -1;
    }
    return 0;
  }
  const int A = alg->algorithm;
  if (A < 1 || A > 4) return fail("unknown algorithm %d", A);
  if (alg->objective == 0 && !c->amp) return fail("amplitudes not set");
  if (alg->objective == 1 && !c->pamp) return fail("phased amplitudes not set");
  if ((alg->constraints & C_MARGIN) && (!c->amin || !c->amax)) return fail("amplitude margins not set");
  const size_t nc = sizeof(float2) * (size_t)c->ntot;
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
  a.inv_size_pow2 = (c->n & (c->n - 1)) == 0 ? (float)(1.0 / (double)c->n) : 0.0f;
  // small square patterns: every iteration of the call in one launch, one
  // block per start with its spectrum resident
  if (persist_wanted(c, alg)) {
    if (upload_betas(c, beta, iterations)) return -1;
    PassArgs p = a;
    p.beta_tab = c->beta_dev;
    p.beta_base = c->beta_zero;
    p.dst = c->X;
    p.gp = c->gp;
    CK(launch_persist(c->ax.lp, p, c->g[0], c->g[1], c->cur, iterations, keep_gp, c->nb, c->st));
    c->launches++;
    c->cur ^= (iterations & 1);
    c->xf_valid = 0;
    return 0;
  }
  // a short call (one support period, typically) runs as one captured graph
  if (c->use_graphs && !c->prof.on && c->warm_alg[A] && iterations >= 2 && iterations <= kWholeGraphMax) {
    GraphEntry *g = find_graph(c, alg, iterations, keep_gp);
    if (!g) {
      g = new_graph_slot(c, alg);
      if (capture_graph(c, a, *g, iterations, keep_gp)) {
        g->used = false;
        return -1;
      }
    }
    if (upload_betas(c, beta, iterations)) return -1;
    CK(cudaGraphLaunch(g->exec, c->st));
    c->launches += g->nodes;
    c->cur ^= (iterations & 1);
    if (A != ALG_DM) c->xf_valid = 0;
    return 0;
  }
  // iterations [0, ngraph) by graph replays, the rest launched directly (the
  // last one stores gp when asked)
  const int direct_tail = keep_gp ? 1 : 0;
  int ngraph = 0;
  if (c->use_graphs && !c->prof.on) ngraph = ((iterations - direct_tail) / kGraphIters) * kGraphIters;
  int it = 0;
  if (ngraph > 0) {
    GraphEntry *g = find_graph(c, alg);
    if (!g) {
      // kernels get their launch attributes from one direct iteration first
      if (!c->warm_alg[A]) {
        a.beta = (A == ALG_ER) ? 0.0f : beta[0];
        if (one_iteration(c, a, nullptr)) return -1;
        c->warm_alg[A] = 1;
        it = 1;
        ngraph = ((iterations - it - direct_tail) / kGraphIters) * kGraphIters;
      }
      if (ngraph > 0) {
        g = new_graph_slot(c, alg);
        if (capture_graph(c, a, *g)) {
          g->used = false;
          return -1;
        }
      }
    }
    if (ngraph > 0) {
      if (upload_betas(c, beta, iterations)) return -1;
      add_int_kernel<<<1, 1, 0, c->st>>>(c->beta_base, it, 1);
      CK(cudaGetLastError());
      c->launches++;
      for (int k = 0; k < ngraph; k += kGraphIters) {
        CK(cudaGraphLaunch(g->exec, c->st));
        c->launches += g->nodes;
      }
      it += ngraph;
    }
  }
  for (; it < iterations; it++) {
    a.beta = (A == ALG_ER) ? 0.0f : beta[it];
    if (one_iteration(c, a, (keep_gp && it == iterations - 1) ? c->gp : nullptr)) return -1;
    c->warm_alg[A] = 1;
  }
  if (A != ALG_DM) c->xf_valid = 0;
  return 0;
}

// the blur factor table of a's radius; a then looks factors up in it
static int gauss_table(spb_ctx *c, PassArgs &a) {
  a.blur_tab = nullptr;
  CK(launch_gauss_table(a, c->gtab, c->st));
  c->launches++;
  a.blur_tab = c->gtab;
  return 0;
}

// blur |g1| of every start (or |img| when img != nullptr) into c->absb
static int blur_abs(spb_ctx *c, const float2 *img, float radius, const double *r2_dev = nullptr) {
  PassArgs a = base_args(c);
  a.src = img ? img : c->g[c->cur];
  a.dst = c->T;
  if (row(c, ROW_FWD_DEPHASE, a)) return -1;
  a.blur_c0 = -2. * pow(3.14159265358979323846, 2);
  a.blur_r2 = pow((double)radius, 2);
  a.blur_r2_dev = r2_dev;
  if (gauss_table(c, a)) return -1;
  if (middle(c, COL_BLUR, c->T, c->T, a)) return -1;
  a.src = c->T;
  a.absout = c->absb;
  if (row(c, ROW_INV_ABS, a)) return -1;
  return 0;
}

// Area rule: threshold = k-th largest |blur| with k = (int)(N * area) (float
// product, as the reference indexes its descending sort); k is clamped to
// N-1 where the reference would read past the end.  Threshold rule: max|blur|
// times value.  Then inside = |blur| > threshold.  nb starts of n pixels,
// each with its own selection state.
static long long area_rank(long long n, float area) {
  long long k = (long long)(int)((float)n * area);
  if (k >= n) k = n - 1;
  if (k < 0) k = 0;
  return k;
}

// dev: when set, the rank (area rule) or the relative threshold is read from
// it at run time (captured support updates).  pdl: launch with programmatic
// dependent launch (context streams with it enabled).
static int select_and_mask_on(cudaStream_t st, SelectState *sel, const float *absv, long long n, int nb, int type,
                              float value, uint8_t *flags, const SupportParams *dev = nullptr, bool pdl = false,
                              bool cluster = false) {
  if (cluster && select_cluster_fits(n) && (type == SPB_SUPPORT_AREA || type == SPB_SUPPORT_THRESHOLD)) {
    const bool area = type == SPB_SUPPORT_AREA;
    const cudaError_t e = launch_select_mask_cluster(
        absv, n, nb, area ? 0 : 1, area ? (unsigned long long)area_rank(n, value) : 0ULL,
        area && dev ? &dev->rank : nullptr, area ? 0.0f : value, !area && dev ? &dev->rel : nullptr, sel, flags, st,
        pdl);
    if (e == cudaSuccess) return 0;
    if (e != cudaErrorNotSupported) CK(e);
  }
  if (type == SPB_SUPPORT_AREA) {
    CK(launch_select_kth_desc(absv, n, nb, area_rank(n, value), sel, st, dev ? &dev->rank : nullptr, pdl));
    CK(launch_mask_from_abs(absv, sel, 0.0f, 0, flags, n, nb, st, nullptr, pdl));
  } else if (type == SPB_SUPPORT_THRESHOLD) {
    CK(launch_max_abs(absv, n, nb, sel, st, pdl));
    CK(launch_mask_from_abs(absv, sel, value, 1, flags, n, nb, st, dev ? &dev->rel : nullptr, pdl));
  } else {
    return fail("unknown support update type %d", type);
  }
  return 0;
}

static int select_and_mask(spb_ctx *c, const float *absv, long long n, int nb, int type, float value,
                           uint8_t *flags, const SupportParams *dev = nullptr) {
  if (prof_begin(c)) return -1;
  const bool cluster = c->tune[SPB_TUNE_SELECT] == 2 && select_cluster_fits(n);
  if (select_and_mask_on(c->st, c->sel, absv, n, nb, type, value, flags, dev, c->tune[SPB_TUNE_NO_PDL] == 0, cluster))
    return -1;
  // one cluster launch | init, four histogram passes, mask | init, max, finish, mask
  c->launches += cluster ? 1 : (type == SPB_SUPPORT_AREA) ? 6 : 4;
  return prof_end(c, type == SPB_SUPPORT_AREA ? 16 : 17);
}

// support-update parameters into the device block (pinned staging ring; an
// unchanged block is not copied again)
static int upload_support_params(spb_ctx *c, const SupportParams &p) {
  if (c->spar_valid && memcmp(&p, &c->spar_shadow, sizeof(p)) == 0) return 0;
  const int seg = c->spar_seg;
  c->spar_seg = (seg + 1) % kParamRing;
  CK(cudaEventSynchronize(c->spar_ev[seg]));
  c->spar_pinned[seg] = p;
  CK(cudaMemcpyAsync(c->spar, c->spar_pinned + seg, sizeof(p), cudaMemcpyHostToDevice, c->st));
  CK(cudaEventRecord(c->spar_ev[seg], c->st));
  c->spar_shadow = p;
  c->spar_valid = true;
  return 0;
}

// The support update of every start; after a first direct run of a rule, it
// runs as a captured graph (one per rule and iterate parity) whose kernels
// read the blur radius and rank or threshold from the device block.
extern "C" int spb_ctx_support_update(spb_ctx *c, int type, float radius, float value) {
  if (type != SPB_SUPPORT_AREA && type != SPB_SUPPORT_THRESHOLD) return fail("unknown support update type %d", type);
  if (c->use_graphs && !c->prof.on && c->warm_sup[type]) {
    SupportParams p;
    memset(&p, 0, sizeof(p));
    p.r2 = pow((double)radius, 2);
    if (type == SPB_SUPPORT_AREA) p.rank = (unsigned long long)area_rank(c->n, value);
    else p.rel = value;
    if (upload_support_params(c, p)) return -1;
    SupportGraph &g = c->sup_graph[type][c->cur];
    if (!g.exec) {
      cudaGraph_t graph = nullptr;
      CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
      const long long l0 = c->launches;
      int rc = blur_abs(c, nullptr, radius, &c->spar->r2);
      if (!rc) rc = select_and_mask(c, c->absb, c->n, c->nb, type, value, c->flags, c->spar);
      const cudaError_t ee = cudaStreamEndCapture(c->st, &graph);
      g.nodes = c->launches - l0;
      c->launches = l0;
      if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
      }
      if (ee != cudaSuccess) return fail("cudaStreamEndCapture: %s", cudaGetErrorString(ee));
      const cudaError_t ie = cudaGraphInstantiate(&g.exec, graph, 0);
      cudaGraphDestroy(graph);
      if (ie != cudaSuccess) {
        g.exec = nullptr;
        return fail("cudaGraphInstantiate: %s", cudaGetErrorString(ie));
      }
    }
    CK(cudaGraphLaunch(g.exec, c->st));
    c->launches += g.nodes;
    c->xf_valid = 0;
    return 0;
  }
  if (blur_abs(c, nullptr, radius)) return -1;
  if (select_and_mask(c, c->absb, c->n, c->nb, type, value, c->flags)) return -1;
  c->warm_sup[type] = 1;
  c->xf_valid = 0;
  return 0;
}

// Patterson support of the shared pattern, computed once on start 0's slot
// and copied to every start.
extern "C" int spb_ctx_support_patterson(spb_ctx *c, float value) {
  const int nb = c->nb;
  const long long ntot = c->ntot;
  c->nb = 1;  // single-start geometry for the passes below
  c->ntot = c->n;
  int rc = 0;
  int axes[2];
  const int k = other_axes(c, axes);
  PassArgs a = base_args(c);
  a.f32src = c->amp;
  if (k == 0) {
    rc = col(c, 0, COL_INV_SQUARE_F32, nullptr, c->T, a);
  } else {
    rc = col(c, axes[k - 1], COL_INV_SQUARE_F32, nullptr, c->T, a);
    for (int i = k - 2; i >= 0 && !rc; i--) rc = col(c, axes[i], COL_INV, c->T, c->T, a);
  }
  a.src = c->T;
  a.absout = c->absb;
  if (!rc) rc = row(c, ROW_INV_ABS, a);
  if (!rc) rc = select_and_mask(c, c->absb, c->n, 1, SPB_SUPPORT_THRESHOLD, value, c->flags);
  c->nb = nb;
  c->ntot = ntot;
  if (rc) return -1;
  if (nb > 1) {
    broadcast_flags_kernel<<<592, 256, 0, c->st>>>(c->flags, c->n, nb, FLAG_INSIDE);
    CK(cudaGetLastError());
    c->launches++;
  }
  c->xf_valid = 0;
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

namespace spb {
// One dilation (dilate = 1) or erosion of the support bit of every start over
// the 6-neighbourhood; neighbours outside the start's array are left out.
// The other flag bits are copied unchanged.
__global__ void support_morph_kernel(const uint8_t *__restrict__ src, uint8_t *__restrict__ dst, int nx, int ny,
                                     int nz, long long n, long long ntot, int dilate) {
  const long long nxy = (long long)nx * ny;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < ntot; k += (long long)gridDim.x * blockDim.x) {
    const long long i = k % n;
    const int z = (int)(i / nxy), y = (int)((i % nxy) / nx), x = (int)(i % nx);
    const uint8_t c = src[k];
    bool in;
    if (dilate) {
      in = (c & FLAG_INSIDE) || (x > 0 && (src[k - 1] & FLAG_INSIDE)) || (x < nx - 1 && (src[k + 1] & FLAG_INSIDE)) ||
           (y > 0 && (src[k - nx] & FLAG_INSIDE)) || (y < ny - 1 && (src[k + nx] & FLAG_INSIDE)) ||
           (z > 0 && (src[k - nxy] & FLAG_INSIDE)) || (z < nz - 1 && (src[k + nxy] & FLAG_INSIDE));
    } else {
      in = (c & FLAG_INSIDE) && !(x > 0 && !(src[k - 1] & FLAG_INSIDE)) &&
           !(x < nx - 1 && !(src[k + 1] & FLAG_INSIDE)) && !(y > 0 && !(src[k - nx] & FLAG_INSIDE)) &&
           !(y < ny - 1 && !(src[k + nx] & FLAG_INSIDE)) && !(z > 0 && !(src[k - nxy] & FLAG_INSIDE)) &&
           !(z < nz - 1 && !(src[k + nxy] & FLAG_INSIDE));
    }
    dst[k] = in ? (uint8_t)(c | FLAG_INSIDE) : (uint8_t)(c & ~FLAG_INSIDE);
  }
}

// support bit of every start = absv[i] > t (absv holds one start's values)
__global__ void support_from_abs_kernel(const float *__restrict__ absv, float t, uint8_t *flags, long long n,
                                        long long ntot) {
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < ntot; k += (long long)gridDim.x * blockDim.x) {
    const uint8_t f = flags[k];
    flags[k] = absv[k % n] > t ? (uint8_t)(f | FLAG_INSIDE) : (uint8_t)(f & ~FLAG_INSIDE);
  }
}
}  // namespace spb

// Support closing of every start: `size` dilations, then `size` erosions.
// The passes alternate between the flags and a scratch copy held in the
// |blur| buffer (an even number of passes ends in the flags).
extern "C" int spb_ctx_support_close(spb_ctx *c, int size) {
  if (size < 0) return fail("negative closing size %d", size);
  uint8_t *scratch = reinterpret_cast<uint8_t *>(c->absb);
  for (int pass = 0; pass < 2 * size; pass++) {
    const uint8_t *src = (pass & 1) ? scratch : c->flags;
    uint8_t *dst = (pass & 1) ? c->flags : scratch;
    support_morph_kernel<<<1184, 256, 0, c->st>>>(src, dst, c->nx, c->ny, c->nz, c->n, c->ntot, pass < size);
    CK(cudaGetLastError());
    c->launches++;
  }
  c->xf_valid = 0;
  return 0;
}

// Support bit of every start = abs_values[i] > threshold, abs_values one
// start's values on the host (a fixed template).
extern "C" int spb_ctx_support_from_abs(spb_ctx *c, const float *abs_values, float threshold) {
  CK(cudaMemcpyAsync(c->absb, abs_values, sizeof(float) * (size_t)c->n, cudaMemcpyHostToDevice, c->st));
  support_from_abs_kernel<<<1184, 256, 0, c->st>>>(c->absb, threshold, c->flags, c->n, c->ntot);
  CK(cudaGetLastError());
  c->launches++;
  CK(cudaStreamSynchronize(c->st));
  c->xf_valid = 0;
  return 0;
}

// ---------------------------------------------------------------- autotuner
// Launch shapes chosen by measurement: for each candidate (row lines per
// block, programmatic dependent launch on or off) the context runs `calls`
// timed calls of `iterations` iterations of the given algorithm (graph
// replays, as in production) and keeps the fastest.  The model, iterates,
// support and parity are saved before and restored after, so tuning leaves the
// reconstruction where it was.  Choices are cached per process by (shape,
// starts, algorithm).
namespace {
struct TuneKey {
  int nx, ny, nz, nb, alg, constraints, objective;
  bool operator<(const TuneKey &o) const {
    const int a[7] = {nx, ny, nz, nb, alg, constraints, objective};
    const int b[7] = {o.nx, o.ny, o.nz, o.nb, o.alg, o.constraints, o.objective};
    for (int i = 0; i < 7; i++)
      if (a[i] != b[i]) return a[i] < b[i];
    return false;
  }
};
std::mutex g_tune_mu;
struct TuneChoice {
  int lines, nopdl, g0, split, persist, colw, tma;
};
std::map<TuneKey, TuneChoice> g_tune_cache;

int apply_choice(spb_ctx *c, const TuneChoice &t) {
  if (spb_ctx_set_tuning(c, SPB_TUNE_ROW_LINES, t.lines) || spb_ctx_set_tuning(c, SPB_TUNE_NO_PDL, t.nopdl) ||
      spb_ctx_set_tuning(c, SPB_TUNE_ROW_G0, t.g0) || spb_ctx_set_tuning(c, SPB_TUNE_SPLIT, t.split) ||
      spb_ctx_set_tuning(c, SPB_TUNE_PERSIST, t.persist) || spb_ctx_set_tuning(c, SPB_TUNE_COL_WIDTH, t.colw) ||
      spb_ctx_set_tuning(c, SPB_TUNE_TMA, t.tma))
    return -1;
  return 0;
}
}  // namespace

extern "C" int spb_ctx_autotune(spb_ctx *c, const spb_alg_desc *alg, int iterations, int calls, int force,
                                double *best_ms) {
  if (iterations < 2 || iterations > kWholeGraphMax) return fail("autotune: 2..%d iterations per call", kWholeGraphMax);
  if (calls < 1) calls = 1;
  const TuneKey key{c->nx, c->ny, c->nz, c->nb, alg->algorithm, alg->constraints, alg->objective};
  if (!force) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      if (best_ms) *best_ms = -1.0;
      return apply_choice(c, it->second);
    }
  }
  // save the state the timed iterations overwrite
  const size_t nc = sizeof(float2) * (size_t)c->ntot;
  float2 *save = nullptr;
  uint8_t *save_flags = nullptr;
  CK(cudaStreamSynchronize(c->st));
  CK(cudaMalloc(&save, 4 * nc));
  if (cudaMalloc(&save_flags, (size_t)c->ntot) != cudaSuccess) {
    cudaFree(save);
    return fail("autotune: no memory for the saved state");
  }
  const int cur0 = c->cur, xv0 = c->x_valid, xfv0 = c->xf_valid;
  const float xfg0 = c->xf_gamma1;
  const TuneChoice knob0{c->tune[SPB_TUNE_ROW_LINES], c->tune[SPB_TUNE_NO_PDL], c->tune[SPB_TUNE_ROW_G0],
                         c->tune[SPB_TUNE_SPLIT], c->tune[SPB_TUNE_PERSIST], c->tune[SPB_TUNE_COL_WIDTH],
                         c->tune[SPB_TUNE_TMA]};
  int rc = 0;
  const float2 *bufs[4] = {c->g[0], c->g[1], c->gp, c->X};
  for (int k = 0; k < 4 && !rc; k++)
    if (cudaMemcpyAsync(save + (size_t)k * c->ntot, bufs[k], nc, cudaMemcpyDeviceToDevice, c->st) != cudaSuccess)
      rc = fail("autotune: save failed");
  if (!rc && cudaMemcpyAsync(save_flags, c->flags, (size_t)c->ntot, cudaMemcpyDeviceToDevice, c->st) != cudaSuccess)
    rc = fail("autotune: save failed");
  std::vector<float> beta((size_t)iterations, 0.9f);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (!rc && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess))
    rc = fail("autotune: cudaEventCreate failed");
  const int T = c->nx >= 16 ? c->nx / 16 : 1;
  const int lpb_max = 256 / T > 0 ? 256 / T : 1;
  double best = 1e30;
  TuneChoice bestc{0, 0, 0, 0, 1, 0, 0};
  // 8-point kernels exist for these row (x) and projection-axis lengths
  auto split_len = [](int n) { return n == 256 || n == 512 || n == 1024 || n == 4096; };
  const int plen = c->nz > 1 ? c->nz : c->ny;
  const bool can_split = split_len(c->nx) || split_len(plen);
  const bool can_persist = persist_wanted_shape(c, alg);
  // time one candidate: the model, iterates and support are restored after the search
  auto time_choice = [&](const TuneChoice &t) {
    if (apply_choice(c, t)) {
      rc = -1;
      return;
    }
    // warm-up: a direct call, then the graph capture
    for (int w = 0; w < 2 && !rc; w++) rc = spb_ctx_iterate(c, alg, beta.data(), iterations, 1);
    if (rc) return;
    if (cudaEventRecord(e0, c->st) != cudaSuccess) rc = fail("autotune: event");
    for (int k = 0; k < calls && !rc; k++) rc = spb_ctx_iterate(c, alg, beta.data(), iterations, 1);
    if (!rc && cudaEventRecord(e1, c->st) != cudaSuccess) rc = fail("autotune: event");
    float ms = 0.0f;
    if (!rc && (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
      rc = fail("autotune: timing failed");
    if (!rc && ms < best) {
      best = ms;
      bestc = t;
    }
  };
  // 1. the two-pass launch shapes: row lines per block x dependent launch x
  //    g0 staging, and the 8-point passes (one block shape of their own)
  std::vector<TuneChoice> cands;
  for (int li = 0; li < 16; li++) {
    const int lines = li ? 1 << (li - 1) : 0;
    if (lines > lpb_max) continue;  // (0 is the built-in choice, which may be lpb_max or fewer)
    for (int sp = 1; sp <= 2; sp++) {
      if (sp == 2 && (!can_split || li != 0)) continue;
      for (int g0 = 1; g0 <= 2; g0++)
        for (int nopdl = 0; nopdl <= 1; nopdl++) cands.push_back(TuneChoice{lines, nopdl, g0, sp, 1, 0, 0});
    }
  }
  for (const TuneChoice &t : cands) {
    if (rc) break;
    time_choice(t);
  }
  // 2. with the best of those, the projection pass's columns per block
  //    (plain loads; the built-in width is timed above with its TMA tile
  //    where that fits, and here with plain loads too)
  if (!rc && bestc.split == 1) {
    const TuneChoice base = bestc;
    {
      TuneChoice t = base;
      t.tma = 1;
      time_choice(t);
    }
    for (int w = 1; w <= 16 && !rc; w <<= 1)
      if (col_width_ok(plen, w)) {
        TuneChoice t = base;
        t.colw = w;
        t.tma = 1;
        time_choice(t);
      }
  }
  // 3. the persistent form, where it applies (no launch-shape knobs)
  if (!rc && can_persist) time_choice(TuneChoice{0, 0, 1, 1, 2, 0, 0});
  // restore the state and apply the choice (or the previous knobs on error)
  for (int k = 0; k < 4; k++)
    cudaMemcpyAsync((void *)bufs[k], save + (size_t)k * c->ntot, nc, cudaMemcpyDeviceToDevice, c->st);
  cudaMemcpyAsync(c->flags, save_flags, (size_t)c->ntot, cudaMemcpyDeviceToDevice, c->st);
  cudaStreamSynchronize(c->st);
  cudaFree(save);
  cudaFree(save_flags);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  c->cur = cur0;
  c->x_valid = xv0;
  c->xf_valid = 0;  // the difference map's second transform is recomputed from the model
  (void)xfv0;
  (void)xfg0;
  if (rc) {
    apply_choice(c, knob0);
    return -1;
  }
  if (apply_choice(c, bestc)) return -1;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = bestc;
  }
  if (best_ms) *best_ms = best / (double)((size_t)calls * iterations);
  return 0;
}

static int fmodel_into_T(spb_ctx *c) {
  if (ensure_x(c)) return -1;
  return forward_rest(c, c->X, c->T);
}

extern "C" int spb_ctx_get_start_image(spb_ctx *c, int start, int which, float *out) {
  if (check_start(c, start)) return -1;
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
  return download(c, out, src + (size_t)start * c->n, nc);
}

extern "C" int spb_ctx_get_image(spb_ctx *c, int which, float *out) {
  return spb_ctx_get_start_image(c, 0, which, out);
}

// sums[b*4 + k] for every start
extern "C" int spb_ctx_batch_efourier_sums(spb_ctx *c, double *sums) {
  if (fmodel_into_T(c)) return -1;
  CK(launch_reduce_efourier(c->T, c->amp, c->flags, c->n, c->nb, c->red, c->st));
  c->launches += 2;
  return download(c, sums, c->red, sizeof(double) * 4 * (size_t)c->nb);
}

extern "C" int spb_ctx_batch_ereal_sums(spb_ctx *c, double *sums) {
  CK(launch_reduce_ereal(c->gp, c->flags, c->n, c->nb, c->red, c->st));
  c->launches += 2;
  return download(c, sums, c->red, sizeof(double) * 4 * (size_t)c->nb);
}

// counts[b] = pixels inside start b's support
extern "C" int spb_ctx_batch_support_counts(spb_ctx *c, long long *counts) {
  CK(launch_count_inside(c->flags, c->n, c->nb, c->red, c->st));
  c->launches += 2;
  std::vector<double> h((size_t)c->nb * 4);
  if (download(c, h.data(), c->red, sizeof(double) * h.size())) return -1;
  for (int b = 0; b < c->nb; b++) counts[b] = (long long)h[(size_t)b * 4];
  return 0;
}

extern "C" int spb_ctx_efourier_sums(spb_ctx *c, double sums[4]) {
  std::vector<double> h((size_t)c->nb * 4);
  if (spb_ctx_batch_efourier_sums(c, h.data())) return -1;
  for (int k = 0; k < 4; k++) sums[k] = h[k];
  return 0;
}

extern "C" int spb_ctx_ereal_sums(spb_ctx *c, double sums[2]) {
  std::vector<double> h((size_t)c->nb * 4);
  if (spb_ctx_batch_ereal_sums(c, h.data())) return -1;
  sums[0] = h[0];
  sums[1] = h[1];
  return 0;
}

namespace spb {
// ORs 1 into *flag when any of the n complex values is NaN or infinite
__global__ void nonfinite_kernel(const float2 *__restrict__ g, long long n, unsigned *flag) {
  unsigned bad = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 v = g[i];
    bad |= (isfinite(v.x) && isfinite(v.y)) ? 0u : 1u;
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1u);
}
}  // namespace spb

extern "C" int spb_ctx_nonfinite_async(spb_ctx *c, int reset, unsigned *host_flag) {
  if (!host_flag) return fail("spb_ctx_nonfinite_async: null flag");
  if (reset) CK(cudaMemsetAsync(c->nonfinite, 0, sizeof(unsigned), c->st));
  long long blocks = (c->ntot + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  nonfinite_kernel<<<(unsigned)blocks, 256, 0, c->st>>>(c->g[c->cur], c->ntot, c->nonfinite);
  CK(cudaGetLastError());
  c->launches++;
  CK(cudaMemcpyAsync(host_flag, c->nonfinite, sizeof(unsigned), cudaMemcpyDeviceToHost, c->st));
  return 0;
}

extern "C" int spb_ctx_support_count(spb_ctx *c, long long *count) {
  std::vector<long long> h((size_t)c->nb);
  if (spb_ctx_batch_support_counts(c, h.data())) return -1;
  *count = h[0];
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
    if (!rc && gauss_table(c, a)) rc = -1;
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
  if (select_and_mask_on(st, sel, dabs, n, 1, type, value, dflags)) return -1;
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

// ------------------------------------------- support mask without allocation
// spb_support_from_blur_noalloc: the same computation as
// spb_support_from_blur_host for callers that must not allocate device
// memory: a process whose HBM is reserved up front by another allocator (a
// framework's caching allocator, a serving loop's job pool), where a
// cudaMalloc of its own fails or fragments that pool, and latency-bound loops
// that cannot take cudaFree's device-wide synchronisation.  Its device
// scratch is one fixed file-scope array instead of per-call allocations.
//
// Scratch layout (byte offsets, each 256-aligned): the selection state, then
// blur (complex), |blur| (f32), the caller's int flags and their u8 form, each
// sized for kNoAllocMaxPixels.  Every call shares the array and finds the
// previous call's contents there: the selection launchers clear the state's
// histogram, prefix and rank before use, and every other region is written
// for the call's n pixels before it is read.  Calls that overlap on the GPU
// (from several host threads, or on several streams) race on the array.
namespace {
constexpr long long kNoAllocMaxPixels = 1LL << 16;  // 256 x 256
constexpr size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t kNaSel = 0;
constexpr size_t kNaBlur = align256(kNaSel + sizeof(SelectState));
constexpr size_t kNaAbs = align256(kNaBlur + sizeof(float2) * kNoAllocMaxPixels);
constexpr size_t kNaIntFlags = align256(kNaAbs + sizeof(float) * kNoAllocMaxPixels);
constexpr size_t kNaFlags = align256(kNaIntFlags + sizeof(int) * kNoAllocMaxPixels);
constexpr size_t kNoAllocScratchBytes = align256(kNaFlags + kNoAllocMaxPixels);  // 1,122,560 bytes
constexpr int kNoAllocMaxDevices = 64;
static_assert(kNoAllocScratchBytes == 1122560, "scratch size is stated in spb_device.h");
}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

static std::mutex g_noalloc_mu;
static unsigned char *g_noalloc_ptr[kNoAllocMaxDevices];

// Device address of the scratch array on the current device, looked up once
// per device (the first call on a device does this set-up).
static unsigned char *noalloc_scratch() {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    fail("cudaGetDevice: %s", cudaGetErrorString(e));
    return nullptr;
  }
  if (dev < 0 || dev >= kNoAllocMaxDevices) {
    fail("device %d is beyond the %d devices spb_support_from_blur_noalloc tracks", dev, kNoAllocMaxDevices);
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      fail("cudaGetSymbolAddress(scratch) on device %d: %s", dev, cudaGetErrorString(e));
      return nullptr;
    }
    g_noalloc_ptr[dev] = (unsigned char *)p;
  }
  return g_noalloc_ptr[dev];
}

namespace spb {
__global__ void flags_to_u8_kernel(const int *in, uint8_t *out, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = (uint8_t)(in[i] & 3);
}
__global__ void flags_to_int_kernel(const uint8_t *in, int *out, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = in[i];
}
}  // namespace spb

extern "C" int spb_support_from_blur_noalloc(long long n, const float *blur, int type, float value, int *flags) {
  if (n < 1) return fail("invalid size %lld", n);
  if (n > kNoAllocMaxPixels)
    return fail("%lld pixels exceed the %lld-pixel limit of spb_support_from_blur_noalloc (fixed %zu-byte device "
                "scratch); use spb_support_from_blur_host",
                n, kNoAllocMaxPixels, kNoAllocScratchBytes);
  if (type != SPB_SUPPORT_AREA && type != SPB_SUPPORT_THRESHOLD) return fail("unknown support update type %d", type);
  unsigned char *s = noalloc_scratch();
  if (!s) return -1;
  SelectState *sel = reinterpret_cast<SelectState *>(s + kNaSel);
  float2 *dblur = reinterpret_cast<float2 *>(s + kNaBlur);
  float *dabs = reinterpret_cast<float *>(s + kNaAbs);
  int *diflags = reinterpret_cast<int *>(s + kNaIntFlags);
  uint8_t *dflags = s + kNaFlags;
  const cudaStream_t st = 0;  // legacy default stream: no stream object is created
  // Every failure after the first enqueue waits for the work already queued,
  // so that no copy still reads or writes the caller's buffers (or the shared
  // scratch) once the call has returned.
  int rc = 0;
#define NA_CK(call)                                                      \
  do {                                                                   \
    cudaError_t e_ = (call);                                             \
    if (e_ != cudaSuccess) {                                             \
      rc = fail("%s: %s", #call, cudaGetErrorString(e_));                \
      goto drain;                                                        \
    }                                                                    \
  } while (0)
  NA_CK(cudaMemcpyAsync(dblur, blur, sizeof(float2) * (size_t)n, cudaMemcpyHostToDevice, st));
  NA_CK(cudaMemcpyAsync(diflags, flags, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, st));
  flags_to_u8_kernel<<<148, 256, 0, st>>>(diflags, dflags, n);
  abs_kernel<<<148, 256, 0, st>>>(dblur, dabs, n);
  NA_CK(cudaGetLastError());
  if (select_and_mask_on(st, sel, dabs, n, 1, type, value, dflags)) {
    rc = -1;
    goto drain;
  }
  flags_to_int_kernel<<<148, 256, 0, st>>>(dflags, diflags, n);
  NA_CK(cudaGetLastError());
  NA_CK(cudaMemcpyAsync(flags, diflags, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, st));
  NA_CK(cudaStreamSynchronize(st));
  return 0;
#undef NA_CK
drain:
  cudaStreamSynchronize(st);  // the error text of the first failure is kept
  return rc;
}

// ------------------------------------------------------------------ PRTF
// Phase-retrieval transfer function of n reconstructions, the reference's
// Python prtf (src/_spimage_prtf.py:17-106) on the device: each image after
// the first is superimposed on the running sum (sp_image_superimpose,
// src/image_util.c:2974-3007: cross-correlation of the moduli, optionally the
// convolution for the enantiomorph, argmax, reflection, wrap-around
// translation), phase-matched to it (sp_image_phase_match weighted by |sum|^2,
// src/image_util.c:3160-3186) and added; the PRTF is |mean of the unit
// phasors of the images' spectra|, zero where any spectrum vanishes.
namespace spb {
__global__ void prtf_modulus_kernel(const float2 *in, float2 *out, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = make_float2(cabs_ref(in[i]), 0.0f);
}
// C = A * conj(B) (correlation) or A * B (convolution), sp_cmul's operation order
__global__ void prtf_cmul_kernel(const float2 *A, const float2 *B, float2 *C, long long n, int conj) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 a = A[i];
    float2 b = B[i];
    if (conj) b.y = -b.y;
    C[i] = make_float2(fsub(fmul(a.x, b.x), fmul(a.y, b.y)), fadd(fmul(a.x, b.y), fmul(b.x, a.y)));
  }
}
// per block: largest |v*s| (sp_cscale then sp_cabs) and its first index
__global__ void prtf_argmax_kernel(const float2 *v, long long n, float s, float *bval, long long *bidx) {
  float best = -1.0f;
  long long bi = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 x = v[i];
    const float m = cabs_ref(make_float2(fmul(x.x, s), fmul(x.y, s)));
    if (m > best) {
      best = m;
      bi = i;
    }
  }
  __shared__ float sv[256];
  __shared__ long long si[256];
  sv[threadIdx.x] = best;
  si[threadIdx.x] = bi;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      const float o = sv[threadIdx.x + w];
      const long long oi = si[threadIdx.x + w];
      if (o > sv[threadIdx.x] || (o == sv[threadIdx.x] && oi < si[threadIdx.x])) {
        sv[threadIdx.x] = o;
        si[threadIdx.x] = oi;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    bval[blockIdx.x] = sv[0];
    bidx[blockIdx.x] = si[0];
  }
}
// sp_image_reflect(SP_ORIGO) of the data (not the mask): both axes in 2-D; in
// 3-D every plane mirrored through the centre except, for an odd depth, the
// middle plane, which the reference's pairwise swap loop leaves unchanged
__global__ void prtf_reflect_kernel(const float2 *in, float2 *out, int nx, int ny, int nz) {
  const long long n = (long long)nx * ny * nz;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / ((long long)nx * ny));
    if (nz > 1 && (nz & 1) && z == (nz - 1) / 2) {
      out[i] = in[i];
    } else {
      const int zz = nz > 1 ? nz - 1 - z : z;
      out[i] = in[((long long)zz * ny + (ny - 1 - y)) * nx + (nx - 1 - x)];
    }
  }
}
// wrap-around translation by (dx,dy,dz) of data and mask (sp_image_translate)
__global__ void prtf_translate_kernel(const float2 *in, const int *min_, float2 *out, int *mout, int nx, int ny,
                                      int nz, int dx, int dy, int dz) {
  const long long n = (long long)nx * ny * nz;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / ((long long)nx * ny));
    const int sx = ((x - dx) % nx + nx) % nx, sy = ((y - dy) % ny + ny) % ny, sz = ((z - dz) % nz + nz) % nz;
    const long long s = ((long long)sz * ny + sy) * nx + sx;
    out[i] = in[s];
    mout[i] = min_[s];
  }
}
// phase match: sum of |a|^2 exp(i(arg a - arg b)) (sums in double)
__global__ void prtf_phase_sum_kernel(const float2 *a, const float2 *b, long long n, double *part) {
  double sx = 0.0, sy = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 av = a[i], bv = b[i];
    const float angle = (float)(atan2((double)av.y, (double)av.x) - atan2((double)bv.y, (double)bv.x));
    const float mag = fadd(fmul(av.x, av.x), fmul(av.y, av.y));
    sx += (double)(float)(cos((double)angle) * mag);
    sy += (double)(float)(sin((double)angle) * mag);
  }
  __shared__ double s0[256], s1[256];
  s0[threadIdx.x] = sx;
  s1[threadIdx.x] = sy;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      s0[threadIdx.x] += s0[threadIdx.x + w];
      s1[threadIdx.x] += s1[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = s0[0];
    part[2 * blockIdx.x + 1] = s1[0];
  }
}
__global__ void prtf_phase_apply_kernel(float2 *b, long long n, float phi) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 v = b[i];
    const float angle = (float)(atan2((double)v.y, (double)v.x) + (double)phi);
    const float mag = cabs_ref(v);
    b[i] = make_float2((float)(cos((double)angle) * mag), (float)(sin((double)angle) * mag));
  }
}
// sum += img (sp_image_add); counts[mask == 0] += 1 when the support is not empty
__global__ void prtf_add_kernel(float2 *sum, const float2 *img, const int *mask, float *counts, long long n,
                                int count_mask) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 s = sum[i], v = img[i];
    sum[i] = make_float2(fadd(s.x, v.x), fadd(s.y, v.y));
    if (count_mask && mask[i] == 0) counts[i] = fadd(counts[i], 1.0f);
  }
}
// unit phasors of a spectrum into the phasor sum; spectra that vanish count zeros
__global__ void prtf_phasor_kernel(const float2 *F, float2 *sum, int *zeros, long long n, int init) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 f = F[i];
    const float m = cabs_ref(f);
    float2 u = make_float2(0.0f, 0.0f);
    if (m > 0.0f) u = make_float2(__fdiv_rn(f.x, m), __fdiv_rn(f.y, m));
    if (init) {
      sum[i] = u;
      zeros[i] = m > 0.0f ? 0 : 1;
    } else {
      const float2 s = sum[i];
      sum[i] = make_float2(fadd(s.x, u.x), fadd(s.y, u.y));
      if (!(m > 0.0f)) zeros[i] += 1;
    }
  }
}
__global__ void prtf_final_kernel(const float2 *sum, const int *zeros, const float *counts, float *prtf, int *smask,
                                  long long n, float nimg) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 s = sum[i];
    const float2 v = make_float2(__fdiv_rn(s.x, nimg), __fdiv_rn(s.y, nimg));
    prtf[i] = zeros[i] > 0 ? 0.0f : cabs_ref(v);
    smask[i] = counts[i] > 0.0f ? 1 : 0;
  }
}
}  // namespace spb

namespace {
// forward / backward unnormalised transform of a whole context-sized buffer
int prtf_fft(spb_ctx *c, const float2 *src, float2 *dst, int sign) {
  PassArgs a = base_args(c);
  if (sign < 0) {
    a.src = src;
    a.dst = dst;
    if (row(c, ROW_FWD, a)) return -1;
    return forward_rest(c, dst, dst);
  }
  if (backward_rest(c, src, c->T)) return -1;
  a.src = c->T;
  a.dst = dst;
  return row(c, ROW_INV, a);
}

// largest |v * s| and its first index
int prtf_argmax(spb_ctx *c, const float2 *v, float s, float *bval, long long *bidx, float *hval, long long *hidx,
                float *best, long long *best_i) {
  const int nblk = 296;
  prtf_argmax_kernel<<<nblk, 256, 0, c->st>>>(v, c->n, s, bval, bidx);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(hval, bval, sizeof(float) * nblk, cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(hidx, bidx, sizeof(long long) * nblk, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  float bv = -1.0f;
  long long bi = 0;
  for (int k = 0; k < nblk; k++)
    if (hval[k] > bv || (hval[k] == bv && hidx[k] < bi)) {
      bv = hval[k];
      bi = hidx[k];
    }
  *best = bv;
  *best_i = bi;
  return 0;
}
}  // namespace

extern "C" int spb_prtf_host(int nx, int ny, int nz, int n, const float *images, const int *supports, int flags,
                             float *prtf, float *super_image, int *super_mask) {
  if (n < 1) return fail("prtf of %d images", n);
  spb_ctx *c = nullptr;
  if (spb_ctx_create(&c, nx, ny, nz)) return -1;
  const long long N = c->n;
  const size_t nc = sizeof(float2) * (size_t)N;
  const int nblk = 296;
  float2 *scratch = nullptr;
  int *mask = nullptr, *mask2 = nullptr, *zeros = nullptr, *smask = nullptr;
  float *counts = nullptr, *bval = nullptr, *dprtf = nullptr;
  long long *bidx = nullptr;
  double *part = nullptr;
  std::vector<float> hval(nblk);
  std::vector<long long> hidx(nblk);
  std::vector<double> hpart(2 * nblk);
  int rc = 0;
  auto alloc = [&](void **p, size_t bytes) {
    if (!rc && cudaMalloc(p, bytes) != cudaSuccess) rc = fail("prtf: cudaMalloc(%zu) failed", bytes);
  };
  alloc((void **)&scratch, nc);
  alloc((void **)&mask, sizeof(int) * N);
  alloc((void **)&mask2, sizeof(int) * N);
  alloc((void **)&zeros, sizeof(int) * N);
  alloc((void **)&smask, sizeof(int) * N);
  alloc((void **)&counts, sizeof(float) * N);
  alloc((void **)&dprtf, sizeof(float) * N);
  alloc((void **)&bval, sizeof(float) * nblk);
  alloc((void **)&bidx, sizeof(long long) * nblk);
  alloc((void **)&part, sizeof(double) * 2 * nblk);
  float2 *avg = c->g[0], *img = c->g[1], *A = c->X, *B = c->Y, *C = c->T, *sum = c->gp;
  const float inv_n = (float)(1.0 / (double)N);
  const int translate = flags & 1, enantio = flags & 2;
  // image 0: the running sum and the first unit phasors
  if (!rc && cudaMemcpyAsync(avg, images, nc, cudaMemcpyHostToDevice, c->st) != cudaSuccess) rc = fail("prtf: upload");
  if (!rc && cudaMemsetAsync(counts, 0, sizeof(float) * N, c->st) != cudaSuccess) rc = fail("prtf: memset");
  if (!rc) rc = prtf_fft(c, avg, scratch, -1);
  if (!rc) {
    prtf_phasor_kernel<<<1184, 256, 0, c->st>>>(scratch, sum, zeros, N, 1);
    if (cudaGetLastError() != cudaSuccess) rc = fail("prtf: phasor kernel");
  }
  for (int i = 1; i < n && !rc; i++) {
    const float *hi = images + 2 * (size_t)N * i;
    const int *hm = supports + (size_t)N * i;
    long long msum = 0;
    for (long long k = 0; k < N; k++) msum += hm[k];
    if (cudaMemcpyAsync(img, hi, nc, cudaMemcpyHostToDevice, c->st) != cudaSuccess ||
        cudaMemcpyAsync(mask, hm, sizeof(int) * N, cudaMemcpyHostToDevice, c->st) != cudaSuccess) {
      rc = fail("prtf: upload");
      break;
    }
    if (translate) {
      // cross-correlation and (optionally) convolution of the moduli
      prtf_modulus_kernel<<<1184, 256, 0, c->st>>>(avg, scratch, N);
      if (prtf_fft(c, scratch, A, -1)) { rc = -1; break; }
      prtf_modulus_kernel<<<1184, 256, 0, c->st>>>(img, scratch, N);
      if (prtf_fft(c, scratch, B, -1)) { rc = -1; break; }
      prtf_cmul_kernel<<<1184, 256, 0, c->st>>>(A, B, scratch, N, 1);
      if (prtf_fft(c, scratch, C, 1)) { rc = -1; break; }
      float m1, m2 = -1.0f;
      long long i1, i2 = 0;
      if (prtf_argmax(c, C, inv_n, bval, bidx, hval.data(), hidx.data(), &m1, &i1)) { rc = -1; break; }
      long long x = i1 % nx, y = (i1 / nx) % ny, z = i1 / ((long long)nx * ny);
      bool reflect = false;
      if (enantio) {
        prtf_cmul_kernel<<<1184, 256, 0, c->st>>>(A, B, scratch, N, 0);
        if (prtf_fft(c, scratch, C, 1)) { rc = -1; break; }
        if (prtf_argmax(c, C, inv_n, bval, bidx, hval.data(), hidx.data(), &m2, &i2)) { rc = -1; break; }
        if (m2 > m1) {
          reflect = true;
          x = i2 % nx + 1;
          y = (i2 / nx) % ny + 1;
          z = i2 / ((long long)nx * ny) + 1;
        }
      }
      if (reflect) {
        prtf_reflect_kernel<<<1184, 256, 0, c->st>>>(img, scratch, nx, ny, nz);
        if (cudaMemcpyAsync(img, scratch, nc, cudaMemcpyDeviceToDevice, c->st) != cudaSuccess) { rc = fail("prtf"); break; }
      }
      prtf_translate_kernel<<<1184, 256, 0, c->st>>>(img, mask, scratch, mask2, nx, ny, nz, (int)x, (int)y, (int)z);
      if (cudaMemcpyAsync(img, scratch, nc, cudaMemcpyDeviceToDevice, c->st) != cudaSuccess ||
          cudaMemcpyAsync(mask, mask2, sizeof(int) * N, cudaMemcpyDeviceToDevice, c->st) != cudaSuccess) {
        rc = fail("prtf: translate");
        break;
      }
      // phase match to the running sum
      prtf_phase_sum_kernel<<<nblk, 256, 0, c->st>>>(avg, img, N, part);
      if (cudaMemcpyAsync(hpart.data(), part, sizeof(double) * 2 * nblk, cudaMemcpyDeviceToHost, c->st) != cudaSuccess ||
          cudaStreamSynchronize(c->st) != cudaSuccess) {
        rc = fail("prtf: phase sum");
        break;
      }
      double sx = 0.0, sy = 0.0;
      for (int k = 0; k < nblk; k++) {
        sx += hpart[2 * k];
        sy += hpart[2 * k + 1];
      }
      const float phi = (float)atan2((double)(float)sy, (double)(float)sx);
      prtf_phase_apply_kernel<<<1184, 256, 0, c->st>>>(img, N, phi);
    }
    prtf_add_kernel<<<1184, 256, 0, c->st>>>(avg, img, mask, counts, N, msum > 0);
    if (prtf_fft(c, img, scratch, -1)) { rc = -1; break; }
    prtf_phasor_kernel<<<1184, 256, 0, c->st>>>(scratch, sum, zeros, N, 0);
    if (cudaGetLastError() != cudaSuccess) rc = fail("prtf: kernel launch failed");
  }
  if (!rc) {
    prtf_final_kernel<<<1184, 256, 0, c->st>>>(sum, zeros, counts, dprtf, smask, N, (float)n);
    if (cudaGetLastError() != cudaSuccess) rc = fail("prtf: kernel launch failed");
  }
  if (!rc && prtf && cudaMemcpyAsync(prtf, dprtf, sizeof(float) * N, cudaMemcpyDeviceToHost, c->st) != cudaSuccess)
    rc = fail("prtf: download");
  if (!rc && super_image && cudaMemcpyAsync(super_image, avg, nc, cudaMemcpyDeviceToHost, c->st) != cudaSuccess)
    rc = fail("prtf: download");
  if (!rc && super_mask && cudaMemcpyAsync(super_mask, smask, sizeof(int) * N, cudaMemcpyDeviceToHost, c->st) != cudaSuccess)
    rc = fail("prtf: download");
  if (!rc && cudaStreamSynchronize(c->st) != cudaSuccess) rc = fail("prtf: device error");
  void *ptrs[] = {scratch, mask, mask2, zeros, smask, counts, dprtf, bval, bidx, part};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  spb_ctx_destroy(c);
  return rc;
}

// --------------------------------- fractional superposition and the C PRTFs
// sp_image_superimpose_fractional (src/image_util.c:3024-3066), sp_prtf_basic
// and sp_prtf_advanced (src/prtf.c:6-78) on the device.  The correlation
// surfaces are the reference's bit for bit (same FFTs, same products and
// scaling), so the argmax, the enantiomorph choice and the translation are the
// reference's; the phase of the peak is taken on the host with the C library's
// atan2 from the same float values.  The Fourier translation and the phase
// shift evaluate cos, sin and atan2 in double on the GPU (the reference calls
// the C library), so those steps agree to rounding, not always bit for bit.
namespace spb {
// zero_pad_shifted_image: source index along one axis of length n padded to p
// (the spectrum split through its middle into the corners), -1 for a new zero
__device__ __forceinline__ int pad_src(int x, int n, int p) {
  if ((double)x < n / 2.0) return x;
  if ((double)(p - x - 1) < (n - 1) / 2.0) return (n - 1) - (p - x - 1);
  return -1;
}
__global__ void pad_shifted_kernel(const float2 *in, float2 *out, int nx, int ny, int nz, int px, int py, int pz) {
  const long long n = (long long)px * py * pz;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % px), y = (int)((i / px) % py), z = (int)(i / ((long long)px * py));
    const int sx = pad_src(x, nx, px), sy = pad_src(y, ny, py), sz = pad_src(z, nz, pz);
    out[i] = (sx < 0 || sy < 0 || sz < 0) ? make_float2(0.0f, 0.0f) : in[((long long)sz * ny + sy) * nx + sx];
  }
}
__global__ void conj_kernel(float2 *v, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    v[i].y = -v[i].y;
}
// sp_image_fourier_translate's multiplier (src/image_util.c:3249-3290): the
// phase f_x*t_x*(1/nx)*2pi + f_y*t_y*(1/ny)*2pi + f_z*t_z*(1/nz)*2pi in float,
// left to right, with f = k for k < n/2 else k - n (an axis of length 1 has
// f = -1); (cos, -sin) in double rounded to float; sp_cmul's operation order
__global__ void fourier_translate_kernel(float2 *F, int nx, int ny, int nz, float tx, float ty, float tz, float nxi,
                                         float nyi, float nzi, float two_pi) {
  const long long n = (long long)nx * ny * nz;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / ((long long)nx * ny));
    const int fx = x < nx / 2 ? x : -(nx - x), fy = y < ny / 2 ? y : -(ny - y), fz = z < nz / 2 ? z : -(nz - z);
    const float ax = fmul(fmul(fmul((float)fx, tx), nxi), two_pi);
    const float ay = fmul(fmul(fmul((float)fy, ty), nyi), two_pi);
    const float az = fmul(fmul(fmul((float)fz, tz), nzi), two_pi);
    const float arg = fadd(fadd(ax, ay), az);
    const float c = (float)cos((double)arg), s = (float)(-sin((double)arg));
    const float2 a = F[i];
    F[i] = make_float2(fsub(fmul(a.x, c), fmul(a.y, s)), fadd(fmul(a.x, s), fmul(c, a.y)));
  }
}
// sp_image_phase_shift in place (src/image_util.c:3413-3426)
__global__ void phase_shift_kernel(float2 *v, long long n, float phi) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 a = v[i];
    const float mag = cabs_ref(a);
    const float arg = (float)atan2((double)a.y, (double)a.x);
    const float t = fadd(arg, phi);
    v[i] = make_float2((float)((double)mag * cos((double)t)), (float)((double)mag * sin((double)t)));
  }
}
// sp_prtf_basic (src/prtf.c:6-34): per pixel the sum of the n images (added
// in order to zeros) and the sum of their moduli; the sum scaled by 1/that
// where it is not zero
__global__ void prtf_basic_kernel(const float2 *imgs, long long N, int n, float2 *out) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    float2 s = make_float2(0.0f, 0.0f);
    float div = 0.0f;
    for (int j = 0; j < n; j++) {
      const float2 v = imgs[(long long)j * N + i];
      s = make_float2(fadd(s.x, v.x), fadd(s.y, v.y));
    }
    for (int j = 0; j < n; j++) div = fadd(div, cabs_ref(imgs[(long long)j * N + i]));
    if (div != 0.0f) {
      const float sc = (float)__ddiv_rn(1.0, (double)div);  // 1.0/div in double, passed on as float
      s = make_float2(fmul(s.x, sc), fmul(s.y, sc));
    }
    out[i] = s;
  }
}
}  // namespace spb

namespace {
struct Superimposer {
  spb_ctx *c = nullptr;   // the images' size
  spb_ctx *cp = nullptr;  // the padded correlation size
  float2 *PA = nullptr, *PB = nullptr, *PC = nullptr, *U = nullptr;
  float *bval = nullptr;
  long long *bidx = nullptr;
  std::vector<float> hval;
  std::vector<long long> hidx;
  int precision = 1, pz = 1;
  ~Superimposer() {
    for (void *p : {(void *)PA, (void *)PB, (void *)PC, (void *)U, (void *)bval, (void *)bidx})
      if (p) cudaFree(p);
    spb_ctx_destroy(cp);
    spb_ctx_destroy(c);
  }
  int init(int nx, int ny, int nz, int prec) {
    if (prec < 1) return fail("superposition precision %d", prec);
    precision = prec;
    pz = nz > 1 ? prec : 1;  // 2-D images are not padded along z
    if (spb_ctx_create(&c, nx, ny, nz) || spb_ctx_create(&cp, nx * prec, ny * prec, nz * pz)) return -1;
    cp->st = c->st;  // one stream for both
    const size_t np = sizeof(float2) * (size_t)cp->n;
    CK(cudaMalloc(&PA, np));
    CK(cudaMalloc(&PB, np));
    CK(cudaMalloc(&PC, np));
    CK(cudaMalloc(&U, sizeof(float2) * (size_t)c->n));
    CK(cudaMalloc(&bval, sizeof(float) * 296));
    CK(cudaMalloc(&bidx, sizeof(long long) * 296));
    hval.resize(296);
    hidx.resize(296);
    return 0;
  }
  // sp_image_fft of an image, padded into the correlation grid
  int padded_spectrum(const float2 *img, float2 *out) {
    if (prtf_fft(c, img, U, -1)) return -1;
    pad_shifted_kernel<<<1184, 256, 0, c->st>>>(U, out, c->nx, c->ny, c->nz, cp->nx, cp->ny, cp->nz);
    CK(cudaGetLastError());
    return 0;
  }
  // sp_image_convolute_fractional (src/image_util.c:1380-1461) of the padded
  // spectra, then sp_image_max: largest modulus of the scaled surface, its
  // first index and the scaled value there
  int overlap(int conj, float *best, long long *best_i, float2 *val) {
    prtf_cmul_kernel<<<1184, 256, 0, c->st>>>(PA, PB, PC, cp->n, conj);
    CK(cudaGetLastError());
    if (prtf_fft(cp, PC, PC, 1)) return -1;
    const float s = (float)(1.0 / (double)c->n);  // the input's size scales, not the padded one
    if (prtf_argmax(cp, PC, s, bval, bidx, hval.data(), hidx.data(), best, best_i)) return -1;
    float2 raw;  // (prtf_argmax has synchronised the stream)
    CK(cudaMemcpyAsync(&raw, PC + *best_i, sizeof(float2), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    *val = make_float2(raw.x * s, raw.y * s);
    return 0;
  }
  // superimposes b (device, the images' size) on a: src/image_util.c:3024-3066
  int run(const float2 *a, float2 *b, int flags) {
    if (padded_spectrum(a, PA) || padded_spectrum(b, PB)) return -1;
    float m1, m2;
    long long i1, i2;
    float2 v1, v2;
    if (overlap(1, &m1, &i1, &v1)) return -1;
    const long long pxy = (long long)cp->nx * cp->ny;
    int x = (int)(i1 % cp->nx), y = (int)((i1 % pxy) / cp->nx), z = (int)(i1 / pxy);
    float phase = (float)atan2((double)v1.y, (double)v1.x);
    bool flip = false;
    if (flags & 1) {  // SpEnantiomorph
      if (overlap(0, &m2, &i2, &v2)) return -1;
      if (m2 > m1) {
        x = (int)(i2 % cp->nx) + precision;
        y = (int)((i2 % pxy) / cp->nx) + precision;
        z = (int)(i2 / pxy) + precision;
        phase = (float)atan2((double)v2.y, (double)v2.x);
        flip = true;
      }
    }
    if (flip) {  // the enantiomorph: reflected through the origin and conjugated
      prtf_reflect_kernel<<<1184, 256, 0, c->st>>>(b, U, c->nx, c->ny, c->nz);
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(b, U, sizeof(float2) * (size_t)c->n, cudaMemcpyDeviceToDevice, c->st));
      conj_kernel<<<1184, 256, 0, c->st>>>(b, c->n);
      CK(cudaGetLastError());
    }
    // sp_image_fourier_translate(b, x/p, y/p, z/p)
    if (prtf_fft(c, b, U, -1)) return -1;
    const float two_pi = (float)(2 * M_PI);
    fourier_translate_kernel<<<1184, 256, 0, c->st>>>(
        U, c->nx, c->ny, c->nz, (float)x / (float)precision, (float)y / (float)precision, (float)z / (float)precision,
        (float)(1.0 / c->nx), (float)(1.0 / c->ny), (float)(1.0 / c->nz), two_pi);
    CK(cudaGetLastError());
    if (prtf_fft(c, U, b, 1)) return -1;
    CK(launch_scale_cmul(b, c->n, (float)(1.0 / (double)c->n), c->st));  // sp_image_scale
    if (flags & 2) {  // SpCorrectPhaseShift
      phase_shift_kernel<<<1184, 256, 0, c->st>>>(b, c->n, phase);
      CK(cudaGetLastError());
    }
    return 0;
  }
};
}  // namespace

extern "C" int spb_superimpose_fractional_host(int nx, int ny, int nz, const float *a, float *b, int flags,
                                               int precision) {
  Superimposer s;
  if (s.init(nx, ny, nz, precision)) return -1;
  const size_t nc = sizeof(float2) * (size_t)s.c->n;
  float2 *da = nullptr, *db = nullptr;
  int rc = 0;
  if (cudaMalloc(&da, nc) != cudaSuccess || cudaMalloc(&db, nc) != cudaSuccess) rc = fail("superimpose: cudaMalloc");
  // everything on the context's stream (non-blocking: the legacy stream
  // would not wait for it)
  if (!rc && (cudaMemcpyAsync(da, a, nc, cudaMemcpyHostToDevice, s.c->st) != cudaSuccess ||
              cudaMemcpyAsync(db, b, nc, cudaMemcpyHostToDevice, s.c->st) != cudaSuccess))
    rc = fail("superimpose: upload");
  if (!rc) rc = s.run(da, db, flags);
  if (!rc && cudaMemcpyAsync(b, db, nc, cudaMemcpyDeviceToHost, s.c->st) != cudaSuccess) rc = fail("superimpose: download");
  if (cudaStreamSynchronize(s.c->st) != cudaSuccess && !rc) rc = fail("superimpose: device error");
  if (da) cudaFree(da);
  if (db) cudaFree(db);
  return rc;
}

extern "C" int spb_prtf_basic_host(int nx, int ny, int nz, int n, const float *images, float *out) {
  if (n < 1) return fail("prtf of %d images", n);
  const long long N = (long long)nx * ny * nz;
  if (N < 1) return fail("invalid image size");
  float2 *d = nullptr, *o = nullptr;
  int rc = 0;
  if (cudaMalloc(&d, sizeof(float2) * (size_t)(N * n)) != cudaSuccess || cudaMalloc(&o, sizeof(float2) * (size_t)N) != cudaSuccess)
    rc = fail("prtf_basic: cudaMalloc");
  if (!rc && cudaMemcpy(d, images, sizeof(float2) * (size_t)(N * n), cudaMemcpyHostToDevice) != cudaSuccess)
    rc = fail("prtf_basic: upload");
  if (!rc) {
    prtf_basic_kernel<<<1184, 256>>>(d, N, n, o);
    if (cudaGetLastError() != cudaSuccess) rc = fail("prtf_basic: launch");
  }
  if (!rc && cudaMemcpy(out, o, sizeof(float2) * (size_t)N, cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = fail("prtf_basic: download");
  if (d) cudaFree(d);
  if (o) cudaFree(o);
  return rc;
}

extern "C" int spb_prtf_advanced_host(int nx, int ny, int nz, int n, float *images, int space, int write_back,
                                      float *prtf) {
  if (n < 1) return fail("prtf of %d images", n);
  if (space != 1 && space != 2) return fail("prtf_advanced: space must be 1 (Fourier) or 2 (real)");
  Superimposer s;
  if (s.init(nx, ny, nz, 4)) return -1;
  spb_ctx *c = s.c;
  const long long N = c->n;
  const size_t all = sizeof(float2) * (size_t)(N * n);
  float2 *R = nullptr, *F = nullptr, *o = nullptr;
  int rc = 0;
  if (cudaMalloc(&R, all) != cudaSuccess || cudaMalloc(&F, all) != cudaSuccess ||
      cudaMalloc(&o, sizeof(float2) * (size_t)N) != cudaSuccess)
    rc = fail("prtf_advanced: cudaMalloc");
  if (!rc && cudaMemcpyAsync(R, images, all, cudaMemcpyHostToDevice, c->st) != cudaSuccess) rc = fail("prtf_advanced: upload");
  // images in Fourier space: their unnormalised inverse transforms (sp_image_ifft)
  for (int i = 0; i < n && !rc && space == 1; i++) rc = prtf_fft(c, R + (size_t)i * N, R + (size_t)i * N, 1);
  // every image superimposed on the first (SpCorrectPhaseShift | SpEnantiomorph, precision 4)
  for (int i = 1; i < n && !rc; i++) rc = s.run(R, R + (size_t)i * N, 3);
  // spectra scaled by 1/N (sp_image_fft, sp_image_scale), then sp_prtf_basic
  for (int i = 0; i < n && !rc; i++) {
    rc = prtf_fft(c, R + (size_t)i * N, F + (size_t)i * N, -1);
    if (!rc && launch_scale_cmul(F + (size_t)i * N, N, (float)(1.0 / (double)N), c->st) != cudaSuccess)
      rc = fail("prtf_advanced: scale");
  }
  if (!rc) {
    prtf_basic_kernel<<<1184, 256, 0, c->st>>>(F, N, n, o);
    if (cudaGetLastError() != cudaSuccess) rc = fail("prtf_advanced: launch");
  }
  if (!rc && cudaMemcpyAsync(prtf, o, sizeof(float2) * (size_t)N, cudaMemcpyDeviceToHost, c->st) != cudaSuccess)
    rc = fail("prtf_advanced: download");
  if (!rc && write_back &&
      cudaMemcpyAsync(images, space == 1 ? F : R, all, cudaMemcpyDeviceToHost, c->st) != cudaSuccess)
    rc = fail("prtf_advanced: download");
  if (cudaStreamSynchronize(c->st) != cudaSuccess && !rc) rc = fail("prtf_advanced: device error");
  for (void *p : {(void *)R, (void *)F, (void *)o})
    if (p) cudaFree(p);
  return rc;
}
