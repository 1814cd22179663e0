/*
 * spfft -- CPU single-precision FFT used by the oracle.  See spfft.h for the
 * exact algorithm.  Build with -ffp-contract=off (no fused multiply-add): the
 * arithmetic below is the specification that the device FFT reproduces.
 *
 * Lines are processed BLK at a time in a structure-of-arrays work buffer so
 * the compiler can vectorise across lines without changing any rounding.
 */
#include "spfft.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define BLK 8

#define C8 0.70710678118654752440f
#define C16 0.92387953251128675613f
#define S16 0.38268343236508977173f
#define S3 0.86602540378443864676f
#define C51 0.30901699437494742410f
#define C52 (-0.80901699437494742410f)
#define S51 0.95105651629515357212f
#define S52 0.58778525229247312917f

int spfft_radix_plan(int n, int *radix) {
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

spfft_plan *spfft_plan_create(int n) {
  spfft_plan *p = (spfft_plan *)calloc(1, sizeof(spfft_plan));
  p->n = n;
  p->nstages = spfft_radix_plan(n, p->radix);
  p->tw = (spfft_cpx *)malloc(sizeof(spfft_cpx) * (size_t)(n > 0 ? n : 1));
  for (int i = 0; i < n; i++) {
    double ang = (2.0 * 3.14159265358979323846 * (double)i) / (double)n;
    p->tw[i].re = (float)cos(ang);
    p->tw[i].im = (float)(-sin(ang));
  }
  return p;
}

void spfft_plan_destroy(spfft_plan *p) {
  if (!p) return;
  free(p->tw);
  free(p);
}

typedef float lane_t[BLK];

/* ---- butterflies on rows of lanes (in place) ---- */

static inline void cmul_rows(lane_t *ar, lane_t *ai, int r, float wr, float wi) {
  for (int l = 0; l < BLK; l++) {
    float xr = ar[r][l], xi = ai[r][l];
    float t1 = xr * wr;
    float t2 = xi * wi;
    float t3 = xr * wi;
    float t4 = xi * wr;
    ar[r][l] = t1 - t2;
    ai[r][l] = t3 + t4;
  }
}

/* multiply by W4^1 (forward -i, backward +i) */
static inline void mulw4_rows(lane_t *ar, lane_t *ai, int r, int inv) {
  for (int l = 0; l < BLK; l++) {
    float xr = ar[r][l], xi = ai[r][l];
    if (!inv) { ar[r][l] = xi; ai[r][l] = -xr; }
    else { ar[r][l] = -xi; ai[r][l] = xr; }
  }
}

/* multiply by W8^1 */
static inline void mulw8_1_rows(lane_t *ar, lane_t *ai, int r, int inv) {
  for (int l = 0; l < BLK; l++) {
    float xr = ar[r][l], xi = ai[r][l];
    if (!inv) { ar[r][l] = (xr + xi) * C8; ai[r][l] = (xi - xr) * C8; }
    else { ar[r][l] = (xr - xi) * C8; ai[r][l] = (xr + xi) * C8; }
  }
}

/* multiply by W8^3 */
static inline void mulw8_3_rows(lane_t *ar, lane_t *ai, int r, int inv) {
  for (int l = 0; l < BLK; l++) {
    float xr = ar[r][l], xi = ai[r][l];
    if (!inv) { ar[r][l] = (xi - xr) * C8; ai[r][l] = -((xr + xi) * C8); }
    else { ar[r][l] = -((xr + xi) * C8); ai[r][l] = (xr - xi) * C8; }
  }
}

static inline void bf2(lane_t *ar, lane_t *ai, int i0, int i1) {
  for (int l = 0; l < BLK; l++) {
    float a0r = ar[i0][l], a0i = ai[i0][l], a1r = ar[i1][l], a1i = ai[i1][l];
    ar[i0][l] = a0r + a1r; ai[i0][l] = a0i + a1i;
    ar[i1][l] = a0r - a1r; ai[i1][l] = a0i - a1i;
  }
}

static inline void bf4(lane_t *ar, lane_t *ai, int i0, int i1, int i2, int i3, int inv) {
  for (int l = 0; l < BLK; l++) {
    float a0r = ar[i0][l], a0i = ai[i0][l];
    float a1r = ar[i1][l], a1i = ai[i1][l];
    float a2r = ar[i2][l], a2i = ai[i2][l];
    float a3r = ar[i3][l], a3i = ai[i3][l];
    float t0r = a0r + a2r, t0i = a0i + a2i;
    float t1r = a0r - a2r, t1i = a0i - a2i;
    float t2r = a1r + a3r, t2i = a1i + a3i;
    float dr = a1r - a3r, di = a1i - a3i;
    float t3r, t3i;
    if (!inv) { t3r = di; t3i = -dr; } else { t3r = -di; t3i = dr; }
    ar[i0][l] = t0r + t2r; ai[i0][l] = t0i + t2i;
    ar[i1][l] = t1r + t3r; ai[i1][l] = t1i + t3i;
    ar[i2][l] = t0r - t2r; ai[i2][l] = t0i - t2i;
    ar[i3][l] = t1r - t3r; ai[i3][l] = t1i - t3i;
  }
}

static void bf8(lane_t *ar, lane_t *ai, int inv) {
  lane_t tr[8], ti[8];
  bf4(ar, ai, 0, 2, 4, 6, inv);  /* e_k at 2k */
  bf4(ar, ai, 1, 3, 5, 7, inv);  /* o_k at 2k+1 */
  mulw8_1_rows(ar, ai, 3, inv);
  mulw4_rows(ar, ai, 5, inv);
  mulw8_3_rows(ar, ai, 7, inv);
  for (int k = 0; k < 4; k++)
    for (int l = 0; l < BLK; l++) {
      float er = ar[2 * k][l], ei = ai[2 * k][l];
      float orr = ar[2 * k + 1][l], oi = ai[2 * k + 1][l];
      tr[k][l] = er + orr; ti[k][l] = ei + oi;
      tr[k + 4][l] = er - orr; ti[k + 4][l] = ei - oi;
    }
  memcpy(ar, tr, sizeof(tr));
  memcpy(ai, ti, sizeof(ti));
}

static void bf16(lane_t *ar, lane_t *ai, int inv) {
  lane_t tr[16], ti[16];
  const float s = inv ? -1.0f : 1.0f;
  /* step 1: DFT4 over q1 for each q2; b[q2][k1] lands at q2 + 4*k1 */
  for (int q2 = 0; q2 < 4; q2++) bf4(ar, ai, q2, q2 + 4, q2 + 8, q2 + 12, inv);
  /* step 2: twiddles W16^(q2*k1) */
  cmul_rows(ar, ai, 1 + 4 * 1, C16, -S16 * s);   /* W^1 */
  mulw8_1_rows(ar, ai, 1 + 4 * 2, inv);          /* W^2 */
  cmul_rows(ar, ai, 1 + 4 * 3, S16, -C16 * s);   /* W^3 */
  mulw8_1_rows(ar, ai, 2 + 4 * 1, inv);          /* W^2 */
  mulw4_rows(ar, ai, 2 + 4 * 2, inv);            /* W^4 */
  mulw8_3_rows(ar, ai, 2 + 4 * 3, inv);          /* W^6 */
  cmul_rows(ar, ai, 3 + 4 * 1, S16, -C16 * s);   /* W^3 */
  mulw8_3_rows(ar, ai, 3 + 4 * 2, inv);          /* W^6 */
  cmul_rows(ar, ai, 3 + 4 * 3, -C16, S16 * s);   /* W^9 */
  /* step 3: DFT4 over q2 for each k1; X[k1 + 4*k2] lands at 4*k1 + k2 */
  for (int k1 = 0; k1 < 4; k1++) bf4(ar, ai, 4 * k1, 4 * k1 + 1, 4 * k1 + 2, 4 * k1 + 3, inv);
  for (int k1 = 0; k1 < 4; k1++)
    for (int k2 = 0; k2 < 4; k2++)
      for (int l = 0; l < BLK; l++) {
        tr[k1 + 4 * k2][l] = ar[4 * k1 + k2][l];
        ti[k1 + 4 * k2][l] = ai[4 * k1 + k2][l];
      }
  memcpy(ar, tr, sizeof(tr));
  memcpy(ai, ti, sizeof(ti));
}

static void bf3(lane_t *ar, lane_t *ai, int inv) {
  for (int l = 0; l < BLK; l++) {
    float a0r = ar[0][l], a0i = ai[0][l];
    float a1r = ar[1][l], a1i = ai[1][l];
    float a2r = ar[2][l], a2i = ai[2][l];
    float t1r = a1r + a2r, t1i = a1i + a2i;
    float dr = a1r - a2r, di = a1i - a2i;
    float mr = a0r - t1r * 0.5f, mi = a0i - t1i * 0.5f;
    float t3r, t3i;
    if (!inv) { t3r = di * S3; t3i = -(dr * S3); }
    else { t3r = -(di * S3); t3i = dr * S3; }
    ar[0][l] = a0r + t1r; ai[0][l] = a0i + t1i;
    ar[1][l] = mr + t3r; ai[1][l] = mi + t3i;
    ar[2][l] = mr - t3r; ai[2][l] = mi - t3i;
  }
}

static void bf5(lane_t *ar, lane_t *ai, int inv) {
  for (int l = 0; l < BLK; l++) {
    float a0r = ar[0][l], a0i = ai[0][l];
    float a1r = ar[1][l], a1i = ai[1][l];
    float a2r = ar[2][l], a2i = ai[2][l];
    float a3r = ar[3][l], a3i = ai[3][l];
    float a4r = ar[4][l], a4i = ai[4][l];
    float b1r = a1r + a4r, b1i = a1i + a4i;
    float b2r = a2r + a3r, b2i = a2i + a3i;
    float d1r = a1r - a4r, d1i = a1i - a4i;
    float d2r = a2r - a3r, d2i = a2i - a3i;
    float y0r = (a0r + b1r) + b2r, y0i = (a0i + b1i) + b2i;
    float m1r = (a0r + b1r * C51) + b2r * C52, m1i = (a0i + b1i * C51) + b2i * C52;
    float m2r = (a0r + b1r * C52) + b2r * C51, m2i = (a0i + b1i * C52) + b2i * C51;
    float n1r = d1r * S51 + d2r * S52, n1i = d1i * S51 + d2i * S52;
    float n2r = d1r * S52 - d2r * S51, n2i = d1i * S52 - d2i * S51;
    ar[0][l] = y0r; ai[0][l] = y0i;
    if (!inv) {
      ar[1][l] = m1r + n1i; ai[1][l] = m1i - n1r;
      ar[4][l] = m1r - n1i; ai[4][l] = m1i + n1r;
      ar[2][l] = m2r + n2i; ai[2][l] = m2i - n2r;
      ar[3][l] = m2r - n2i; ai[3][l] = m2i + n2r;
    } else {
      ar[1][l] = m1r - n1i; ai[1][l] = m1i + n1r;
      ar[4][l] = m1r + n1i; ai[4][l] = m1i - n1r;
      ar[2][l] = m2r - n2i; ai[2][l] = m2i + n2r;
      ar[3][l] = m2r + n2i; ai[3][l] = m2i - n2r;
    }
  }
}

/* generic prime radix r: y_m = a_0 + sum_{q=1}^{r-1} a_q * W_r^{(m q) mod r}, summed left to right */
static void bfgen(lane_t *ar, lane_t *ai, int r, const spfft_plan *p, int inv, lane_t *tr, lane_t *ti) {
  const int step = p->n / r;
  for (int l = 0; l < BLK; l++) {
    float accr = ar[0][l], acci = ai[0][l];
    for (int q = 1; q < r; q++) { accr = accr + ar[q][l]; acci = acci + ai[q][l]; }
    tr[0][l] = accr; ti[0][l] = acci;
  }
  for (int m = 1; m < r; m++) {
    for (int l = 0; l < BLK; l++) {
      float accr = ar[0][l], acci = ai[0][l];
      for (int q = 1; q < r; q++) {
        int e = (int)(((long)m * q) % r);
        float wr = p->tw[e * step].re;
        float wi = inv ? -p->tw[e * step].im : p->tw[e * step].im;
        float xr = ar[q][l], xi = ai[q][l];
        float t1 = xr * wr, t2 = xi * wi, t3 = xr * wi, t4 = xi * wr;
        accr = accr + (t1 - t2);
        acci = acci + (t3 + t4);
      }
      tr[m][l] = accr; ti[m][l] = acci;
    }
  }
  memcpy(ar, tr, sizeof(lane_t) * (size_t)r);
  memcpy(ai, ti, sizeof(lane_t) * (size_t)r);
}

static int max_radix(const spfft_plan *p) {
  int m = 16;
  for (int s = 0; s < p->nstages; s++) if (p->radix[s] > m) m = p->radix[s];
  return m;
}

static void run_stage(const spfft_plan *p, int ns, int r, int inv, const float *xr, const float *xi,
                      float *yr, float *yi, lane_t *ar, lane_t *ai, lane_t *tr, lane_t *ti) {
  const int n = p->n, nr = n / r, L = ns * r, tstep = n / L;
  for (int j = 0; j < nr; j++) {
    const int k = j % ns;
    for (int m = 0; m < r; m++) {
      const float *sr = xr + (size_t)(j + m * nr) * BLK, *si = xi + (size_t)(j + m * nr) * BLK;
      for (int l = 0; l < BLK; l++) { ar[m][l] = sr[l]; ai[m][l] = si[l]; }
    }
    if (k) {
      for (int m = 1; m < r; m++) {
        const spfft_cpx w = p->tw[m * k * tstep];
        cmul_rows(ar, ai, m, w.re, inv ? -w.im : w.im);
      }
    }
    switch (r) {
      case 2: bf2(ar, ai, 0, 1); break;
      case 3: bf3(ar, ai, inv); break;
      case 4: bf4(ar, ai, 0, 1, 2, 3, inv); break;
      case 5: bf5(ar, ai, inv); break;
      case 8: bf8(ar, ai, inv); break;
      case 16: bf16(ar, ai, inv); break;
      default: bfgen(ar, ai, r, p, inv, tr, ti); break;
    }
    const int base = (j / ns) * L + k;
    for (int m = 0; m < r; m++) {
      float *dr = yr + (size_t)(base + m * ns) * BLK, *di = yi + (size_t)(base + m * ns) * BLK;
      for (int l = 0; l < BLK; l++) { dr[l] = ar[m][l]; di[l] = ai[m][l]; }
    }
  }
}

typedef struct {
  const spfft_plan *p;
  int inv;
  spfft_cpx *data;
  long h0, h1, stride, dist;
} lines_job;

static void *lines_worker(void *arg) {
  lines_job *jb = (lines_job *)arg;
  const spfft_plan *p = jb->p;
  const int n = p->n, R = max_radix(p);
  float *buf = (float *)calloc((size_t)4 * n * BLK, sizeof(float));
  lane_t *scratch = (lane_t *)calloc((size_t)4 * R, sizeof(lane_t));
  lane_t *ar = scratch, *ai = scratch + R, *tr = scratch + 2 * R, *ti = scratch + 3 * R;
  for (long h = jb->h0; h < jb->h1; h += BLK) {
    const int B = (int)((jb->h1 - h) < BLK ? (jb->h1 - h) : BLK);
    float *xr = buf, *xi = buf + (size_t)n * BLK, *yr = buf + (size_t)2 * n * BLK, *yi = buf + (size_t)3 * n * BLK;
    for (int i = 0; i < n; i++)
      for (int l = 0; l < B; l++) {
        const spfft_cpx v = jb->data[(h + l) * jb->dist + (long)i * jb->stride];
        xr[(size_t)i * BLK + l] = v.re;
        xi[(size_t)i * BLK + l] = v.im;
      }
    int ns = 1;
    for (int s = 0; s < p->nstages; s++) {
      const int r = p->radix[s];
      run_stage(p, ns, r, jb->inv, xr, xi, yr, yi, ar, ai, tr, ti);
      ns *= r;
      float *t = xr; xr = yr; yr = t;
      t = xi; xi = yi; yi = t;
    }
    for (int i = 0; i < n; i++)
      for (int l = 0; l < B; l++) {
        spfft_cpx *d = &jb->data[(h + l) * jb->dist + (long)i * jb->stride];
        d->re = xr[(size_t)i * BLK + l];
        d->im = xi[(size_t)i * BLK + l];
      }
  }
  free(scratch);
  free(buf);
  return NULL;
}

void spfft_lines(const spfft_plan *p, int sign, spfft_cpx *data, long howmany, long stride, long dist,
                 int nthreads) {
  if (p->n <= 1 || howmany <= 0) return;
  const int inv = sign > 0;
  long blocks = (howmany + BLK - 1) / BLK;
  int nt = nthreads < 1 ? 1 : nthreads;
  if (nt > blocks) nt = (int)blocks;
  if (nt <= 1) {
    lines_job jb = {p, inv, data, 0, howmany, stride, dist};
    lines_worker(&jb);
    return;
  }
  lines_job *jobs = (lines_job *)calloc((size_t)nt, sizeof(lines_job));
  pthread_t *th = (pthread_t *)calloc((size_t)nt, sizeof(pthread_t));
  for (int t = 0; t < nt; t++) {
    long b0 = blocks * t / nt, b1 = blocks * (t + 1) / nt;
    long h0 = b0 * BLK, h1 = b1 * BLK;
    if (h1 > howmany) h1 = howmany;
    jobs[t] = (lines_job){p, inv, data, h0, h1, stride, dist};
  }
  for (int t = 1; t < nt; t++) pthread_create(&th[t], NULL, lines_worker, &jobs[t]);
  lines_worker(&jobs[0]);
  for (int t = 1; t < nt; t++) pthread_join(th[t], NULL);
  free(th);
  free(jobs);
}

/* ---- small plan cache (plans are immutable once built) ---- */
#define CACHE_N 16
static spfft_plan *g_cache[CACHE_N];
static int g_cache_next;
static pthread_mutex_t g_cache_mu = PTHREAD_MUTEX_INITIALIZER;

static const spfft_plan *cached_plan(int n) {
  pthread_mutex_lock(&g_cache_mu);
  for (int i = 0; i < CACHE_N; i++)
    if (g_cache[i] && g_cache[i]->n == n) {
      pthread_mutex_unlock(&g_cache_mu);
      return g_cache[i];
    }
  spfft_plan *p = spfft_plan_create(n);
  /* evicted plans are leaked on purpose: another thread may still use them */
  g_cache[g_cache_next] = p;
  g_cache_next = (g_cache_next + 1) % CACHE_N;
  pthread_mutex_unlock(&g_cache_mu);
  return p;
}

void spfft_nd(int rank, const int *dims, int sign, const spfft_cpx *in, spfft_cpx *out, int nthreads) {
  long total = 1;
  for (int a = 0; a < rank; a++) total *= dims[a];
  if (in != out) memmove(out, in, sizeof(spfft_cpx) * (size_t)total);
  for (int t = 0; t < rank; t++) {
    const int a = sign < 0 ? rank - 1 - t : t; /* forward: fastest axis first */
    const int n = dims[a];
    if (n <= 1) continue;
    long inner = 1;
    for (int b = a + 1; b < rank; b++) inner *= dims[b];
    const long outer = total / (inner * n);
    const spfft_plan *p = cached_plan(n);
    if (inner == 1) {
      spfft_lines(p, sign, out, outer, 1, n, nthreads);
    } else {
      for (long o = 0; o < outer; o++)
        spfft_lines(p, sign, out + o * n * inner, inner, inner, 1, nthreads);
    }
  }
}
