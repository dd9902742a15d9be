/*
 * fftw3_shim.c — test-infrastructure FP64 FFT behind the FFTW3 API subset in
 * fftw3.h. NOT part of the product: only the oracle build links it.
 *
 * Power-of-two sizes use an out-of-place Stockham autosort FFT (radix-4 passes,
 * one radix-2 pass when log2(n) is odd) with per-pass twiddle tables computed
 * from libm cos/sin in FP64 at plan time. Other sizes fall back to a direct
 * O(n^2) DFT with an exact (t*k mod n) twiddle index. Transforms are
 * unnormalised, as in FFTW.
 *
 * Thread safety: a plan is read-only after creation; the ping-pong scratch is
 * thread-local, so the reference may execute different plans (or the same
 * plan) concurrently from OpenMP threads, as it does in
 * src/MultimodePropagation_CPU.cpp:114-119 and :136-163.
 */
#define _POSIX_C_SOURCE 200112L /* posix_memalign under -std=c11 */
#include "fftw3.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct { double re, im; } cplx;

struct mmp_shim_plan_s {
  int n;
  int sign;        /* -1 forward, +1 backward */
  int pow2;
  int n_passes;    /* Stockham passes */
  int radix[40];   /* radix of each pass (4 or 2) */
  cplx* tw;        /* concatenated per-pass tables: w1, w2, w3 for radix 4; w1 for radix 2 */
  size_t tw_off[40];
  cplx* dft_tw;    /* direct-DFT table for non-power-of-two sizes, length n */
  fftw_complex* in;   /* the arrays the plan was made for (fftw_execute) */
  fftw_complex* out;
};

static const double kTwoPi = 6.283185307179586476925286766559;

int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int nthreads) { (void)nthreads; }
void fftw_cleanup_threads(void) {}

void* fftw_malloc(size_t n) {
  void* p = NULL;
  if (posix_memalign(&p, 64, n ? n : 64) != 0) return NULL;
  return p;
}
void fftw_free(void* p) { free(p); }

static cplx unit_root(double num, double den, int sign) {
  /* exp(sign * 2*pi*i * num/den) */
  double a = kTwoPi * num / den;
  cplx w;
  w.re = cos(a);
  w.im = (double)sign * sin(a);
  return w;
}

fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned flags) {
  (void)flags;
  if (n <= 0) return NULL;
  struct mmp_shim_plan_s* p = (struct mmp_shim_plan_s*)calloc(1, sizeof(*p));
  p->n = n;
  p->in = in;
  p->out = out;
  p->sign = (sign < 0) ? -1 : 1;
  p->pow2 = (n & (n - 1)) == 0;
  if (p->pow2) {
    /* pass sizes: current sub-transform length m runs n, n/4, ... */
    int m = n;
    size_t total = 0;
    int np = 0;
    while (m >= 4) { p->radix[np++] = 4; total += 3 * (size_t)(m / 4); m /= 4; }
    if (m == 2) { p->radix[np++] = 2; total += 1; }
    p->n_passes = np;
    p->tw = (cplx*)malloc((total ? total : 1) * sizeof(cplx));
    m = n;
    size_t off = 0;
    for (int s = 0; s < np; ++s) {
      p->tw_off[s] = off;
      if (p->radix[s] == 4) {
        int q = m / 4;
        for (int j = 0; j < q; ++j) {
          p->tw[off + j] = unit_root((double)j, (double)m, p->sign);
          p->tw[off + q + j] = unit_root(2.0 * j, (double)m, p->sign);
          p->tw[off + 2 * q + j] = unit_root(3.0 * j, (double)m, p->sign);
        }
        off += 3 * (size_t)q;
        m /= 4;
      } else {
        p->tw[off] = unit_root(0.0, 2.0, p->sign);
        off += 1;
        m /= 2;
      }
    }
  } else {
    p->dft_tw = (cplx*)malloc((size_t)n * sizeof(cplx));
    for (int k = 0; k < n; ++k) p->dft_tw[k] = unit_root((double)k, (double)n, p->sign);
  }
  return p;
}

void fftw_destroy_plan(fftw_plan p) {
  if (!p) return;
  free(p->tw);
  free(p->dft_tw);
  free(p);
}

/* thread-local scratch, grown on demand */
static __thread cplx* tl_scratch = NULL;
static __thread size_t tl_scratch_len = 0;

static cplx* scratch(size_t need) {
  if (tl_scratch_len < need) {
    free(tl_scratch);
    tl_scratch = (cplx*)malloc(need * sizeof(cplx));
    tl_scratch_len = need;
  }
  return tl_scratch;
}

/* One radix-4 Stockham pass: sub-transform length m, stride s (m*s == n). */
static void pass4(const cplx* x, cplx* y, int m, int s, const cplx* w1t, const cplx* w2t,
                  const cplx* w3t, int sign) {
  const int q = m / 4;
  for (int j = 0; j < q; ++j) {
    const cplx w1 = w1t[j], w2 = w2t[j], w3 = w3t[j];
    const cplx* x0 = x + (size_t)s * j;
    const cplx* x1 = x + (size_t)s * (j + q);
    const cplx* x2 = x + (size_t)s * (j + 2 * q);
    const cplx* x3 = x + (size_t)s * (j + 3 * q);
    cplx* y0 = y + (size_t)s * (4 * j);
    cplx* y1 = y0 + s;
    cplx* y2 = y1 + s;
    cplx* y3 = y2 + s;
    for (int k = 0; k < s; ++k) {
      const cplx a = x0[k], b = x1[k], c = x2[k], d = x3[k];
      const double apc_re = a.re + c.re, apc_im = a.im + c.im;
      const double amc_re = a.re - c.re, amc_im = a.im - c.im;
      const double bpd_re = b.re + d.re, bpd_im = b.im + d.im;
      /* rot = sign * i * (b - d) */
      const double bmd_re = b.re - d.re, bmd_im = b.im - d.im;
      const double rot_re = -(double)sign * bmd_im, rot_im = (double)sign * bmd_re;
      const double t0_re = apc_re + bpd_re, t0_im = apc_im + bpd_im;
      const double t1_re = amc_re + rot_re, t1_im = amc_im + rot_im;
      const double t2_re = apc_re - bpd_re, t2_im = apc_im - bpd_im;
      const double t3_re = amc_re - rot_re, t3_im = amc_im - rot_im;
      y0[k].re = t0_re;
      y0[k].im = t0_im;
      y1[k].re = t1_re * w1.re - t1_im * w1.im;
      y1[k].im = t1_re * w1.im + t1_im * w1.re;
      y2[k].re = t2_re * w2.re - t2_im * w2.im;
      y2[k].im = t2_re * w2.im + t2_im * w2.re;
      y3[k].re = t3_re * w3.re - t3_im * w3.im;
      y3[k].im = t3_re * w3.im + t3_im * w3.re;
    }
  }
}

/* The final radix-2 pass (m == 2): twiddle is 1. */
static void pass2(const cplx* x, cplx* y, int s) {
  for (int k = 0; k < s; ++k) {
    const cplx a = x[k], b = x[k + s];
    y[k].re = a.re + b.re;
    y[k].im = a.im + b.im;
    y[k + s].re = a.re - b.re;
    y[k + s].im = a.im - b.im;
  }
}

static void exec_pow2(const struct mmp_shim_plan_s* p, const cplx* in, cplx* out) {
  const int n = p->n;
  if (n == 1) { out[0] = in[0]; return; }
  cplx* buf = scratch((size_t)2 * n);
  cplx* tmp = buf;
  const cplx* src = in;
  if (in == out) {
    memcpy(buf + n, in, (size_t)n * sizeof(cplx));
    src = buf + n;
  }
  /* choose the first destination so that the last pass lands in `out` */
  cplx* dst = (p->n_passes % 2 == 1) ? out : tmp;
  int m = n, s = 1;
  for (int ps = 0; ps < p->n_passes; ++ps) {
    if (p->radix[ps] == 4) {
      const int q = m / 4;
      const cplx* t = p->tw + p->tw_off[ps];
      pass4(src, dst, m, s, t, t + q, t + 2 * q, p->sign);
      m /= 4;
      s *= 4;
    } else {
      pass2(src, dst, s);
      m /= 2;
      s *= 2;
    }
    src = dst;
    dst = (dst == out) ? tmp : out;
  }
}

static void exec_direct(const struct mmp_shim_plan_s* p, const cplx* in, cplx* out) {
  const int n = p->n;
  cplx* buf = scratch((size_t)n);
  for (int k = 0; k < n; ++k) {
    double re = 0.0, im = 0.0;
    long long idx = 0;
    for (int t = 0; t < n; ++t) {
      const cplx w = p->dft_tw[idx];
      re += in[t].re * w.re - in[t].im * w.im;
      im += in[t].re * w.im + in[t].im * w.re;
      idx += k;
      if (idx >= n) idx -= n;
    }
    buf[k].re = re;
    buf[k].im = im;
  }
  memcpy(out, buf, (size_t)n * sizeof(cplx));
}

void fftw_execute_dft(const fftw_plan p, fftw_complex* in, fftw_complex* out) {
  if (!p) return;
  if (p->pow2)
    exec_pow2(p, (const cplx*)in, (cplx*)out);
  else
    exec_direct(p, (const cplx*)in, (cplx*)out);
}

/* FFTW's fftw_execute: the plan on the arrays it was made for */
void fftw_execute(const fftw_plan p) {
  if (p) fftw_execute_dft(p, p->in, p->out);
}
