/* Drives the oracle's FFTW-API shim (oracle/fftw_shim) under AddressSanitizer and
 * UndefinedBehaviorSanitizer: plans of every power-of-two size the oracle uses (and a few
 * more), execution on the planned arrays and on other arrays, in place and out of place,
 * both directions, against a naive DFT. Exit status 0 when every transform matched. */
#include <math.h>
#include <stdio.h>
#include <string.h>

#include "fftw3.h"

#if !defined(__SANITIZE_ADDRESS__)
#error "shim_fft.c is built with -fsanitize=address (tests/test_host_sanitize.py)"
#endif

static double naive_err(int n, int sign, const fftw_complex* x, const fftw_complex* y) {
  double err = 0.0, mag = 0.0;
  for (int k = 0; k < n; ++k) {
    double re = 0.0, im = 0.0;
    for (int t = 0; t < n; ++t) {
      const double a = sign * 2.0 * M_PI * (double)((long)t * k % n) / n;
      re += x[t][0] * cos(a) - x[t][1] * sin(a);
      im += x[t][0] * sin(a) + x[t][1] * cos(a);
    }
    err = fmax(err, fmax(fabs(re - y[k][0]), fabs(im - y[k][1])));
    mag = fmax(mag, fmax(fabs(re), fabs(im)));
  }
  return err / (mag > 0 ? mag : 1.0);
}

int main(void) {
  int bad = 0;
  fftw_init_threads();
  fftw_plan_with_nthreads(4);
  for (int n = 1; n <= 4096; n *= 2) {
    fftw_complex* x = (fftw_complex*)fftw_malloc(sizeof(fftw_complex) * n);
    fftw_complex* y = (fftw_complex*)fftw_malloc(sizeof(fftw_complex) * n);
    fftw_complex* z = (fftw_complex*)fftw_malloc(sizeof(fftw_complex) * n);
    fftw_complex* keep = (fftw_complex*)fftw_malloc(sizeof(fftw_complex) * n);
    for (int t = 0; t < n; ++t) {
      x[t][0] = sin(0.37 * t + 0.1);
      x[t][1] = cos(0.11 * t * t);
    }
    for (int sign = -1; sign <= 1; sign += 2) {
      fftw_plan p = fftw_plan_dft_1d(n, x, y, sign, FFTW_ESTIMATE);
      memcpy(keep, x, sizeof(fftw_complex) * n);
      fftw_execute(p);  /* on the planned arrays: the input is kept */
      if (n <= 1024 && naive_err(n, sign, x, y) > 1e-12) { printf("n=%d sign=%d: wrong\n", n, sign); ++bad; }
      if (memcmp(keep, x, sizeof(fftw_complex) * n)) { printf("n=%d: input changed\n", n); ++bad; }
      memcpy(z, x, sizeof(fftw_complex) * n);
      fftw_execute_dft(p, z, z);  /* another array, in place */
      for (int k = 0; k < n; ++k)
        if (fabs(z[k][0] - y[k][0]) > 1e-12 * (1 + fabs(y[k][0])) || fabs(z[k][1] - y[k][1]) > 1e-12 * (1 + fabs(y[k][1]))) {
          printf("n=%d: in-place result differs\n", n);
          ++bad;
          break;
        }
      fftw_destroy_plan(p);
    }
    fftw_free(x);
    fftw_free(y);
    fftw_free(z);
    fftw_free(keep);
  }
  fftw_cleanup_threads();
  if (!bad) printf("fftw shim: all checks passed\n");
  return bad ? 1 : 0;
}
