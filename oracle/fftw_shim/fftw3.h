/*
 * fftw3.h — test-infrastructure shim, NOT part of the product.
 *
 * FFTW3 is not installed on this image and there is no network, so the
 * reference's CPU path (src/DiscreteFourierTransform.cpp:4-37 of
 * alexandreroget/MM_Propagation) is linked against this header instead. It
 * declares exactly the subset of FFTW3's public C API that the reference calls,
 * with the meaning FFTW's manual gives it:
 *   - fftw_complex is double[2] (re, im);
 *   - FFTW_FORWARD = -1 computes X[k] = sum_t x[t] exp(-2*pi*i*t*k/n),
 *     FFTW_BACKWARD = +1 the same with exp(+...), both UNNORMALISED;
 *   - fftw_execute_dft(plan, in, out) applies a plan to other arrays of the
 *     same size and preserves the input when in != out;
 *   - planning flags and thread counts are accepted and have no effect
 *     (one transform always runs on the calling thread).
 * The arithmetic behind it is our own FP64 Stockham FFT (fftw3_shim.c).
 * FFTW itself is a third-party dependency the reference does not vendor or pin
 * (CMakeLists.txt:28 uses find_package(FFTW)); results through this shim agree
 * with numpy.fft (pocketfft) to ~1e-15 relative, checked in tests/.
 */
#ifndef MMP_ORACLE_FFTW3_SHIM_H
#define MMP_ORACLE_FFTW3_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct mmp_shim_plan_s* fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
void fftw_cleanup_threads(void);

void* fftw_malloc(size_t n);
void fftw_free(void* p);

fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_execute_dft(const fftw_plan p, fftw_complex* in, fftw_complex* out);
void fftw_destroy_plan(fftw_plan p);

#ifdef __cplusplus
}
#endif

#endif
