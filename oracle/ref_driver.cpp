/*
 * ref_driver.cpp — test infrastructure, NOT part of the product.
 *
 * A C entry point over the reference's OWN, unmodified CPU solver classes
 * (alexandreroget/MM_Propagation, src/MultimodePropagation_CPU.cpp), compiled
 * from the reference sources in place by oracle/Makefile into
 * oracle/_ref/libmmref.so. Tests, smoke() and bench.py's CPU-baseline leg load
 * it with ctypes; nothing in the product links it.
 *
 * It only translates the flat mmp_params (include/mmp.h) into the reference's
 * struct SimulationParameters (include/MultimodePropagation.hpp:16-33), runs
 * the solver the way the reference's drivers do (simulations/main.cpp:94-99,
 * matlab/mm_propagation.cpp:59-92) and copies getResult() out.
 */
#include <chrono>
#include <complex>
#include <cstring>
#include <vector>

#include "MultimodePropagation_CPU.hpp"
#include "mmp.h"

namespace {

/* The reference's FFT wrapper calls omp_set_num_threads(max_threads / M) as a
 * process-wide side effect (src/DiscreteFourierTransform.cpp:6), so a second
 * solver in the same process would start from the reduced count. Each run
 * therefore starts again from the thread count seen when the library loaded. */
const int g_initial_threads = omp_get_max_threads();

SimulationParameters to_reference(const mmp_params* prm) {
  SimulationParameters in;
  const unsigned M = prm->n_modes, nt = prm->nt, L = prm->n_beta;
  in.n_modes = M;
  in.fiber_length = prm->fiber_length;
  in.dispersion_coefficients.assign(M, std::vector<double>(L));
  for (unsigned p = 0; p < M; ++p)
    for (unsigned i = 0; i < L; ++i) in.dispersion_coefficients[p][i] = prm->dispersion[p * L + i];
  in.coupling_coefficients.assign(M, Sparse3DArray());
  for (unsigned j = 0; j < prm->n_nonzeros; ++j) {
    const mmp_nz& e = prm->coupling[j];
    NonZeroValue nzv = {{e.k, e.l, e.m}, e.value};
    in.coupling_coefficients[e.p].addNonZeroValue(nzv);
  }
  in.nt = nt;
  in.time_window = prm->time_window;
  in.pulse_width = prm->pulse_width;
  in.initial_fields = ComplexArraysContainer(nt, M);
  for (unsigned p = 0; p < M; ++p)
    for (unsigned t = 0; t < nt; ++t)
      in.initial_fields[p][t] = std::complex<double>(prm->initial_fields[2 * (size_t(p) * nt + t)],
                                                     prm->initial_fields[2 * (size_t(p) * nt + t) + 1]);
  in.n_steps = prm->n_steps;
  in.method_order = prm->method_order;
  in.nonlinearity_const = prm->nonlinearity_const;
  in.raman_proportion = prm->raman_proportion;
  in.raman_response.assign(nt, 0.0);
  if (prm->raman_response)
    for (unsigned t = 0; t < nt; ++t) in.raman_response[t] = prm->raman_response[t];
  return in;
}

}  // namespace

extern "C" {

/* Construct the reference solver (RamanON when prm->raman != 0), call
 * computeLawsonRK(chunks[c]) for each chunk in order (0xFFFFFFFF means the
 * no-argument computeLawsonRK()), then getResult() into out[M][NT][2].
 * *seconds receives the wall time of the computeLawsonRK calls plus getResult,
 * excluding construction (planning, setup). Returns 0, or -1 on bad input. */
int mmref_run(const mmp_params* prm, const unsigned* chunks, unsigned n_chunks, double* out,
              double* seconds) {
  if (!prm || !prm->n_modes || !prm->nt || !prm->dispersion || !prm->initial_fields) return -1;
  omp_set_num_threads(g_initial_threads);
  SimulationParameters in = to_reference(prm);
  MultimodePropagation* solver = nullptr;
  if (prm->raman)
    solver = new MultimodePropagationCPU_RamanON(in);
  else
    solver = new MultimodePropagationCPU_RamanOFF(in);
  auto t0 = std::chrono::steady_clock::now();
  for (unsigned c = 0; c < n_chunks; ++c) {
    if (chunks[c] == 0xFFFFFFFFu)
      solver->computeLawsonRK();
    else
      solver->computeLawsonRK(chunks[c]);
  }
  ComplexArraysContainer phi = solver->getResult();
  auto t1 = std::chrono::steady_clock::now();
  if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
  const unsigned M = prm->n_modes, nt = prm->nt;
  for (unsigned p = 0; p < M; ++p)
    for (unsigned t = 0; t < nt; ++t) {
      out[2 * (size_t(p) * nt + t)] = phi[p][t].real();
      out[2 * (size_t(p) * nt + t) + 1] = phi[p][t].imag();
    }
  delete solver;
  return 0;
}

/* The FFTW-API shim the reference is linked against, exposed for its own
 * check against numpy.fft: sign -1 forward, +1 backward, unnormalised. */
int mmref_fft(int n, int sign, const double* in, double* out) {
  fftw_complex* a = (fftw_complex*)fftw_malloc(sizeof(fftw_complex) * n);
  fftw_complex* b = (fftw_complex*)fftw_malloc(sizeof(fftw_complex) * n);
  std::memcpy(a, in, sizeof(fftw_complex) * n);
  fftw_plan plan = fftw_plan_dft_1d(n, a, b, sign, FFTW_ESTIMATE);
  fftw_execute_dft(plan, a, b);
  std::memcpy(out, b, sizeof(fftw_complex) * n);
  fftw_destroy_plan(plan);
  fftw_free(a);
  fftw_free(b);
  return 0;
}

/* Threads the reference's parallel regions use for an M-mode solve:
 * max(1, initial / M) (src/MultimodePropagation_CPU.cpp:13-15). */
int mmref_initial_threads(void) { return g_initial_threads; }
int mmref_effective_threads(unsigned M) {
  int n = g_initial_threads / (int)(M ? M : 1);
  return n > 0 ? n : 1;
}

}  // extern "C"
