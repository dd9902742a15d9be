// A user driver in the style the reference documents (README.md:125-187): it fills
// a SimulationParameters, builds a solver, runs computeLawsonRK and getResult.
// Compiled twice from this one file: against the reference's own CPU classes
// (-DMMP_REFERENCE_BUILD, to make the golden output) and against this project's
// drop-in headers, where the only differences are the header and the class name.
//
// usage: two_mode_driver <output file>   (writes "re im" per sample, mode by mode)
#include <cmath>
#include <cstdio>

#ifdef MMP_REFERENCE_BUILD
#include "MultimodePropagation_CPU.hpp"
#define SOLVER_CLASS MultimodePropagationCPU_RamanON
#else
#include "MultimodePropagation_B200.hpp"
#define SOLVER_CLASS MultimodePropagationB200_RamanON
#endif

static ComplexArray sech_pulse(unsigned nt, double window, double width, double peak, double shift,
                               double chirp_free_phase) {
  ComplexArray a(nt);
  const std::complex<double> i(0., 1.);
  for (unsigned j = 0; j < nt; ++j) {
    const double t = -window / 2 + j * window / nt - shift;
    a[j] = std::sqrt(peak) / std::cosh(t / width) * std::exp(i * chirp_free_phase);
  }
  return a;
}

int main(int argc, char** argv) {
  const unsigned nt = 1024;
  const double window = 8.0;  // ps
  struct SimulationParameters in;
  in.n_modes = 2;
  in.fiber_length = 0.05;
  in.nt = nt;
  in.time_window = window;
  in.pulse_width = 0.08;
  in.n_steps = 200;
  in.method_order = 4;
  in.nonlinearity_const = 1.4e-13;
  in.raman_proportion = 0.18;

  in.dispersion_coefficients.push_back(std::vector<double>({0., 0., 0.0189, 2e-5}));
  in.dispersion_coefficients.push_back(std::vector<double>({250., 5e-4, 0.0186, -1e-5}));

  const double S = 6.4e12;
  // fully symmetric two-mode overlap tensor, entries listed in (k, l, m) order per p
  const double q[5] = {S, S / 3, S / 2, S / 4, 0.8 * S};
  for (unsigned p = 0; p < 2; ++p) {
    Sparse3DArray Q;
    for (unsigned k = 0; k < 2; ++k)
      for (unsigned l = 0; l < 2; ++l)
        for (unsigned m = 0; m < 2; ++m) {
          struct NonZeroValue nzv = {{k, l, m}, q[p + k + l + m]};
          Q.addNonZeroValue(nzv);
        }
    in.coupling_coefficients.push_back(Q);
  }

  in.raman_response = std::vector<double>(nt);
  const double dt = window / nt, tau1 = 12.2e-3, tau2 = 32e-3;
  double norm = 0.;
  for (unsigned j = 0; j < nt; ++j) {
    const double t = (double)j * dt;
    in.raman_response[j] = std::exp(-t / tau2) * std::sin(t / tau1);
    norm += in.raman_response[j] * dt;
  }
  for (unsigned j = 0; j < nt; ++j) in.raman_response[j] /= norm;

  in.initial_fields = ComplexArraysContainer(nt, 2);
  in.initial_fields[0] = sech_pulse(nt, window, 0.08, 60.0, -0.6, 0.3);
  in.initial_fields[1] = sech_pulse(nt, window, 0.1, 25.0, 0.7, -1.1);

  MultimodePropagation* solver = new SOLVER_CLASS(in);
  solver->computeLawsonRK(in.n_steps);
  ComplexArraysContainer out(nt, 2);
  out = solver->getResult();

  FILE* f = std::fopen(argc > 1 ? argv[1] : "two_mode_out.txt", "w");
  if (!f) return 1;
  for (unsigned p = 0; p < 2; ++p)
    for (unsigned j = 0; j < nt; ++j) std::fprintf(f, "%.17g %.17g\n", out[p][j].real(), out[p][j].imag());
  std::fclose(f);
  delete solver;
  return 0;
}
