// RungeKutta.hpp — drop-in for the reference's Butcher tableau builders
// (include/RungeKutta.hpp:10-22). The coefficients come from the library
// (mmp_tableau), i.e. exactly the tableaus the solver integrates with.
#ifndef MMPROP_B200_RUNGE_KUTTA_HPP
#define MMPROP_B200_RUNGE_KUTTA_HPP

#include <stdexcept>
#include <vector>

#include "mmp.h"

typedef std::vector<double> doubleArray;

struct RungeKuttaCoefficients {
  unsigned int s;
  std::vector<doubleArray> a;  // row i holds a_ij for j < max(i, 1), as in the reference
  doubleArray b;
  doubleArray c;
};

namespace mmprop_detail {
inline void fill_tableau(RungeKuttaCoefficients& RK, unsigned order, int variant, double lam, double mu) {
  uint32_t s = 0;
  double a[121], b[11], c[11];
  if (mmp_tableau(order, variant, lam, mu, &s, a, b, c) != MMP_OK) throw std::runtime_error("mmp_tableau failed");
  RK.s = s;
  RK.a.assign(s, doubleArray());
  for (unsigned i = 0; i < s; ++i) {
    const unsigned len = i == 0 ? 1 : i;
    for (unsigned j = 0; j < len; ++j) RK.a[i].push_back(a[i * 11 + j]);
  }
  RK.b.assign(b, b + s);
  RK.c.assign(c, c + s);
}
}  // namespace mmprop_detail

inline void Butcher4(RungeKuttaCoefficients& RK) { mmprop_detail::fill_tableau(RK, 4, MMP_RK_BY_ORDER, 0, 0); }
// The solver only ever uses nu = 1 (src/MultimodePropagation.cpp:20).
inline void Butcher7(RungeKuttaCoefficients& RK, const double nu) {
  if (nu != 1.0) throw std::invalid_argument("Butcher7(nu): this build provides nu = 1, the value the solver uses");
  mmprop_detail::fill_tableau(RK, 6, MMP_RK_BY_ORDER, 0, 0);
}
inline void Butcher7(RungeKuttaCoefficients& RK, const double lambda, const double mu) {
  mmprop_detail::fill_tableau(RK, 6, MMP_RK_BUTCHER7_LAMBDA_MU, lambda, mu);
}
inline void Butcher11(RungeKuttaCoefficients& RK) { mmprop_detail::fill_tableau(RK, 8, MMP_RK_BY_ORDER, 0, 0); }

#endif
