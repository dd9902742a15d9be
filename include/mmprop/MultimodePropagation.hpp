// MultimodePropagation.hpp — drop-in for the reference's solver interface
// (include/MultimodePropagation.hpp:16-94): struct SimulationParameters (also
// available as InputParameters, README.md:71) and the abstract solver with
// computeLawsonRK(nz), computeLawsonRK() and getResult(). The destructor is
// virtual here (drivers delete through the base pointer, simulations/main.cpp:107).
#ifndef MMPROP_B200_MULTIMODE_PROPAGATION_HPP
#define MMPROP_B200_MULTIMODE_PROPAGATION_HPP

#include <algorithm>
#include <fstream>
#include <iostream>

#include "ComplexArraysContainer.hpp"
#include "RungeKutta.hpp"
#include "Sparse3DArray.hpp"

typedef std::vector<double> doubleArray;

struct SimulationParameters {
  unsigned int n_modes;
  double fiber_length;
  std::vector<doubleArray> dispersion_coefficients;
  std::vector<Sparse3DArray> coupling_coefficients;

  unsigned int nt;
  double time_window;
  double pulse_width;
  ComplexArraysContainer initial_fields;

  unsigned int n_steps;
  unsigned int method_order;
  double nonlinearity_const;
  double raman_proportion;
  doubleArray raman_response;
};

// `struct InputParameters input;` as in the reference's README.
struct InputParameters : SimulationParameters {};

class MultimodePropagation {
 public:
  virtual ~MultimodePropagation() {}
  virtual void computeLawsonRK(const unsigned int nz) = 0;
  // nz = floor(z_final / delta_z) (src/MultimodePropagation.cpp:213-216)
  void computeLawsonRK() { computeLawsonRK(default_steps_); }
  virtual ComplexArraysContainer getResult() = 0;

 protected:
  unsigned int default_steps_ = 0;
};

#endif
