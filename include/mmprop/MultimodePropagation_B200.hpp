// MultimodePropagation_B200.hpp — the B200 solver behind the reference's class
// interface. A driver written for MultimodePropagationCPU_RamanOFF/ON or
// MultimodePropagationGPU_RamanOFF/ON (include/MultimodePropagation_CPU.hpp:31-53,
// include/MultimodePropagation_GPU.cuh:54-85) switches by including this header and
// naming MultimodePropagationB200_RamanOFF/ON. Everything runs in libmmp_b200.so
// (link -lmmp_b200); errors throw std::runtime_error with the library's message.
//
// The optional `flags` argument takes MMP_F_* values from mmp.h, e.g. MMP_F_FP64
// for all-FP64 arithmetic or MMP_F_CONTINUOUS to carry z across calls.
#ifndef MMPROP_B200_MULTIMODE_PROPAGATION_B200_HPP
#define MMPROP_B200_MULTIMODE_PROPAGATION_B200_HPP

#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

#include "MultimodePropagation.hpp"
#include "mmp.h"

class MultimodePropagationB200 : public MultimodePropagation {
 public:
  using MultimodePropagation::computeLawsonRK;

  MultimodePropagationB200(const SimulationParameters& in, bool raman, unsigned int flags = 0) {
    const unsigned M = in.n_modes, nt = in.nt;
    if (in.dispersion_coefficients.size() != M || in.coupling_coefficients.size() != M)
      throw std::invalid_argument("dispersion_coefficients and coupling_coefficients need n_modes entries");
    const unsigned L = M ? (unsigned)in.dispersion_coefficients[0].size() : 0;
    beta_.resize((size_t)M * L);
    for (unsigned p = 0; p < M; ++p) {
      if (in.dispersion_coefficients[p].size() != L)
        throw std::invalid_argument("every mode needs the same number of dispersion coefficients");
      for (unsigned i = 0; i < L; ++i) beta_[(size_t)p * L + i] = in.dispersion_coefficients[p][i];
    }
    for (unsigned p = 0; p < M; ++p) {
      const Sparse3DArray& Q = in.coupling_coefficients[p];
      for (unsigned j = 0; j < Q.getNumberOfNonZeroValues(); ++j) {
        const NonZeroValue v = Q.getNonZeroValue(j);
        mmp_nz e = {p, v.index[0], v.index[1], v.index[2], v.value};
        nz_.push_back(e);
      }
    }
    ComplexArraysContainer fields = in.initial_fields;
    if (fields.getNumberOfArrays() != M || fields.getArraySize() != nt)
      throw std::invalid_argument("initial_fields must be a ComplexArraysContainer(nt, n_modes)");
    phi0_.resize((size_t)2 * M * nt);
    for (unsigned p = 0; p < M; ++p)
      for (unsigned t = 0; t < nt; ++t) {
        phi0_[2 * ((size_t)p * nt + t)] = fields[p][t].real();
        phi0_[2 * ((size_t)p * nt + t) + 1] = fields[p][t].imag();
      }
    if (raman && in.raman_response.size() < nt)
      throw std::invalid_argument("raman_response needs nt samples for a Raman-on solver");
    mmp_params prm = {};
    prm.n_modes = M;
    prm.nt = nt;
    prm.n_beta = L;
    prm.dispersion = beta_.data();
    prm.n_nonzeros = (uint32_t)nz_.size();
    prm.coupling = nz_.empty() ? nullptr : nz_.data();
    prm.initial_fields = phi0_.data();
    prm.time_window = in.time_window;
    prm.pulse_width = in.pulse_width;
    prm.fiber_length = in.fiber_length;
    prm.n_steps = in.n_steps;
    prm.method_order = in.method_order;
    prm.nonlinearity_const = in.nonlinearity_const;
    prm.raman_proportion = in.raman_proportion;
    prm.raman_response = raman ? in.raman_response.data() : nullptr;
    prm.raman = raman ? 1 : 0;
    prm.flags = flags;
    check(mmp_solver_create(&prm, &s_), "mmp_solver_create");
    mmp_info info;
    check(mmp_get_info(s_, &info), "mmp_get_info");
    M_ = M;
    nt_ = nt;
    default_steps_ = (unsigned)std::floor(info.z_final / info.delta_z);
  }

  ~MultimodePropagationB200() override { mmp_solver_destroy(s_); }
  MultimodePropagationB200(const MultimodePropagationB200&) = delete;
  MultimodePropagationB200& operator=(const MultimodePropagationB200&) = delete;

  void computeLawsonRK(const unsigned int nz) override { check(mmp_propagate(s_, nz), "computeLawsonRK"); }

  ComplexArraysContainer getResult() override {
    std::vector<double> out((size_t)2 * M_ * nt_);
    check(mmp_get_result(s_, out.data()), "getResult");
    ComplexArraysContainer phi(nt_, M_);
    for (unsigned p = 0; p < M_; ++p)
      for (unsigned t = 0; t < nt_; ++t)
        phi[p][t] = Complex(out[2 * ((size_t)p * nt_ + t)], out[2 * ((size_t)p * nt_ + t) + 1]);
    return phi;
  }

  // FP64 energy (pJ) after each step since construction.
  std::vector<double> getEnergyMonitor() {
    mmp_info info;
    check(mmp_get_info(s_, &info), "mmp_get_info");
    std::vector<double> e(info.steps_done ? info.steps_done : 1);
    uint64_t n = 0;
    check(mmp_get_monitors(s_, e.data(), nullptr, info.steps_done, &n), "mmp_get_monitors");
    e.resize(n);
    return e;
  }

  // The MEX front end's n_save loop (matlab/mm_propagation.cpp:61-91): the result
  // after each of n_save chunks of n_steps / n_save steps (the last one takes the
  // remainder) with its position Z (m) and the seconds since the call began.
  // referenceZ = true restarts z at each chunk as the reference's computeLawsonRK does;
  // the default carries z on, so every snapshot is the field at its Z.
  struct Snapshot {
    double Z;
    ComplexArraysContainer fields;
    double cpu_time;
  };
  std::vector<Snapshot> computeSnapshots(unsigned int n_save, bool referenceZ = false) {
    std::vector<double> f((size_t)2 * M_ * nt_ * (n_save ? n_save : 1)), z(n_save ? n_save : 1),
        t(n_save ? n_save : 1);
    check(mmp_propagate_snapshots(s_, n_save, referenceZ ? 1 : 0, f.data(), z.data(), t.data()),
          "computeSnapshots");
    std::vector<Snapshot> out;
    for (unsigned i = 0; i < n_save; ++i) {
      ComplexArraysContainer phi(nt_, M_);
      const double* a = f.data() + (size_t)i * 2 * M_ * nt_;
      for (unsigned p = 0; p < M_; ++p)
        for (unsigned s = 0; s < nt_; ++s) phi[p][s] = Complex(a[2 * ((size_t)p * nt_ + s)], a[2 * ((size_t)p * nt_ + s) + 1]);
      out.push_back(Snapshot{z[i], phi, t[i]});
    }
    return out;
  }

  mmp_solver* handle() { return s_; }

 private:
  static void check(int rc, const char* where) {
    if (rc != MMP_OK)
      throw std::runtime_error(std::string(where) + ": " + mmp_strerror(rc) + ": " + mmp_last_error());
  }
  mmp_solver* s_ = nullptr;
  unsigned M_ = 0, nt_ = 0;
  std::vector<double> beta_, phi0_;
  std::vector<mmp_nz> nz_;
};

class MultimodePropagationB200_RamanOFF : public MultimodePropagationB200 {
 public:
  explicit MultimodePropagationB200_RamanOFF(const SimulationParameters& in, unsigned int flags = 0)
      : MultimodePropagationB200(in, false, flags) {}
};

class MultimodePropagationB200_RamanON : public MultimodePropagationB200 {
 public:
  explicit MultimodePropagationB200_RamanON(const SimulationParameters& in, unsigned int flags = 0)
      : MultimodePropagationB200(in, true, flags) {}
};

#endif
