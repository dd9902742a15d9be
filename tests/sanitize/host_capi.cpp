// Drives the C ABI's host-only paths (no device needed) for a build of the library's host
// code under AddressSanitizer and UndefinedBehaviorSanitizer: parameter validation (valid
// and malformed inputs), RK tableaus, dense-coupling conversion, the MAT-file and text
// writers and the error strings. Exit status 0 when every call returned what it should;
// the sanitizers abort the process on the first error they find.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "mmp.h"

#if !defined(__SANITIZE_ADDRESS__)
#error "host_capi.cpp is built with -fsanitize=address (tests/test_host_sanitize.py)"
#endif

static int failures = 0;
#define CHECK(cond)                                                        \
  do {                                                                     \
    if (!(cond)) {                                                         \
      std::fprintf(stderr, "check failed at line %d: %s\n", __LINE__, #cond); \
      ++failures;                                                          \
    }                                                                      \
  } while (0)

int main(int argc, char** argv) {
  const std::string dir = argc > 1 ? argv[1] : ".";
  const uint32_t M = 3, NT = 256, L = 4;
  std::vector<double> beta(M * L, 0.0);
  for (uint32_t p = 0; p < M; ++p) {
    beta[p * L + 0] = 10.0 * p;
    beta[p * L + 1] = 1e-3 * p;
    beta[p * L + 2] = 0.02;
    beta[p * L + 3] = 5e-5;
  }
  std::vector<mmp_nz> q;
  for (uint32_t p = 0; p < M; ++p)
    for (uint32_t k = 0; k < M; ++k) q.push_back(mmp_nz{p, k, (p + k) % M, (p + 2 * k) % M, 1e12 * (1 + p + k)});
  std::vector<double> phi0(2 * M * NT), hr(NT);
  for (uint32_t i = 0; i < 2 * M * NT; ++i) phi0[i] = std::sin(0.01 * i);
  for (uint32_t i = 0; i < NT; ++i) hr[i] = std::exp(-0.05 * i) * std::sin(0.2 * i);
  mmp_params p;
  std::memset(&p, 0, sizeof(p));
  p.n_modes = M;
  p.nt = NT;
  p.n_beta = L;
  p.dispersion = beta.data();
  p.n_nonzeros = (uint32_t)q.size();
  p.coupling = q.data();
  p.initial_fields = phi0.data();
  p.time_window = 10.0;
  p.pulse_width = 0.1;
  p.fiber_length = 0.1;
  p.n_steps = 100;
  p.method_order = 4;
  p.nonlinearity_const = 1e-13;
  p.raman = 1;
  p.raman_proportion = 0.18;
  p.raman_response = hr.data();
  char msg[256];
  CHECK(mmp_validate_params(&p, msg, sizeof(msg)) == MMP_OK);
  CHECK(mmp_validate_params(&p, msg, 1) == MMP_OK);  // a one-byte message buffer

  // malformed inputs: each is rejected with a message, and nothing reads past its arrays
  {
    mmp_params b = p;
    b.nt = 100;
    CHECK(mmp_validate_params(&b, msg, sizeof(msg)) != MMP_OK && msg[0]);
    b = p;
    b.dispersion = nullptr;
    CHECK(mmp_validate_params(&b, msg, sizeof(msg)) == MMP_EINVAL);
    b = p;
    b.n_beta = 2;
    CHECK(mmp_validate_params(&b, msg, sizeof(msg)) == MMP_EINVAL);
    std::vector<mmp_nz> bad = q;
    bad.back().l = M;  // index out of range
    b = p;
    b.coupling = bad.data();
    CHECK(mmp_validate_params(&b, msg, sizeof(msg)) == MMP_EINVAL);
    std::vector<double> nan_beta = beta;
    nan_beta[5] = std::nan("");
    b = p;
    b.dispersion = nan_beta.data();
    CHECK(mmp_validate_params(&b, msg, sizeof(msg)) == MMP_EINVAL);
    std::vector<double> inf_phi = phi0;
    inf_phi[2 * M * NT - 1] = INFINITY;
    b = p;
    b.initial_fields = inf_phi.data();
    CHECK(mmp_validate_params(&b, msg, sizeof(msg)) == MMP_EINVAL);
    b = p;
    b.raman_response = nullptr;
    CHECK(mmp_validate_params(&b, msg, sizeof(msg)) == MMP_EINVAL);
    CHECK(mmp_validate_params(nullptr, msg, sizeof(msg)) == MMP_EINVAL);
    CHECK(mmp_validate_params(&p, nullptr, 0) == MMP_OK);
  }

  // RK tableaus
  for (uint32_t order : {4u, 6u, 8u}) {
    uint32_t s = 0;
    double a[144], b[12], c[12];
    CHECK(mmp_tableau(order, 0, 0.0, 0.0, &s, a, b, c) == MMP_OK && s >= 4 && s <= 12);
    double sb = 0.0;
    for (uint32_t i = 0; i < s; ++i) sb += b[i];
    CHECK(std::fabs(sb - 1.0) < 1e-12);
  }
  {
    uint32_t s = 0;
    double a[144], b[12], c[12];
    CHECK(mmp_tableau(6, MMP_RK_BUTCHER7_LAMBDA_MU, 0.5, 0.25, &s, a, b, c) == MMP_OK);
  }

  // dense coupling -> non-zeros, in MATLAB element order; a buffer of `cap` entries gets at
  // most cap of them (here exactly two entries long, so the sanitizer sees any write
  // beyond), the count is always the full one, and a NULL buffer only counts
  {
    std::vector<double> dense((size_t)M * M * M * M, 0.0);
    for (size_t i = 0; i < dense.size(); i += 7) dense[i] = 1.0 + (double)i;
    const uint32_t want = (uint32_t)((dense.size() + 6) / 7);
    uint32_t n = 0;
    std::vector<mmp_nz> out(dense.size());
    CHECK(mmp_coupling_from_dense(M, dense.data(), out.data(), (uint32_t)out.size(), &n) == MMP_OK && n == want);
    CHECK(out[1].p == 7 % M && out[1].value == 8.0);
    std::vector<mmp_nz> two(2);
    CHECK(mmp_coupling_from_dense(M, dense.data(), two.data(), 2, &n) == MMP_OK && n == want);
    CHECK(mmp_coupling_from_dense(M, dense.data(), nullptr, 0, &n) == MMP_OK && n == want);
    CHECK(mmp_coupling_from_dense(M, nullptr, nullptr, 0, &n) == MMP_EINVAL);
  }

  // writers
  CHECK(mmp_write_abs_text((dir + "/abs.txt").c_str(), M, NT, phi0.data(), phi0.data()) == MMP_OK);
  CHECK(mmp_write_mat((dir + "/out.mat").c_str(), "savename_1", 0.1, M, NT, phi0.data(), 1.5) == MMP_OK);
  CHECK(mmp_write_mat((dir + "/no/such/dir/out.mat").c_str(), "x", 0.1, M, NT, phi0.data(), 1.5) != MMP_OK);
  CHECK(std::strlen(mmp_last_error()) > 0);

  // error strings
  for (int code = 1; code >= -12; --code) CHECK(mmp_strerror(code) != nullptr);
  CHECK(mmp_version() != nullptr);

  if (failures) std::fprintf(stderr, "%d checks failed\n", failures);
  else std::printf("host C ABI: all checks passed\n");
  return failures ? 1 : 0;
}
