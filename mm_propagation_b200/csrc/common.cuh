// common.cuh — complex helpers and per-solve device descriptors shared by every kernel.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace mmp {

template <typename T> struct cvec;
template <> struct cvec<float> { using type = float2; };
template <> struct cvec<double> { using type = double2; };
template <typename T> using c2 = typename cvec<T>::type;

template <typename T> __host__ __device__ __forceinline__ c2<T> mk(T re, T im) {
  c2<T> r; r.x = re; r.y = im; return r;
}
template <typename V> __host__ __device__ __forceinline__ V cadd(V a, V b) { a.x += b.x; a.y += b.y; return a; }
template <typename V> __host__ __device__ __forceinline__ V csub(V a, V b) { a.x -= b.x; a.y -= b.y; return a; }
template <typename V> __host__ __device__ __forceinline__ V cmul(V a, V b) {
  V r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
// a * conj(b)
template <typename V> __host__ __device__ __forceinline__ V cmulc(V a, V b) {
  V r;
  r.x = a.x * b.x + a.y * b.y;
  r.y = a.y * b.x - a.x * b.y;
  return r;
}
template <typename V> __host__ __device__ __forceinline__ V cconj(V a) { a.y = -a.y; return a; }
template <typename V, typename S> __host__ __device__ __forceinline__ V cscale(V a, S s) {
  a.x *= s; a.y *= s; return a;
}
// multiply by i (INV=false: -i, the forward-DFT rotation; INV=true: +i)
template <bool PLUS_I, typename V> __host__ __device__ __forceinline__ V crot(V a) {
  V r;
  if (PLUS_I) { r.x = -a.y; r.y = a.x; }
  else        { r.x = a.y;  r.y = -a.x; }
  return r;
}
__device__ __forceinline__ double2 to_d2(float2 a) { return make_double2(a.x, a.y); }
__device__ __forceinline__ double2 to_d2(double2 a) { return a; }
template <typename T> __device__ __forceinline__ c2<T> from_d2(double2 a);
template <> __device__ __forceinline__ float2 from_d2<float>(double2 a) { return make_float2((float)a.x, (float)a.y); }
template <> __device__ __forceinline__ double2 from_d2<double>(double2 a) { return a; }

// Padded shared-memory index: one spare element per 32 keeps the Stockham
// passes' strided stores free of bank conflicts for 8- and 16-byte elements.
__host__ __device__ __forceinline__ int pad(int i) { return i + (i >> 5); }
__host__ __device__ constexpr int padded_len(int n) { return n + (n >> 5); }

// SolveDesc::status bits
constexpr int kStatusNonFinite = 1;  // the field became NaN/Inf
constexpr int kStatusTimeout = 2;    // a bounded device-side wait gave up
constexpr int kStatusDrift = 4;      // the FP64 energy left the band set by drift_tol

// Maximum number of RK stages (Butcher11) and dispersion orders handled.
constexpr int kMaxStages = 11;
constexpr int kMaxBeta = 13;

// One contraction term of sigma_p = sum Q * U_k * W (16 bytes), with
//   Raman off: W = U_l conj(U_m)
//   Raman on:  W = (1 - fR) U_l conj(U_m) + R_pair, R_pair the Raman convolution of the
//              pair field l<=m; for l > m the stored pair is (m, l) and R is conjugated
//              (R_lm = conj(R_ml) because h_R is real).
// pc = pair index | (conj << 15).
struct Term {
  unsigned short k;
  unsigned short l;
  unsigned short m;
  unsigned short pc;
  double q;
};
static_assert(sizeof(Term) == 16, "Term layout");

// Everything a kernel needs about one solve. Lives in device memory (an array
// of these per batch); kernels index it with blockIdx.y.
struct SolveDesc {
  int M;            // modes
  int P;            // distinct pair fields (l <= m) formed on the device
  int n_beta;       // polynomial coefficients per mode
  int raman;        // 1: Raman on (contraction adds R = h_R (*) V to (1-fR) V)
  double alpha_scale;   // 2*pi / t_final
  double dz;            // h (dimensionless)
  double sgn_gamma;     // +1 / -1
  double one_minus_fR;  // 1 - f_R (Raman on)
  double inv_nt;        // 1 / NT
  double result_scale;  // 1 / (NT * conversion_factor)
  double energy_scale;  // converts sum |psi_hat|^2 into pJ
  double omega0_T0;     // dimensionless carrier, 0 disables the photon monitor
  double photon_scale;
  const double* poly;   // [M][n_beta]: Im L_p(alpha) = sum_j poly[p][j] alpha^j
  double2* psi_hat;     // [M][NT] interaction-picture field, frequency domain, FP64
  // [M][NT] psi_hat rounded to T, written wherever psi_hat is (the intermediate stages
  // read it: they round psi_hat to T anyway); psi_hat itself in FP64 solves
  void* psi_t;
  void* Nh;             // [s][M][NT] stage derivatives, frequency domain (T2)
  void* U;              // [M][NT] stage field, time domain (T2)
  void* W;              // [P][NT] Raman-convolved pair fields R, time domain (T2)
  void* sigma;          // [M][NT] contraction output, time domain (T2)
  const void* H;        // [NT] scaled Raman spectrum (T2) or null
  double2* io;          // [M][NT] FP64 staging for upload / result
  const int2* pairs;    // [P] (l, m)
  const Term* terms;    // sorted by p
  const int* term_off;  // [M+1]
  unsigned long long* step;   // steps since the last z reset
  unsigned long long* total;  // steps since creation (monitor index)
  unsigned int* done_ctr;     // last-CTA counter of the final stage
  double* energy;             // [mon_cap]
  double* photons;            // [mon_cap]
  unsigned long long mon_cap;
  int* status;                // kStatus* bits
  int monitors;               // 1: accumulate monitors
  // Polls the contraction kernels give the first wait for their tile copy before they
  // report kStatusTimeout (they then still wait, with the full bound, for the copy to
  // land before leaving). The host sets it far above any copy time.
  unsigned tile_wait_polls;
  // Stage kernels do nothing for this solve once *step >= step_limit (a solve in a
  // served pool stops at its own step count while the pool's graph keeps running).
  unsigned long long step_limit;
  // Raman response as a damped sinusoid h_i = Im(c lambda^i) (k_raman_scan): iir = 1
  // when the sampled h_R fits it; kappa = Delta_t T0 f_R c (1 - lambda^NT),
  // inv_one_minus = 1 / (1 - lambda^NT).
  int iir;
  int pad2_;
  double2 iir_lambda;
  double2 iir_kappa;
  double2 iir_inv_one_minus;
  // [kRamanPow] (T complex): lambda^j, j < kRamanPow, computed once in FP64 (iir solves)
  const void* raman_pow;
  // [P][NT/16][2] (T complex): per contraction tile and pair field, the recurrence's
  // tile aggregate (k_raman_agg), then the state entering the tile (k_raman_carry)
  void* raman_tiles;
  // Dense form of the contraction (M <= kDenseMaxModes), T values [M][P][2 kDenseMaxModes]:
  // entry (p, q, k) sums Q over the terms of p with U_k and pair field q, entry
  // (p, q, kDenseMaxModes + k) the same with the sign of conj-read terms; null if unused
  const void* dense_q;
  // The same coefficients for the tensor-core form (FP32 solves): per chunk of kTcChunk pair
  // fields, four K-major matrices [Re hi, Re lo, Im hi, Im lo][kTcChunk/4][16 M][4] of
  // TF32 values (x = hi + lo), row (p, k) = 16 p + k; null if unused
  const float* dense_tc;
  // Energy drift check (0 = off): the last CTA of each step's final stage compares the
  // step's FP64 energy with *drift_ref (the first step's energy after creation or
  // set_fields) and sets kStatusDrift when |E - E_ref| > drift_tol E_ref.
  double drift_tol;
  double* drift_ref;
  // The contraction's terms merged per (p, k, pair field q) for k_contract_sr: a term
  // reading W_q and one reading conj(W_q) with the same k add up to
  //   U_k (a Re W_q + i b Im W_q),  a = Q1 + Q2, b = Q1 - Q2,
  // sorted by p; sr_coef holds (a, b) in T, sr_kq = q | k << 16. sr_plan assigns the modes'
  // term ranges to the kernel's groups of eight lanes, sr_rounds rounds of kSrGroups groups:
  // (p, first term, end, role), role 0 a whole mode, 1 and 2 the lower and upper halves of a
  // split one (the upper half hands its sums to the lower), 3 an empty group.
  const void* sr_coef;
  const unsigned* sr_kq;
  const int4* sr_plan;
  int sr_terms;
  int sr_rounds;
};

// Largest mode count of the dense contraction form (its accumulators live in registers),
// and the coefficient rows a warp stages in shared memory per chunk.
constexpr int kDenseMaxModes = 16;
// Powers of the Raman recurrence's lambda kept per solve (the largest contraction tile).
constexpr int kRamanPow = 256;
constexpr int kDenseChunk = 16;
// Tensor-core form of the dense contraction: samples per tile (the MMA's M), pair fields
// per K chunk, and the fewest modes a solve needs for it (from 6 modes, 21 pair fields,
// on; below that the register-blocked form costs less than a tile's MMA pipeline).
constexpr int kTcTile = 128;
constexpr int kTcChunk = 16;
constexpr int kTcMinModes = 6;

// RK tableau passed by value to the stage kernels (identical for a batch).
struct Tableau {
  int s;
  int last_b;                 // index of the last stage with b != 0
  double a[kMaxStages][kMaxStages];
  double b[kMaxStages];
  double c[kMaxStages];
};

}  // namespace mmp
