// stage_kernels.cuh — the fused Lawson–RK stage kernels.
//
// The solver keeps the interaction-picture field in the FREQUENCY domain
// (psi_hat = FFT(psi), FP64). The reference keeps psi in the time domain and
// runs FFT -> *E_i -> IFFT on it in every stage
// (src/MultimodePropagation_CPU.cpp:114-119); since the FFT is linear,
// FFT(psi + h sum a_ij N_j) = psi_hat + h sum a_ij N_hat_j, so each stage needs
// one inverse transform per mode to get U and one forward transform per mode
// to turn sigma into N_hat, instead of two of each.
//
// One RK stage i of step n is, with Raman on and h_R a damped sinusoid (every workload),
// four launches; two with Raman off:
//   k_raman_agg    per time tile:   the Raman recurrence's aggregate over the tile for
//                                   every pair field V = U_l conj(U_m)
//   k_raman_carry  per pair field:  tile aggregates -> the state entering each tile
//   k_contract     per time tile:   R through the tile from that state, then
//                                   sigma_p = sum Q U_k [(1-fR) V_lm + R_lm] (all p)
//                  (k_contract_pc for tiles with too many pair fields to hold at once,
//                   k_contract_tc for dense Q on the tensor cores)
//   k_nu           per mode p:      FFT(sigma_p) -> N_hat_i = i sgn(gamma) conj(E_i) *.,
//                                   [last stage: psi_hat += h sum b_j N_hat_j, monitors],
//                                   x_hat = psi_hat + h sum a_{i+1,j} N_hat_j,
//                                   * E_{i+1} -> IFFT -> U for the next stage
// Any other h_R takes k_pair (V -> FFT -> * H_R -> IFFT = R per pair field) instead of
// the first two, and k_contract reads R as rows. k_prime makes U for stage 0 when a
// propagate call starts. E_i = exp(i Im L_p(w) z) is never stored: the phase
// Im L_p(w) * (z_n + c_i h) is evaluated in FP64, reduced in FP64 and only then passed
// to sin/cos in T.
#pragma once

#include <type_traits>

#include "fft.cuh"
#include "tc_sm100.cuh"

namespace mmp {

struct KParams {
  const SolveDesc* descs;
  TwTables tw;
  Tableau tab;
  int stage;
  int pad_;
};

// Im L_p(alpha) by Horner over the per-mode polynomial (FP64).
__device__ __forceinline__ double im_L(const double* poly, int nb, double alpha) {
  double r = poly[nb - 1];
  for (int j = nb - 2; j >= 0; --j) r = fma(r, alpha, poly[j]);
  return r;
}

// Small integer -> double without the conversion unit: the bits 0x43300000:(j + 2^31) are
// the double 2^52 + 2^31 + j (exact for |j| < 2^31), so one subtraction leaves j.
__device__ __forceinline__ double int_to_double(int j) {
  return __hiloint2double(0x43300000, (int)((unsigned)j ^ 0x80000000u)) - 4503601774854144.0;
}

__device__ __forceinline__ double alpha_of(int k, int nt, double alpha_scale) {
  // src/MultimodePropagation.cpp:167-171: index j <= nt/2 -> j, else j - nt
  const int kk = (k <= (nt >> 1)) ? k : k - nt;
  return alpha_scale * int_to_double(kk);
}

// exp(i theta) with theta reduced in FP64 (Cody–Waite with a two-part constant).
// FP32: reduced by pi/2 to x in [-pi/4, pi/4] and quadrant n mod 4 (n = theta 2/pi rounded
// by adding 1.5 * 2^52, whose ulp is 1: n and its low bits come out of one FMA, with
// no conversion instruction; valid for |theta 2/pi| < 2^51), then the Taylor
// series of sin and cos to x^9 and x^10 (truncation below 2e-9 on that interval),
// evaluated by Horner in x^2 in FP32; the quadrant swaps and negates. Short, branch-free
// code with no large-argument path (the argument is already small). FP64: reduced by
// 2 pi, then sincos.
template <typename T> __device__ __forceinline__ c2<T> expi(double theta) {
  if constexpr (sizeof(T) == 4) {
    constexpr double k2OverPi = 0.63661977236758134308;
    constexpr double kHalfPiHi = 1.57079632679489655800;    // nearest double to pi/2
    constexpr double kHalfPiLo = 6.12323399573676603587e-17;  // pi/2 - kHalfPiHi
    constexpr double kRound = 6755399441055744.0;  // 1.5 * 2^52
    const double t = fma(theta, k2OverPi, kRound);
    const double n = t - kRound;
    const double r = fma(-n, kHalfPiLo, fma(-n, kHalfPiHi, theta));
    const float x = (float)r, x2 = x * x;
    // sin x = x (1 - x^2/3! + x^4/5! - x^6/7! + x^8/9!), cos x = 1 - x^2/2! + ... - x^10/10!
    const float sp =
        x * fmaf(x2, fmaf(x2, fmaf(x2, fmaf(x2, 1.0f / 362880.0f, -1.0f / 5040.0f), 1.0f / 120.0f), -1.0f / 6.0f), 1.0f);
    const float cp = fmaf(
        x2, fmaf(x2, fmaf(x2, fmaf(x2, fmaf(x2, -1.0f / 3628800.0f, 1.0f / 40320.0f), -1.0f / 720.0f), 1.0f / 24.0f),
                 -0.5f),
        1.0f);
    const int q = __double2loint(t) & 3;
    const float c = (q & 1) ? sp : cp, s = (q & 1) ? cp : sp;
    return make_float2((q == 1 || q == 2) ? -c : c, (q >= 2) ? -s : s);
  } else {
    constexpr double kInv2Pi = 0.15915494309189533577;
    constexpr double kTwoPiHi = 6.28318530717958623200;   // nearest double to 2 pi
    constexpr double kTwoPiLo = 2.4492935982947063697e-16;  // 2 pi - kTwoPiHi
    const double n = rint(theta * kInv2Pi);
    double r = fma(-n, kTwoPiHi, theta);
    r = fma(-n, kTwoPiLo, r);
    double s, c;
    sincos(r, &s, &c);
    return make_double2(c, s);
  }
}

template <typename T> __device__ __forceinline__ c2<T>* as_t2(void* p) { return reinterpret_cast<c2<T>*>(p); }
template <typename T> __device__ __forceinline__ const c2<T>* as_t2(const void* p) { return reinterpret_cast<const c2<T>*>(p); }

// two adjacent complex samples (one 16-byte access in FP32; p 16-byte aligned)
template <typename T>
__device__ __forceinline__ void ld2(const c2<T>* p, c2<T>& a, c2<T>& b) {
  a = p[0];
  b = p[1];
}
template <>
__device__ __forceinline__ void ld2<float>(const float2* p, float2& a, float2& b) {
  const float4 v = *reinterpret_cast<const float4*>(p);
  a = make_float2(v.x, v.y);
  b = make_float2(v.z, v.w);
}
template <typename T>
__device__ __forceinline__ void st2(c2<T>* p, c2<T> a, c2<T> b) {
  p[0] = a;
  p[1] = b;
}
template <>
__device__ __forceinline__ void st2<float>(float2* p, float2 a, float2 b) {
  *reinterpret_cast<float4*>(p) = make_float4(a.x, a.y, b.x, b.y);
}

__device__ __forceinline__ void load_poly(double* poly, const SolveDesc& d, int p) {
  if (threadIdx.x < d.n_beta) poly[threadIdx.x] = d.poly[p * d.n_beta + threadIdx.x];
  __syncthreads();
}

// One warp copies this CTA's solve descriptor into shared memory in a single round
// trip, instead of every field becoming its own dependent global load. The caller
// synchronises before reading it.
static_assert(sizeof(SolveDesc) % 8 == 0, "descriptor copied in 8-byte words");
__device__ __forceinline__ void stage_desc(SolveDesc* dst, const SolveDesc* src) {
  constexpr int W = (int)(sizeof(SolveDesc) / 8);
  for (int i = threadIdx.x; i < W; i += blockDim.x)
    reinterpret_cast<unsigned long long*>(dst)[i] = __ldg(reinterpret_cast<const unsigned long long*>(src) + i);
}

// Ask the TMA engine to pull [p, p + bytes) into L2 without waiting for it
// (p 16-byte aligned, bytes a multiple of 16). Used to have a row ready in L2 by the
// time a kernel's epilogue reads it.
__device__ __forceinline__ void prefetch_l2(const void* p, unsigned bytes) {
  constexpr unsigned kPiece = 64u * 1024u;
  const char* c = static_cast<const char*>(p);
  for (unsigned off = 0; off < bytes; off += kPiece) {
    const unsigned n = bytes - off < kPiece ? bytes - off : kPiece;
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(c + off), "r"(n) : "memory");
  }
}

// Ampere-style asynchronous copies global -> shared (both addresses aligned to the size),
// grouped and waited for per thread: the loads are in flight without holding registers.
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gmem_src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(gmem_src) : "memory");
}
// one complex value of T
template <typename T> __device__ __forceinline__ void cp_async_c2(c2<T>* smem_dst, const c2<T>* gmem_src) {
  if constexpr (sizeof(c2<T>) == 8) cp_async8(smem_dst, gmem_src);
  else cp_async16(smem_dst, gmem_src);
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <typename G> __device__ __forceinline__ int cluster_rank() {
  if constexpr (G::C == 1) return 0;
  else return (int)cg::this_cluster().block_rank();
}

// Common start of a row kernel: shared memory (the row, then the twiddle table).
#define MMP_ROW_SMEM()                                                 \
  extern __shared__ __align__(128) unsigned char smem_raw[];            \
  V* s = reinterpret_cast<V*>(smem_raw);

// ---- k_prime: U for stage `stage` from psi_hat (and the stored N_hat_j) -------------------
template <typename T, int LOGN, int XC>
__global__ void __launch_bounds__(Geo<T, LOGN, XC>::NTHR, Geo<T, LOGN, XC>::MIN_BLOCKS) k_prime(const KParams kp) {
  using Gm = Geo<T, LOGN, XC>;
  using V = c2<T>;
  MMP_ROW_SMEM();
  __shared__ double poly[kMaxBeta];
  __shared__ SolveDesc sdesc;
  stage_desc(&sdesc, kp.descs + blockIdx.y);
  const V* sq = load_twiddles<T, LOGN, XC>(smem_raw, kp.tw);
  __syncthreads();
  const SolveDesc& d = sdesc;
  const int p = blockIdx.x / Gm::C;
  if (p >= d.M) return;  // uniform over the cluster
  const int rank = cluster_rank<Gm>();
  const int tid = threadIdx.x;
  load_poly(poly, d, p);
  const int i = kp.stage;
  const unsigned long long n = __ldcg(d.step);
  const double zs = ((double)n + kp.tab.c[i]) * d.dz;
  const size_t row = (size_t)p * Gm::N;
  const size_t mstride = (size_t)d.M * Gm::N;
  const V* Nh = as_t2<T>(d.Nh);
#pragma unroll 2
  for (int li = tid; li < Gm::NL; li += Gm::NTHR) {
    const int k = Gm::freq_of(rank, li);
    double2 x = d.psi_hat[row + k];
    for (int j = 0; j < i; ++j) {
      const double aij = kp.tab.a[i][j];
      if (aij != 0.0) {
        const double2 nj = to_d2(Nh[(size_t)j * mstride + row + k]);
        x.x = fma(aij * d.dz, nj.x, x.x);
        x.y = fma(aij * d.dz, nj.y, x.y);
      }
    }
    const double th = im_L(poly, d.n_beta, alpha_of(k, Gm::N, d.alpha_scale)) * zs;
    s[Gm::sidx(li)] = cmul(from_d2<T>(x), expi<T>(th));
  }
  inverse<T, LOGN, XC>(s, sq, kp.tw);
  V* U = as_t2<T>(d.U);
  const T inv = (T)d.inv_nt;
#pragma unroll 8
  for (int w = tid; w < Gm::NL; w += Gm::NTHR) U[row + Gm::time_of_w(rank, w)] = cscale(s[Gm::sidx(Gm::local_of_w(w))], inv);
}

// ---- k_pair: R_q = IFFT(FFT(V_q) * H), V_q = U_l conj(U_m) -------------------------------
template <typename T, int LOGN, int XC>
__global__ void __launch_bounds__(Geo<T, LOGN, XC>::NTHR, Geo<T, LOGN, XC>::MIN_BLOCKS) k_pair(const KParams kp) {
  using Gm = Geo<T, LOGN, XC>;
  using V = c2<T>;
  MMP_ROW_SMEM();
  __shared__ SolveDesc sdesc;
  stage_desc(&sdesc, kp.descs + blockIdx.y);
  const V* sq = load_twiddles<T, LOGN, XC>(smem_raw, kp.tw);
  __syncthreads();
  const SolveDesc& d = sdesc;
  const int q = blockIdx.x / Gm::C;
  if (q >= d.P || __ldcg(d.step) >= d.step_limit) return;  // uniform over the cluster
  const int rank = cluster_rank<Gm>();
  const int tid = threadIdx.x;
  const int2 lm = d.pairs[q];
  const V* U = as_t2<T>(d.U);
  const size_t rl = (size_t)lm.x * Gm::N, rm = (size_t)lm.y * Gm::N;
  if constexpr (Gm::C == 1 && sizeof(T) == 4) {
    // one CTA per row: two consecutive samples per 16-byte load
    const float4* Ul = reinterpret_cast<const float4*>(U + rl);
    const float4* Um = reinterpret_cast<const float4*>(U + rm);
#pragma unroll 8
    for (int u2 = tid; u2 < Gm::NL / 2; u2 += Gm::NTHR) {
      const float4 a = Ul[u2], b = Um[u2];
      s[pad(2 * u2)] = cmulc(make_float2(a.x, a.y), make_float2(b.x, b.y));
      s[pad(2 * u2 + 1)] = cmulc(make_float2(a.z, a.w), make_float2(b.z, b.w));
    }
  } else {
#pragma unroll 8
    for (int w = tid; w < Gm::NL; w += Gm::NTHR) {
      const int t = Gm::time_of_w(rank, w);
      s[Gm::sidx(Gm::local_of_w(w))] = cmulc(U[rl + t], U[rm + t]);
    }
  }
  forward<T, LOGN, XC>(s, sq, kp.tw);
  const V* H = as_t2<T>(d.H);
  if constexpr (Gm::C == 1 && sizeof(T) == 4) {
    const float4* H4 = reinterpret_cast<const float4*>(H);
#pragma unroll 8
    for (int k2 = tid; k2 < Gm::NL / 2; k2 += Gm::NTHR) {
      const float4 hh = __ldg(&H4[k2]);
      s[pad(2 * k2)] = cmul(s[pad(2 * k2)], make_float2(hh.x, hh.y));
      s[pad(2 * k2 + 1)] = cmul(s[pad(2 * k2 + 1)], make_float2(hh.z, hh.w));
    }
  } else {
#pragma unroll 4
    for (int li = tid; li < Gm::NL; li += Gm::NTHR) s[Gm::sidx(li)] = cmul(s[Gm::sidx(li)], __ldg(&H[Gm::freq_of(rank, li)]));
  }
  inverse<T, LOGN, XC>(s, sq, kp.tw);
  // R_q = (H_R conv V_q); the Kerr part (1 - fR) V_q is formed by the contraction from
  // the U tile it already holds
  V* R = as_t2<T>(d.W) + (size_t)q * Gm::N;
#pragma unroll 8
  for (int w = tid; w < Gm::NL; w += Gm::NTHR) R[Gm::time_of_w(rank, w)] = s[Gm::sidx(Gm::local_of_w(w))];
}

// ---- k_raman_scan: R_q = h_R (*) V_q as a periodic linear recurrence ----------------------
// Used instead of k_pair when the sampled Raman response is a damped sinusoid,
// h_i = Im(c lambda^i) for every i < NT (the model simulations/main.cpp:67-75 samples;
// the host checks the fit to 1e-10 of max|h|). With V = a + i b (a, b real) and
// w = Delta_t T0 f_R,
//   R[n] = w sum_i h_i V[(n - i) mod NT] = Im(kappa S_a[n]) + i Im(kappa S_b[n]),
//   S[n] = lambda S[n-1] + x[n]  (x = a or b, periodic in n), kappa = w c (1 - lambda^NT):
// the same circular convolution k_pair evaluates by FFT, in O(NT) per row.
// Each thread owns E consecutive samples in sub-chunks of 8. Sub-chunk scans run in T
// from zero; carries between sub-chunks and threads are FP64: a block-wide scan of
// the affine maps s -> A s + B (A = lambda^E) gives every thread the state entering its
// samples, and the periodic start S[-1] = S_lin[NT-1] / (1 - lambda^NT) closes the circle.
struct Affine {  // s -> a s + (ba, bb) for the two scans
  double2 a, ba, bb;
};
__device__ __forceinline__ Affine affine_then(const Affine& first, const Affine& second) {
  Affine r;
  r.a = cmul(first.a, second.a);
  r.ba = cadd(cmul(second.a, first.ba), second.ba);
  r.bb = cadd(cmul(second.a, first.bb), second.bb);
  return r;
}
__device__ __forceinline__ double2 shfl_up_d2(double2 v, int off, unsigned mask) {
  v.x = __shfl_up_sync(mask, v.x, off);
  v.y = __shfl_up_sync(mask, v.y, off);
  return v;
}
__device__ __forceinline__ Affine shfl_up_affine(const Affine& v, int off, unsigned mask) {
  Affine r;
  r.a = shfl_up_d2(v.a, off, mask);
  r.ba = shfl_up_d2(v.ba, off, mask);
  r.bb = shfl_up_d2(v.bb, off, mask);
  return r;
}
// inclusive scan over the lanes of a warp (lanes >= n hold identities)
__device__ __forceinline__ Affine warp_scan_affine(Affine v, int lane) {
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const Affine o = shfl_up_affine(v, off, 0xffffffffu);
    if (lane >= off) v = affine_then(o, v);
  }
  return v;
}

// Block-wide exclusive scan of the threads' maps (in thread order): returns the map of
// all earlier threads; *total receives the composition over the whole block.
__device__ __forceinline__ Affine affine_identity() {
  Affine r;
  r.a = make_double2(1.0, 0.0);
  r.ba = r.bb = make_double2(0.0, 0.0);
  return r;
}
// warp_tot holds 17 entries: per-warp totals, then (after the scan) per-warp exclusive
// prefixes in [0, 16) and the block total in [16].
__device__ __forceinline__ Affine block_scan_affine(const Affine& mine, Affine* warp_tot, Affine* total) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  const Affine incl = warp_scan_affine(mine, lane);
  if (lane == 31) warp_tot[warp] = incl;
  __syncthreads();
  if (warp == 0) {  // one warp scans the warp totals
    const Affine wt = lane < nwarps ? warp_tot[lane] : affine_identity();
    const Affine wi = warp_scan_affine(wt, lane);
    Affine we = shfl_up_affine(wi, 1, 0xffffffffu);
    if (lane == 0) we = affine_identity();
    __syncwarp();
    if (lane < nwarps) warp_tot[lane] = we;
    if (lane == 31) warp_tot[16] = wi;
  }
  __syncthreads();
  const Affine wpre = warp_tot[warp];
  *total = warp_tot[16];
  Affine lpre = shfl_up_affine(incl, 1, 0xffffffffu);  // earlier lanes of this warp
  if (lane == 0) lpre = affine_identity();
  __syncthreads();  // warp_tot is reused by the next scan
  return affine_then(wpre, lpre);
}

// Rows are processed in segments of `seg` samples (the whole row when it fits the
// 128 KB staging buffer): V = U_l conj(U_m) of a segment is formed in shared memory from
// coalesced loads, every thread scans its E consecutive samples from there, and the
// outputs are written back in place and stored coalesced. With one segment the staged
// V serves both passes; with several, pass 1 records each segment's map and pass 2
// stages every segment again.
template <typename T>
__global__ void __launch_bounds__(512) k_raman_scan(const SolveDesc* __restrict__ descs, int nt, int seg) {
  using V = c2<T>;
  constexpr int kMaxSeg = 16;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  V* sv = reinterpret_cast<V*>(smem_raw);  // padded: element i at pad(i)
  __shared__ Affine warp_tot[17];
  __shared__ Affine seg_map[kMaxSeg];
  const SolveDesc& d = descs[blockIdx.y];
  const int q = blockIdx.x;
  if (q >= d.P || __ldcg(d.step) >= d.step_limit) return;  // uniform over the CTA
  const int tid = threadIdx.x;
  const int nthr = blockDim.x;                   // 32..512, a power of two
  const int nseg = nt / seg;                     // <= kMaxSeg
  const int act = min(nthr, seg >> 3);           // threads that own samples
  const int E = seg / act;                       // a multiple of 8
  const int myE = tid < act ? E : 0;
  const int off = min(tid, act - 1) * E;
  const int2 lm = d.pairs[q];
  const V* Ul = as_t2<T>(d.U) + (size_t)lm.x * nt;
  const V* Um = as_t2<T>(d.U) + (size_t)lm.y * nt;
  V* R = as_t2<T>(d.W) + (size_t)q * nt;
  const double2 lam = d.iir_lambda;
  V pw[8];  // lambda^(k+1)
  double2 lam8;
  {
    double2 p = lam;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      pw[k] = from_d2<T>(p);
      lam8 = p;
      p = cmul(p, lam);
    }
  }
  const V lt = from_d2<T>(lam);
  // s <- lambda s + x for a real input x (two dependent FMAs per component)
  auto step = [&](V s, T x) {
    return mk<T>(fma(lt.x, s.x, fma(-lt.y, s.y, x)), fma(lt.x, s.y, lt.y * s.x));
  };
  // stage V of segment g into shared memory (coalesced: two samples per thread per load)
  auto stage = [&](int g) {
    const size_t base = (size_t)g * seg;
#pragma unroll 8
    for (int i2 = tid; i2 < (seg >> 1); i2 += nthr) {
      V ul0, ul1, um0, um1;
      ld2<T>(Ul + base + 2 * i2, ul0, ul1);
      ld2<T>(Um + base + 2 * i2, um0, um1);
      sv[pad(2 * i2)] = cmulc(ul0, um0);
      sv[pad(2 * i2 + 1)] = cmulc(ul1, um1);
    }
    __syncthreads();
  };
  // this thread's map s -> lambda^E s + (S_a, S_b) over its samples of the staged segment
  auto thread_map = [&]() {
    Affine mine;
    mine.a = make_double2(1.0, 0.0);
    mine.ba = make_double2(0.0, 0.0);
    mine.bb = make_double2(0.0, 0.0);
    for (int j = 0; j < myE; j += 8) {
      V la = mk<T>(0, 0), lb = mk<T>(0, 0);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const V x = sv[pad(off + j + k)];
        la = step(la, x.x);
        lb = step(lb, x.y);
      }
      mine.a = cmul(mine.a, lam8);
      mine.ba = cadd(cmul(lam8, mine.ba), to_d2(la));
      mine.bb = cadd(cmul(lam8, mine.bb), to_d2(lb));
    }
    return mine;
  };
  // pass 1: every segment's map (a single segment stays staged for pass 2)
  Affine pre, tot;
  for (int g = 0; g < nseg; ++g) {
    stage(g);
    pre = block_scan_affine(thread_map(), warp_tot, &tot);
    if (tid == 0) seg_map[g] = tot;
    if (nseg > 1) __syncthreads();  // the next segment overwrites sv
  }
  __syncthreads();
  // periodic start: S[-1] = S_lin[NT-1] / (1 - lambda^NT)
  Affine row;
  row.a = make_double2(1.0, 0.0);
  row.ba = row.bb = make_double2(0.0, 0.0);
  for (int g = 0; g < nseg; ++g) row = affine_then(row, seg_map[g]);
  const double2 inv = d.iir_inv_one_minus;
  double2 sa = cmul(row.ba, inv), sb = cmul(row.bb, inv);  // state entering segment 0
  const double2 kap = d.iir_kappa;
  const V kt = from_d2<T>(kap);
  // pass 2: outputs R = Im(kappa s), s = local + lambda^(k+1) C within each sub-chunk
  for (int g = 0; g < nseg; ++g) {
    if (nseg > 1) {
      stage(g);
      pre = block_scan_affine(thread_map(), warp_tot, &tot);
    }
    double2 Ca = cadd(cmul(pre.a, sa), pre.ba);
    double2 Cb = cadd(cmul(pre.a, sb), pre.bb);
    for (int j = 0; j < myE; j += 8) {
      const V kca = from_d2<T>(cmul(kap, Ca)), kcb = from_d2<T>(cmul(kap, Cb));
      V la = mk<T>(0, 0), lb = mk<T>(0, 0);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        V& cell = sv[pad(off + j + k)];
        const V x = cell;
        la = step(la, x.x);
        lb = step(lb, x.y);
        // Im(kappa local) + Im(lambda^(k+1) kappa C)
        cell = mk<T>(fma(kt.x, la.y, fma(kt.y, la.x, fma(pw[k].x, kca.y, pw[k].y * kca.x))),
                     fma(kt.x, lb.y, fma(kt.y, lb.x, fma(pw[k].x, kcb.y, pw[k].y * kcb.x))));
      }
      Ca = cadd(cmul(lam8, Ca), to_d2(la));
      Cb = cadd(cmul(lam8, Cb), to_d2(lb));
    }
    __syncthreads();
    const size_t base = (size_t)g * seg;
    for (int i2 = tid; i2 < (seg >> 1); i2 += nthr) st2<T>(R + base + 2 * i2, sv[pad(2 * i2)], sv[pad(2 * i2 + 1)]);
    // state entering the next segment
    const double2 na = cadd(cmul(seg_map[g].a, sa), seg_map[g].ba);
    const double2 nb = cadd(cmul(seg_map[g].a, sb), seg_map[g].bb);
    sa = na;
    sb = nb;
    if (nseg > 1) __syncthreads();
  }
}

// ---- k_nu: sigma_p -> N_hat_i, final accumulation, next stage's U ------------------------
// BODY: the stage arithmetic of an intermediate stage that reads n stored N_hat_j terms
// (BODY = n), of a last stage that reads n (BODY = kNuLastBody + n), or of any stage (-1).
// The host launches the instantiation that matches each stage of its tableau (RK4: 0 at
// the intermediate stages, kNuLastBody + 3 at the last), so each kernel carries one body.
constexpr int kNuLastBody = 10;
template <typename T, int LOGN, int XC, int BODY>
__global__ void __launch_bounds__(Geo<T, LOGN, XC>::NTHR, Geo<T, LOGN, XC>::MIN_BLOCKS) k_nu(const KParams kp) {
  using Gm = Geo<T, LOGN, XC>;
  using V = c2<T>;
  MMP_ROW_SMEM();
  __shared__ double poly[kMaxBeta];
  __shared__ double red[2][32];
  __shared__ SolveDesc sdesc;
  const int p = blockIdx.x / Gm::C;
  const int rank = cluster_rank<Gm>();
  const int tid = threadIdx.x;
  // The sigma row and the twiddle table start on their way first, as asynchronous copies
  // into shared memory (all of a thread's elements in flight, no registers held): the row's
  // address and the mode count come straight from the descriptor in global memory, so
  // the descriptor and polynomial round trips below overlap the row's.
  V* sq = reinterpret_cast<V*>(smem_raw + Gm::DATA_BYTES);
  {
    const c2<T>* g = tw_table<T>(kp.tw, Gm::LOGNLG);
    for (int m = tid; m < Gm::NTW; m += Gm::NTHR) cp_async_c2<T>(&sq[pad(m)], &g[m]);
    const SolveDesc* gd = kp.descs + blockIdx.y;
    if (p < __ldg(&gd->M)) {
      const V* sg = as_t2<T>(reinterpret_cast<const void*>(__ldg(reinterpret_cast<const unsigned long long*>(&gd->sigma)))) +
                    (size_t)p * Gm::N;
      for (int w = tid; w < Gm::NL; w += Gm::NTHR)
        cp_async_c2<T>(&s[Gm::sidx(Gm::local_of_w(w))], sg + Gm::time_of_w(rank, w));
    }
    cp_async_commit();
  }
  stage_desc(&sdesc, kp.descs + blockIdx.y);
  __syncthreads();
  const SolveDesc& d = sdesc;
  if (p >= d.M) {  // empty slot (its descriptor is zero); uniform over the cluster
    cp_async_wait<0>();  // no copy may land after the CTA has left
    return;
  }
  // the step counters in one round trip, shared by the finished-solve check and thread
  // 0's setup below
  const unsigned long long n_step = __ldcg(d.step), n_total = __ldcg(d.total);
  if (n_step >= d.step_limit) {  // finished solve; uniform over the cluster
    cp_async_wait<0>();
    return;
  }
  load_poly(poly, d, p);
  // Scalars needed after the forward transform live in shared memory rather than in
  // registers, so the (out-of-line) transform call has little to save and restore.
  __shared__ unsigned long long s_cnt[2];  // step since z reset, steps since creation
  __shared__ double s_z[2];               // z at this stage, z at the next stage
  // Stage-combination list: the stored N_hat_j entering x_hat (or, at the last stage,
  // psi_{n+1} = psi_n + h sum_j b_j N_j, src/MultimodePropagation_CPU.cpp:75-85) with
  // their coefficients h*a or h*b; N_hat_i itself comes from registers (cself).
  // Once the sigma loads are issued, the CTA's threads start L2 prefetches of the psi_hat
  // the cluster reads after its forward transform, so it arrives while the transform runs.
  __shared__ int s_jq[kMaxStages];
  __shared__ double s_cq[kMaxStages];
  __shared__ int s_nq;
  if (tid == 0) {
    const int i = kp.stage;
    const int S = kp.tab.s;
    const bool last = (i == S - 1);
    const double h = d.dz;
    const unsigned long long n = n_step;
    s_cnt[0] = n;
    s_cnt[1] = n_total;
    s_z[0] = ((double)n + kp.tab.c[i]) * h;
    s_z[1] = last ? ((double)(n + 1)) * h : ((double)n + kp.tab.c[i + 1]) * h;
    int nq = 0;
    if (last) {
      for (int j = 0; j < S; ++j)
        if (j != i && kp.tab.b[j] != 0.0) { s_jq[nq] = j; s_cq[nq] = kp.tab.b[j] * h; ++nq; }
    } else {
      for (int j = 0; j < i; ++j)
        if (kp.tab.a[i + 1][j] != 0.0) { s_jq[nq] = j; s_cq[nq] = kp.tab.a[i + 1][j] * h; ++nq; }
    }
    s_nq = nq;
  }
  {
    // the row's psi_hat (FP64 at the last stage, in T at the others), 1/C of it per CTA of
    // the cluster (together the frequencies every CTA reads), one piece of at most 32 KB
    // per thread. The N_hat_j are not prefetched: a wave's rows of them do not fit in L2
    // beside the rest, and measured, prefetching them too was slower.
    const bool lastp = kp.stage == kp.tab.s - 1;
    const unsigned esz = lastp ? (unsigned)sizeof(double2) : (unsigned)sizeof(V);
    const unsigned bytes = Gm::NL * esz;
    const unsigned piece = bytes < 32u * 1024u ? bytes : 32u * 1024u;
    const char* base = reinterpret_cast<const char*>(lastp ? (const void*)d.psi_hat : d.psi_t) +
                       ((size_t)p * Gm::N + (size_t)rank * Gm::NL) * esz;
    for (unsigned t = tid; t < bytes / piece; t += Gm::NTHR) prefetch_l2(base + (size_t)t * piece, piece);
  }
  cp_async_wait<0>();                  // this thread's sigma and twiddle copies
  forward<T, LOGN, XC>(s, sq, kp.tw);  // its barriers publish them and the values thread 0 wrote
  const int i = kp.stage;
  const int S = kp.tab.s;
  // a specialised BODY serves intermediate or last stages only: fixed at compile time, so
  // each instantiation carries only its half of the stage arithmetic
  const bool last = BODY < 0 ? (i == S - 1) : (BODY >= kNuLastBody);
  const double h = d.dz;
  const size_t row = (size_t)p * Gm::N;
  const size_t mstride = (size_t)d.M * Gm::N;
  V* Nh = as_t2<T>(d.Nh);
  V* psiT = as_t2<T>(d.psi_t);
  // FP32 stage bodies of one kind read psi_hat's T copy at the intermediate stages; the
  // FP64 ones (psi_t is psi_hat) and the any-stage body read psi_hat
  constexpr bool kReadT = sizeof(T) == 4 && BODY >= 0;
  const double zi = s_z[0], znext = s_z[1];
  double e_part = 0.0, p_part = 0.0;
  bool finite = true;
  const int nq = s_nq;
  const double cself = (last ? kp.tab.b[i] : kp.tab.a[i + 1][i]) * h;
  // spectrum entering the inverse transform: conjugated when it runs as a forward one
  auto spec_in = [](V v) { return Gm::C == 1 ? cconj(v) : v; };
  constexpr int MAXQ = 6;
  // Fast path, one body per count of stored terms (no predicated dead work): all loads
  // of a chunk of frequencies are issued before its math. Intermediate stages combine
  // x_hat in T (it only feeds the nonlinearity, which runs in T); the last stage
  // accumulates psi_{n+1} in FP64.
  // E_{i+1} = E_i when z does not move between the stages (RK4: c_2 = c_3, c_4 = 1)
  const bool same_z = zi == znext;
  float p_part_f = 0.0f;
  const float w0f = (float)d.omega0_T0, asf = (float)d.alpha_scale;
  // NQ: the (compile-time) most stored terms the body reads; nqr: how many it reads
  auto body = [&](auto nqc, int nqr) {
    constexpr int NQ = decltype(nqc)::value;
    // frequencies per chunk: all of a chunk's loads are in flight together (8 when the
    // stage reads only psi_hat; 4 also with 4 or 5 stored terms, where 2 was measured 3%
    // slower on the 28-mode sweep and 2% on the 6-mode order-6 batch)
    constexpr int CHK0 = NQ == 0 ? 8 : 4;
    constexpr int CHK = CHK0 < Gm::E ? CHK0 : Gm::E;
    const double nb3 = d.n_beta == 3;
#pragma unroll 1
    for (int e0 = 0; e0 < Gm::E; e0 += CHK) {
      int kk[CHK];
      double2 ps[CHK];  // last stage: psi_hat in FP64
      V pt[CHK];        // other stages: psi_hat in T
      V sv[CHK];
      V nj[CHK][NQ > 0 ? NQ : 1];
#pragma unroll
      for (int c = 0; c < CHK; ++c) {
        const int li = tid + (e0 + c) * Gm::NTHR;
        kk[c] = Gm::freq_of(rank, li);
        if constexpr (!kReadT) ps[c] = d.psi_hat[row + kk[c]];
        else if (last) ps[c] = d.psi_hat[row + kk[c]];
        else pt[c] = psiT[row + kk[c]];
        sv[c] = s[Gm::sidx(li)];
#pragma unroll
        for (int q = 0; q < NQ; ++q)
          if (q < nqr) nj[c][q] = Nh[(size_t)s_jq[q] * mstride + row + kk[c]];
      }
#pragma unroll
      for (int c = 0; c < CHK; ++c) {
        const int li = tid + (e0 + c) * Gm::NTHR;
        const int k = kk[c];
        const double alpha = alpha_of(k, Gm::N, d.alpha_scale);
        const double L = nb3 ? fma(fma(poly[2], alpha, poly[1]), alpha, poly[0]) : im_L(poly, d.n_beta, alpha);
        // N_hat_i = i sgn(gamma) conj(E_i) FFT(sigma)   (src/MultimodePropagation_CPU.cpp:231-237)
        const V ei = expi<T>(L * zi);
        const V xe = cmulc(sv[c], ei);
        V nh;
        nh.x = (T)(-d.sgn_gamma) * xe.y;
        nh.y = (T)(d.sgn_gamma) * xe.x;
        Nh[(size_t)i * mstride + row + k] = nh;
        V xt;
        if (last && sizeof(T) == 4) {
          // psi_{n+1} = psi_n + inc in FP64; the increment h sum_j b_j N_j is formed in
          // FP32 from the FP32 N_j (its rounding is that of the N_j themselves), so the
          // only conversions are inc -> FP64 and psi_{n+1} -> FP32
          V inc = mk<T>((T)cself * nh.x, (T)cself * nh.y);
#pragma unroll
          for (int q = 0; q < NQ; ++q) {
            if (q < nqr) {
              const T cq = (T)s_cq[q];
              inc.x = fma(cq, nj[c][q].x, inc.x);
              inc.y = fma(cq, nj[c][q].y, inc.y);
            }
          }
          const double2 x = make_double2(ps[c].x + (double)inc.x, ps[c].y + (double)inc.y);
          d.psi_hat[row + k] = x;
          const double a2 = x.x * x.x + x.y * x.y;
          finite = finite && isfinite(a2);
          e_part += a2;
          xt = from_d2<T>(x);
          psiT[row + k] = xt;
          // photon monitor in FP32 (per-thread partial sums; FP64 across threads)
          if (w0f != 0.0f) {
            const int kk = (k <= (Gm::N >> 1)) ? k : k - Gm::N;
            const float af = __int_as_float(0x4B400000 + kk) - 12582912.0f;  // kk as float, exact
            p_part_f += __fdividef(xt.x * xt.x + xt.y * xt.y, fmaf(asf, af, w0f));
          }
        } else if (last) {
          const double2 nhd = to_d2(nh);
          double2 x = ps[c];
          x.x = fma(cself, nhd.x, x.x);
          x.y = fma(cself, nhd.y, x.y);
#pragma unroll
          for (int q = 0; q < NQ; ++q) {
            if (q < nqr) {
              const double2 v = to_d2(nj[c][q]);
              x.x = fma(s_cq[q], v.x, x.x);
              x.y = fma(s_cq[q], v.y, x.y);
            }
          }
          d.psi_hat[row + k] = x;
          const double a2 = x.x * x.x + x.y * x.y;
          finite = finite && isfinite(a2);
          e_part += a2;
          if (d.omega0_T0 != 0.0) p_part += a2 / (d.omega0_T0 + alpha);
          xt = from_d2<T>(x);
        } else {
          if constexpr (!kReadT) xt = from_d2<T>(ps[c]);
          else xt = pt[c];  // = psi_hat rounded to T
          const T cs = (T)cself;
          xt.x = fma(cs, nh.x, xt.x);
          xt.y = fma(cs, nh.y, xt.y);
#pragma unroll
          for (int q = 0; q < NQ; ++q) {
            if (q < nqr) {
              const T cq = (T)s_cq[q];
              xt.x = fma(cq, nj[c][q].x, xt.x);
              xt.y = fma(cq, nj[c][q].y, xt.y);
            }
          }
        }
        V en;
        if (same_z) en = ei;
        else en = expi<T>(L * znext);
        s[Gm::sidx(li)] = spec_in(cmul(xt, en));
      }
    }
  };
  // One body per kernel: every extra copy of this loop grows the kernel, and a larger
  // kernel runs its transforms slower (measured: the forward transform ran ~50% slower
  // with seven copies). The generic instantiation (stages of the order-6 and order-8
  // tableaus) runs the same body with the count at run time (at most kFastQ stored terms,
  // loads predicated), and an element-wise loop beyond that.
  constexpr int kFastQ = 5;
  if constexpr (BODY >= 0) {
    constexpr int NQB = BODY >= kNuLastBody ? BODY - kNuLastBody : BODY;
    body(std::integral_constant<int, NQB>{}, NQB);
  } else if (nq <= kFastQ) {
    body(std::integral_constant<int, kFastQ>{}, nq);
  } else {
#pragma unroll 2
  for (int li = tid; li < Gm::NL; li += Gm::NTHR) {
    const int k = Gm::freq_of(rank, li);
    const double alpha = alpha_of(k, Gm::N, d.alpha_scale);
    const double L = im_L(poly, d.n_beta, alpha);
    // N_hat_i = i sgn(gamma) conj(E_i) FFT(sigma)   (src/MultimodePropagation_CPU.cpp:231-237)
    const V xe = cmulc(s[Gm::sidx(li)], expi<T>(L * zi));
    V nh;
    nh.x = (T)(-d.sgn_gamma) * xe.y;
    nh.y = (T)(d.sgn_gamma) * xe.x;
    Nh[(size_t)i * mstride + row + k] = nh;
    const double2 nhd = to_d2(nh);
    double2 x = d.psi_hat[row + k];
    if (last) {
      // psi_{n+1} = psi_n + h sum_j b_j N_j  (src/MultimodePropagation_CPU.cpp:75-85), FP64
      for (int j = 0; j < S; ++j) {
        const double bj = kp.tab.b[j];
        if (bj != 0.0) {
          const double2 nj = (j == i) ? nhd : to_d2(Nh[(size_t)j * mstride + row + k]);
          x.x = fma(bj * h, nj.x, x.x);
          x.y = fma(bj * h, nj.y, x.y);
        }
      }
      d.psi_hat[row + k] = x;
      if constexpr (sizeof(T) == 4) psiT[row + k] = from_d2<T>(x);
      const double a2 = x.x * x.x + x.y * x.y;
      finite = finite && isfinite(a2);
      e_part += a2;
      if (d.omega0_T0 != 0.0) p_part += a2 / (d.omega0_T0 + alpha);
    } else {
      for (int j = 0; j <= i; ++j) {
        const double aij = kp.tab.a[i + 1][j];
        if (aij != 0.0) {
          const double2 nj = (j == i) ? nhd : to_d2(Nh[(size_t)j * mstride + row + k]);
          x.x = fma(aij * h, nj.x, x.x);
          x.y = fma(aij * h, nj.y, x.y);
        }
      }
    }
    s[Gm::sidx(li)] = spec_in(cmul(from_d2<T>(x), expi<T>(L * znext)));
  }
  }
  p_part += (double)p_part_f;
  if (last) {
    // Block reduction of the monitors, then the last CTA of this solve advances the
    // step. Done before the inverse transform, so none of it is live across that call;
    // every CTA of the solve read the step counter at its start, and the next launch
    // starts only after this one has finished.
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      e_part += __shfl_xor_sync(0xffffffffu, e_part, o);
      p_part += __shfl_xor_sync(0xffffffffu, p_part, o);
    }
    const int finite_all = __syncthreads_and(finite ? 1 : 0);
    if ((tid & 31) == 0) { red[0][tid >> 5] = e_part; red[1][tid >> 5] = p_part; }
    __syncthreads();
    if (tid == 0) {
      const unsigned long long n = s_cnt[0], total = s_cnt[1];
      double es = 0.0, ps = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { es += red[0][w]; ps += red[1][w]; }
      if (!finite_all) atomicOr(d.status, kStatusNonFinite);
      if (d.monitors && total < d.mon_cap) {
        atomicAdd(&d.energy[total], es * d.energy_scale);
        if (d.omega0_T0 != 0.0) atomicAdd(&d.photons[total], ps * d.photon_scale);
      }
      __threadfence();
      const unsigned prev = atomicAdd(d.done_ctr, 1u);
      if (prev == (unsigned)(d.M * Gm::C) - 1u) {
        *d.done_ctr = 0u;
        *d.step = n + 1;
        *d.total = total + 1;
        if (d.drift_tol > 0.0 && d.monitors && total < d.mon_cap) {
          // every CTA's energy sum is in (their adds precede their counter increments)
          const double en = __ldcg(&d.energy[total]), e0 = *d.drift_ref;
          if (e0 == 0.0) *d.drift_ref = en;
          else if (!(fabs(en - e0) <= d.drift_tol * e0)) atomicOr(d.status, kStatusDrift);
        }
        __threadfence();
      }
    }
  }
  V* U = as_t2<T>(d.U);
  const T inv = (T)d.inv_nt;
  if constexpr (Gm::C == 1) {
    // inverse transform as conj(FFT(conj(x))): the spectrum was stored conjugated, so
    // this kernel carries the forward transform's code only (a smaller kernel runs its
    // transforms faster)
    forward<T, LOGN, XC>(s, sq, kp.tw);
#pragma unroll 8
    for (int u = tid; u < Gm::NL; u += Gm::NTHR) U[(size_t)p * Gm::N + u] = cscale(cconj(s[pad(u)]), inv);
  } else {
    inverse<T, LOGN, XC>(s, sq, kp.tw);
#pragma unroll 8
    for (int w = tid; w < Gm::NL; w += Gm::NTHR)
      U[(size_t)p * Gm::N + Gm::time_of_w(rank, w)] = cscale(s[Gm::sidx(Gm::local_of_w(w))], inv);
  }
}

// ---- k_result: phi_p = IFFT(exp(L_p z) psi_hat_p) / conversion_factor -> io (FP64) --------
template <typename T, int LOGN, int XC>
__global__ void __launch_bounds__(Geo<T, LOGN, XC>::NTHR, Geo<T, LOGN, XC>::MIN_BLOCKS) k_result(const KParams kp) {
  using Gm = Geo<T, LOGN, XC>;
  using V = c2<T>;
  MMP_ROW_SMEM();
  __shared__ double poly[kMaxBeta];
  __shared__ SolveDesc sdesc;
  stage_desc(&sdesc, kp.descs + blockIdx.y);
  const V* sq = load_twiddles<T, LOGN, XC>(smem_raw, kp.tw);
  __syncthreads();
  const SolveDesc& d = sdesc;
  const int p = blockIdx.x / Gm::C;
  if (p >= d.M) return;  // uniform over the cluster
  const int rank = cluster_rank<Gm>();
  const int tid = threadIdx.x;
  load_poly(poly, d, p);
  const unsigned long long n = __ldcg(d.step);
  const double z = (double)n * d.dz;
  const size_t row = (size_t)p * Gm::N;
#pragma unroll 2
  for (int li = tid; li < Gm::NL; li += Gm::NTHR) {
    const int k = Gm::freq_of(rank, li);
    const double th = im_L(poly, d.n_beta, alpha_of(k, Gm::N, d.alpha_scale)) * z;
    s[Gm::sidx(li)] = cmul(from_d2<T>(d.psi_hat[row + k]), expi<T>(th));
  }
  inverse<T, LOGN, XC>(s, sq, kp.tw);
#pragma unroll 8
  for (int w = tid; w < Gm::NL; w += Gm::NTHR) {
    const double2 r = to_d2(s[Gm::sidx(Gm::local_of_w(w))]);
    d.io[row + Gm::time_of_w(rank, w)] = make_double2(r.x * d.result_scale, r.y * d.result_scale);
  }
}

// ---- k_dft: rows of FP64 samples -> transform in precision T -> rows of FP64 -------------
// Forward (INV=false): out = scale * FFT(in). Inverse: out = scale * sum_k in[k] e^{+...}.
struct DftArgs {
  const double2* in;
  double2* out;
  int rows;
  int pad_;
  double scale;
  TwTables tw;
};

template <typename T, int LOGN, int XC, bool INV>
__global__ void __launch_bounds__(Geo<T, LOGN, XC>::NTHR, Geo<T, LOGN, XC>::MIN_BLOCKS) k_dft(const DftArgs a) {
  using Gm = Geo<T, LOGN, XC>;
  using V = c2<T>;
  MMP_ROW_SMEM();
  const int r = blockIdx.x / Gm::C;
  if (r >= a.rows) return;
  const int rank = cluster_rank<Gm>();
  const int tid = threadIdx.x;
  const V* sq = load_twiddles<T, LOGN, XC>(smem_raw, a.tw);
  const size_t row = (size_t)r * Gm::N;
  if constexpr (!INV) {
#pragma unroll 8
    for (int w = tid; w < Gm::NL; w += Gm::NTHR) s[Gm::sidx(Gm::local_of_w(w))] = from_d2<T>(a.in[row + Gm::time_of_w(rank, w)]);
    forward<T, LOGN, XC>(s, sq, a.tw);
#pragma unroll 8
    for (int li = tid; li < Gm::NL; li += Gm::NTHR) {
      const double2 x = to_d2(s[Gm::sidx(li)]);
      a.out[row + Gm::freq_of(rank, li)] = make_double2(x.x * a.scale, x.y * a.scale);
    }
  } else {
#pragma unroll 8
    for (int li = tid; li < Gm::NL; li += Gm::NTHR) s[Gm::sidx(li)] = from_d2<T>(a.in[row + Gm::freq_of(rank, li)]);
    inverse<T, LOGN, XC>(s, sq, a.tw);
#pragma unroll 8
    for (int w = tid; w < Gm::NL; w += Gm::NTHR) {
      const double2 x = to_d2(s[Gm::sidx(Gm::local_of_w(w))]);
      a.out[row + Gm::time_of_w(rank, w)] = make_double2(x.x * a.scale, x.y * a.scale);
    }
  }
}

// ---- bulk-async copies (TMA engine) into shared memory, completing on an mbarrier -------
__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
// global -> this CTA's shared memory; dst, src 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
// Wait for phase `parity` of the mbarrier, giving up after `max_iter` polls.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, unsigned max_iter) {
  const unsigned a = smem_addr(bar);
  for (unsigned it = 0; it < max_iter; ++it) {
    unsigned done;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
constexpr unsigned kMaxWaitPolls = 1u << 24;  // far above any copy time; then report, not hang

// ---- the Raman recurrence inside a contraction tile ---------------------------------------
// With h_R a damped sinusoid (see k_raman_scan) the pair fields' convolutions need no
// row pass at all: per tile of TT = 32 c samples (2 <= c <= 8)
//   k_raman_agg    the recurrence's aggregate over the tile from a zero start,
//   k_raman_carry  per pair row, a scan of the tile aggregates (periodic start): the
//                  state entering every tile,
//   k_contract     (mode 2) runs the recurrence through its own tile from that state
//                  and forms W = (1 - f_R) V + R in shared memory; R never leaves the SM.
// Within a tile one warp handles one pair field at a time, lane L owning samples
// [c L, c L + c). The pair field row is written once, coalesced, in a swizzled layout
// (wsw) in which a lane's c samples are also conflict-free 16-byte loads; the lane keeps
// them in registers through the scan and writes W back in place, in the same layout.
template <typename T> struct TileScan {
  using V = c2<T>;
  V lt, kt;
  V rw[8];      // lambda^(c-1-k): weights of the lane's local aggregate
  V lvl[5];     // lambda^(c 2^j): the multipliers of the lane scan's levels
  V lane_pow;   // lambda^(c lane): carries the tile's entering state to this lane
  int c;
  __device__ __forceinline__ void init(const SolveDesc& d, int c_, int lane) {
    c = c_;
    const double2 lam = d.iir_lambda;
    lt = from_d2<T>(lam);
    kt = from_d2<T>(d.iir_kappa);
    double2 p = make_double2(1.0, 0.0);
#pragma unroll
    for (int k = 7; k >= 0; --k) {
      rw[k] = from_d2<T>(p);
      if (k < c) p = cmul(p, lam);
    }
    // p = lambda^c
    double2 lp = make_double2(1.0, 0.0);
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      lvl[j] = from_d2<T>(p);
      if ((lane >> j) & 1) lp = cmul(lp, p);
      p = cmul(p, p);
    }
    lane_pow = from_d2<T>(lp);
  }
  // inclusive scan over the lanes of (la, lb): s_L = lambda^c s_{L-1} + local_L
  __device__ __forceinline__ void lane_scan(V& a, V& b, int lane) const {
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      const int o = 1 << j;
      V pa, pb;
      pa.x = __shfl_up_sync(0xffffffffu, a.x, o);
      pa.y = __shfl_up_sync(0xffffffffu, a.y, o);
      pb.x = __shfl_up_sync(0xffffffffu, b.x, o);
      pb.y = __shfl_up_sync(0xffffffffu, b.y, o);
      if (lane >= o) {
        a = cadd(cmul(lvl[j], pa), a);
        b = cadd(cmul(lvl[j], pb), b);
      }
    }
  }
  __device__ __forceinline__ V step(V s, T x) const {
    return mk<T>(fma(lt.x, s.x, fma(-lt.y, s.y, x)), fma(lt.x, s.y, lt.y * s.x));
  }
};

// Position of the sample pair (2h, 2h + 1) in a pair-field row of the contraction tile:
// 16-byte chunk h ^ ((h >> 3) & mask). With mask = TT/64 - 1 (TT = 128, 256) both a
// warp's 32 consecutive chunks and lane L's chunks [g L, g L + g) (g = TT/64) fall on
// distinct banks per quarter warp; mask 0 is the plain layout.
__device__ __forceinline__ int wsw(int h, int mask) { return h ^ ((h >> 3) & mask); }

// The states entering tile `tile` for pair fields 0..P-1 (k_raman_carry's output) into
// shared memory, [q][Re V, Im V]; published by the caller's next barrier.
template <typename T>
__device__ __forceinline__ void stage_tile_carries(c2<T>* sC, const SolveDesc& d, int P, int ntiles, int tile) {
  const c2<T>* tiles = as_t2<T>(d.raman_tiles);
  for (int i = threadIdx.x; i < 2 * P; i += blockDim.x)
    sC[i] = tiles[((size_t)(i >> 1) * ntiles + tile) * 2 + (i & 1)];
}

// The recurrence through one pair field of a contraction tile, by one warp (TT = 32 c
// samples, 64 <= TT <= 256): V = U_l conj(U_m) is written coalesced to row (pair positions
// swizzled by wmask), each lane takes its c samples into registers, the lanes' aggregates
// are scanned, every lane runs the recurrence from the state entering it (carry[0..1]: the
// states entering the tile for Re V and Im V) and hands W = (1 - f_R) V + R for its samples
// c lane .. c lane + c - 1 to fin(x) (tile_pair_recurrence: back into row, in place). With
// DIRECT each lane forms V for its own samples straight from U (row unused).
template <typename T, bool DIRECT = false, typename Fin>
__device__ __forceinline__ void tile_pair_recurrence_to(const TileScan<T>& ts, const c2<T>* sU, int TT, int2 lm,
                                                        c2<T>* row, int wmask, const c2<T>* carry, T kerr,
                                                        int lane, Fin&& fin) {
  using V = c2<T>;
  const int H = TT >> 1, c = ts.c, g = c >> 1;
  V x[8];
  if constexpr (!DIRECT) {
    // V = U_l conj(U_m), coalesced over the sample pairs, then each lane's own samples
    for (int h = lane; h < H; h += 32) {
      V ul0, ul1, um0, um1;
      ld2<T>(sU + lm.x * TT + 2 * h, ul0, ul1);
      ld2<T>(sU + lm.y * TT + 2 * h, um0, um1);
      st2<T>(row + 2 * wsw(h, wmask), cmulc(ul0, um0), cmulc(ul1, um1));
    }
    __syncwarp();
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (j < g) ld2<T>(row + 2 * wsw(g * lane + j, wmask), x[2 * j], x[2 * j + 1]);
  } else {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if (j < g) {
        V ul0, ul1, um0, um1;
        ld2<T>(sU + lm.x * TT + 2 * (g * lane + j), ul0, ul1);
        ld2<T>(sU + lm.y * TT + 2 * (g * lane + j), um0, um1);
        x[2 * j] = cmulc(ul0, um0);
        x[2 * j + 1] = cmulc(ul1, um1);
      }
    }
  }
  // this lane's aggregate from a zero start: sum_k lambda^(c-1-k) x_k, x_k = Re or Im V
  V la = mk<T>(0, 0), lb = mk<T>(0, 0);
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    if (k < c) {
      la = mk<T>(fma(ts.rw[k].x, x[k].x, la.x), fma(ts.rw[k].y, x[k].x, la.y));
      lb = mk<T>(fma(ts.rw[k].x, x[k].y, lb.x), fma(ts.rw[k].y, x[k].y, lb.y));
    }
  }
  ts.lane_scan(la, lb, lane);
  // state entering this lane's samples: lambda^(c lane) C_tile + earlier lanes
  V ea, eb;
  ea.x = __shfl_up_sync(0xffffffffu, la.x, 1);
  ea.y = __shfl_up_sync(0xffffffffu, la.y, 1);
  eb.x = __shfl_up_sync(0xffffffffu, lb.x, 1);
  eb.y = __shfl_up_sync(0xffffffffu, lb.y, 1);
  if (lane == 0) ea = eb = mk<T>(0, 0);
  V sa = cadd(cmul(ts.lane_pow, carry[0]), ea);
  V sb = cadd(cmul(ts.lane_pow, carry[1]), eb);
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    if (k < c) {
      sa = ts.step(sa, x[k].x);
      sb = ts.step(sb, x[k].y);
      // R = Im(kappa S), W = (1 - f_R) V + R
      x[k] = mk<T>(fma(kerr, x[k].x, fma(ts.kt.x, sa.y, ts.kt.y * sa.x)),
                   fma(kerr, x[k].y, fma(ts.kt.x, sb.y, ts.kt.y * sb.x)));
    }
  }
  fin(x);
}
template <typename T>
__device__ __forceinline__ void tile_pair_recurrence(const TileScan<T>& ts, const c2<T>* sU, int TT, int2 lm,
                                                     c2<T>* row, int wmask, const c2<T>* carry, T kerr,
                                                     int lane) {
  const int g = ts.c >> 1;
  tile_pair_recurrence_to<T>(ts, sU, TT, lm, row, wmask, carry, kerr, lane, [&](const c2<T>* x) {
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (j < g) st2<T>(row + 2 * wsw(g * lane + j, wmask), x[2 * j], x[2 * j + 1]);
  });
}

template <typename T>
__global__ void __launch_bounds__(256) k_raman_agg(const SolveDesc* __restrict__ descs, int nt, int TT) {
  using V = c2<T>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const SolveDesc& d = descs[blockIdx.y];
  const int tile = blockIdx.x, t0 = tile * TT;
  if (t0 >= nt || d.M == 0) return;  // empty slot
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  V* sU = reinterpret_cast<V*>(smem_raw);
  V* sp = sU + (size_t)d.M * TT;  // lambda^j, j < TT
  {  // the U tile and the powers of lambda as 16-byte asynchronous copies, before the step check
    const V* U = as_t2<T>(d.U);
    const int per_row = TT * (int)sizeof(V) / 16;
    for (int idx = threadIdx.x; idx < (d.M + 1) * per_row; idx += blockDim.x) {
      const int r = idx / per_row, c = idx - r * per_row;
      const V* src = r < d.M ? U + (size_t)r * nt + t0 : as_t2<T>(d.raman_pow);
      cp_async16(reinterpret_cast<char*>(sU + (size_t)r * TT) + 16 * c, reinterpret_cast<const char*>(src) + 16 * c);
    }
    cp_async_commit();
  }
  if (__ldcg(d.step) >= d.step_limit) {  // finished solve: the copies land before the CTA leaves
    cp_async_wait<0>();
    return;
  }
  // The aggregate over the tile from a zero start is a weighted sum,
  //   S_end = sum_t lambda^(TT-1-t) x_t   (x = Re or Im of U_l conj(U_m)),
  // so it needs no sequential pass: each lane sums sample pairs (2h, 2h + 1), h = lane,
  // lane + 32, ..., weighted from the table of powers, and the warp adds the lanes.
  cp_async_wait<0>();
  __syncthreads();
  const int ntiles = nt / TT;
  V* out = as_t2<T>(d.raman_tiles);
  for (int q = warp; q < d.P; q += nwarps) {
    const int2 lm = d.pairs[q];
    V sa = mk<T>(0, 0), sb = mk<T>(0, 0);
    for (int h = lane; h < (TT >> 1); h += 32) {
      V ul0, ul1, um0, um1, wb, wa;
      ld2<T>(sU + lm.x * TT + 2 * h, ul0, ul1);
      ld2<T>(sU + lm.y * TT + 2 * h, um0, um1);
      ld2<T>(sp + TT - 2 - 2 * h, wb, wa);  // lambda^(TT-2-2h) for sample 2h+1, lambda^(TT-1-2h) for 2h
      const V x0 = cmulc(ul0, um0), x1 = cmulc(ul1, um1);
      sa = mk<T>(fma(wa.x, x0.x, fma(wb.x, x1.x, sa.x)), fma(wa.y, x0.x, fma(wb.y, x1.x, sa.y)));
      sb = mk<T>(fma(wa.x, x0.y, fma(wb.x, x1.y, sb.x)), fma(wa.y, x0.y, fma(wb.y, x1.y, sb.y)));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      sa.x += __shfl_xor_sync(0xffffffffu, sa.x, o);
      sa.y += __shfl_xor_sync(0xffffffffu, sa.y, o);
      sb.x += __shfl_xor_sync(0xffffffffu, sb.x, o);
      sb.y += __shfl_xor_sync(0xffffffffu, sb.y, o);
    }
    if (lane == 0) {
      out[((size_t)q * ntiles + tile) * 2] = sa;
      out[((size_t)q * ntiles + tile) * 2 + 1] = sb;
    }
  }
}

// one warp per (pair field, solve): tile aggregates -> states entering the tiles
template <typename T>
__global__ void __launch_bounds__(32) k_raman_carry(const SolveDesc* __restrict__ descs, int nt, int TT) {
  using V = c2<T>;
  const SolveDesc& d = descs[blockIdx.y];
  const int q = blockIdx.x;
  if (q >= d.P || d.M == 0 || __ldcg(d.step) >= d.step_limit) return;
  const int lane = threadIdx.x;
  const int ntiles = nt / TT;
  const int per = (ntiles + 31) / 32;  // tiles per lane
  const int first = min(lane * per, ntiles), last = min(first + per, ntiles);
  double2 lamT = d.iir_lambda;  // lambda^TT (TT a power of two)
  for (int s = 1; s < TT; s <<= 1) lamT = cmul(lamT, lamT);
  V* tiles = as_t2<T>(d.raman_tiles) + (size_t)q * ntiles * 2;
  Affine mine = affine_identity();
  for (int i = first; i < last; ++i) {
    mine.a = cmul(mine.a, lamT);
    mine.ba = cadd(cmul(lamT, mine.ba), to_d2(tiles[2 * i]));
    mine.bb = cadd(cmul(lamT, mine.bb), to_d2(tiles[2 * i + 1]));
  }
  const Affine incl = warp_scan_affine(mine, lane);
  Affine pre = shfl_up_affine(incl, 1, 0xffffffffu);
  if (lane == 0) pre = affine_identity();
  const Affine tot = [&] {
    Affine t;
    t.a = make_double2(__shfl_sync(0xffffffffu, incl.a.x, 31), __shfl_sync(0xffffffffu, incl.a.y, 31));
    t.ba = make_double2(__shfl_sync(0xffffffffu, incl.ba.x, 31), __shfl_sync(0xffffffffu, incl.ba.y, 31));
    t.bb = make_double2(__shfl_sync(0xffffffffu, incl.bb.x, 31), __shfl_sync(0xffffffffu, incl.bb.y, 31));
    return t;
  }();
  const double2 inv = d.iir_inv_one_minus;
  double2 ca = cadd(cmul(pre.a, cmul(tot.ba, inv)), pre.ba);
  double2 cb = cadd(cmul(pre.a, cmul(tot.bb, inv)), pre.bb);
  for (int i = first; i < last; ++i) {
    const double2 ga = to_d2(tiles[2 * i]), gb = to_d2(tiles[2 * i + 1]);
    tiles[2 * i] = from_d2<T>(ca);
    tiles[2 * i + 1] = from_d2<T>(cb);
    ca = cadd(cmul(lamT, ca), ga);
    cb = cadd(cmul(lamT, cb), gb);
  }
}

// ---- k_contract: sigma_p(t) = sum_terms Q U_k(t) W(t) over a tile of t, all p ----------
// The U tile [M][TT] and the R tile [P][TT] (Raman on) arrive in shared memory as
// one bulk-async copy per row segment (TT contiguous samples), issued by the
// threads of the CTA and counted on one mbarrier. Then
//   1. every pair field of the tile is formed once, in place:
//        W_lm = (1 - f_R) U_l conj(U_m) + R_lm      (Raman off: U_l conj(U_m)),
//   2. each thread accumulates sigma_p for two adjacent samples over p's terms,
//        sigma_p += q U_k W_pair   (conj(W_pair) for terms whose (l, m) is (m, l) of the
//        stored pair: R_ml = conj(R_lm) as h_R is real, and the Kerr part likewise).
// A warp covers 64 consecutive t of one p (TT >= 64), so term reads are warp-uniform
// and tile reads are conflict-free; terms are staged in shared memory with the
// coefficient already in T.
template <typename T> struct StagedTerm {
  unsigned short k, pc;
  T q;
};

// 16 consecutive values of T from 16-byte aligned shared memory, by 16-byte loads
template <typename T> __device__ __forceinline__ void lds16(const T* a, T* v);
template <> __device__ __forceinline__ void lds16<float>(const float* a, float* v) {
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const float4 x = reinterpret_cast<const float4*>(a)[j];
    v[4 * j] = x.x; v[4 * j + 1] = x.y; v[4 * j + 2] = x.z; v[4 * j + 3] = x.w;
  }
}
template <> __device__ __forceinline__ void lds16<double>(const double* a, double* v) {
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const double2 x = reinterpret_cast<const double2*>(a)[j];
    v[2 * j] = x.x; v[2 * j + 1] = x.y;
  }
}

// Resident CTAs per SM the FP32 build is held to (registers): 3 for the term loop, 2 for the
// dense form (its accumulators), none for FP64.
template <typename T, int DENSE> constexpr int contract_min_blocks() {
  return sizeof(T) == 4 ? (DENSE == 0 ? 3 : 2) : 1;
}

// raman_mode: 0 Raman off; 1 the convolutions R arrive as rows (k_pair / k_raman_scan);
// 2 the recurrence runs through the tile here from the carries of k_raman_carry.
// DENSE = 1: the contraction in its dense form (SolveDesc::dense_q, M <= 16, TT >= 64);
// DENSE = 2: per solve, the dense form where dense_q is set and the term loop elsewhere
// (a batch that mixes both; each solve runs the same arithmetic as on its own):
//   T_pk(t) = sum_q A_re[p][q][k] Re W_q(t) + i sum_q A_im[p][q][k] Im W_q(t),
//   sigma_p(t) = sum_k U_k(t) T_pk(t),
// one warp per (p, 64 samples), each lane two samples with all k in registers: a
// register-blocked matrix product instead of one complex triple product per term.
template <typename T, int DENSE>
__global__ void __launch_bounds__(256, (contract_min_blocks<T, DENSE>())) k_contract(const SolveDesc* __restrict__ descs, int nt, int TT,
                                                  int stage_terms, int raman_mode) {
  using V = c2<T>;
  using ST = StagedTerm<T>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) unsigned long long bar;
  V* sU = reinterpret_cast<V*>(smem_raw);
  const SolveDesc& d = descs[blockIdx.y];
  const int t0 = blockIdx.x * TT;
  if (t0 >= nt || d.M == 0) return;  // empty slot
  const int M = d.M;
  const int raman = raman_mode;
  const int P = d.P;                          // pair fields formed in this tile
  const int Pl = raman == 1 ? P : 0;          // pair rows loaded (Raman convolutions)
  // The tile's rows are requested first, before the step check and the term staging
  const V* U = as_t2<T>(d.U);
  const V* R = as_t2<T>(d.W);
  const unsigned row_bytes = (unsigned)(TT * sizeof(V));
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_arrive_expect_tx(&bar, (unsigned)(M + Pl) * row_bytes);
  }
  __syncthreads();
  for (int r = threadIdx.x; r < M + Pl; r += blockDim.x) {
    const V* src = (r < M) ? U + (size_t)r * nt + t0 : R + (size_t)(r - M) * nt + t0;
    bulk_g2s(sU + (size_t)r * TT, src, row_bytes, &bar);
  }
  if (__ldcg(d.step) >= d.step_limit) {  // finished solve: the copies land before the CTA leaves
    mbar_wait(&bar, 0, kMaxWaitPolls);
    return;
  }
  const T kerr = (T)d.one_minus_fR;
  V* sW = sU + (size_t)M * TT;
  const int n_terms = d.term_off[M];
  // pair-field rows: swizzled (wsw) when the recurrence runs here, else plain
  const int wmask = raman == 2 ? max(TT >> 6, 1) - 1 : 0;
  // raman_mode 2: the states entering this tile per pair field (Re V, Im V), staged while
  // the tile lands
  V* sC = sW + (size_t)P * TT;
  // dense form: per warp, two chunks of kDenseChunk coefficient rows (cp.async double buffer)
  T* sA = reinterpret_cast<T*>(sC + (raman == 2 ? 2 * (size_t)P : 0));
  if (raman == 2) stage_tile_carries<T>(sC, d, P, nt / TT, blockIdx.x);
  const size_t dense_elems = DENSE ? (size_t)(blockDim.x >> 5) * 2 * kDenseChunk * 2 * kDenseMaxModes : 0;
  ST* st = reinterpret_cast<ST*>(sA + dense_elems);
  if (stage_terms) {
    for (int j = threadIdx.x; j < n_terms; j += blockDim.x) {
      const Term tm = d.terms[j];
      ST s;
      s.k = tm.k;
      s.pc = tm.pc;
      s.q = (T)tm.q;
      st[j] = s;
    }
  }
  // every thread polls with a bound; the barrier makes the outcome CTA-uniform and
  // also publishes the staged terms
  const bool landed = mbar_wait(&bar, 0, d.tile_wait_polls);
  if (!__syncthreads_and(landed ? 1 : 0)) {
    if (threadIdx.x == 0) atomicOr(d.status, kStatusTimeout);
    // give the copies a second bounded chance to land before the CTA leaves
    mbar_wait(&bar, 0, kMaxWaitPolls);
    return;
  }
  const int H = TT >> 1;  // sample pairs per row
  // 1. pair fields
  if (raman != 2) {  // two samples per thread
    for (int idx = threadIdx.x; idx < P * H; idx += blockDim.x) {
      const int q = idx / H, tt = 2 * (idx - q * H);
      const int2 lm = d.pairs[q];
      V ul0, ul1, um0, um1;
      ld2<T>(sU + lm.x * TT + tt, ul0, ul1);
      ld2<T>(sU + lm.y * TT + tt, um0, um1);
      V w0 = cmulc(ul0, um0), w1 = cmulc(ul1, um1);
      if (raman) {
        V r0, r1;
        ld2<T>(sW + q * TT + tt, r0, r1);
        w0 = mk<T>(fma(kerr, w0.x, r0.x), fma(kerr, w0.y, r0.y));
        w1 = mk<T>(fma(kerr, w1.x, r1.x), fma(kerr, w1.y, r1.y));
      }
      st2<T>(sW + q * TT + tt, w0, w1);
    }
  } else {  // one warp per pair field: the recurrence through the tile, then W in place
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    TileScan<T> ts;
    ts.init(d, TT >> 5, lane);
    for (int q = warp; q < P; q += nwarps)
      tile_pair_recurrence<T>(ts, sU, TT, d.pairs[q], sW + (size_t)q * TT, wmask, sC + 2 * q, kerr, lane);
  }
  __syncthreads();
  // 2. contraction
  V* sigma = as_t2<T>(d.sigma);
  if (DENSE == 1 || (DENSE == 2 && d.dense_q != nullptr)) {
    constexpr int K = kDenseMaxModes;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    constexpr int ROW = 2 * K;                       // values per coefficient row (p, q)
    constexpr int CH = kDenseChunk;                  // rows per staged chunk
    constexpr int PIECES = CH * ROW * (int)sizeof(T) / 16;  // 16-byte copies per chunk
    const T* A = static_cast<const T*>(d.dense_q);
    T* sAw = sA + (size_t)warp * 2 * CH * ROW;       // this warp's two chunk buffers
    const int chunks = TT >> 6;
    const int nchunk = (P + CH - 1) / CH;
    for (int item = warp; item < M * chunks; item += nwarps) {
      const int p = item / chunks, tt = ((item - p * chunks) << 6) + 2 * lane;
      const int tw = 2 * wsw(tt >> 1, wmask);
      T re0[K], re1[K], im0[K], im1[K];
#pragma unroll
      for (int k = 0; k < K; ++k) re0[k] = re1[k] = im0[k] = im1[k] = 0;
      const T* Ap = A + (size_t)p * P * ROW;
      // rows q0 .. q0 + CH - 1 (clamped to P) into buffer buf, as one cp.async group
      auto stage_rows = [&](int buf, int q0) {
        const int rows = min(CH, P - q0);
        const int pieces = rows * ROW * (int)sizeof(T) / 16;
        const char* src = reinterpret_cast<const char*>(Ap + (size_t)q0 * ROW);
        char* dst = reinterpret_cast<char*>(sAw + (size_t)buf * CH * ROW);
        for (int i = lane; i < pieces && i < PIECES; i += 32) cp_async16(dst + 16 * i, src + 16 * i);
        cp_async_commit();
      };
      __syncwarp();  // the previous item's reads of both buffers are done
      stage_rows(0, 0);
      for (int c = 0; c < nchunk; ++c) {
        if (c + 1 < nchunk) {
          stage_rows((c + 1) & 1, (c + 1) * CH);
          cp_async_wait<1>();
        } else {
          cp_async_wait<0>();
        }
        __syncwarp();  // every lane's copies of chunk c have landed
        const T* rowp = sAw + (size_t)(c & 1) * CH * ROW;
        const int q0 = c * CH, rows = min(CH, P - q0);
#pragma unroll 2
        for (int r = 0; r < rows; ++r) {
          V w0, w1;
          ld2<T>(sW + (q0 + r) * TT + tw, w0, w1);
          T ar[K], ai[K];  // the same addresses on every lane: broadcasts, 16 bytes per load
          lds16<T>(rowp + r * ROW, ar);
          lds16<T>(rowp + r * ROW + K, ai);
#pragma unroll
          for (int k = 0; k < K; ++k) {
            re0[k] = fma(ar[k], w0.x, re0[k]);
            re1[k] = fma(ar[k], w1.x, re1[k]);
            im0[k] = fma(ai[k], w0.y, im0[k]);
            im1[k] = fma(ai[k], w1.y, im1[k]);
          }
        }
        __syncwarp();  // reads of buffer c & 1 done before chunk c + 2 is staged into it
      }
      T sx0 = 0, sy0 = 0, sx1 = 0, sy1 = 0;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if (k < M) {
          V u0, u1;
          ld2<T>(sU + k * TT + tt, u0, u1);
          sx0 = fma(u0.x, re0[k], fma(-u0.y, im0[k], sx0));
          sy0 = fma(u0.x, im0[k], fma(u0.y, re0[k], sy0));
          sx1 = fma(u1.x, re1[k], fma(-u1.y, im1[k], sx1));
          sy1 = fma(u1.x, im1[k], fma(u1.y, re1[k], sy1));
        }
      }
      st2<T>(sigma + (size_t)p * nt + t0 + tt, mk<T>(sx0, sy0), mk<T>(sx1, sy1));
    }
    return;
  }
  for (int idx = threadIdx.x; idx < M * H; idx += blockDim.x) {
    const int p = idx / H, tt = 2 * (idx - p * H);
    const int tw = 2 * wsw(tt >> 1, wmask);
    T ax0 = 0, ay0 = 0, ax1 = 0, ay1 = 0;
    const int j1 = d.term_off[p + 1];
    for (int j = d.term_off[p]; j < j1; ++j) {
      unsigned short k, pc;
      T qv;
      if (stage_terms) {
        const ST s = st[j];
        k = s.k; pc = s.pc; qv = s.q;
      } else {
        const Term tm = d.terms[j];
        k = tm.k; pc = tm.pc; qv = (T)tm.q;
      }
      V u0, u1, w0, w1;
      ld2<T>(sU + k * TT + tt, u0, u1);
      ld2<T>(sW + (pc & 0x7fff) * TT + tw, w0, w1);
      if (pc & 0x8000) {
        w0.y = -w0.y;
        w1.y = -w1.y;
      }
      const V a0 = cmul(u0, w0), a1 = cmul(u1, w1);
      ax0 = fma(qv, a0.x, ax0);
      ay0 = fma(qv, a0.y, ay0);
      ax1 = fma(qv, a1.x, ax1);
      ay1 = fma(qv, a1.y, ay1);
    }
    st2<T>(sigma + (size_t)p * nt + t0 + tt, mk<T>(ax0, ay0), mk<T>(ax1, ay1));
  }
}

// ---- k_contract_pc: the term loop with the Raman recurrence in the tiles, for tiles with
// too many pair fields to hold at once (tall tiles). Only `pc` pair fields live in shared
// memory at a time: per chunk the warps run the recurrence for the chunk's fields, then
// every thread advances each of its (p, two samples) items through the terms of p whose
// pair field lies in the chunk, accumulating in registers. The terms of each p are sorted
// by pair field, so one cursor per item walks them chunk by chunk. At most kPcItems items
// per thread (M * TT / 2 <= kPcItems * blockDim.x), every term staged in shared memory.
constexpr int kPcItems = 4;
template <typename T>
__global__ void __launch_bounds__(256, (sizeof(T) == 4 ? 3 : 2)) k_contract_pc(const SolveDesc* __restrict__ descs,
                                                                              int nt, int TT, int pc) {
  using V = c2<T>;
  using ST = StagedTerm<T>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) unsigned long long bar;
  V* sU = reinterpret_cast<V*>(smem_raw);  // [M][TT]
  const SolveDesc& d = descs[blockIdx.y];
  const int t0 = blockIdx.x * TT;
  if (t0 >= nt || d.M == 0) return;  // empty slot
  const int M = d.M, P = d.P;
  const unsigned row_bytes = (unsigned)(TT * sizeof(V));
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_arrive_expect_tx(&bar, (unsigned)M * row_bytes);
  }
  __syncthreads();
  for (int r = threadIdx.x; r < M; r += blockDim.x)
    bulk_g2s(sU + (size_t)r * TT, as_t2<T>(d.U) + (size_t)r * nt + t0, row_bytes, &bar);
  if (__ldcg(d.step) >= d.step_limit) {  // finished solve: the copies land before the CTA leaves
    mbar_wait(&bar, 0, kMaxWaitPolls);
    return;
  }
  V* sW = sU + (size_t)M * TT;                             // [pc][TT], pair positions swizzled
  ST* st = reinterpret_cast<ST*>(sW + (size_t)pc * TT);   // every term, sorted by (p, pair field)
  const int n_terms = d.term_off[M];
  V* sC = reinterpret_cast<V*>(st + n_terms);               // states entering the tile, [P][2]
  stage_tile_carries<T>(sC, d, P, nt / TT, blockIdx.x);
  for (int j = threadIdx.x; j < n_terms; j += blockDim.x) {
    const Term tm = d.terms[j];
    ST x;
    x.k = tm.k;
    x.pc = tm.pc;
    x.q = (T)tm.q;
    st[j] = x;
  }
  const bool landed = mbar_wait(&bar, 0, d.tile_wait_polls);
  if (!__syncthreads_and(landed ? 1 : 0)) {
    if (threadIdx.x == 0) atomicOr(d.status, kStatusTimeout);
    mbar_wait(&bar, 0, kMaxWaitPolls);
    return;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int H = TT >> 1, nitems = M * H;
  const int wmask = max(TT >> 6, 1) - 1;
  const T kerr = (T)d.one_minus_fR;
  TileScan<T> ts;
  ts.init(d, TT >> 5, lane);
  T acc[kPcItems][4];
  int cur[kPcItems], end[kPcItems];
#pragma unroll
  for (int i = 0; i < kPcItems; ++i) {
    const int idx = threadIdx.x + i * blockDim.x;
    const int p = idx < nitems ? idx / H : 0;
    cur[i] = idx < nitems ? d.term_off[p] : 0;
    end[i] = idx < nitems ? d.term_off[p + 1] : 0;
    acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0;
  }
  for (int c0 = 0; c0 < P; c0 += pc) {
    const int c1 = min(P, c0 + pc);
    for (int q = c0 + warp; q < c1; q += nwarps)
      tile_pair_recurrence<T>(ts, sU, TT, d.pairs[q], sW + (size_t)(q - c0) * TT, wmask, sC + 2 * q, kerr, lane);
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kPcItems; ++i) {
      const int idx = threadIdx.x + i * blockDim.x;
      if (idx >= nitems) continue;
      const int p = idx / H, tt = 2 * (idx - p * H);
      const int tw = 2 * wsw(tt >> 1, wmask);
      int j = cur[i];
      for (; j < end[i]; ++j) {
        const ST x = st[j];
        const int q = x.pc & 0x7fff;
        if (q >= c1) break;
        V u0, u1, w0, w1;
        ld2<T>(sU + x.k * TT + tt, u0, u1);
        ld2<T>(sW + (q - c0) * TT + tw, w0, w1);
        if (x.pc & 0x8000) {
          w0.y = -w0.y;
          w1.y = -w1.y;
        }
        const V a0 = cmul(u0, w0), a1 = cmul(u1, w1);
        acc[i][0] = fma(x.q, a0.x, acc[i][0]);
        acc[i][1] = fma(x.q, a0.y, acc[i][1]);
        acc[i][2] = fma(x.q, a1.x, acc[i][2]);
        acc[i][3] = fma(x.q, a1.y, acc[i][3]);
      }
      cur[i] = j;
    }
    __syncthreads();  // the chunk's fields are read before the next chunk overwrites them
  }
  V* sigma = as_t2<T>(d.sigma);
#pragma unroll
  for (int i = 0; i < kPcItems; ++i) {
    const int idx = threadIdx.x + i * blockDim.x;
    if (idx >= nitems) continue;
    const int p = idx / H, tt = 2 * (idx - p * H);
    st2<T>(sigma + (size_t)p * nt + t0 + tt, mk<T>(acc[i][0], acc[i][1]), mk<T>(acc[i][2], acc[i][3]));
  }
}

// ---- k_contract_sr: the term loop with the Raman recurrence run serially per pair field --
// For tall tiles (more pair fields than k_contract holds in a tile). A CTA owns TB
// consecutive samples of one solve and walks them in sub-blocks of kSrSub = 16 samples:
//   staging  U of the next sub-block is loaded from global memory while this one is
//            worked on, into a double buffer in which each sample pair (t, t + 1) of a
//            row is stored as (Re t, Re t+1, Im t, Im t+1);
//   phase A  each thread owns one or two pair fields q = (l, m) for the whole tile and runs
//            the Raman recurrence S = lambda S + x (x = Re V and Im V, V = U_l conj(U_m))
//            sample after sample from the state entering the tile (k_raman_carry); the
//            state stays in registers from one sub-block to the next, and
//            W_q = (1 - f_R) V + Im(kappa S) for the sub-block goes to shared memory
//            (Raman off: W_q = V);
//   phase B  sigma_p(t) = sum over p's merged terms of U_k (a Re W_q + i b Im W_q)
//            (SolveDesc::sr_coef), eight lanes (one per sample pair) per group; a plan
//            made on the host (SolveDesc::sr_plan) gives each group a mode, or half of a
//            mode with many terms (the two halves sit in one warp and are added by a
//            shuffle), so the longest group's term loop is about half as long as the
//            heaviest mode's; groups of similar length share a warp.
// Per term a lane reads U_k and W_q (16 bytes each for its two samples) and the 8-byte
// coefficient from shared memory, whose bandwidth bounds the kernel.
// Compared with the warp-per-field scan, a sample costs one step of each recurrence and no
// scan levels. FP32 solves use the packed two-lane FMA (fma.rn.f32x2): phase A packs the
// two recurrences (Re V and Im V share lambda), phase B the two samples of a pair; each
// lane rounds exactly as the scalar FMA does. No asynchronous copies and no waits besides
// __syncthreads.
constexpr int kSrSub = 16;
constexpr int kSrThreads = 256;
constexpr int kSrPairsPerThread = 2;  // pair fields per thread: P <= 512
constexpr int kSrMaxModes = 64;       // staging: M * kSrSub / 2 <= 2 kSrThreads

__device__ __forceinline__ float2 pk_fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 pk_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ double2 pk_fma(double2 a, double2 b, double2 c) {
  return make_double2(fma(a.x, b.x, c.x), fma(a.y, b.y, c.y));
}
__device__ __forceinline__ double2 pk_mul(double2 a, double2 b) { return make_double2(a.x * b.x, a.y * b.y); }

// A sample pair (t, t + 1) of one row: re = (Re t, Re t+1), im = (Im t, Im t+1).
template <typename T> struct SrPair {
  c2<T> re, im;
};
template <typename T> __device__ __forceinline__ SrPair<T> ld_pair(const SrPair<T>* p) {
  if constexpr (sizeof(T) == 4) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    SrPair<T> r;
    r.re = make_float2(v.x, v.y);
    r.im = make_float2(v.z, v.w);
    return r;
  } else {
    return *p;
  }
}
template <typename T> __device__ __forceinline__ void st_pair(SrPair<T>* p, c2<T> re, c2<T> im) {
  if constexpr (sizeof(T) == 4) {
    *reinterpret_cast<float4*>(p) = make_float4(re.x, re.y, im.x, im.y);
  } else {
    p->re = re;
    p->im = im;
  }
}
constexpr int kSrGroups = (kSrThreads / 32) * 4;  // groups of eight lanes in phase B

// One merged term as k_contract_sr keeps it in shared memory: the coefficients (a, b) and
// q | k << 16 in one record of 2 complex values (16 bytes in FP32, 32 in FP64), so that a
// term costs one shared-memory access (two in FP64).
template <typename T> struct SrRec {
  c2<T> ab;
  unsigned kq;
  unsigned pad[sizeof(T) == 4 ? 1 : 3];
};
static_assert(sizeof(SrRec<float>) == 16 && sizeof(SrRec<double>) == 32, "SrRec layout");
template <typename T> __device__ __forceinline__ void ld_rec(const SrRec<T>* r, c2<T>& ab, unsigned& kq) {
  if constexpr (sizeof(T) == 4) {
    const float4 v = *reinterpret_cast<const float4*>(r);
    ab = make_float2(v.x, v.y);
    kq = __float_as_uint(v.z);
  } else {
    ab = r->ab;
    kq = r->kq;
  }
}

template <typename V> __device__ __forceinline__ V shfl_down_c(V v, int d) {
  v.x = __shfl_down_sync(0xffffffffu, v.x, d);
  v.y = __shfl_down_sync(0xffffffffu, v.y, d);
  return v;
}

// raman_mode: 0 Raman off, 2 the recurrence from the tile carries of k_raman_carry (tiles of TB)
template <typename T>
__global__ void __launch_bounds__(kSrThreads, (sizeof(T) == 4 ? 3 : 1))
    k_contract_sr(const SolveDesc* __restrict__ descs, int nt, int TB, int raman_mode) {
  using V = c2<T>;
  using SP = SrPair<T>;
  using CF = c2<T>;              // merged coefficient (a, b)
  constexpr int J = kSrSub / 2;  // sample pairs per sub-block
  constexpr int RS = J + 1;      // row stride in sample pairs: consecutive rows start 16 bytes apart
                                 // mod 128, so a quarter warp's rows fall on different banks
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const SolveDesc& d = descs[blockIdx.y];
  const int t0 = blockIdx.x * TB;
  if (t0 >= nt || d.M == 0) return;               // empty slot
  if (__ldcg(d.step) >= d.step_limit) return;     // finished solve (nothing is in flight yet)
  const int M = d.M, P = d.P, nterm = d.sr_terms, rounds = d.sr_rounds;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // shared memory: U [2][M][RS], W [P][RS], group plan [rounds kSrGroups], merged terms
  // [nterm] (coefficients and q | k << 16)
  SP* sU = reinterpret_cast<SP*>(smem_raw);
  SP* sW = sU + 2 * (size_t)M * RS;
  int4* sPlan = reinterpret_cast<int4*>(sW + (size_t)P * RS);
  SrRec<T>* sRec = reinterpret_cast<SrRec<T>*>(sPlan + rounds * kSrGroups);
  {
    const CF* gCf = static_cast<const CF*>(d.sr_coef);
    for (int i = tid; i < nterm; i += kSrThreads) {
      SrRec<T> r = {};
      r.ab = gCf[i];
      r.kq = d.sr_kq[i];
      sRec[i] = r;
    }
    for (int i = tid; i < rounds * kSrGroups; i += kSrThreads) sPlan[i] = d.sr_plan[i];
  }
  // U staging: sample pair j of row r is item r J + j; a thread carries at most two
  const V* U = as_t2<T>(d.U);
  const int nu = M * J;
  V pre[2][2];
  auto fetch = [&](int sub) {
    const int ts = t0 + sub * kSrSub;
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int idx = tid + r * kSrThreads;
      if (idx < nu) {
        const int row = idx / J, j = idx - row * J;
        ld2<T>(U + (size_t)row * nt + ts + 2 * j, pre[r][0], pre[r][1]);
      }
    }
  };
  auto park = [&](int buf) {
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int idx = tid + r * kSrThreads;
      if (idx < nu) {
        const int row = idx / J, j = idx - row * J;
        st_pair<T>(sU + ((size_t)buf * M + row) * RS + j, mk<T>(pre[r][0].x, pre[r][1].x),
                   mk<T>(pre[r][0].y, pre[r][1].y));
      }
    }
  };
  // phase A: this thread's pair fields and their recurrence states, packed as
  // sr = (Re S_a, Re S_b), si = (Im S_a, Im S_b) (S_a for Re V, S_b for Im V)
  int pl[kSrPairsPerThread], pm[kSrPairsPerThread];
  V sr[kSrPairsPerThread], si[kSrPairsPerThread];
  const int ntiles = nt / TB;
#pragma unroll
  for (int i = 0; i < kSrPairsPerThread; ++i) {
    const int q = tid + i * kSrThreads;
    pl[i] = pm[i] = 0;
    sr[i] = si[i] = mk<T>(0, 0);
    if (q < P) {
      const int2 lm = d.pairs[q];
      pl[i] = lm.x;
      pm[i] = lm.y;
      if (raman_mode == 2) {
        const V* tiles = as_t2<T>(d.raman_tiles) + ((size_t)q * ntiles + blockIdx.x) * 2;
        const V ca = tiles[0], cb = tiles[1];
        sr[i] = mk<T>(ca.x, cb.x);
        si[i] = mk<T>(ca.y, cb.y);
      }
    }
  }
  const T lr = (T)d.iir_lambda.x, li = (T)d.iir_lambda.y;
  const V lr2 = mk<T>(lr, lr), li2 = mk<T>(li, li), nli2 = mk<T>(-li, -li);
  const V kr2 = mk<T>((T)d.iir_kappa.x, (T)d.iir_kappa.x), ki2 = mk<T>((T)d.iir_kappa.y, (T)d.iir_kappa.y);
  const T kerr = (T)d.one_minus_fR;
  const V kerr2 = mk<T>(kerr, kerr);
  V* sigma = as_t2<T>(d.sigma);
  const int nsub = TB / kSrSub;
  fetch(0);
  park(0);
  __syncthreads();  // U of sub-block 0, the terms
  for (int sub = 0; sub < nsub; ++sub) {
    const int buf = sub & 1;
    if (sub + 1 < nsub) fetch(sub + 1);  // lands while this sub-block is worked on
    const SP* uc = sU + (size_t)buf * M * RS;
    // phase A
#pragma unroll
    for (int i = 0; i < kSrPairsPerThread; ++i) {
      const int q = tid + i * kSrThreads;
      if (q < P) {
        const SP* ul = uc + pl[i] * RS;
        const SP* um = uc + pm[i] * RS;
        SP* wq = sW + (size_t)q * RS;
        V Sr = sr[i], Si = si[i];
#pragma unroll
        for (int j = 0; j < J; ++j) {
          const SP a = ld_pair<T>(ul + j), b = ld_pair<T>(um + j);
          V w[2];
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const V ue = e ? mk<T>(a.re.y, a.im.y) : mk<T>(a.re.x, a.im.x);
            const V me = e ? mk<T>(b.re.y, b.im.y) : mk<T>(b.re.x, b.im.x);
            const V x = cmulc(ue, me);  // V = U_l conj(U_m): (Re V, Im V)
            if (raman_mode == 2) {
              // S <- lambda S + x for both recurrences, then W = (1 - f_R) V + Im(kappa S)
              const V t = pk_mul(li2, Sr);
              Sr = pk_fma(lr2, Sr, pk_fma(nli2, Si, x));
              Si = pk_fma(lr2, Si, t);
              w[e] = pk_fma(kerr2, x, pk_fma(kr2, Si, pk_mul(ki2, Sr)));
            } else {
              w[e] = x;
            }
          }
          st_pair<T>(wq + j, mk<T>(w[0].x, w[1].x), mk<T>(w[0].y, w[1].y));
        }
        sr[i] = Sr;
        si[i] = Si;
      }
    }
    __syncthreads();  // W of this sub-block is complete
    // phase B
    {
      const int j = lane & 7;
      const int ts = t0 + sub * kSrSub;
      for (int r = 0; r < rounds; ++r) {
        const int4 pl = sPlan[r * kSrGroups + warp * 4 + (lane >> 3)];  // p, first term, end, role
        // sigma = U X summed over the terms: Re = a1 - a2, Im = a3 + a4 with a1 = sum Re U Re X,
        // a2 = sum Im U Im X, a3 = sum Re U Im X, a4 = sum Im U Re X (packed over the pair)
        V a1 = mk<T>(0, 0), a2 = a1, a3 = a1, a4 = a1;
        // a mode's terms are sorted by k: U_k is read again only when k changes
        SP u = {};
        int kprev = -1;
#pragma unroll 2
        for (int n = pl.y; n < pl.z; ++n) {
          CF c;
          unsigned kq;
          ld_rec<T>(sRec + n, c, kq);
          const int k = (int)(kq >> 16);
          if (k != kprev) {
            u = ld_pair<T>(uc + k * RS + j);
            kprev = k;
          }
          const SP w = ld_pair<T>(sW + (kq & 0xffffu) * RS + j);
          const V xr = pk_mul(mk<T>(c.x, c.x), w.re), xi = pk_mul(mk<T>(c.y, c.y), w.im);  // X
          a1 = pk_fma(u.re, xr, a1);
          a2 = pk_fma(u.im, xi, a2);
          a3 = pk_fma(u.re, xi, a3);
          a4 = pk_fma(u.im, xr, a4);
        }
        // the upper half of a split mode (the next group, 8 lanes up) adds into the lower half
        const V b1 = shfl_down_c(a1, 8), b2 = shfl_down_c(a2, 8), b3 = shfl_down_c(a3, 8), b4 = shfl_down_c(a4, 8);
        if (pl.w == 1) {
          a1 = cadd(a1, b1);
          a2 = cadd(a2, b2);
          a3 = cadd(a3, b3);
          a4 = cadd(a4, b4);
        }
        if (pl.w <= 1)
          st2<T>(sigma + (size_t)pl.x * nt + ts + 2 * j, mk<T>(a1.x - a2.x, a3.x + a4.x), mk<T>(a1.y - a2.y, a3.y + a4.y));
      }
    }
    // buffer buf ^ 1 was last read in the previous sub-block, which ended at a barrier
    if (sub + 1 < nsub) park(buf ^ 1);
    __syncthreads();  // W is free again; the next U is in place
  }
}

// ---- k_raman_agg_sr: the tile aggregates for k_contract_sr's tiles ------------------------
// One thread per pair field: the aggregate of the recurrence over the tile from a zero
// start, S_end = sum_t lambda^(TB-1-t) x_t (x = Re V, Im V, V = U_l conj(U_m)), run as
// S <- lambda S + x sample after sample (the arithmetic of k_contract_sr's phase A without
// the output), U arriving in sub-blocks of kSrSub samples through the same double buffer.
// k_raman_carry turns the aggregates into the states entering the tiles.
template <typename T>
__global__ void __launch_bounds__(kSrThreads, (sizeof(T) == 4 ? 4 : 2))
    k_raman_agg_sr(const SolveDesc* __restrict__ descs, int nt, int TB) {
  using V = c2<T>;
  using SP = SrPair<T>;
  constexpr int J = kSrSub / 2;
  constexpr int RS = J + 1;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const SolveDesc& d = descs[blockIdx.y];
  const int t0 = blockIdx.x * TB;
  if (t0 >= nt || d.M == 0) return;            // empty slot
  if (__ldcg(d.step) >= d.step_limit) return;  // finished solve
  const int M = d.M, P = d.P, tid = threadIdx.x;
  SP* sU = reinterpret_cast<SP*>(smem_raw);  // [2][M][RS]
  const V* U = as_t2<T>(d.U);
  const int nu = M * J;
  V pre[2][2];
  auto fetch = [&](int sub) {
    const int ts = t0 + sub * kSrSub;
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int idx = tid + r * kSrThreads;
      if (idx < nu) {
        const int row = idx / J, j = idx - row * J;
        ld2<T>(U + (size_t)row * nt + ts + 2 * j, pre[r][0], pre[r][1]);
      }
    }
  };
  auto park = [&](int buf) {
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int idx = tid + r * kSrThreads;
      if (idx < nu) {
        const int row = idx / J, j = idx - row * J;
        st_pair<T>(sU + ((size_t)buf * M + row) * RS + j, mk<T>(pre[r][0].x, pre[r][1].x),
                   mk<T>(pre[r][0].y, pre[r][1].y));
      }
    }
  };
  int pl[kSrPairsPerThread], pm[kSrPairsPerThread];
  V sr[kSrPairsPerThread], si[kSrPairsPerThread];
#pragma unroll
  for (int i = 0; i < kSrPairsPerThread; ++i) {
    const int q = tid + i * kSrThreads;
    pl[i] = pm[i] = 0;
    sr[i] = si[i] = mk<T>(0, 0);
    if (q < P) {
      const int2 lm = d.pairs[q];
      pl[i] = lm.x;
      pm[i] = lm.y;
    }
  }
  const T lr = (T)d.iir_lambda.x, li = (T)d.iir_lambda.y;
  const V lr2 = mk<T>(lr, lr), li2 = mk<T>(li, li), nli2 = mk<T>(-li, -li);
  const int nsub = TB / kSrSub;
  fetch(0);
  park(0);
  __syncthreads();
  for (int sub = 0; sub < nsub; ++sub) {
    const int buf = sub & 1;
    if (sub + 1 < nsub) fetch(sub + 1);
    const SP* uc = sU + (size_t)buf * M * RS;
#pragma unroll
    for (int i = 0; i < kSrPairsPerThread; ++i) {
      if (tid + i * kSrThreads < P) {
        const SP* ul = uc + pl[i] * RS;
        const SP* um = uc + pm[i] * RS;
        V Sr = sr[i], Si = si[i];
#pragma unroll
        for (int j = 0; j < J; ++j) {
          const SP a = ld_pair<T>(ul + j), b = ld_pair<T>(um + j);
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const V x = cmulc(e ? mk<T>(a.re.y, a.im.y) : mk<T>(a.re.x, a.im.x),
                              e ? mk<T>(b.re.y, b.im.y) : mk<T>(b.re.x, b.im.x));
            const V t = pk_mul(li2, Sr);
            Sr = pk_fma(lr2, Sr, pk_fma(nli2, Si, x));
            Si = pk_fma(lr2, Si, t);
          }
        }
        sr[i] = Sr;
        si[i] = Si;
      }
    }
    // buffer buf ^ 1 was last read in the previous sub-block, which ended at this barrier
    if (sub + 1 < nsub) park(buf ^ 1);
    __syncthreads();
  }
  const int ntiles = nt / TB;
  V* out = as_t2<T>(d.raman_tiles);
#pragma unroll
  for (int i = 0; i < kSrPairsPerThread; ++i) {
    const int q = tid + i * kSrThreads;
    if (q < P) {
      out[((size_t)q * ntiles + blockIdx.x) * 2] = mk<T>(sr[i].x, si[i].x);      // Re V recurrence
      out[((size_t)q * ntiles + blockIdx.x) * 2 + 1] = mk<T>(sr[i].y, si[i].y);  // Im V recurrence
    }
  }
}

// ---- k_contract_tc: the dense contraction on the tensor cores (FP32 solves, M <= 16) -----
// Per tile of kTcTile = 128 samples the dense form is two real matrix products over the
// pair fields q,
//   T_re[t][(p, k)] = sum_q Re W_q(t) A_re[p][q][k],   T_im[t][(p, k)] = sum_q Im W_q(t) A_im[p][q][k],
// followed by sigma_p(t) = sum_k U_k(t) (T_re + i T_im) (the k_contract<T, 1> arithmetic).
// The products are tcgen05 TF32 MMAs: M = 128 samples (TMEM lane = sample), N = 16 M
// columns (p, k) per product (Re in TMEM columns [0, N), Im in [256, 256 + N)), K = the pair
// fields in chunks of kTcChunk = 16. Both operands are split x = hi + lo into TF32 parts
// and every product is formed as hi hi + hi lo + lo hi with FP32 accumulation: relative
// error about 2^-21 (plain TF32 would leave 2^-11).
// Per chunk c the 16 warps build the chunk's pair fields W, one field each (the Raman
// recurrence through the tile, raman_mode 2, or V = U_l conj(U_m), raman_mode 0), and each
// lane writes its 4 consecutive samples, split into TF32 hi and lo, straight into the A
// operands (buffer c % 2) in the MN-major TF32 layout (samples contiguous: the 4 samples of
// one field are one 16-byte chunk per matrix); one thread issues the chunk's 12 MMAs and
// commits them to an mbarrier; the chunk's split coefficients (SolveDesc::dense_tc, K-major)
// arrive by one bulk copy issued when the chunk starts. The MMAs of chunk c run while the
// warps build chunk c + 1. Every wait is bounded: on a timeout the CTA flags kStatusTimeout,
// waits once more for its MMAs and frees its TMEM.
template <typename T>
__global__ void __launch_bounds__(512, 1) k_contract_tc(const SolveDesc* __restrict__ descs, int nt, int raman_mode) {
  static_assert(sizeof(T) == 4, "TF32 operands come from FP32 solves");
  using V = float2;
  constexpr int TT = kTcTile, KC = kTcChunk, WMASK = TT / 64 - 1;
  // A operand (MN-major TF32 layout): 32-sample atoms 512 bytes apart, 4-field groups 2048
  static_assert(TT == 128 && KC % 8 == 0, "one MMA covers the tile's 128 samples");
  constexpr uint32_t A_LBO = 512, A_SBO = 2048;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) unsigned long long bar_u, bar_b[2], bar_m[2];
  __shared__ uint32_t s_tmem;
  const SolveDesc& d = descs[blockIdx.y];
  const int t0 = blockIdx.x * TT;
  if (t0 >= nt || d.M == 0) return;  // empty slot
  const int M = d.M, P = d.P, N = 16 * M;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  V* sU = reinterpret_cast<V*>(smem_raw);                        // [M][TT]
  // [2][4][KC * TT] MN-major operands, on the next 1024-byte boundary (the swizzle pattern's
  // alignment; the launch reserves the slack)
  unsigned char* after_u = reinterpret_cast<unsigned char*>(sU + (size_t)M * TT);
  float* sA = reinterpret_cast<float*>(after_u + ((1024u - (tc::smem_u32(after_u) & 1023u)) & 1023u));
  float* sB = sA + 2 * 4 * KC * TT;                              // [2][4][KC/4][N][4]
  V* sC = reinterpret_cast<V*>(sB + 2 * 4 * KC * N);              // states entering the tile, [P][2]
  if (tid == 0) {
    mbar_init(&bar_u, 1);
    for (int i = 0; i < 2; ++i) {
      mbar_init(&bar_b[i], 1);
      mbar_init(&bar_m[i], 1);
    }
    mbar_arrive_expect_tx(&bar_u, (unsigned)(M * TT * sizeof(V)));
  }
  __syncthreads();
  if (tid < M) bulk_g2s(sU + (size_t)tid * TT, as_t2<float>(d.U) + (size_t)tid * nt + t0, TT * sizeof(V), &bar_u);
  if (__ldcg(d.step) >= d.step_limit) {  // finished solve: the copies land before the CTA leaves
    mbar_wait(&bar_u, 0, kMaxWaitPolls);
    return;
  }
  if (raman_mode == 2) stage_tile_carries<float>(sC, d, P, nt / TT, blockIdx.x);
  if (warp == 0) {
    tc::alloc(&s_tmem, 512);
    tc::relinquish();
  }
  tc::fence_before_sync();
  bool ok = __syncthreads_and(mbar_wait(&bar_u, 0, d.tile_wait_polls) ? 1 : 0);
  const bool u_landed = ok;
  int b_issued = -1;  // last chunk whose coefficient copy was issued
  tc::fence_after_sync();
  const uint32_t tmem = s_tmem;
  TileScan<float> ts;
  if (raman_mode == 2) ts.init(d, TT >> 5, lane);
  const float kerr = (float)d.one_minus_fR;
  const int nch = (P + KC - 1) / KC;
  const unsigned bbytes = (unsigned)(4 * KC * N * sizeof(float));
  const uint32_t idesc = tc::idesc_tf32(TT, N, true);
  int committed = -1;  // last chunk whose MMAs were committed
  for (int c = 0; c < nch && ok; ++c) {
    const int buf = c & 1;
    float* A = sA + (size_t)buf * 4 * KC * TT;
    float* B = sB + (size_t)buf * 4 * KC * N;
    if (c >= 2) {  // chunk c - 2's MMAs read this buffer pair: wait for them
      ok = __syncthreads_and(mbar_wait(&bar_m[buf], ((c - 2) >> 1) & 1, kMaxWaitPolls) ? 1 : 0);
      if (!ok) break;
      tc::fence_after_sync();
    }
    if (tid == 0) {
      mbar_arrive_expect_tx(&bar_b[buf], bbytes);
      bulk_g2s(B, d.dense_tc + (size_t)c * 4 * KC * N, bbytes, &bar_b[buf]);
    }
    b_issued = c;
    for (int j = warp; j < KC; j += nwarps) {  // pair field q = c KC + j, one warp each
      const int q = c * KC + j;
      // lane L's samples 4L .. 4L + 3 of field j: one 16-byte chunk of each operand matrix
      float* a0 = A + tc::mn_tf32_offset(4 * lane, j, A_LBO, A_SBO) / 4;
      auto put = [&](const V* x) {
        float rh[4], rl[4], ih[4], il[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          rh[e] = tc::tf32_hi(x[e].x);
          rl[e] = x[e].x - rh[e];
          ih[e] = tc::tf32_hi(x[e].y);
          il[e] = x[e].y - ih[e];
        }
        *reinterpret_cast<float4*>(a0) = make_float4(rh[0], rh[1], rh[2], rh[3]);
        *reinterpret_cast<float4*>(a0 + KC * TT) = make_float4(rl[0], rl[1], rl[2], rl[3]);
        *reinterpret_cast<float4*>(a0 + 2 * KC * TT) = make_float4(ih[0], ih[1], ih[2], ih[3]);
        *reinterpret_cast<float4*>(a0 + 3 * KC * TT) = make_float4(il[0], il[1], il[2], il[3]);
      };
      if (q >= P) {  // past the last field: zeros (the buffers start uninitialised)
        const V z[4] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
        put(z);
      } else if (raman_mode == 2) {
        tile_pair_recurrence_to<float, true>(ts, sU, TT, d.pairs[q], nullptr, WMASK, sC + 2 * q, kerr, lane, put);
      } else {
        const int2 lm = d.pairs[q];
        V x[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) x[e] = cmulc(sU[lm.x * TT + 4 * lane + e], sU[lm.y * TT + 4 * lane + e]);
        put(x);
      }
    }
    tc::fence_proxy_async();
    // the chunk's coefficients have landed and every thread's operand writes are done
    ok = __syncthreads_and(mbar_wait(&bar_b[buf], (c >> 1) & 1, kMaxWaitPolls) ? 1 : 0);
    if (!ok) break;
    b_issued = -1;  // landed
    tc::fence_after_sync();
    if (tid == 0) {
      // Re: (A Re hi, B Re hi), (Re hi, Re lo), (Re lo, Re hi); Im likewise
      constexpr int ta[3] = {0, 0, 1}, tb[3] = {0, 1, 0};
#pragma unroll
      for (int part = 0; part < 2; ++part)
#pragma unroll
        for (int term = 0; term < 3; ++term)
#pragma unroll
          for (int ks = 0; ks < KC / 8; ++ks) {
            const float* a = A + (size_t)(2 * part + ta[term]) * KC * TT + ks * 2 * A_SBO / 4;
            const float* b = B + (size_t)(2 * part + tb[term]) * KC * N + ks * 2 * N * 4;
            tc::mma_tf32(tmem + 256u * part, tc::desc_mn_tf32(a, A_LBO, A_SBO), tc::desc_kmajor(b, N * 16, 128),
                         idesc, (c > 0 || term > 0 || ks > 0) ? 1u : 0u);
          }
      tc::commit(&bar_m[buf]);
    }
    committed = c;
  }
  // the last chunk's MMAs complete after all earlier ones (in-order issue, one thread)
  if (ok && committed >= 0)
    ok = __syncthreads_and(mbar_wait(&bar_m[committed & 1], (committed >> 1) & 1, kMaxWaitPolls) ? 1 : 0);
  tc::fence_after_sync();
  if (ok) {
    // sigma_p(t) = sum_k U_k(t) (T_re + i T_im): warp w reads TMEM lanes 32 (w % 4) .. + 31
    const int quad = warp & 3, t = quad * 32 + lane;
    const uint32_t tl = tmem + ((uint32_t)(quad * 32) << 16);
    V* sigma = as_t2<float>(d.sigma);
    for (int p = warp >> 2; p < M; p += nwarps >> 2) {
      float re[16], im[16];
      tc::ld16(tl + 16u * p, re);
      tc::ld16(tl + 256u + 16u * p, im);
      float sx = 0.f, sy = 0.f;
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        if (k < M) {
          const V u = sU[k * TT + t];
          sx = fmaf(u.x, re[k], fmaf(-u.y, im[k], sx));
          sy = fmaf(u.x, im[k], fmaf(u.y, re[k], sy));
        }
      }
      sigma[(size_t)p * nt + t0 + t] = make_float2(sx, sy);
    }
  } else {
    if (tid == 0) atomicOr(d.status, kStatusTimeout);
    // nothing may still be writing this CTA's shared memory or TMEM when it leaves: the
    // tile and coefficient copies in flight, the MMAs in flight (each waited for once more)
    if (!u_landed) mbar_wait(&bar_u, 0, kMaxWaitPolls);
    if (b_issued >= 0) mbar_wait(&bar_b[b_issued & 1], (b_issued >> 1) & 1, kMaxWaitPolls);
    if (committed >= 0) mbar_wait(&bar_m[committed & 1], (committed >> 1) & 1, kMaxWaitPolls);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::dealloc(tmem, 512);
}

// FP64 rows -> T rows (used for the Raman spectrum)
template <typename T>
__global__ void k_to_t2(const double2* __restrict__ in, c2<T>* __restrict__ out, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = from_d2<T>(in[i]);
}

}  // namespace mmp
