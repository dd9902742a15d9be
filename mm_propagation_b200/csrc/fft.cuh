// fft.cuh — shared-memory Stockham FFT for one row per CTA, or one row per
// thread-block cluster (rows larger than 128 KB), built for sm_100a.
//
// Row of N = 2^LOGN complex samples in precision T (float or double).
//  * C = 2^LOGC CTAs (a cluster) share a row when N * sizeof(T2) > 128 KB.
//    CTA c holds the decimated sub-sequence x[c + C*u], u < NL = N / C, in its
//    shared memory and transforms it locally; a radix-C butterfly across the
//    cluster, reading and writing peer CTAs' shared memory (DSMEM), combines
//    the C local spectra (decimation in time). The inverse runs the same steps
//    backwards (split across the cluster, then local inverse transforms).
//  * The local transform is an in-place Stockham autosort FFT in padded
//    shared memory: each thread keeps E = 2^LOGE samples in registers per pass,
//    runs radix-2^r butterflies on them, and writes them back in Stockham order,
//    so no bit reversal is needed and input and output are both in natural order.
//  * Twiddles come from per-size tables w_n[m] = exp(-2 pi i m / n), computed in
//    FP64 on the host and rounded to T.
//
// Frequency-domain samples are handed between the FFT and the kernels'
// point-wise math in registers: register slot i of a thread holds frequency
// freq_index(i) (see Geo). Time-domain samples stay in shared memory: local
// index u holds time t = rank + C*u.
#pragma once

#include <cooperative_groups.h>

#include "common.cuh"

namespace mmp {
namespace cg = cooperative_groups;

// cos(2*pi*k/32) for any integer k, exact to double rounding.
__host__ __device__ constexpr double cos32(int k) {
  k = ((k % 32) + 32) % 32;
  if (k > 16) k = 32 - k;            // cos is even around 0 (mod 32)
  const bool neg = k > 8;
  if (neg) k = 16 - k;               // cos(pi - x) = -cos(x)
  constexpr double t[9] = {1.0,
                           0.98078528040323044912618223613424,
                           0.92387953251128675612818318939679,
                           0.83146961230254523707878837761791,
                           0.70710678118654752440084436210485,
                           0.55557023301960222474283081394853,
                           0.38268343236508977172845998403040,
                           0.19509032201612826784828486847702,
                           0.0};
  return neg ? -t[k] : t[k];
}

// Multiply v by w_R^e = exp(sgn * 2*pi*i*e / R), sgn = -1 forward, +1 inverse.
// Exact special cases for multiples of pi/4.
template <int R, int E_, bool INV, typename V>
__device__ __forceinline__ V twiddle_const(V v) {
  constexpr int e = ((E_ % R) + R) % R;
  if constexpr (e == 0) {
    return v;
  } else if constexpr ((4 * e) % R == 0) {
    constexpr int quarter = (4 * e) / R;  // 1, 2, 3 quarter turns
    if constexpr (quarter == 2) {
      v.x = -v.x; v.y = -v.y; return v;
    } else {
      // forward: quarter 1 -> -i, quarter 3 -> +i ; inverse: mirrored
      constexpr bool plus_i = (quarter == 1) == INV;
      return crot<plus_i>(v);
    }
  } else {
    using S = decltype(v.x);
    constexpr int k32 = e * (32 / R);
    constexpr double cr = cos32(k32);
    constexpr double si = cos32(k32 - 8);  // sin(2 pi k/32)
    const S c = (S)cr;
    const S s = INV ? (S)si : (S)(-si);
    V r;
    r.x = v.x * c - v.y * s;
    r.y = v.x * s + v.y * c;
    return r;
  }
}

// In-register DFT of size R (power of two <= 32), natural order in and out.
template <int R, bool INV> struct RegDFT;

template <bool INV> struct RegDFT<1, INV> {
  template <typename V> __device__ __forceinline__ static void run(V*) {}
};
template <bool INV> struct RegDFT<2, INV> {
  template <typename V> __device__ __forceinline__ static void run(V* v) {
    const V a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};
template <bool INV> struct RegDFT<4, INV> {
  template <typename V> __device__ __forceinline__ static void run(V* v) {
    const V a = v[0], b = v[1], c = v[2], d = v[3];
    const V apc = cadd(a, c), amc = csub(a, c), bpd = cadd(b, d);
    const V rot = crot<INV>(csub(b, d));  // forward: -i (b-d); inverse: +i (b-d)
    v[0] = cadd(apc, bpd);
    v[1] = cadd(amc, rot);
    v[2] = csub(apc, bpd);
    v[3] = csub(amc, rot);
  }
};
// R = A * B with A = 4 (or 2 for R = 8 ... kept at 4 where possible):
// t = a + A*b, k = B*ka + kb:  X[B ka + kb] = sum_a w_A^{a ka} w_R^{a kb} sum_b x[a + A b] w_B^{b kb}
template <int R, bool INV> struct RegDFT {
  static constexpr int A = (R % 4 == 0 && R > 4) ? 4 : 2;
  static constexpr int B = R / A;
  template <typename V> __device__ __forceinline__ static void run(V* v) {
    V y[R];
#pragma unroll
    for (int a = 0; a < A; ++a) {
      V col[B];
#pragma unroll
      for (int b = 0; b < B; ++b) col[b] = v[a + A * b];
      RegDFT<B, INV>::run(col);
#pragma unroll
      for (int kb = 0; kb < B; ++kb) y[a * B + kb] = col[kb];
    }
    apply_tw<0, 0>(y);
#pragma unroll
    for (int kb = 0; kb < B; ++kb) {
      V row[A];
#pragma unroll
      for (int a = 0; a < A; ++a) row[a] = y[a * B + kb];
      RegDFT<A, INV>::run(row);
#pragma unroll
      for (int ka = 0; ka < A; ++ka) v[B * ka + kb] = row[ka];
    }
  }
  // compile-time walk over (a, kb) applying w_R^{a*kb}
  template <int a, int kb, typename V> __device__ __forceinline__ static void apply_tw(V* y) {
    if constexpr (a < A) {
      if constexpr (kb < B) {
        y[a * B + kb] = twiddle_const<R, a * kb, INV>(y[a * B + kb]);
        apply_tw<a, kb + 1>(y);
      } else {
        apply_tw<a + 1, 0>(y);
      }
    }
  }
};


// Twiddle tables: tw.f[L] / tw.d[L] point at 2^L entries exp(-2 pi i m / 2^L).
struct TwTables {
  const float2* f[17];
  const double2* d[17];
};
template <typename T> __device__ __forceinline__ const c2<T>* tw_table(const TwTables& t, int L);
template <> __device__ __forceinline__ const float2* tw_table<float>(const TwTables& t, int L) { return t.f[L]; }
template <> __device__ __forceinline__ const double2* tw_table<double>(const TwTables& t, int L) { return t.d[L]; }

// Geometry of one row transform.
template <typename T, int LOGN_, int XC_ = 0> struct Geo {
  static constexpr int LOGN = LOGN_;
  static constexpr int N = 1 << LOGN;
  static constexpr int LOGSZ = sizeof(c2<T>) == 8 ? 3 : 4;
  static constexpr int LOGC = ((LOGN + LOGSZ > 17) ? (LOGN + LOGSZ - 17) : 0) + XC_;  // <= 128 KB of row per CTA, times 2^XC_ CTAs
  static constexpr int C = 1 << LOGC;
  static constexpr int LOGL = LOGN - LOGC;
  static constexpr int NL = 1 << LOGL;
  static constexpr int LOGE_PREF = (sizeof(T) == 4 && LOGL >= 13) ? 5 : 4;
  static constexpr int LOGE_CAP = LOGL - 5 > 1 ? LOGL - 5 : 1;  // keep >= 32 threads
  static constexpr int LOGE = LOGE_PREF < LOGE_CAP ? LOGE_PREF : LOGE_CAP;
  static constexpr int E = 1 << LOGE;
  static constexpr int NTHR = NL / E;
  static constexpr int LOGCH = LOGL - LOGC;
  static constexpr int CH = NL / C;       // frequencies k a CTA combines
  static constexpr int LOGQ = LOGL - 2;   // quarter-wave twiddle table: NL/4 entries
  static constexpr int DATA_BYTES = padded_len(NL) * (int)sizeof(c2<T>);
  static constexpr int TWQ_BYTES = padded_len(NL / 4) * (int)sizeof(c2<T>);
  static constexpr int SMEM_BYTES = DATA_BYTES + TWQ_BYTES;
  // split rows (XC_ > 0) are sized so that two CTAs share an SM
  static constexpr int MIN_BLOCKS = (XC_ > 0 && SMEM_BYTES <= 110 * 1024 && NTHR <= 512) ? 2 : 1;
  static_assert(LOGE >= LOGC, "each thread must combine at least one frequency per CTA");
  static_assert(NTHR >= 32 && NTHR <= 1024, "block size");
  static_assert(DATA_BYTES % 16 == 0, "twiddle table alignment");

  // Spectrum layout in shared memory after a forward transform ("combined layout"):
  // local index i holds frequency rank*CH + (i mod CH) + NL*(i div CH); for C = 1
  // that is just i.
  __device__ __forceinline__ static int freq_of(int rank, int i) {
    if constexpr (C == 1) return i;
    else return rank * CH + (i & (CH - 1)) + NL * (i >> LOGCH);
  }
  // Time layout: local index u holds time rank + C*u.
  __device__ __forceinline__ static int time_of(int rank, int u) { return rank + C * u; }
};

// exp(-2 pi i m / NL) (conjugated for INV) from the quarter-wave table
// sq[pad(m')] = exp(-2 pi i m' / NL), m' < NL/4: w(m) = (-i)^(m div NL/4) * sq[m mod NL/4].
// The table uses the same padded index as the data: the Stockham passes read it at
// strides of 2^a entries, which would otherwise land in one bank.
template <typename V, bool INV, int LOGQ>
__device__ __forceinline__ V tw_quarter(const V* __restrict__ sq, int m) {
  const int q = m >> LOGQ;
  const V w = sq[pad(m & ((1 << LOGQ) - 1))];
  V r;
  r.x = (q & 1) ? w.y : w.x;
  r.y = (q & 1) ? -w.x : w.y;
  if (q & 2) { r.x = -r.x; r.y = -r.y; }
  if (INV) r.y = -r.y;
  return r;
}

// Copy the first quarter of the size-NL table into shared memory.
template <typename T, int LOGN, int XC>
__device__ __forceinline__ c2<T>* load_twiddles(unsigned char* smem_raw, const TwTables& tw) {
  using Gm = Geo<T, LOGN, XC>;
  c2<T>* sq = reinterpret_cast<c2<T>*>(smem_raw + Gm::DATA_BYTES);
  const c2<T>* g = tw_table<T>(tw, Gm::LOGL);
#pragma unroll 4
  for (int m = threadIdx.x; m < Gm::NL / 4; m += Gm::NTHR) sq[pad(m)] = __ldg(&g[m]);
  return sq;
}

// One in-place Stockham pass of radix 2^LOGR at stride Ns = 2^logns (runtime).
template <typename T, int LOGL, int LOGE, int LOGR, bool INV>
__device__ __forceinline__ void stockham_pass(c2<T>* __restrict__ s, const c2<T>* __restrict__ sq, int logns) {
  using V = c2<T>;
  constexpr int NL = 1 << LOGL, E = 1 << LOGE, NTHR = NL / E;
  constexpr int R = 1 << LOGR, NB = E / R, LOGQ = LOGL - 2;
  const int tid = threadIdx.x;
  V v[E];
#pragma unroll
  for (int bf = 0; bf < NB; ++bf) {
    const int j = tid + bf * NTHR;
#pragma unroll
    for (int r = 0; r < R; ++r) v[bf * R + r] = s[pad(j + r * (NL / R))];
  }
  __syncthreads();
  const int nsm = (1 << logns) - 1;
#pragma unroll
  for (int bf = 0; bf < NB; ++bf) {
    const int j = tid + bf * NTHR;
    const int jm = j & nsm;
    if (logns > 0) {
      const int step = jm << (LOGL - logns - LOGR);  // jm * NL / (Ns * R)
#pragma unroll
      for (int r = 1; r < R; ++r) v[bf * R + r] = cmul(v[bf * R + r], tw_quarter<V, INV, LOGQ>(sq, r * step));
    }
    RegDFT<R, INV>::run(&v[bf * R]);
    const int idxD = ((j >> logns) << (logns + LOGR)) + jm;
#pragma unroll
    for (int r = 0; r < R; ++r) s[pad(idxD + (r << logns))] = v[bf * R + r];
  }
  __syncthreads();
}

// Local transform of the NL samples in shared memory (natural order in and out,
// unnormalised). One pass body per radix keeps the instruction footprint small.
template <typename T, int LOGN, int XC, bool INV>
__device__ __noinline__ void local_fft(c2<T>* __restrict__ s, const c2<T>* __restrict__ sq) {
  using Gm = Geo<T, LOGN, XC>;
  constexpr int FULL = Gm::LOGL / Gm::LOGE, REM = Gm::LOGL % Gm::LOGE;
  __syncthreads();
  int logns = 0;
#pragma unroll 1
  for (int p = 0; p < FULL; ++p) {
    stockham_pass<T, Gm::LOGL, Gm::LOGE, Gm::LOGE, INV>(s, sq, logns);
    logns += Gm::LOGE;
  }
  if constexpr (REM > 0) stockham_pass<T, Gm::LOGL, Gm::LOGE, REM, INV>(s, sq, logns);
}

// Forward transform of the time samples in shared memory (local u = time rank + C*u);
// leaves the spectrum in shared memory in the combined layout (Geo::freq_of).
template <typename T, int LOGN, int XC>
__device__ __forceinline__ void forward(c2<T>* __restrict__ s, const c2<T>* __restrict__ sq, const TwTables& tw) {
  using Gm = Geo<T, LOGN, XC>;
  using V = c2<T>;
  local_fft<T, LOGN, XC, false>(s, sq);
  if constexpr (Gm::C > 1) {
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    const int tid = threadIdx.x;
    const V* twN = tw_table<T>(tw, Gm::LOGN);
    V out[Gm::E];
    cl.sync();  // every CTA finished its local transform
#pragma unroll
    for (int jj = 0; jj < Gm::E / Gm::C; ++jj) {
      const int k = rank * Gm::CH + tid + jj * Gm::NTHR;
      V vals[Gm::C];
#pragma unroll
      for (int c = 0; c < Gm::C; ++c) {
        const V* peer = cl.map_shared_rank(s, c);
        V f = peer[pad(k)];
        if (c > 0) f = cmul(f, __ldg(&twN[c * k]));
        vals[c] = f;
      }
      RegDFT<Gm::C, false>::run(vals);
#pragma unroll
      for (int q = 0; q < Gm::C; ++q) out[jj * Gm::C + q] = vals[q];
    }
    cl.sync();  // all peer reads done before shared memory is overwritten
#pragma unroll
    for (int jj = 0; jj < Gm::E / Gm::C; ++jj) {
      const int kl = tid + jj * Gm::NTHR;
#pragma unroll
      for (int q = 0; q < Gm::C; ++q) s[pad(kl + Gm::CH * q)] = out[jj * Gm::C + q];
    }
    __syncthreads();
  }
}

// Inverse transform of a spectrum in shared memory in the combined layout; leaves
// the (unnormalised) time samples in shared memory, local u = time rank + C*u.
template <typename T, int LOGN, int XC>
__device__ __forceinline__ void inverse(c2<T>* __restrict__ s, const c2<T>* __restrict__ sq, const TwTables& tw) {
  using Gm = Geo<T, LOGN, XC>;
  using V = c2<T>;
  if constexpr (Gm::C > 1) {
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    const int tid = threadIdx.x;
    const V* twN = tw_table<T>(tw, Gm::LOGN);
    V out[Gm::E];
    __syncthreads();  // the caller's writes of the spectrum are complete
#pragma unroll
    for (int jj = 0; jj < Gm::E / Gm::C; ++jj) {
      const int kl = tid + jj * Gm::NTHR;
      const int k = rank * Gm::CH + kl;
      V vals[Gm::C];
#pragma unroll
      for (int q = 0; q < Gm::C; ++q) vals[q] = s[pad(kl + Gm::CH * q)];
      RegDFT<Gm::C, true>::run(vals);
#pragma unroll
      for (int c = 0; c < Gm::C; ++c) {
        V f = vals[c];
        if (c > 0) f = cmulc(f, __ldg(&twN[c * k]));
        out[jj * Gm::C + c] = f;
      }
    }
    cl.sync();  // every CTA is running and has read its own spectrum
#pragma unroll
    for (int jj = 0; jj < Gm::E / Gm::C; ++jj) {
      const int k = rank * Gm::CH + tid + jj * Gm::NTHR;
#pragma unroll
      for (int c = 0; c < Gm::C; ++c) {
        V* peer = cl.map_shared_rank(s, c);
        peer[pad(k)] = out[jj * Gm::C + c];
      }
    }
    cl.sync();  // all peer writes landed
  }
  local_fft<T, LOGN, XC, true>(s, sq);
}

}  // namespace mmp
