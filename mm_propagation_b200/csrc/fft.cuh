// fft.cuh — shared-memory Stockham FFT for one row per CTA, or one row per
// thread-block cluster (rows larger than 128 KB), built for sm_100a.
//
// Row of N = 2^LOGN complex samples in precision T (float or double).
//  * C = 2^LOGC CTAs (a cluster) share a row when N * sizeof(T2) > 128 KB.
//    The row is cut into runs of G consecutive samples, G * sizeof(T2) = 32 bytes (one
//    DRAM sector: G = 4 in FP32, 2 in FP64), dealt out to the CTAs in turn: CTA r holds
//    the samples t = g + G (r + C v), g < G, v < NL/G (NL = N / C), so that its global
//    loads and stores move whole sectors. In shared memory they are G rows of NL/G:
//    row g is the sub-sequence x_g[s] = x[g + G s] at s = r + C v, decimated over the
//    cluster. Forward: every CTA transforms its G rows locally (NL/G points each); a
//    radix-(C G) butterfly combines, per frequency, the partial spectra of the G rows
//    of all C CTAs, read through distributed shared memory (decimation in time over
//    the C G sub-sequences x[n + C G u]). The inverse runs the same steps backwards.
//    With C = 1, G = 1 and the row is one local transform.
//  * The local transform is an in-place Stockham autosort FFT in padded
//    shared memory: each thread keeps E = 2^LOGE samples in registers per pass,
//    runs radix-2^r butterflies on them, and writes them back in Stockham order,
//    so no bit reversal is needed and input and output are both in natural order.
//  * Twiddles come from per-size tables w_n[m] = exp(-2 pi i m / n), computed in
//    FP64 on the host and rounded to T.
//
// Frequency-domain samples stay in shared memory in the "combined layout" (Geo::freq_of:
// C G spans of CH consecutive frequencies per CTA). Time-domain samples: local row g,
// column v holds time g + G (rank + C v); kernels walk them in time order with
// Geo::time_of_w / Geo::local_of_w, so that a warp's accesses cover whole sectors.
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
// cf[L][xc] / cd[L][xc]: the cluster combine's twiddles of a split row of 2^L samples
// (row split xc), [n][kl] = exp(-2 pi i n kl / 2^L) for n < CG, kl < 2^L / CG (CG = C G of
// that geometry), so that a warp's lanes (consecutive kl) read consecutive entries; null
// where not built (the combine then reads the 2^L table at n kl).
struct TwTables {
  const float2* f[17];
  const double2* d[17];
  const float2* cf[17][2];
  const double2* cd[17][2];
};
template <typename T> __device__ __forceinline__ const c2<T>* tw_table(const TwTables& t, int L);
template <> __device__ __forceinline__ const float2* tw_table<float>(const TwTables& t, int L) { return t.f[L]; }
template <> __device__ __forceinline__ const double2* tw_table<double>(const TwTables& t, int L) { return t.d[L]; }
template <typename T> __device__ __forceinline__ const c2<T>* cmb_table(const TwTables& t, int L, int xc);
template <> __device__ __forceinline__ const float2* cmb_table<float>(const TwTables& t, int L, int xc) { return t.cf[L][xc]; }
template <> __device__ __forceinline__ const double2* cmb_table<double>(const TwTables& t, int L, int xc) { return t.cd[L][xc]; }

// Geometry of one row transform.
template <typename T, int LOGN_, int XC_ = 0> struct Geo {
  using Real = T;
  static constexpr int LOGN = LOGN_;
  static constexpr int N = 1 << LOGN;
  static constexpr int LOGSZ = sizeof(c2<T>) == 8 ? 3 : 4;
  static constexpr int LOGC = ((LOGN + LOGSZ > 17) ? (LOGN + LOGSZ - 17) : 0) + XC_;  // <= 128 KB of row per CTA, times 2^XC_ CTAs
  static constexpr int C = 1 << LOGC;
  static constexpr int LOGL = LOGN - LOGC;
  static constexpr int NL = 1 << LOGL;
  // runs of G samples (32 bytes) per CTA on split rows; G rows of NLG in shared memory
  static constexpr int LOGG = LOGC > 0 ? 5 - LOGSZ : 0;
  static constexpr int G = 1 << LOGG;
  static constexpr int LOGNLG = LOGL - LOGG;
  static constexpr int NLG = 1 << LOGNLG;
  static constexpr int LOGE_PREF = (sizeof(T) == 4 && LOGL >= 13) ? 5 : 4;
  static constexpr int LOGE_CAP = LOGL - 5 > 1 ? LOGL - 5 : 1;  // keep >= 32 threads
  static constexpr int LOGE = LOGE_PREF < LOGE_CAP ? LOGE_PREF : LOGE_CAP;
  static constexpr int E = 1 << LOGE;
  static constexpr int NTHR = NL / E;
  static constexpr int LOGCH = LOGNLG - LOGC;
  static constexpr int CH = 1 << LOGCH;  // frequencies per span: C G spans per CTA
  // twiddle table of the local size in shared memory: half a wave (one sign flip per
  // lookup) where that is at most 32 KB, else a quarter wave (a quadrant fold per lookup;
  // a 64 KB table cost the 16384-sample single-CTA rows ~5% in loading it)
  static constexpr bool TW_HALF = (NLG / 2) * (int)sizeof(c2<T>) <= 32 * 1024;
  static constexpr int LOGH = TW_HALF ? LOGNLG - 1 : LOGNLG - 2;  // log2 of the table's entries
  static constexpr int NTW = 1 << LOGH;
  // rows g > 0 start SKEW elements later (mod 128 bytes), so that a warp walking the
  // samples in time order (row g = lane mod G) reads and writes without bank conflicts
  static constexpr int SKEW = LOGG > 0 ? 4 : 0;
  static constexpr int DATA_BYTES = (padded_len(NL) + (G - 1) * SKEW) * (int)sizeof(c2<T>);
  static constexpr int TW_BYTES = padded_len(NTW) * (int)sizeof(c2<T>);
  static constexpr int SMEM_BYTES = DATA_BYTES + TW_BYTES;
  // split rows (XC_ > 0) are sized so that two CTAs share an SM
  static constexpr int MIN_BLOCKS = (XC_ > 0 && SMEM_BYTES <= 110 * 1024 && NTHR <= 512) ? 2 : 1;
  static_assert(LOGE >= LOGC + LOGG, "each thread must combine at least one frequency per CTA");
  static_assert(LOGNLG - LOGE >= 5 || LOGG == 0, "a warp's butterflies stay within one row");
  static_assert(NTHR >= 32 && NTHR <= 1024, "block size");
  static_assert(DATA_BYTES % 16 == 0, "twiddle table alignment");

  // shared-memory offset of local index i (row i >> LOGNLG)
  __host__ __device__ __forceinline__ static int sidx(int i) { return pad(i) + (i >> LOGNLG) * SKEW; }
  // Spectrum layout in shared memory after a forward transform ("combined layout"):
  // local index i holds frequency rank*CH + (i mod CH) + NLG*(i div CH); for C = 1
  // that is just i.
  __device__ __forceinline__ static int freq_of(int rank, int i) {
    if constexpr (C == 1) return i;
    else return rank * CH + (i & (CH - 1)) + NLG * (i >> LOGCH);
  }
  // The CTA's time samples in time order, w < NL: time and local index of the w-th.
  __device__ __forceinline__ static int time_of_w(int rank, int w) {
    if constexpr (C == 1) return w;
    else return ((((w >> LOGG) << LOGC) + rank) << LOGG) + (w & (G - 1));
  }
  __device__ __forceinline__ static int local_of_w(int w) {
    if constexpr (C == 1) return w;
    else return ((w & (G - 1)) << LOGNLG) + (w >> LOGG);
  }
};

// exp(-2 pi i m / NLG) (conjugated for INV), m < NLG, from the table
// sh[pad(m')] = exp(-2 pi i m' / NLG), m' < 2^LOGH: a half wave (w(m) = -sh[m - NLG/2] from
// NLG/2 on) or a quarter wave (w(m) = (-i)^(m div NLG/4) sh[m mod NLG/4]).
// The table uses the same padded index as the data: the Stockham passes read it at
// strides of 2^a entries, which would otherwise land in one bank.
template <typename V, bool INV, bool HALF, int LOGH>
__device__ __forceinline__ V tw_lookup(const V* __restrict__ sh, int m) {
  const int q = m >> LOGH;
  V w = sh[pad(m & ((1 << LOGH) - 1))];
  if constexpr (HALF) {
    if (q) { w.x = -w.x; w.y = -w.y; }
  } else {
    const V w0 = w;
    w.x = (q & 1) ? w0.y : w0.x;
    w.y = (q & 1) ? -w0.x : w0.y;
    if (q & 2) { w.x = -w.x; w.y = -w.y; }
  }
  if (INV) w.y = -w.y;
  return w;
}

// Copy the first 2^LOGH entries of the local transform's table (NLG points) into shared memory.
template <typename T, int LOGN, int XC>
__device__ __forceinline__ c2<T>* load_twiddles(unsigned char* smem_raw, const TwTables& tw) {
  using Gm = Geo<T, LOGN, XC>;
  c2<T>* sq = reinterpret_cast<c2<T>*>(smem_raw + Gm::DATA_BYTES);
  const c2<T>* g = tw_table<T>(tw, Gm::LOGNLG);
#pragma unroll 4
  for (int m = threadIdx.x; m < Gm::NTW; m += Gm::NTHR) sq[pad(m)] = __ldg(&g[m]);
  return sq;
}

// One in-place Stockham pass of radix 2^LOGR at stride Ns = 2^logns (runtime) over the
// rows of Gm (G rows of NLG samples; a thread's butterflies j < NL/R, row j / (NLG/R)).
// Shared-memory offsets: where a butterfly's R elements lie 32·c apart within a row, the
// padded offset advances by a constant (pad(i + 32c) = pad(i) + 33c), so only the first
// is computed.
template <typename Gm, int LOGR, bool INV>
__device__ __forceinline__ void stockham_pass(c2<typename Gm::Real>* __restrict__ s,
                                              const c2<typename Gm::Real>* __restrict__ sq, int logns) {
  using V = c2<typename Gm::Real>;
  constexpr int LOGB = Gm::LOGNLG;  // row length
  constexpr int NB = 1 << LOGB, E = Gm::E, NTHR = Gm::NTHR;
  constexpr int R = 1 << LOGR, NBF = E / R;
  constexpr int LOGJ = LOGB - LOGR;  // butterflies per row
  constexpr int S = NB / R;          // read stride
  const int tid = threadIdx.x;
  V v[E];
#pragma unroll
  for (int bf = 0; bf < NBF; ++bf) {
    const int ja = tid + bf * NTHR;
    const int base = (ja >> LOGJ) << LOGB, j = ja & ((1 << LOGJ) - 1);
    if constexpr (S % 32 == 0) {
      const int a0 = Gm::sidx(base + j);
#pragma unroll
      for (int r = 0; r < R; ++r) v[bf * R + r] = s[a0 + r * (S + S / 32)];
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) v[bf * R + r] = s[Gm::sidx(base + j + r * S)];
    }
  }
  __syncthreads();
  const int nsm = (1 << logns) - 1;
#pragma unroll
  for (int bf = 0; bf < NBF; ++bf) {
    const int ja = tid + bf * NTHR;
    const int base = (ja >> LOGJ) << LOGB, j = ja & ((1 << LOGJ) - 1);
    const int jm = j & nsm;
    if (logns > 0) {
      const int step = jm << (LOGB - logns - LOGR);  // jm * NB / (Ns * R)
#pragma unroll
      for (int r = 1; r < R; ++r) v[bf * R + r] = cmul(v[bf * R + r], tw_lookup<V, INV, Gm::TW_HALF, Gm::LOGH>(sq, r * step));
    }
    RegDFT<R, INV>::run(&v[bf * R]);
    const int idxD = ((j >> logns) << (logns + LOGR)) + jm;
    const int w0 = Gm::sidx(base + idxD);
    if (logns >= 5) {  // R elements Ns apart, Ns a multiple of 32
      const int st = (1 << logns) + (1 << (logns - 5));
#pragma unroll
      for (int r = 0; r < R; ++r) s[w0 + r * st] = v[bf * R + r];
    } else if (logns == 0) {  // R consecutive elements from a multiple of R (R <= 32)
#pragma unroll
      for (int r = 0; r < R; ++r) s[w0 + r] = v[bf * R + r];
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) s[Gm::sidx(base + idxD + (r << logns))] = v[bf * R + r];
    }
  }
  __syncthreads();
}

// Local transform of the G rows of NLG samples in shared memory (natural order in and
// out, unnormalised). One pass body per radix keeps the instruction footprint small.
template <typename T, int LOGN, int XC, bool INV>
__device__ __noinline__ void local_fft(c2<T>* __restrict__ s, const c2<T>* __restrict__ sq) {
  using Gm = Geo<T, LOGN, XC>;
  constexpr int FULL = Gm::LOGNLG / Gm::LOGE, REM = Gm::LOGNLG % Gm::LOGE;
  __syncthreads();
  int logns = 0;
#pragma unroll 1
  for (int p = 0; p < FULL; ++p) {
    stockham_pass<Gm, Gm::LOGE, INV>(s, sq, logns);
    logns += Gm::LOGE;
  }
  if constexpr (REM > 0) stockham_pass<Gm, REM, INV>(s, sq, logns);
}

// w[n] = w_N^{n kl}, 0 < n < CG: row n of the combine table at kl, or the N-point table
// at n kl where no combine table is given.
template <typename Gm>
__device__ __forceinline__ void combine_twiddles(c2<typename Gm::Real>* w, const c2<typename Gm::Real>* twc,
                                                 const c2<typename Gm::Real>* twN, int kl) {
  constexpr int CG = Gm::C * Gm::G;
  if (twc) {
#pragma unroll
    for (int n = 1; n < CG; ++n) w[n] = __ldg(&twc[n * Gm::NLG + kl]);
  } else {
#pragma unroll
    for (int n = 1; n < CG; ++n) w[n] = __ldg(&twN[n * kl]);
  }
}

// Forward transform of the time samples in shared memory (row g, column v: time
// g + G (rank + C v)); leaves the spectrum in shared memory in the combined layout
// (Geo::freq_of). Row g of CTA c is the sub-sequence x[n + CG u], n = g + G c, u < NLG
// (CG = C G), so with F_n its local NLG-point spectrum (decimation in time):
//   X[kl + NLG j] = sum_n w_CG^{n j} w_N^{n kl} F_n[kl],  kl < NLG, j < CG.
// A thread handles K = E / CG values kl = rank CH + i, i = tid + jj NTHR: CG inputs each
// (G rows in each of the C CTAs), one radix-CG DFT, CG outputs, all of them frequencies
// this CTA keeps (span j, offset i). Every remote read is issued before the cluster
// barrier that lets the CTAs overwrite their rows. Out of line: its registers are its own.
template <typename T, int LOGN, int XC>
__device__ __noinline__ void combine_fwd(c2<T>* __restrict__ s, const TwTables& tw) {
  using Gm = Geo<T, LOGN, XC>;
  using V = c2<T>;
  if constexpr (Gm::C > 1) {
    constexpr int C = Gm::C, G = Gm::G, CG = C * G, K = Gm::E / CG;
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    const int tid = threadIdx.x;
    const V* twN = tw_table<T>(tw, Gm::LOGN);
    V v[K][CG];
    cl.sync();  // every CTA finished its local transforms
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const V* peer = cl.map_shared_rank(s, c);
#pragma unroll
      for (int jj = 0; jj < K; ++jj) {
        const int kl = rank * Gm::CH + tid + jj * Gm::NTHR;
#pragma unroll
        for (int g = 0; g < G; ++g) v[jj][g + G * c] = peer[Gm::sidx(g * Gm::NLG + kl)];
      }
    }
    const V* twc = cmb_table<T>(tw, Gm::LOGN, XC);
#pragma unroll
    for (int jj = 0; jj < K; ++jj) {
      const int kl = rank * Gm::CH + tid + jj * Gm::NTHR;
      V w[CG];
      combine_twiddles<Gm>(w, twc, twN, kl);
#pragma unroll
      for (int n = 1; n < CG; ++n) v[jj][n] = cmul(v[jj][n], w[n]);
      RegDFT<CG, false>::run(v[jj]);
    }
    cl.sync();  // all peer reads done before shared memory is overwritten
#pragma unroll
    for (int jj = 0; jj < K; ++jj) {
      const int i = tid + jj * Gm::NTHR;
#pragma unroll
      for (int j = 0; j < CG; ++j) s[Gm::sidx(j * Gm::CH + i)] = v[jj][j];
    }
    __syncthreads();
  }
}
template <typename T, int LOGN, int XC>
__device__ __forceinline__ void forward(c2<T>* __restrict__ s, const c2<T>* __restrict__ sq, const TwTables& tw) {
  local_fft<T, LOGN, XC, false>(s, sq);
  if constexpr (Geo<T, LOGN, XC>::C > 1) combine_fwd<T, LOGN, XC>(s, tw);
}

// Inverse transform of a spectrum in shared memory in the combined layout; leaves
// the (unnormalised) time samples in shared memory (row g, column v: time
// g + G (rank + C v)): the forward steps backwards with conjugate twiddles.
template <typename T, int LOGN, int XC>
__device__ __noinline__ void combine_inv(c2<T>* __restrict__ s, const TwTables& tw) {
  using Gm = Geo<T, LOGN, XC>;
  using V = c2<T>;
  if constexpr (Gm::C > 1) {
    constexpr int C = Gm::C, G = Gm::G, CG = C * G, K = Gm::E / CG;
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    const int tid = threadIdx.x;
    const V* twN = tw_table<T>(tw, Gm::LOGN);
    V v[K][CG];
    __syncthreads();  // the caller's writes of the spectrum are complete
    const V* twc = cmb_table<T>(tw, Gm::LOGN, XC);
#pragma unroll
    for (int jj = 0; jj < K; ++jj) {
      const int i = tid + jj * Gm::NTHR;
      const int kl = rank * Gm::CH + i;
#pragma unroll
      for (int j = 0; j < CG; ++j) v[jj][j] = s[Gm::sidx(j * Gm::CH + i)];
      RegDFT<CG, true>::run(v[jj]);
      V w[CG];
      combine_twiddles<Gm>(w, twc, twN, kl);
#pragma unroll
      for (int n = 1; n < CG; ++n) v[jj][n] = cmulc(v[jj][n], w[n]);
    }
    cl.sync();  // every CTA is running and has read its own spectrum
#pragma unroll
    for (int c = 0; c < C; ++c) {
      V* peer = cl.map_shared_rank(s, c);
#pragma unroll
      for (int jj = 0; jj < K; ++jj) {
        const int kl = rank * Gm::CH + tid + jj * Gm::NTHR;
#pragma unroll
        for (int g = 0; g < G; ++g) peer[Gm::sidx(g * Gm::NLG + kl)] = v[jj][g + G * c];
      }
    }
    cl.sync();  // all peer writes landed
  }
}
template <typename T, int LOGN, int XC>
__device__ __forceinline__ void inverse(c2<T>* __restrict__ s, const c2<T>* __restrict__ sq, const TwTables& tw) {
  if constexpr (Geo<T, LOGN, XC>::C > 1) combine_inv<T, LOGN, XC>(s, tw);
  local_fft<T, LOGN, XC, true>(s, sq);
}

}  // namespace mmp
