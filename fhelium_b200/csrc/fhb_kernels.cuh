// CKKS evaluation kernels for sm_100a (device code).
//
// Residue tensors are the reference layout: contiguous [*batch, limb, N]
// with limb j belonging to prime id (row_start + j) of the level-zero chain
// [Q | P] (fhelium/core/ciphertext.py:26-67).  A ciphertext component at
// level l holds prime ids [l, num_q); its Q+P extension holds [l, num_q+num_p).
#pragma once
#include "fhb_context.h"
#include "fhb_ntt.cuh"

namespace fhb {

enum InverseOut : int { kInvMontgomery = 0, kInvStandardLazy = 1, kInvStandard = 2, kInvCentered = 3 };

// ---- thread-contiguous vector access (E residues per thread) ----------------------------
template <typename T, int E>
__device__ __forceinline__ void load16(const T* p, T (&v)[E]) {
  if constexpr (sizeof(T) == 8) {
    const ulonglong2* q = reinterpret_cast<const ulonglong2*>(p);
#pragma unroll
    for (int i = 0; i < E / 2; ++i) {
      const ulonglong2 x = q[i];
      v[2 * i] = x.x;
      v[2 * i + 1] = x.y;
    }
  } else {
    const uint4* q = reinterpret_cast<const uint4*>(p);
#pragma unroll
    for (int i = 0; i < E / 4; ++i) {
      const uint4 x = q[i];
      v[4 * i] = x.x; v[4 * i + 1] = x.y; v[4 * i + 2] = x.z; v[4 * i + 3] = x.w;
    }
  }
}
template <typename T, int E>
__device__ __forceinline__ void store16(T* p, const T (&v)[E]) {
  if constexpr (sizeof(T) == 8) {
    ulonglong2* q = reinterpret_cast<ulonglong2*>(p);
#pragma unroll
    for (int i = 0; i < E / 2; ++i) q[i] = make_ulonglong2(v[2 * i], v[2 * i + 1]);
  } else {
    uint4* q = reinterpret_cast<uint4*>(p);
#pragma unroll
    for (int i = 0; i < E / 4; ++i) q[i] = make_uint4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
  }
}

template <typename T, int LOGN>
__device__ __forceinline__ int cluster_rank() {
  if constexpr (NttGeom<T, LOGN>::kC > 1) return int(cg::this_cluster().block_rank());
  return 0;
}

// ---------------------------------------------------------------------------
// Plain forward NTT: standard -> NTT/Montgomery (x R) or Montgomery -> NTT.
// Output lazy [0, 2q) as in csrc/ops/ntt/forward_ntt.cpp:19-22.
// Source of a plain forward transform: the input row, optionally taken to
// Montgomery form on the fly.  Plain loads: `in` may alias the output.
template <typename T, bool TO_MONT>
struct RowSource {
  const T* in;
  T c, cs, q;
  template <int C>
  __device__ __forceinline__ void column(int m, int stride, T (&x)[C]) const {
#pragma unroll
    for (int k = 0; k < C; ++k) {
      T v = in[k * stride + m];
      if constexpr (TO_MONT) v = Word<T>::shoup(v, c, cs, q);
      x[k] = v;
    }
  }
};

// FP64 forms of the transforms for the rows of primes below 2^42: residues
// as exact integers in doubles, Word<double> products on the FP64 pipe,
// 64-bit words in memory, converted on load and store.
template <bool TO_MONT>
struct U64MontSource {
  const uint64_t* in;
  double c, cs, q;
  template <int C>
  __device__ __forceinline__ void column(int m, int stride, double (&x)[C]) const {
#pragma unroll
    for (int k = 0; k < C; ++k) {
      double v = __ull2double_rn(in[k * stride + m]);
      if constexpr (TO_MONT) v = Word<double>::shoup(v, c, cs, q);
      x[k] = v;
    }
  }
};

template <int E>
__device__ __forceinline__ void store_words(uint64_t* p, const double (&v)[E]) {
  uint64_t w[E];
#pragma unroll
  for (int e = 0; e < E; ++e) w[e] = __double2ull_rz(v[e]);
  store16(p, w);
}

struct F64OutEpilogue {
  uint64_t* dst;
  double q, c, cs;
  int kind;
  __device__ __forceinline__ void operator()(int pos, double v) const {
    v = Word<double>::shoup(v, c, cs, q);  // [0, 2q)
    if (kind >= kInvStandard) v = csub(v, q);
    if (kind == kInvCentered && v > floor(0.5 * q)) {
      dst[pos] = uint64_t(__double2ll_rz(v - q));
      return;
    }
    dst[pos] = __double2ull_rz(v);
  }
};

// Plain forward NTT of `rows`-row groups of polynomials, one cluster per
// polynomial.  SPLIT (int64 chains with FP64 tables): the leading f64_rows
// rows of every group, whose primes are below 2^42, run the transform in
// FP64 arithmetic in the same launch (a cluster-uniform branch); their lazy
// outputs equal the integer transform's modulo q.
template <typename T, int LOGN, bool TO_MONT, int EPT = 0, bool SPLIT = false>
__global__ void __launch_bounds__(NttGeom<T, LOGN, EPT>::kThreads)
k_ntt_forward(const T* __restrict__ in, T* __restrict__ out, int rows, int row_start, ChainTables<T> tabs,
              ChainTables<double> tabs64f, int f64_rows) {
  using G = NttGeom<T, LOGN, EPT>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int rank = cluster_rank<T, LOGN>();
  const int64_t poly = blockIdx.x / G::kC;
  const int row = int(poly % rows), pid = row_start + row;
  T* dst = out + poly * G::kN + int64_t(rank) * G::kM + threadIdx.x * G::kE;
  if constexpr (SPLIT) {
    static_assert(sizeof(T) == 8, "FP64 rows exist in int64 chains only");
    if (row < f64_rows) {
      const PrimeInfo<double> p = tabs64f.prime[pid];
      U64MontSource<TO_MONT> src{reinterpret_cast<const uint64_t*>(in) + poly * G::kN, p.rmod, p.rmod_s, p.q};
      double v[G::kE];
      Ntt<double, LOGN, TwGlobalQ<LOGN>, EPT>::forward_from(
          src, reinterpret_cast<double*>(smem_raw), TwGlobalQ<LOGN>{tabs64f.twv_fwd + int64_t(pid) * G::kN, p.one_s},
          p.q, p.one_s, rank, v);
#pragma unroll
      for (int e = 0; e < G::kE; ++e) v[e] = Word<double>::to_lazy(v[e], p.q, p.one_s);
      store_words(reinterpret_cast<uint64_t*>(dst), v);
      return;
    }
  }
  const PrimeInfo<T> p = tabs.prime[pid];
  RowSource<T, TO_MONT> src{in + poly * G::kN, p.rmod, p.rmod_s, p.q};
  T v[G::kE];
  Ntt<T, LOGN, TwGlobal<T, LOGN>, EPT>::forward_from(src, reinterpret_cast<T*>(smem_raw),
                                                     tabs.tw_fwd + int64_t(pid) * G::kN, p.q, p.twice_q, rank, v);
#pragma unroll
  for (int e = 0; e < G::kE; ++e) v[e] = csub(v[e], p.twice_q);
  store16(dst, v);
}

template <typename T>
struct InvEpilogue {
  T* dst;
  T q;
  T c, cs;
  int kind;
  __device__ __forceinline__ void operator()(int pos, T v) const {
    v = Word<T>::shoup(v, c, cs, q);  // [0, 2q)
    if (kind >= kInvStandard) v = csub(v, q);
    if (kind == kInvCentered) v = v <= (q >> 1) ? v : v - q;
    dst[pos] = v;
  }
};

template <typename T>
__device__ __forceinline__ InvEpilogue<T> make_inv_epilogue(T* dst, const PrimeInfo<T>& p, int kind,
                                                            bool montgomery_input) {
  InvEpilogue<T> e{dst, p.q, p.ninv, p.ninv_s, kind};
  if (kind != kInvMontgomery && montgomery_input) {
    e.c = p.ninv_rinv;
    e.cs = p.ninv_rinv_s;
  }
  return e;
}

// Plain inverse NTT from NTT/Montgomery lazy input.  SPLIT: the leading
// f64_rows rows of every group in FP64 arithmetic, the same output words.
template <typename T, int LOGN, int EPT = 0, bool SPLIT = false>
__global__ void __launch_bounds__(NttGeom<T, LOGN, EPT>::kThreads)
k_ntt_inverse(const T* __restrict__ in, T* __restrict__ out, int rows, int row_start, int kind, ChainTables<T> tabs,
              ChainTables<double> tabs64f, int f64_rows) {
  using G = NttGeom<T, LOGN, EPT>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int rank = cluster_rank<T, LOGN>();
  const int64_t poly = blockIdx.x / G::kC;
  const int row = int(poly % rows), pid = row_start + row;
  T w[G::kE];
  load16(in + poly * G::kN + int64_t(rank) * G::kM + threadIdx.x * G::kE, w);
  if constexpr (SPLIT) {
    static_assert(sizeof(T) == 8, "FP64 rows exist in int64 chains only");
    if (row < f64_rows) {
      const PrimeInfo<double> p = tabs64f.prime[pid];
      double v[G::kE];
#pragma unroll
      for (int e = 0; e < G::kE; ++e) v[e] = __ull2double_rn(w[e]);
      const bool std_out = kind != kInvMontgomery;  // N^-1 R^-1 unless the output stays Montgomery
      F64OutEpilogue epi{reinterpret_cast<uint64_t*>(out) + poly * G::kN, p.q, std_out ? p.ninv_rinv : p.ninv,
                         std_out ? p.ninv_rinv_s : p.ninv_s, kind};
      Ntt<double, LOGN, TwGlobalQ<LOGN>, EPT>::inverse(reinterpret_cast<double*>(smem_raw),
                                                       TwGlobalQ<LOGN>{tabs64f.twv_inv + int64_t(pid) * G::kN, p.one_s},
                                                       p.q, p.one_s, rank, v, epi);
      return;
    }
  }
  const PrimeInfo<T> p = tabs.prime[pid];
  InvEpilogue<T> epi = make_inv_epilogue<T>(out + poly * G::kN, p, kind, true);
  Ntt<T, LOGN, TwGlobal<T, LOGN>, EPT>::inverse(reinterpret_cast<T*>(smem_raw), tabs.tw_inv + int64_t(pid) * G::kN,
                                                p.q, p.twice_q, rank, w, epi);
}

// ---------------------------------------------------------------------------
// Fused tensor product + inverse NTT.
// a, b: [2, B, L, N] NTT/Montgomery lazy; out: [3, B, L, N] coefficient/standard
// canonical = INTT of (a0 b0, a0 b1 + a1 b0, a1 b1)
// (fhelium/engine/ckks_engine.py:1570-1606 then :1655-1660).
template <typename T, int LOGN, int EPT = 0>
__global__ void __launch_bounds__(NttGeom<T, LOGN, EPT>::kThreads)
k_mul_to_coefficient(const T* __restrict__ a, const T* __restrict__ b, T* __restrict__ out,
                     int64_t batch, int limbs, int level, ChainTables<T> tabs) {
  using G = NttGeom<T, LOGN, EPT>;
  using W = Word<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* s = reinterpret_cast<T*>(smem_raw);
  const int rank = cluster_rank<T, LOGN>();
  const int64_t poly = blockIdx.x / G::kC;  // over [3, B, L]
  const int64_t comp_stride = batch * limbs * G::kN;
  const int comp = int(poly / (batch * limbs));
  const int64_t rest = poly % (batch * limbs);
  const int pid = level + int(rest % limbs);
  const PrimeInfo<T> p = tabs.prime[pid];
  const int64_t off = rest * G::kN + int64_t(rank) * G::kM + threadIdx.x * G::kE;
  T v[G::kE], x[G::kE], y[G::kE];
  const T* a0 = a + off;
  const T* a1 = a + comp_stride + off;
  const T* b0 = b + off;
  const T* b1 = b + comp_stride + off;
  load16(comp == 2 ? a1 : a0, x);
  load16(comp == 0 ? b0 : b1, y);
#pragma unroll
  for (int e = 0; e < G::kE; ++e) v[e] = W::mont(x[e], y[e], p.q, p.neg_inv);
  if (comp == 1) {
    load16(a1, x);
    load16(b0, y);
#pragma unroll
    for (int e = 0; e < G::kE; ++e) v[e] = csub(v[e] + W::mont(x[e], y[e], p.q, p.neg_inv), p.twice_q);
  }
  InvEpilogue<T> epi = make_inv_epilogue<T>(out + comp * comp_stride + rest * G::kN, p, kInvStandard, true);
  Ntt<T, LOGN, TwGlobal<T, LOGN>, EPT>::inverse(s, tabs.tw_inv + int64_t(pid) * G::kN, p.q, p.twice_q, rank, v,
                                                epi);
}

// Element-wise kernels over [batch, rows, N]: each thread owns V consecutive
// coefficients of one row (16-byte loads and stores when V > 1) and walks the
// batch items of its z-slice, so the row's constants and the index arithmetic
// are paid once per thread.  Grid: (N / (256 V), rows, z-slices).
constexpr int kEwThreads = 256;

template <typename T, int V>
struct alignas(V * sizeof(T) >= 16 ? 16 : sizeof(T)) EwVec {
  T v[V];
};

template <typename T, int V>
__device__ __forceinline__ EwVec<T, V> ew_load(const T* p) {
  EwVec<T, V> r;
  if constexpr (V * sizeof(T) == 16) {
    *reinterpret_cast<uint4*>(r.v) = *reinterpret_cast<const uint4*>(p);
  } else {
#pragma unroll
    for (int i = 0; i < V; ++i) r.v[i] = p[i];
  }
  return r;
}

template <typename T, int V>
__device__ __forceinline__ void ew_store(T* p, const EwVec<T, V>& r) {
  if constexpr (V * sizeof(T) == 16) {
    *reinterpret_cast<uint4*>(p) = *reinterpret_cast<const uint4*>(r.v);
  } else {
#pragma unroll
    for (int i = 0; i < V; ++i) p[i] = r.v[i];
  }
}

// NTT-domain tensor product only (reference multiply): out [3, B, L, N] lazy.
template <typename T, int V>
__global__ void k_mul_ntt(const T* __restrict__ a, const T* __restrict__ b, T* __restrict__ out,
                          int64_t batch, int limbs, int log_n, int level, ChainTables<T> tabs, int64_t in_pitch,
                          int64_t out_pitch) {
  const int64_t n = int64_t(1) << log_n;
  const int64_t k = (int64_t(blockIdx.x) * kEwThreads + threadIdx.x) * V;
  if (k >= n) return;
  const int row = blockIdx.y;
  const PrimeInfo<T>& pp = tabs.prime[level + row];
  const T q = pp.q, ni = pp.neg_inv, tq = pp.twice_q;
  for (int64_t bi = blockIdx.z; bi < batch; bi += gridDim.z) {
    const int64_t i = (bi * limbs + row) * n + k;
    const EwVec<T, V> x0 = ew_load<T, V>(a + i), x1 = ew_load<T, V>(a + in_pitch + i);
    const EwVec<T, V> y0 = ew_load<T, V>(b + i), y1 = ew_load<T, V>(b + in_pitch + i);
    EwVec<T, V> d0, d1, d2;
#pragma unroll
    for (int e = 0; e < V; ++e) {
      d0.v[e] = Word<T>::mont(x0.v[e], y0.v[e], q, ni);
      d1.v[e] = csub(Word<T>::mont(x0.v[e], y1.v[e], q, ni) + Word<T>::mont(x1.v[e], y0.v[e], q, ni), tq);
      d2.v[e] = Word<T>::mont(x1.v[e], y1.v[e], q, ni);
    }
    ew_store<T, V>(out + i, d0);
    ew_store<T, V>(out + out_pitch + i, d1);
    ew_store<T, V>(out + 2 * out_pitch + i, d2);
  }
}

// ---------------------------------------------------------------------------
// Galois automorphism sigma_g on a coefficient-domain residue: destination j
// reads source (j g^{-1} mod 2N) with a sign flip when that index >= N
// (fhelium/engine/galois.py:49-83, derived in-kernel, no gather table).
__device__ __forceinline__ int galois_source(int j, int log_n, uint32_t ginv, bool& negate) {
  const uint64_t two_n_mask = (uint64_t{2} << log_n) - 1;
  const uint32_t i = uint32_t((uint64_t(j) * ginv) & two_n_mask);
  negate = i >> log_n;
  return int(i & ((1u << log_n) - 1));
}

// Inverse of an odd Galois element modulo 2N (Newton iteration mod 2^32).
__device__ __forceinline__ uint32_t galois_inverse_dev(uint32_t g, int log_n) {
  uint32_t x = 1;
#pragma unroll
  for (int i = 0; i < 5; ++i) x *= 2u - g * x;
  return x & ((2u << log_n) - 1);
}

// NTT-domain automorphism gather (bit-reversed evaluation order):
// destination k reads br(((2 br(k) + 1) g mod 2N - 1) / 2)
// (fhelium/engine/hybrid_keyswitch.py:506-528).
__device__ __forceinline__ int galois_ntt_source(int k, int log_n, uint32_t g) {
  const uint32_t br = __brev(uint32_t(k)) >> (32 - log_n);
  const uint32_t e = uint32_t((uint64_t(2 * br + 1) * g) & ((uint64_t{2} << log_n) - 1));
  return int(__brev((e - 1) >> 1) >> (32 - log_n));
}

// ---------------------------------------------------------------------------
// ModUp stage 1: Garner mixed-radix digits of every active hybrid digit
// (fhelium/engine/hybrid_keyswitch.py:95-170, exact same digits as
// csrc/ops/rns/cpu/rns_arithmetic_cpu.cpp:482-615).  comp: [B, L, N]
// coefficient/standard (canonical or lazy [0, 2q)); digits: [B, L, N],
// row r holds the mixed-radix digit of the prime in row r.  When ginv != 0
// the input is first mapped through sigma_g (rotation).
template <typename T, int V>
__global__ void k_modup_digits(const T* __restrict__ comp, T* __restrict__ digits, int64_t batch,
                               int limbs, int log_n, int level, uint32_t ginv,
                               const uint32_t* __restrict__ item_galois, ChainTables<T> tabs, LevelTables<T> lt) {
  // grid: (N / (256 V), digit, z-slices of the batch); V coefficients per thread
  const int64_t n = int64_t(1) << log_n;
  const int64_t k0 = (int64_t(blockIdx.x) * kEwThreads + threadIdx.x) * V;
  if (k0 >= n) return;
  using W = Word<T>;
  const DigitDesc d = lt.digits[blockIdx.y];
  const TwPair<T>* g = lt.garner + blockIdx.y * kMaxDigitWidth * kMaxDigitWidth;
  for (int64_t bi = blockIdx.z; bi < batch; bi += gridDim.z) {
    // per-item Galois elements (mixed-step rotation batches) override ginv
    const uint32_t gi = item_galois ? (item_galois[bi] == 1 ? 0u : galois_inverse_dev(item_galois[bi], log_n)) : ginv;
    const T* src = comp + bi * limbs * n;
    T* dst = digits + bi * limbs * n;
    EwVec<T, V> dig[kMaxDigitWidth];
    for (int r = 0; r < d.alpha; ++r) {
      const int row = d.prime0 - level + r;
      const T q = tabs.prime[d.prime0 + r].q;
      EwVec<T, V> x;
      if (gi == 0) {
        x = ew_load<T, V>(src + row * n + k0);
#pragma unroll
        for (int e = 0; e < V; ++e) x.v[e] = csub(x.v[e], q);
      } else {
#pragma unroll
        for (int e = 0; e < V; ++e) {
          bool neg = false;
          const int srck = galois_source(int(k0) + e, log_n, gi, neg);
          T y = csub(src[row * n + srck], q);
          x.v[e] = (neg && y) ? q - y : y;
        }
      }
      if (r > 0) {
        const TwPair<T> inv = g[r * kMaxDigitWidth + r];
#pragma unroll
        for (int e = 0; e < V; ++e) {
          T acc = 0;
          for (int i = 0; i < r; ++i) {
            const TwPair<T> c = g[r * kMaxDigitWidth + i];
            acc = csub(acc + csub(W::shoup(dig[i].v[e], c.w, c.wp, q), q), q);
          }
          x.v[e] = csub(W::shoup(csub(x.v[e] + q - acc, q), inv.w, inv.wp, q), q);
        }
      }
      dig[r] = x;
      ew_store<T, V>(dst + row * n + k0, x);
    }
  }
}

// ---------------------------------------------------------------------------
// Twiddle placement for kernels that transform several polynomials of one
// prime (key switching): the CTA's forward (then inverse) twiddles are staged
// once into shared memory when they fit next to the NTT working block.
#ifndef FHB_TW_SMEM
#define FHB_TW_SMEM 0
#endif
template <typename T, int LOGN>
struct KsTw {
  using G = NttGeom<T, LOGN>;
  static constexpr size_t kData = size_t(G::kSmemElems) * sizeof(T);
  static constexpr size_t kTwBytes = size_t(G::kM) * sizeof(TwPair<T>);
  static constexpr bool kShared = FHB_TW_SMEM && kData + kTwBytes <= 227 * 1024;
  const TwPair<T>* gf;
  const TwPair<T>* gi;
  TwPair<T>* st;
  int rank;
  __device__ __forceinline__ KsTw(unsigned char* smem, const TwPair<T>* fwd_row, const TwPair<T>* inv_row, int r)
      : gf(fwd_row), gi(inv_row), st(reinterpret_cast<TwPair<T>*>(smem + kData)), rank(r) {}
  __device__ __forceinline__ void stage(bool inverse) {
    if constexpr (kShared) {
      __syncthreads();
      TwShared<T, LOGN>::stage(st, inverse ? gi : gf, rank, inverse);
      __syncthreads();
    }
  }
  // the transforms' second modulus argument: 2q, or 1/q for the balanced FP64 rows
  __device__ __forceinline__ static T m2(const PrimeInfo<T>& p) {
    if constexpr (std::is_same<T, double>::value) {
      return p.one_s;
    } else {
      return p.twice_q;
    }
  }
  template <class Src>
  __device__ __forceinline__ void forward_from(Src& src, T* data, const PrimeInfo<T>& p, T (&v)[G::kE]) const {
    if constexpr (kShared) {
      Ntt<T, LOGN, TwShared<T, LOGN>>::forward_from(src, data, TwShared<T, LOGN>{gf, st, rank * G::kM}, p.q, m2(p),
                                                    rank, v);
    } else {
      Ntt<T, LOGN>::forward_from(src, data, TwGlobal<T, LOGN>(gf), p.q, m2(p), rank, v);
    }
  }
  template <class Epi>
  __device__ __forceinline__ void inverse(T* data, const PrimeInfo<T>& p, const T (&v)[G::kE], Epi& epi) const {
    if constexpr (kShared) {
      Ntt<T, LOGN, TwShared<T, LOGN>>::inverse(data, TwShared<T, LOGN>{gi, st, rank * G::kM}, p.q, m2(p), rank, v,
                                               epi);
    } else {
      Ntt<T, LOGN>::inverse(data, TwGlobal<T, LOGN>(gi), p.q, m2(p), rank, v, epi);
    }
  }
};

// Key-switch accumulators of one thread: 2 x 16 residues kept in shared
// memory ([element][thread], conflict-free) when the CTA has room next to the
// NTT working block (and the twiddles are not staged there), otherwise in the
// thread's own slots of the output rows.
template <typename T, int LOGN>
struct KsAcc {
  using G = NttGeom<T, LOGN>;
#ifndef FHB_KS_ACC_SMEM
#define FHB_KS_ACC_SMEM 1
#endif
  static constexpr bool kSmem = FHB_KS_ACC_SMEM && !KsTw<T, LOGN>::kShared &&
                                (G::kSmemElems + 2 * G::kM) * sizeof(T) <= 200 * 1024;
  static constexpr size_t smem_bytes() {
    return KsTw<T, LOGN>::kShared ? KsTw<T, LOGN>::kData + KsTw<T, LOGN>::kTwBytes
                                  : (G::kSmemElems + (kSmem ? 2 * G::kM : 0)) * sizeof(T);
  }
  T* c0;
  T* c1;
  int stride;
  __device__ __forceinline__ KsAcc(T* s, T* g0, T* g1) {
    if constexpr (kSmem) {
      c0 = s + G::kSmemElems + threadIdx.x;
      c1 = c0 + G::kM;
      stride = G::kThreads;
    } else {
      c0 = g0;
      c1 = g1;
      stride = 1;
    }
#pragma unroll
    for (int e = 0; e < G::kE; ++e) c0[e * stride] = c1[e * stride] = 0;
  }
  __device__ __forceinline__ void mac(int e, T x, T k0, T k1, const PrimeInfo<T>& p) {
    c0[e * stride] = csub(c0[e * stride] + Word<T>::mont(x, k0, p.q, p.neg_inv), p.twice_q);
    c1[e * stride] = csub(c1[e * stride] + Word<T>::mont(x, k1, p.q, p.neg_inv), p.twice_q);
  }
  // FP64 form (T = double, balanced): forward outputs |x| < 20 q times key
  // words below 2q, quotient from 1/q; each term in (-0.6 q, 0.6 q), summed
  // without reduction (the sum is reduced once before the inverse transform)
  __device__ __forceinline__ void mac_f64(int e, T x, T k0, T k1, T q, T qinv) {
    c0[e * stride] += Word<T>::mul_qinv_bal(x, k0, q, qinv);
    c1[e * stride] += Word<T>::mul_qinv_bal(x, k1, q, qinv);
  }
  __device__ __forceinline__ void get(int which, T (&v)[G::kE]) const {
    const T* c = which ? c1 : c0;
#pragma unroll
    for (int e = 0; e < G::kE; ++e) v[e] = c[e * stride];
  }
};

// Exact basis extension of one hybrid digit to destination prime p, as the
// source of the forward transform: sum_r d_r (M_r mod p), lazy [0, 2p).
// dig: the digit's first mixed-radix row of this ciphertext; ext: the
// extension constants of the digit for prime p (entry r at ext[r * qp0]).
template <typename T>
struct ExtSource {
  const T* dig;
  const TwPair<T>* ext;
  int qp0, alpha, log_n;
  T q, twice_q;
  // x[k] = extension of the digit at position k * stride + m; the digit's
  // rows are the outer loop so each constant is loaded once per column.
  template <int C>
  __device__ __forceinline__ void column(int m, int stride, T (&x)[C]) const {
#pragma unroll
    for (int k = 0; k < C; ++k) x[k] = 0;
    for (int r = 0; r < alpha; ++r) {
      const TwPair<T> c = ext[int64_t(r) * qp0];
      const T* row = dig + (int64_t(r) << log_n) + m;
#pragma unroll
      for (int k = 0; k < C; ++k) x[k] = csub(x[k] + Word<T>::shoup(row[k * stride], c.w, c.wp, q), twice_q);
    }
  }
};

// Work order of the per-(ciphertext, row) clusters of the key-switch kernels:
// order 0 runs the rows of one ciphertext back to back; order 1 runs row j of
// every ciphertext back to back, so concurrently resident clusters read the
// same key rows; order 2 runs row j of a group of kKsGroup ciphertexts back
// to back, group by group, so both the key rows of j (shared by the group)
// and the group's digit rows (read for every destination row) stay in L2
// (chosen by the autotuner).
constexpr int kKsGroup = 4;
__device__ __forceinline__ void ks_work(int64_t cluster, int qp_limbs, int64_t batch, int order, int64_t& poly,
                                        int64_t& bi, int& jrow) {
  if (order == 0) {
    poly = cluster;
    bi = poly / qp_limbs;
    jrow = int(poly % qp_limbs);
  } else if (order == 1) {
    jrow = int(cluster / batch);
    bi = cluster % batch;
    poly = bi * qp_limbs + jrow;
  } else {
    const int64_t full = batch - batch % kKsGroup;  // ciphertexts in whole groups
    if (cluster < full * qp_limbs) {
      const int64_t g = cluster / (int64_t(qp_limbs) * kKsGroup), r = cluster % (int64_t(qp_limbs) * kKsGroup);
      jrow = int(r / kKsGroup);
      bi = g * kKsGroup + r % kKsGroup;
    } else {
      const int64_t c2 = cluster - full * qp_limbs, rest = batch - full;
      jrow = int(c2 / rest);
      bi = full + c2 % rest;
    }
    poly = bi * qp_limbs + jrow;
  }
}

// acc += v * key (both key components), streaming the key rows in 16-byte
// pieces so that only two key words per component are live at a time.
template <typename T, class Acc, int E>
__device__ __forceinline__ void key_mac(Acc& acc, const T (&v)[E], const T* key0, const T* key1,
                                        const PrimeInfo<T>& p) {
  if constexpr (sizeof(T) == 8) {
#pragma unroll
    for (int i = 0; i < E / 2; ++i) {
      const ulonglong2 a = __ldg(reinterpret_cast<const ulonglong2*>(key0) + i);
      const ulonglong2 b = __ldg(reinterpret_cast<const ulonglong2*>(key1) + i);
      acc.mac(2 * i, csub(v[2 * i], p.twice_q), a.x, b.x, p);
      acc.mac(2 * i + 1, csub(v[2 * i + 1], p.twice_q), a.y, b.y, p);
    }
  } else {
#pragma unroll
    for (int i = 0; i < E / 4; ++i) {
      const uint4 a = __ldg(reinterpret_cast<const uint4*>(key0) + i);
      const uint4 b = __ldg(reinterpret_cast<const uint4*>(key1) + i);
      acc.mac(4 * i, csub(v[4 * i], p.twice_q), a.x, b.x, p);
      acc.mac(4 * i + 1, csub(v[4 * i + 1], p.twice_q), a.y, b.y, p);
      acc.mac(4 * i + 2, csub(v[4 * i + 2], p.twice_q), a.z, b.z, p);
      acc.mac(4 * i + 3, csub(v[4 * i + 3], p.twice_q), a.w, b.w, p);
    }
  }
}

// Relinearisation of an NTT-domain ct3 = (c0, c1, c2): for a Q row the
// addends c0, c1 are folded into the key-switch accumulators before their
// inverse NTT, as P c_k, so that ModDown returns KS(c2) + c_k directly
// ((t + P c - [t]_P) / P = (t - [t]_P) / P + c).  c_k is in Montgomery form
// (c R) and P R^{-1} mod q is the Shoup constant.  ct3 points at this
// thread's first element of component 0; comp_stride is the component pitch.
template <typename T, int E>
__device__ __forceinline__ void ks_add_p_scaled(T (&v)[E], int which, const T* ct3, int64_t comp_stride,
                                                const PrimeInfo<T>& p, TwPair<T> ps) {
  using W = Word<T>;
#pragma unroll
  for (int e = 0; e < E; ++e) v[e] = csub(v[e] + W::shoup(ct3[which * comp_stride + e], ps.w, ps.wp, p.q), p.twice_q);
}

// For a Q row that belongs to the digit being processed, the exact extension
// of the digit is c2 itself (modulo that row's prime), so its forward NTT is
// c2's NTT-domain residue: v = c2 R * R^{-1}, standard form, [0, 2q).
template <typename T, int E>
__device__ __forceinline__ void ks_own_digit_ntt(T (&v)[E], const T* ct3, int64_t comp_stride,
                                                 const PrimeInfo<T>& p) {
#pragma unroll
  for (int e = 0; e < E; ++e) v[e] = Word<T>::shoup(ct3[2 * comp_stride + e], p.rinv, p.rinv_s, p.q);
}

// ---------------------------------------------------------------------------
// Fused ModUp stage 2 + forward NTT + key inner product + inverse NTT.
// One cluster per (ciphertext b, destination row j of Q_l P).  For every
// active digit: extend the mixed-radix digits to prime p_j exactly
// (sum_r d_r M_r mod p_j), transform, multiply by the key digit row and
// accumulate; finally inverse-transform both accumulators to
// coefficient/standard canonical rows.  Equals, modulo p_j, the reference's
// per-digit basis extension + forward NTT + keyswitch_accumulate + the
// inverse NTT at the start of ModDown (fhelium/engine/hybrid_keyswitch.py:
// 321-371, 530-546).  key: [D, 2, QP0, N] NTT/Montgomery level-zero rows.
// acc0/acc1: [B, QP_l, N]; they double as accumulation scratch.
// PRE (tensor-core form): `digits` holds the extensions already computed by
// the int8 tensor-core basis conversion, [D_l][B][QP_l][N] in [0, 2p), so
// the source of each forward NTT is a plain row read instead of the
// extension sum.
// One unit (ciphertext bi, row jrow of Q_l P) of the key-switch core.
template <typename T, int LOGN, bool PRE>
__device__ __forceinline__ void ks_core_unit(const T* __restrict__ digits, const T* __restrict__ key,
                                             T* __restrict__ acc0, T* __restrict__ acc1, int64_t batch, int q_limbs,
                                             int qp_limbs, int level, int qp0, const T* __restrict__ ct3,
                                             int64_t ct3_stride, const ChainTables<T>& tabs, const LevelTables<T>& lt,
                                             int64_t bi, int jrow, unsigned char* smem_raw, int rank) {
  using G = NttGeom<T, LOGN>;
  T* s = reinterpret_cast<T*>(smem_raw);
  const int64_t poly = bi * qp_limbs + jrow;
  const int pid = level + jrow;
  const PrimeInfo<T> p = tabs.prime[pid];
  const TwPair<T>* twf = tabs.tw_fwd + int64_t(pid) * G::kN;
  const T* dig = digits + bi * q_limbs * int64_t(G::kN);
  const int64_t own = int64_t(rank) * G::kM + threadIdx.x * G::kE;
  KsAcc<T, LOGN> acc(s, acc0 + poly * G::kN + own, acc1 + poly * G::kN + own);
  KsTw<T, LOGN> tw(smem_raw, twf, tabs.tw_inv + int64_t(pid) * G::kN, rank);
  tw.stage(false);
  const bool add = ct3 != nullptr && jrow < q_limbs;
  const T* ct3_own = add ? ct3 + (bi * q_limbs + jrow) * int64_t(G::kN) + own : nullptr;
  for (int a = 0; a < lt.num_digits; ++a) {
    const DigitDesc d = lt.digits[a];
    const T* key0 = key + ((int64_t(d.key_digit) * 2 + 0) * qp0 + pid) * G::kN + own;
    const T* key1 = key + ((int64_t(d.key_digit) * 2 + 1) * qp0 + pid) * G::kN + own;
    T v[G::kE];
    if (add && pid >= d.prime0 && pid < d.prime0 + d.alpha) {
      // uniform over the cluster: skipping the transform skips its barriers everywhere
      ks_own_digit_ntt(v, ct3_own, ct3_stride, p);
    } else if constexpr (PRE) {
      RowSource<T, false> src{digits + ((int64_t(a) * batch + bi) * qp_limbs + jrow) * G::kN, 0, 0, p.q};
      tw.forward_from(src, s, p, v);
    } else {
      ExtSource<T> src{dig + (int64_t(d.prime0 - level) << LOGN), lt.ext + int64_t(a) * kMaxDigitWidth * qp0 + pid,
                       qp0, d.alpha, LOGN, p.q, p.twice_q};
      tw.forward_from(src, s, p, v);
    }
    key_mac(acc, v, key0, key1, p);
  }
  tw.stage(true);
  T v[G::kE];
  acc.get(0, v);
  if (add) ks_add_p_scaled(v, 0, ct3_own, ct3_stride, p, tabs.p_rinv[pid]);
  InvEpilogue<T> e0 = make_inv_epilogue<T>(acc0 + poly * G::kN, p, kInvStandard, false);
  tw.inverse(s, p, v, e0);
  acc.get(1, v);
  if (add) ks_add_p_scaled(v, 1, ct3_own, ct3_stride, p, tabs.p_rinv[pid]);
  InvEpilogue<T> e1 = make_inv_epilogue<T>(acc1 + poly * G::kN, p, kInvStandard, false);
  tw.inverse(s, p, v, e1);
}

template <typename T, int LOGN, bool PRE = false>
__global__ void __launch_bounds__(NttGeom<T, LOGN>::kThreads)
k_keyswitch_core(const T* __restrict__ digits, const T* __restrict__ key, T* __restrict__ acc0,
                 T* __restrict__ acc1, int64_t batch, int q_limbs, int qp_limbs, int level, int qp0, int order,
                 const unsigned long long* __restrict__ item_keys, const T* __restrict__ ct3, int64_t ct3_stride,
                 ChainTables<T> tabs, LevelTables<T> lt) {
  using G = NttGeom<T, LOGN>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  int64_t poly, bi;
  int jrow;
  ks_work(blockIdx.x / G::kC, qp_limbs, batch, order, poly, bi, jrow);
  if (item_keys) key = reinterpret_cast<const T*>(item_keys[bi]);  // mixed-key batch
  ks_core_unit<T, LOGN, PRE>(digits, key, acc0, acc1, batch, q_limbs, qp_limbs, level, qp0, ct3, ct3_stride, tabs,
                             lt, bi, jrow, smem_raw, cluster_rank<T, LOGN>());
}

// ---------------------------------------------------------------------------
// The key-switch core's rows whose primes are below 2^42, in FP64
// arithmetic (int64 chains, rings up to N = 2^16 so the accumulators live in
// shared memory).  Residues are held as exact integers in doubles and every
// product is Word<double>'s exact product, so the butterflies run on the
// FP64 pipe instead of the integer multiply-add pipe; inputs and outputs
// stay 64-bit words in global memory, converted on load and store.  The key
// words are used as stored (k R, the Montgomery form), so the accumulators
// carry a factor R, removed with N^{-1} R^{-1} in the inverse transform's
// epilogue; for relinearisation the addends enter as P c R (ct3 holds c R,
// tabs.p_rinv holds P mod q in the FP64 tables) and an own-digit row as
// c2 = (c2 R) R^{-1}.  The outputs are the integer core's words.
struct U64RowSource {
  const uint64_t* in;
  template <int C>
  __device__ __forceinline__ void column(int m, int stride, double (&x)[C]) const {
#pragma unroll
    for (int k = 0; k < C; ++k) x[k] = __ull2double_rn(in[k * stride + m]);
  }
};

// Exact extension of one digit to prime p in FP64 (the CUDA-core form's
// source of the forward transform): sum_r d_r (M_r mod p), balanced: every
// term reduced to (-0.6 p, 0.6 p) and summed unreduced (16 terms at most,
// below 9.6 p).  Digit words below 2^42 enter whole; a digit that holds a
// wider prime has its words split into 30-bit halves against
// (M_r mod p) 2^30 and M_r mod p.
struct ExtSourceF64 {
  const uint64_t* dig;        // the digit's first mixed-radix row of this ciphertext
  const TwPair<double>* ext;  // [r][2][qp0] of this digit, offset by the destination prime id
  int qp0, alpha, log_n;
  bool wide;
  double q, twice_q;
  template <int C>
  __device__ __forceinline__ void column(int m, int stride, double (&x)[C]) const {
    using W = Word<double>;
#pragma unroll
    for (int k = 0; k < C; ++k) x[k] = 0.0;
    for (int r = 0; r < alpha; ++r) {
      const TwPair<double> lo = ext[int64_t(r * 2 + 1) * qp0];
      const uint64_t* row = dig + (int64_t(r) << log_n) + m;
      if (wide) {
        const TwPair<double> hi = ext[int64_t(r * 2) * qp0];
#pragma unroll
        for (int k = 0; k < C; ++k) {
          const uint64_t w = row[k * stride];
          x[k] += W::shoup_bal(__ull2double_rn(w >> 30), hi.w, hi.wp, q);
          x[k] += W::shoup_bal(__ull2double_rn(w & ((uint64_t{1} << 30) - 1)), lo.w, lo.wp, q);
        }
      } else {
#pragma unroll
        for (int k = 0; k < C; ++k) x[k] += W::shoup_bal(__ull2double_rn(row[k * stride]), lo.w, lo.wp, q);
      }
    }
  }
};

// Canonical output of a balanced inverse transform: v c mod q in [0, q).
struct F64InvEpilogue {
  uint64_t* dst;
  double q, c, cs;
  __device__ __forceinline__ void operator()(int pos, double v) const {
    v = Word<double>::shoup_bal(v, c, cs, q);
    dst[pos] = __double2ull_rz(v < 0.0 ? v + q : v);
  }
};

template <class Acc, int E>
__device__ __forceinline__ void key_mac_f64(Acc& acc, const double (&v)[E], const uint64_t* key0,
                                            const uint64_t* key1, double q, double qinv) {
#pragma unroll
  for (int i = 0; i < E / 2; ++i) {
    const ulonglong2 a = __ldg(reinterpret_cast<const ulonglong2*>(key0) + i);
    const ulonglong2 b = __ldg(reinterpret_cast<const ulonglong2*>(key1) + i);
    acc.mac_f64(2 * i, v[2 * i], __ull2double_rn(a.x), __ull2double_rn(b.x), q, qinv);
    acc.mac_f64(2 * i + 1, v[2 * i + 1], __ull2double_rn(a.y), __ull2double_rn(b.y), q, qinv);
  }
}

// One unit (ciphertext bi, Q row jrow) of the FP64 core.  PRE (tensor-core
// form): `ext` holds the extensions [D_l][B][QP_l][N] of the tensor-core
// basis conversion.  PRE = false (CUDA-core form): `ext` holds the ModUp
// digits [B][L][N] and the extension is computed in the transform's source
// (ExtSourceF64, constants ext64f [level][digit][r][2][QP] of `ext_digits`
// digits per level; digits that reach prime id f64_end or beyond hold a wide
// prime).
template <int LOGN, bool PRE>
__device__ __forceinline__ void ks_core_unit_f64(const uint64_t* __restrict__ ext, const uint64_t* __restrict__ key,
                                                 uint64_t* __restrict__ acc0, uint64_t* __restrict__ acc1,
                                                 int64_t batch, int q_limbs, int qp_limbs, int level, int qp0,
                                                 const uint64_t* __restrict__ ct3, int64_t ct3_stride,
                                                 const ChainTables<double>& tabs, const LevelTables<uint64_t>& lt,
                                                 const TwPair<double>* __restrict__ ext64f, int ext_digits,
                                                 int f64_end, int64_t bi, int jrow, unsigned char* smem_raw,
                                                 int rank) {
  using G = NttGeom<double, LOGN>;
  using W = Word<double>;
  static_assert(KsAcc<double, LOGN>::kSmem, "the FP64 core keeps its accumulators in shared memory");
  double* s = reinterpret_cast<double*>(smem_raw);
  const int64_t poly = bi * qp_limbs + jrow;
  const int pid = level + jrow;
  const PrimeInfo<double> p = tabs.prime[pid];
  const double q = p.q, twoq = p.twice_q, qinv = p.one_s;
  const int64_t own = int64_t(rank) * G::kM + threadIdx.x * G::kE;
  KsAcc<double, LOGN> acc(s, nullptr, nullptr);
  // (w, w / q) twiddle pairs: the quotient estimate does not wait for the
  // product, which measured faster here than value-only twiddles
  KsTw<double, LOGN> tw(smem_raw, tabs.tw_fwd + int64_t(pid) * G::kN, tabs.tw_inv + int64_t(pid) * G::kN, rank);
  tw.stage(false);
  const bool add = ct3 != nullptr;
  const uint64_t* ct3_own = add ? ct3 + (bi * q_limbs + jrow) * int64_t(G::kN) + own : nullptr;
  for (int a = 0; a < lt.num_digits; ++a) {
    const DigitDesc d = lt.digits[a];
    const uint64_t* key0 = key + ((int64_t(d.key_digit) * 2 + 0) * qp0 + pid) * G::kN + own;
    const uint64_t* key1 = key + ((int64_t(d.key_digit) * 2 + 1) * qp0 + pid) * G::kN + own;
    double v[G::kE];
    if (add && pid >= d.prime0 && pid < d.prime0 + d.alpha) {
      // uniform over the cluster: the own digit's NTT residue is c2 itself
#pragma unroll
      for (int e = 0; e < G::kE; ++e) v[e] = W::shoup(__ull2double_rn(ct3_own[2 * ct3_stride + e]), p.rinv, p.rinv_s, q);
    } else if constexpr (PRE) {
      U64RowSource src{ext + ((int64_t(a) * batch + bi) * qp_limbs + jrow) * G::kN};
      tw.forward_from(src, s, p, v);
    } else {
      ExtSourceF64 src{ext + (bi * q_limbs + (d.prime0 - level)) * int64_t(G::kN),
                       ext64f + (((int64_t(level) * ext_digits + a) * kMaxDigitWidth) * 2) * qp0 + pid, qp0, d.alpha,
                       LOGN, d.prime0 + d.alpha > f64_end, q, twoq};
      tw.forward_from(src, s, p, v);
    }
    key_mac_f64(acc, v, key0, key1, q, qinv);
  }
  tw.stage(true);
  const TwPair<double> pc = tabs.p_rinv[pid];  // P mod q and its companion (FP64 tables)
  for (int c = 0; c < 2; ++c) {
    double v[G::kE];
    acc.get(c, v);
#pragma unroll
    for (int e = 0; e < G::kE; ++e) v[e] = W::reduce_bal(v[e], q, qinv);  // |v| < 0.51 q
    if (add) {
#pragma unroll
      for (int e = 0; e < G::kE; ++e)
        v[e] += W::shoup_bal(__ull2double_rn(ct3_own[c * ct3_stride + e]), pc.w, pc.wp, q);
    }
    F64InvEpilogue epi{(c ? acc1 : acc0) + poly * G::kN, q, p.ninv_rinv, p.ninv_rinv_s};
    tw.inverse(s, p, v, epi);
  }
}

// The whole key-switch core of an int64 chain in one launch: the units of
// the leading f64_rows Q rows (primes below 2^42) run the FP64 body, the
// others (wider Q primes, the P rows) the integer body.  The branch is
// uniform over a cluster, and one launch lets the two kinds of units share
// the GPU instead of running one after the other.
template <int LOGN, bool PRE>
__global__ void __launch_bounds__(NttGeom<double, LOGN>::kThreads)
k_keyswitch_core_split(const uint64_t* __restrict__ digits, const uint64_t* __restrict__ key,
                       uint64_t* __restrict__ acc0, uint64_t* __restrict__ acc1, int64_t batch, int q_limbs,
                       int qp_limbs, int level, int qp0, int order, const unsigned long long* __restrict__ item_keys,
                       const uint64_t* __restrict__ ct3, int64_t ct3_stride, ChainTables<uint64_t> tabs,
                       LevelTables<uint64_t> lt, ChainTables<double> tabs64f, int f64_rows,
                       const TwPair<double>* __restrict__ ext64f, int ext_digits, int f64_end) {
  using G = NttGeom<double, LOGN>;
  static_assert(NttGeom<uint64_t, LOGN>::kC == G::kC && NttGeom<uint64_t, LOGN>::kThreads == G::kThreads,
                "one geometry for both bodies");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  int64_t poly, bi;
  int jrow;
  ks_work(blockIdx.x / G::kC, qp_limbs, batch, order, poly, bi, jrow);
  if (item_keys) key = reinterpret_cast<const uint64_t*>(item_keys[bi]);  // mixed-key batch
  const int rank = cluster_rank<double, LOGN>();
  if (jrow < f64_rows)
    ks_core_unit_f64<LOGN, PRE>(digits, key, acc0, acc1, batch, q_limbs, qp_limbs, level, qp0, ct3, ct3_stride,
                                tabs64f, lt, ext64f, ext_digits, f64_end, bi, jrow, smem_raw, rank);
  else
    ks_core_unit<uint64_t, LOGN, PRE>(digits, key, acc0, acc1, batch, q_limbs, qp_limbs, level, qp0, ct3,
                                      ct3_stride, tabs, lt, bi, jrow, smem_raw, rank);
}

// Sum of key switches of several ciphertexts with their own keys, reduced
// before the inverse NTT: acc = sum_g sum_d NTT(ext_d(digits[g])) * key_g[d]
// for every (ciphertext b, row j) unit, then one inverse NTT of each
// accumulator.  Followed by one ModDown, this is the "lazy ModDown" sum of
// rotations sum_g KS_g(sigma_g(c1_g)) (each term differs from its own ModDown
// by the rounding of the division by P, i.e. the sum is within `giants`
// units of the sum of separately rounded rotations).  digits: [G][B][L][N]
// ModUp digits (sigma_g applied); key_ptrs: device array of G key addresses;
// acc0/acc1: [B][QP_l][N].  Used for the giant steps of bootstrapping's
// linear transforms (the reference rotates and adds each giant step,
// fhelium/experimental/bootstrap/_linear.py:235-393).  PRE (tensor-core
// form): `digits` holds the extensions of the giants' digits,
// [D_l][giants x B][QP_l][N] (giant-major within a digit).
template <typename T, int LOGN, bool PRE = false>
__global__ void __launch_bounds__(NttGeom<T, LOGN>::kThreads)
k_keyswitch_sum(const T* __restrict__ digits, const unsigned long long* __restrict__ key_ptrs, T* __restrict__ acc0,
                T* __restrict__ acc1, int giants, int64_t batch, int q_limbs, int qp_limbs, int level, int qp0,
                int order, ChainTables<T> tabs, LevelTables<T> lt) {
  using G = NttGeom<T, LOGN>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* s = reinterpret_cast<T*>(smem_raw);
  const int rank = cluster_rank<T, LOGN>();
  int64_t poly, bi;
  int jrow;
  ks_work(blockIdx.x / G::kC, qp_limbs, batch, order, poly, bi, jrow);
  const int pid = level + jrow;
  const PrimeInfo<T> p = tabs.prime[pid];
  const int64_t own = int64_t(rank) * G::kM + threadIdx.x * G::kE;
  KsAcc<T, LOGN> acc(s, acc0 + poly * G::kN + own, acc1 + poly * G::kN + own);
  KsTw<T, LOGN> tw(smem_raw, tabs.tw_fwd + int64_t(pid) * G::kN, tabs.tw_inv + int64_t(pid) * G::kN, rank);
  tw.stage(false);
  for (int gi = 0; gi < giants; ++gi) {
    const T* dig = digits + (int64_t(gi) * batch + bi) * q_limbs * int64_t(G::kN);
    const T* key = reinterpret_cast<const T*>(key_ptrs[gi]);
    for (int a = 0; a < lt.num_digits; ++a) {
      const DigitDesc d = lt.digits[a];
      T v[G::kE];
      if constexpr (PRE) {
        RowSource<T, false> src{
            digits + ((int64_t(a) * giants * batch + int64_t(gi) * batch + bi) * qp_limbs + jrow) * G::kN, 0, 0, p.q};
        tw.forward_from(src, s, p, v);
      } else {
        ExtSource<T> src{dig + (int64_t(d.prime0 - level) << LOGN),
                         lt.ext + int64_t(a) * kMaxDigitWidth * qp0 + pid, qp0, d.alpha, LOGN, p.q, p.twice_q};
        tw.forward_from(src, s, p, v);
      }
      key_mac(acc, v, key + ((int64_t(d.key_digit) * 2 + 0) * qp0 + pid) * G::kN + own,
              key + ((int64_t(d.key_digit) * 2 + 1) * qp0 + pid) * G::kN + own, p);
    }
  }
  tw.stage(true);
  T v[G::kE];
  acc.get(0, v);
  InvEpilogue<T> e0 = make_inv_epilogue<T>(acc0 + poly * G::kN, p, kInvStandard, false);
  tw.inverse(s, p, v, e0);
  acc.get(1, v);
  InvEpilogue<T> e1 = make_inv_epilogue<T>(acc1 + poly * G::kN, p, kInvStandard, false);
  tw.inverse(s, p, v, e1);
}

// Hoisting stage 1: materialise NTT-domain extended digits once
// (fhelium/engine/hybrid_keyswitch.py:373-417).  prepared: [D_l, B, QP_l, N]
// standard NTT-domain values in [0, 2p).  SPLIT (int64 chains with FP64
// tables): the units of the leading f64_rows rows (primes below 2^42) run
// the extension and the transform in balanced FP64 arithmetic, the others
// the integer body, in one launch; both store lazy words in [0, 2p) (equal
// modulo p, not word for word).
template <typename T, int LOGN>
__device__ __forceinline__ void prepare_unit(const T* __restrict__ digits, T* __restrict__ prepared, int64_t batch,
                                             int q_limbs, int qp_limbs, int level, int qp0, const ChainTables<T>& tabs,
                                             const LevelTables<T>& lt, int64_t bi, int jrow, unsigned char* smem_raw,
                                             int rank) {
  using G = NttGeom<T, LOGN>;
  T* s = reinterpret_cast<T*>(smem_raw);
  const int64_t poly = bi * qp_limbs + jrow;
  const int pid = level + jrow;
  const PrimeInfo<T> p = tabs.prime[pid];
  const T* dig = digits + bi * q_limbs * int64_t(G::kN);
  const int64_t own = int64_t(rank) * G::kM + threadIdx.x * G::kE;
  KsTw<T, LOGN> tw(smem_raw, tabs.tw_fwd + int64_t(pid) * G::kN, tabs.tw_inv + int64_t(pid) * G::kN, rank);
  tw.stage(false);
  for (int a = 0; a < lt.num_digits; ++a) {
    const DigitDesc d = lt.digits[a];
    ExtSource<T> src{dig + (int64_t(d.prime0 - level) << LOGN), lt.ext + int64_t(a) * kMaxDigitWidth * qp0 + pid,
                     qp0, d.alpha, LOGN, p.q, p.twice_q};
    T v[G::kE];
    tw.forward_from(src, s, p, v);
#pragma unroll
    for (int e = 0; e < G::kE; ++e) v[e] = csub(v[e], p.twice_q);
    store16(prepared + (int64_t(a) * batch * qp_limbs + poly) * G::kN + own, v);
  }
}

template <int LOGN>
__device__ __forceinline__ void prepare_unit_f64(const uint64_t* __restrict__ digits, uint64_t* __restrict__ prepared,
                                                 int64_t batch, int q_limbs, int qp_limbs, int level, int qp0,
                                                 const ChainTables<double>& tabs, const LevelTables<uint64_t>& lt,
                                                 const TwPair<double>* __restrict__ ext64f, int ext_digits,
                                                 int f64_end, int64_t bi, int jrow, unsigned char* smem_raw,
                                                 int rank) {
  using G = NttGeom<double, LOGN>;
  double* s = reinterpret_cast<double*>(smem_raw);
  const int64_t poly = bi * qp_limbs + jrow;
  const int pid = level + jrow;
  const PrimeInfo<double> p = tabs.prime[pid];
  const int64_t own = int64_t(rank) * G::kM + threadIdx.x * G::kE;
  KsTw<double, LOGN> tw(smem_raw, tabs.tw_fwd + int64_t(pid) * G::kN, tabs.tw_inv + int64_t(pid) * G::kN, rank);
  tw.stage(false);
  for (int a = 0; a < lt.num_digits; ++a) {
    const DigitDesc d = lt.digits[a];
    ExtSourceF64 src{digits + (bi * q_limbs + (d.prime0 - level)) * int64_t(G::kN),
                     ext64f + (((int64_t(level) * ext_digits + a) * kMaxDigitWidth) * 2) * qp0 + pid, qp0, d.alpha,
                     LOGN, d.prime0 + d.alpha > f64_end, p.q, p.twice_q};
    double v[G::kE];
    tw.forward_from(src, s, p, v);
#pragma unroll
    for (int e = 0; e < G::kE; ++e) v[e] = Word<double>::to_lazy(v[e], p.q, p.one_s);
    store_words(prepared + (int64_t(a) * batch * qp_limbs + poly) * G::kN + own, v);
  }
}

template <typename T, int LOGN, bool SPLIT = false>
__global__ void __launch_bounds__(NttGeom<T, LOGN>::kThreads)
k_prepare_rotation(const T* __restrict__ digits, T* __restrict__ prepared, int64_t batch, int q_limbs,
                   int qp_limbs, int level, int qp0, int order, ChainTables<T> tabs, LevelTables<T> lt,
                   ChainTables<double> tabs64f, int f64_rows, const TwPair<double>* __restrict__ ext64f,
                   int ext_digits, int f64_end) {
  using G = NttGeom<T, LOGN>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int rank = cluster_rank<T, LOGN>();
  int64_t poly, bi;  // poly over [B, QP_l]
  int jrow;
  ks_work(blockIdx.x / G::kC, qp_limbs, batch, order, poly, bi, jrow);
  if constexpr (SPLIT) {
    static_assert(sizeof(T) == 8, "FP64 rows exist in int64 chains only");
    if (jrow < f64_rows) {
      prepare_unit_f64<LOGN>(reinterpret_cast<const uint64_t*>(digits), reinterpret_cast<uint64_t*>(prepared), batch,
                             q_limbs, qp_limbs, level, qp0, tabs64f, lt, ext64f, ext_digits, f64_end, bi, jrow,
                             smem_raw, rank);
      return;
    }
  }
  prepare_unit<T, LOGN>(digits, prepared, batch, q_limbs, qp_limbs, level, qp0, tabs, lt, bi, jrow, smem_raw, rank);
}

// The NTT-domain automorphism keeps a CTA's block whole: destination k's
// CTA is given by the low log C bits of br(k), and the low log C bits of the
// source's natural index depend only on those.  So the M destinations of
// CTA `rank` read one contiguous block of M source words, which the CTA
// copies into shared memory with 16-byte loads before gathering from it.
template <typename T, int LOGN>
__device__ __forceinline__ int galois_source_block(int rank, uint32_t galois) {
  using G = NttGeom<T, LOGN>;
  return galois_ntt_source(rank * G::kM, LOGN, galois) >> G::kLogM;
}

template <typename T, int LOGN>
__device__ __forceinline__ void stage_block(T* dst, const T* src) {
  using G = NttGeom<T, LOGN>;
  constexpr int kVec = G::kM * int(sizeof(T)) / 16;
  static_assert(kVec % G::kThreads == 0, "whole 16-byte vectors per thread");
#pragma unroll
  for (int i = threadIdx.x; i < kVec; i += G::kThreads)
    reinterpret_cast<uint4*>(dst)[i] = __ldg(reinterpret_cast<const uint4*>(src) + i);
}

// Hoisting stage 2 for rings whose key-switch accumulators live outside
// shared memory (N = 2^17): per rotation step, NTT-domain automorphism of the
// prepared digits + key inner product + inverse NTT of both accumulators
// (fhelium/engine/hybrid_keyswitch.py:419-469).  The automorphism gathers
// from a staged copy of the source block (galois_source_block) in the NTT
// working area, which is free until the inverse transform.  SPLIT: the units
// of the leading f64_rows rows in balanced FP64 arithmetic (the key used as
// stored, k R, and R removed with N^{-1} R^{-1}), the same canonical outputs.
template <typename T, int LOGN, bool SPLIT = false>
__global__ void __launch_bounds__(NttGeom<T, LOGN>::kThreads)
k_apply_prepared_rotation_staged(const T* __restrict__ prepared, const T* __restrict__ key, T* __restrict__ acc0,
                          T* __restrict__ acc1, int64_t batch, int qp_limbs, int level, int qp0,
                          uint32_t galois, int order, ChainTables<T> tabs, LevelTables<T> lt,
                          ChainTables<double> tabs64f, int f64_rows) {
  using G = NttGeom<T, LOGN>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int rank = cluster_rank<T, LOGN>();
  int64_t poly, bi;
  int jrow;
  ks_work(blockIdx.x / G::kC, qp_limbs, batch, order, poly, bi, jrow);
  (void)bi;
  const int pid = level + jrow;
  const int own = rank * G::kM + threadIdx.x * G::kE;
  const int blk = galois ? galois_source_block<T, LOGN>(rank, galois) : rank;
  T* staged = reinterpret_cast<T*>(smem_raw);  // the NTT working area, M words
  if constexpr (SPLIT) {
    static_assert(sizeof(T) == 8, "FP64 rows exist in int64 chains only");
    if (jrow < f64_rows) {
      double* s = reinterpret_cast<double*>(smem_raw);
      const PrimeInfo<double> p = tabs64f.prime[pid];
      const double q = p.q, qinv = p.one_s;
      KsAcc<double, LOGN> acc(s, nullptr, nullptr);
      KsTw<double, LOGN> tw(smem_raw, tabs64f.tw_fwd + int64_t(pid) * G::kN, tabs64f.tw_inv + int64_t(pid) * G::kN,
                            rank);
      for (int a = 0; a < lt.num_digits; ++a) {
        const DigitDesc d = lt.digits[a];
        const T* pr = prepared + (int64_t(a) * batch * qp_limbs + poly) * G::kN;
        const T* key0 = key + ((int64_t(d.key_digit) * 2 + 0) * qp0 + pid) * G::kN + own;
        const T* key1 = key + ((int64_t(d.key_digit) * 2 + 1) * qp0 + pid) * G::kN + own;
        if (galois) {
          __syncthreads();  // the previous digit's gathers are done
          stage_block<T, LOGN>(staged, pr + int64_t(blk) * G::kM);
          __syncthreads();
        }
#pragma unroll 4
        for (int e = 0; e < G::kE; ++e) {
          const T x = galois ? staged[galois_ntt_source(own + e, LOGN, galois) - blk * G::kM] : __ldg(pr + own + e);
          acc.mac_f64(e, __ull2double_rn(x), __ull2double_rn(__ldg(key0 + e)), __ull2double_rn(__ldg(key1 + e)), q,
                      qinv);
        }
      }
      if (galois) __syncthreads();  // the inverse transform reuses the working area
      tw.stage(true);
      for (int c = 0; c < 2; ++c) {
        double v[G::kE];
        acc.get(c, v);
#pragma unroll
        for (int e = 0; e < G::kE; ++e) v[e] = Word<double>::reduce_bal(v[e], q, qinv);
        F64InvEpilogue epi{reinterpret_cast<uint64_t*>(c ? acc1 : acc0) + poly * G::kN, q, p.ninv_rinv,
                           p.ninv_rinv_s};
        tw.inverse(s, p, v, epi);
      }
      return;
    }
  }
  T* s = reinterpret_cast<T*>(smem_raw);
  const PrimeInfo<T> p = tabs.prime[pid];
  KsAcc<T, LOGN> acc(s, acc0 + poly * G::kN + own, acc1 + poly * G::kN + own);
  KsTw<T, LOGN> tw(smem_raw, tabs.tw_fwd + int64_t(pid) * G::kN, tabs.tw_inv + int64_t(pid) * G::kN, rank);
  for (int a = 0; a < lt.num_digits; ++a) {
    const DigitDesc d = lt.digits[a];
    const T* pr = prepared + (int64_t(a) * batch * qp_limbs + poly) * G::kN;
    const T* key0 = key + ((int64_t(d.key_digit) * 2 + 0) * qp0 + pid) * G::kN + own;
    const T* key1 = key + ((int64_t(d.key_digit) * 2 + 1) * qp0 + pid) * G::kN + own;
    if (galois) {
      __syncthreads();
      stage_block<T, LOGN>(staged, pr + int64_t(blk) * G::kM);
      __syncthreads();
    }
#pragma unroll 4
    for (int e = 0; e < G::kE; ++e) {
      const T x = galois ? staged[galois_ntt_source(own + e, LOGN, galois) - blk * G::kM] : __ldg(pr + own + e);
      acc.mac(e, x, __ldg(key0 + e), __ldg(key1 + e), p);
    }
  }
  if (galois) __syncthreads();
  tw.stage(true);
  T v[G::kE];
  acc.get(0, v);
  InvEpilogue<T> e0 = make_inv_epilogue<T>(acc0 + poly * G::kN, p, kInvStandard, false);
  tw.inverse(s, p, v, e0);
  acc.get(1, v);
  InvEpilogue<T> e1 = make_inv_epilogue<T>(acc1 + poly * G::kN, p, kInvStandard, false);
  tw.inverse(s, p, v, e1);
}

// Hoisting stage 2 with the accumulators in registers (rings whose key-
// switch accumulators fit in shared memory, 8 residues per thread): thread
// t of CTA `rank` accumulates destinations base + j * threads + t, so a
// warp covers 32 consecutive destinations, whose sources under the
// NTT-domain automorphism are a permutation of one aligned group of 32
// (the low five bits of k become the top bits of br(k), and the odd g
// permutes them): the gathers, like the key loads, are 256-byte coalesced
// global loads, with no staging and no barrier in the digit loop.  The sums
// then pass through shared memory once (padded, conflict-free) into the
// thread-contiguous layout of the inverse transform.
template <typename T, int LOGN>
struct ApplyRegs {
  using G = NttGeom<T, LOGN>;
  static constexpr bool kOk = KsAcc<T, LOGN>::kSmem && G::kE == 8;
};

template <typename T, int LOGN>
__device__ __forceinline__ void apply_transpose(unsigned char* smem_raw, const T (&a0)[NttGeom<T, LOGN>::kE],
                                                const T (&a1)[NttGeom<T, LOGN>::kE], T* r1) {
  using G = NttGeom<T, LOGN>;
  T* w = reinterpret_cast<T*>(smem_raw);
#pragma unroll
  for (int j = 0; j < G::kE; ++j) {
    w[G::sidx(j * G::kThreads + threadIdx.x)] = a0[j];
    r1[G::sidx(j * G::kThreads + threadIdx.x)] = a1[j];
  }
  __syncthreads();
}

// Hoisting stage 2: per rotation step, NTT-domain automorphism of the
// prepared digits + key inner product + inverse NTT of both accumulators
// (fhelium/engine/hybrid_keyswitch.py:419-469).  SPLIT: the units of the
// leading f64_rows rows in balanced FP64 arithmetic (the key used as stored,
// k R, and R removed with N^{-1} R^{-1}), the same canonical outputs.
template <typename T, int LOGN, bool SPLIT = false>
__global__ void __launch_bounds__(NttGeom<T, LOGN>::kThreads)
k_apply_prepared_rotation(const T* __restrict__ prepared, const T* __restrict__ key, T* __restrict__ acc0,
                          T* __restrict__ acc1, int64_t batch, int qp_limbs, int level, int qp0,
                          uint32_t galois, int order, ChainTables<T> tabs, LevelTables<T> lt,
                          ChainTables<double> tabs64f, int f64_rows) {
  using G = NttGeom<T, LOGN>;
  static_assert(ApplyRegs<T, LOGN>::kOk, "register accumulators need the shared-memory accumulator room");
  constexpr int E = G::kE;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int rank = cluster_rank<T, LOGN>();
  int64_t poly, bi;
  int jrow;
  ks_work(blockIdx.x / G::kC, qp_limbs, batch, order, poly, bi, jrow);
  (void)bi;
  const int pid = level + jrow;
  const int base = rank * G::kM;
  // the second sum's transpose area: the key-switch accumulator room
  T* r1 = reinterpret_cast<T*>(smem_raw) + G::kSmemElems;
  if constexpr (SPLIT) {
    static_assert(sizeof(T) == 8, "FP64 rows exist in int64 chains only");
    if (jrow < f64_rows) {
      const PrimeInfo<double> p = tabs64f.prime[pid];
      const double q = p.q, qinv = p.one_s;
      double a0[E], a1[E];
#pragma unroll
      for (int j = 0; j < E; ++j) a0[j] = a1[j] = 0.0;
      for (int a = 0; a < lt.num_digits; ++a) {
        const DigitDesc d = lt.digits[a];
        const T* pr = prepared + (int64_t(a) * batch * qp_limbs + poly) * G::kN;
        const T* key0 = key + ((int64_t(d.key_digit) * 2 + 0) * qp0 + pid) * G::kN;
        const T* key1 = key + ((int64_t(d.key_digit) * 2 + 1) * qp0 + pid) * G::kN;
#pragma unroll
        for (int j = 0; j < E; ++j) {
          const int dst = base + j * G::kThreads + int(threadIdx.x);
          const int src = galois ? galois_ntt_source(dst, LOGN, galois) : dst;
          const double x = __ull2double_rn(__ldg(pr + src));
          a0[j] += Word<double>::mul_qinv_bal(x, __ull2double_rn(__ldg(key0 + dst)), q, qinv);
          a1[j] += Word<double>::mul_qinv_bal(x, __ull2double_rn(__ldg(key1 + dst)), q, qinv);
        }
      }
#pragma unroll
      for (int j = 0; j < E; ++j) {
        a0[j] = Word<double>::reduce_bal(a0[j], q, qinv);
        a1[j] = Word<double>::reduce_bal(a1[j], q, qinv);
      }
      double* w = reinterpret_cast<double*>(smem_raw);
      double* r1d = reinterpret_cast<double*>(r1);
      apply_transpose<double, LOGN>(smem_raw, a0, a1, r1d);
      KsTw<double, LOGN> tw(smem_raw, tabs64f.tw_fwd + int64_t(pid) * G::kN, tabs64f.tw_inv + int64_t(pid) * G::kN,
                            rank);
      tw.stage(true);
      for (int c = 0; c < 2; ++c) {
        double v[E];
#pragma unroll
        for (int e = 0; e < E; ++e) v[e] = (c ? r1d : w)[G::sidx(int(threadIdx.x) * E + e)];
        if (c == 0) __syncthreads();  // every thread has its values before the transform reuses the area
        F64InvEpilogue epi{reinterpret_cast<uint64_t*>(c ? acc1 : acc0) + poly * G::kN, q, p.ninv_rinv,
                           p.ninv_rinv_s};
        tw.inverse(w, p, v, epi);
      }
      return;
    }
  }
  const PrimeInfo<T> p = tabs.prime[pid];
  T a0[E], a1[E];
#pragma unroll
  for (int j = 0; j < E; ++j) a0[j] = a1[j] = 0;
  for (int a = 0; a < lt.num_digits; ++a) {
    const DigitDesc d = lt.digits[a];
    const T* pr = prepared + (int64_t(a) * batch * qp_limbs + poly) * G::kN;
    const T* key0 = key + ((int64_t(d.key_digit) * 2 + 0) * qp0 + pid) * G::kN;
    const T* key1 = key + ((int64_t(d.key_digit) * 2 + 1) * qp0 + pid) * G::kN;
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int dst = base + j * G::kThreads + int(threadIdx.x);
      const int src = galois ? galois_ntt_source(dst, LOGN, galois) : dst;
      const T x = __ldg(pr + src);
      a0[j] = csub(a0[j] + Word<T>::mont(x, __ldg(key0 + dst), p.q, p.neg_inv), p.twice_q);
      a1[j] = csub(a1[j] + Word<T>::mont(x, __ldg(key1 + dst), p.q, p.neg_inv), p.twice_q);
    }
  }
  T* w = reinterpret_cast<T*>(smem_raw);
  apply_transpose<T, LOGN>(smem_raw, a0, a1, r1);
  KsTw<T, LOGN> tw(smem_raw, tabs.tw_fwd + int64_t(pid) * G::kN, tabs.tw_inv + int64_t(pid) * G::kN, rank);
  tw.stage(true);
  for (int c = 0; c < 2; ++c) {
    T v[E];
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = (c ? r1 : w)[G::sidx(int(threadIdx.x) * E + e)];
    if (c == 0) __syncthreads();
    InvEpilogue<T> epi = make_inv_epilogue<T>((c ? acc1 : acc0) + poly * G::kN, p, kInvStandard, false);
    tw.inverse(w, p, v, epi);
  }
}

// ---------------------------------------------------------------------------
// ModDown by P fused with the final addition and, optionally, the rescale by
// the leading prime.  t0/t1: [B, QP_l, N] canonical coefficient rows;
// add0/add1 (nullable): [B, Q_l, N] canonical, add0 optionally read through
// sigma_g (rotation of c0).  Result per Q row i (prime q):
//   v_i = (t_i - [t]_P) P^{-1} + add_i  (mod q)
// which is exactly the sequential divide-by-p_j chain of
// csrc/ops/ckks/cpu/ckks_cpu.cpp:474-601 (both compute (t - [t]_P)/P over
// the integers), then (when rescale) the nearest-rounded division by the
// leading prime of csrc/ops/ckks/cpu/ckks_cpu.cpp:203-262:
//   out_i = (v_i - v_0) q_0^{-1} + [v_0 > q_0/2]  (mod q_i), i >= 1.
// out: [2, B, Q_l (- 1 if rescale), N] canonical, components out_pitch
// words apart (a slice of a larger batch when the pitch exceeds the slice).
template <typename T>
__global__ void k_moddown(const T* __restrict__ t0, const T* __restrict__ t1, const T* __restrict__ add0,
                          const T* __restrict__ add1, T* __restrict__ out, int64_t batch, int log_n,
                          int level, int num_q, int num_p, uint32_t add0_ginv,
                          const uint32_t* __restrict__ item_galois, int rescale, ChainTables<T> tabs,
                          LevelTables<T> lt, int64_t out_pitch) {
  using W = Word<T>;
  const int64_t n = int64_t(1) << log_n;
  const int q_limbs = num_q - level;
  const int qp_limbs = q_limbs + num_p;
  const int out_limbs = q_limbs - (rescale ? 1 : 0);
  const int64_t total = batch * n;
  const int qp0 = num_q + num_p;
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < total;
       idx += int64_t(gridDim.x) * blockDim.x) {
    const int64_t bi = idx >> log_n;
    const int k = int(idx & (n - 1));
    bool neg = false;
    const uint32_t gi =
        item_galois ? (item_galois[bi] == 1 ? 0u : galois_inverse_dev(item_galois[bi], log_n)) : add0_ginv;
    const int ak = gi ? galois_source(k, log_n, gi, neg) : k;
    for (int c = 0; c < 2; ++c) {
      const T* t = (c == 0 ? t0 : t1) + bi * qp_limbs * n;
      const T* ad = c == 0 ? add0 : add1;
      const int kk = c == 0 ? ak : k;
      const bool nn = c == 0 ? neg : false;
      // Garner digits of the P part
      T e[kMaxDigitWidth];
      for (int r = 0; r < num_p; ++r) {
        const PrimeInfo<T> p = tabs.prime[num_q + r];
        T x = t[(q_limbs + r) * n + k];
        T acc = 0;
        for (int i = 0; i < r; ++i) {
          const TwPair<T> g = tabs.p_garner[r * kMaxDigitWidth + i];
          acc = csub(acc + csub(W::shoup(e[i], g.w, g.wp, p.q), p.q), p.q);
        }
        if (r > 0) {
          const TwPair<T> inv = tabs.p_garner[r * kMaxDigitWidth + r];
          x = csub(W::shoup(csub(x + p.q - acc, p.q), inv.w, inv.wp, p.q), p.q);
        }
        e[r] = x;
      }
      T* o = out + int64_t(c) * out_pitch + bi * out_limbs * n;
      T v0 = 0;
      for (int i = 0; i < q_limbs; ++i) {
        const int pid = level + i;
        const PrimeInfo<T> p = tabs.prime[pid];
        T sub = 0;
        for (int r = 0; r < num_p; ++r) {
          const TwPair<T> m = tabs.p_mix[r * qp0 + pid];
          sub = csub(sub + csub(W::shoup(e[r], m.w, m.wp, p.q), p.q), p.q);
        }
        const TwPair<T> pinv = tabs.p_inv[pid];
        T v = csub(t[i * n + k] + p.q - sub, p.q);
        v = csub(W::shoup(v, pinv.w, pinv.wp, p.q), p.q);
        if (ad) {
          T x = csub(ad[(bi * q_limbs + i) * n + kk], p.q);
          if (nn && x) x = p.q - x;
          v = csub(v + x, p.q);
        }
        if (!rescale) {
          o[i * n + k] = v;
        } else if (i == 0) {
          v0 = v;
        } else {
          const T x0 = reduce_any(v0, p);
          const TwPair<T> inv = lt.rescale_inv[pid];
          T r = csub(W::shoup(csub(v + p.q - x0, p.q), inv.w, inv.wp, p.q), p.q);
          r += (v0 > (tabs.prime[level].q >> 1)) ? 1 : 0;
          o[(i - 1) * n + k] = csub(r, p.q);
        }
      }
    }
  }
}

// Standalone rescale of coefficient/standard components: in [K, L, N] ->
// out [K, L-1, N] (csrc/ops/ckks/cpu/ckks_cpu.cpp:203-262).
template <typename T>
__global__ void k_rescale(const T* __restrict__ in, T* __restrict__ out, int64_t polys, int limbs, int log_n,
                          int level, int nearest, ChainTables<T> tabs, LevelTables<T> lt) {
  using W = Word<T>;
  const int64_t n = int64_t(1) << log_n;
  const int64_t total = polys * (limbs - 1) * n;
  const T half = tabs.prime[level].q >> 1;
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < total;
       idx += int64_t(gridDim.x) * blockDim.x) {
    const int k = int(idx & (n - 1));
    const int64_t rowi = idx >> log_n;
    const int i = int(rowi % (limbs - 1)) + 1;
    const int64_t pl = rowi / (limbs - 1);
    const int pid = level + i;
    const PrimeInfo<T> p = tabs.prime[pid];
    const T v0 = in[pl * limbs * n + k];
    const T x0 = reduce_any(v0, p);
    const T v = reduce_any(in[(pl * limbs + i) * n + k], p);
    const TwPair<T> inv = lt.rescale_inv[pid];
    T r = csub(W::shoup(csub(v + p.q - x0, p.q), inv.w, inv.wp, p.q), p.q);
    if (nearest) r += (v0 > half) ? 1 : 0;
    out[idx] = csub(r, p.q);
  }
}

// Coefficient-domain automorphism: out = sigma_g(in), canonical
// (csrc/ops/ckks/cpu/ckks_cpu.cpp:287-380).
template <typename T>
__global__ void k_automorphism(const T* __restrict__ in, T* __restrict__ out, int64_t batch, int rows,
                               int row_start, int log_n, uint32_t ginv, ChainTables<T> tabs) {
  const int64_t n = int64_t(1) << log_n;
  const int64_t total = batch * rows * n;
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < total;
       idx += int64_t(gridDim.x) * blockDim.x) {
    const int k = int(idx & (n - 1));
    const int64_t row = idx >> log_n;
    const PrimeInfo<T> p = tabs.prime[row_start + int(row % rows)];
    bool neg = false;
    const int src = galois_source(k, log_n, ginv, neg);
    T x = csub(in[row * n + src], p.q);
    if (neg && x) x = p.q - x;
    out[idx] = x;
  }
}

// Pointwise RNS arithmetic over [batch, rows, N] whose rows are prime ids
// [row_start, row_start + rows) (fhelium_rns_ops.montgomery_mul / add_lazy /
// sub_lazy / add_canonical / sub_canonical, csrc/ops/rns/rns_arithmetic.cpp:
// 30-72, rns_canonical_arithmetic.cpp:15-23).  b_mode 0: b has a's shape;
// 1: b is [rows, N] shared by every batch item; 2: b is [rows] (one scalar
// per row, montgomery_mul_row_scalars_).
enum RnsOp : int { kOpMontMul = 0, kOpAddLazy = 1, kOpSubLazy = 2, kOpAddCanon = 3, kOpSubCanon = 4,
                   kOpNegCanon = 5 };

template <typename T, int V>
__global__ void k_rns_binary(const T* __restrict__ a, const T* __restrict__ b, T* __restrict__ out, int64_t batch,
                             int rows, int row_start, int log_n, int op, int b_mode, ChainTables<T> tabs) {
  const int64_t n = int64_t(1) << log_n;
  const int64_t k = (int64_t(blockIdx.x) * kEwThreads + threadIdx.x) * V;
  if (k >= n) return;
  const int row = blockIdx.y;
  const PrimeInfo<T> p = tabs.prime[row_start + row];
  const int64_t per = int64_t(rows) * n, off = int64_t(row) * n + k;
  EwVec<T, V> y;
  if (op == kOpNegCanon) {
#pragma unroll
    for (int e = 0; e < V; ++e) y.v[e] = T(0);
  } else if (b_mode == 1) {
    y = ew_load<T, V>(b + off);
  } else if (b_mode == 2) {
#pragma unroll
    for (int e = 0; e < V; ++e) y.v[e] = b[row];
  }
  for (int64_t bi = blockIdx.z; bi < batch; bi += gridDim.z) {
    const int64_t idx = bi * per + off;
    const EwVec<T, V> x = ew_load<T, V>(a + idx);
    if (b_mode == 0 && op != kOpNegCanon) y = ew_load<T, V>(b + idx);
    EwVec<T, V> r;
#pragma unroll
    for (int e = 0; e < V; ++e) {
      const T xv = x.v[e], yv = y.v[e];
      switch (op) {
        case kOpMontMul: r.v[e] = Word<T>::mont(xv, yv, p.q, p.neg_inv); break;
        case kOpAddLazy: r.v[e] = csub(xv + yv, p.twice_q); break;
        case kOpSubLazy: r.v[e] = csub(xv + p.twice_q - yv, p.twice_q); break;
        case kOpAddCanon: r.v[e] = csub(reduce_any(xv, p) + reduce_any(yv, p), p.q); break;
        case kOpSubCanon: r.v[e] = csub(reduce_any(xv, p) + p.q - reduce_any(yv, p), p.q); break;
        default: { const T c = reduce_any(xv, p); r.v[e] = c ? p.q - c : T(0); }
      }
    }
    ew_store<T, V>(out + idx, r);
  }
}

// Baby-step/giant-step inner products of a diagonal linear transform, all
// giant steps of one transform group in one pass:
//   out[k] = sum_b rot[b] (.) pts[table[k][b]]      (NTT/Montgomery, lazy)
// rot: [babies][polys][rows][N] baby rotations; pts: [entries][rows][N]
// diagonal plaintexts shared by every poly; table: [giants][babies] entry
// index or -1.  Each baby residue is read once and multiplied into up to 16
// giant accumulators held in registers.  Replaces the per-diagonal
// plaintext product + add of the reference's BSGS evaluation
// (fhelium/experimental/bootstrap/_linear.py:235-393).
template <typename T>
__global__ void k_bsgs_inner(const T* __restrict__ rot, int64_t rot_stride, const T* __restrict__ pts,
                             int64_t pt_stride, const int* __restrict__ table, int giants, int babies,
                             T* __restrict__ out, int64_t out_stride, int64_t polys, int rows, int row_start,
                             int log_n, ChainTables<T> tabs) {
  constexpr int kAcc = 16;
  const int64_t n = int64_t(1) << log_n;
  const int64_t per = int64_t(rows) * n;
  const int64_t total = polys * per;
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < total;
       idx += int64_t(gridDim.x) * blockDim.x) {
    const int64_t in_poly = idx % per;  // row * N + coefficient
    const int row = int(in_poly >> log_n);
    const PrimeInfo<T> p = tabs.prime[row_start + row];
    for (int g0 = 0; g0 < giants; g0 += kAcc) {
      T acc[kAcc];
#pragma unroll
      for (int j = 0; j < kAcc; ++j) acc[j] = 0;
      for (int b = 0; b < babies; ++b) {
        const T x = rot[b * rot_stride + idx];
#pragma unroll
        for (int j = 0; j < kAcc; ++j) {
          if (g0 + j >= giants) break;
          const int e = table[(g0 + j) * babies + b];
          if (e >= 0)
            acc[j] = csub(acc[j] + Word<T>::mont(x, pts[e * pt_stride + in_poly], p.q, p.neg_inv), p.twice_q);
        }
      }
#pragma unroll
      for (int j = 0; j < kAcc; ++j)
        if (g0 + j < giants) out[(g0 + j) * out_stride + idx] = acc[j];
    }
  }
}

// Same inner products with the plaintext rows staged in shared memory, so
// that each plaintext residue leaves HBM once however many polynomials share
// it.  One block per (row, 32 consecutive coefficients): the block stages
// the 32-coefficient slice of every plaintext entry (entries * 32 words),
// then each warp takes polynomials warp, warp + 8, ... with lane = the
// coefficient.  Requires entries * 32 * sizeof(T) of dynamic shared memory.
template <typename T>
__global__ void __launch_bounds__(256)
k_bsgs_inner_staged(const T* __restrict__ rot, int64_t rot_stride, const T* __restrict__ pts, int64_t pt_stride,
                    int entries, const int* __restrict__ table, int giants, int babies, T* __restrict__ out,
                    int64_t out_stride, int64_t polys, int rows, int row_start, int log_n, ChainTables<T> tabs) {
  constexpr int kAcc = 16;
  constexpr int kTile = 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sp = reinterpret_cast<T*>(smem_raw);  // [entries][kTile]
  const int64_t n = int64_t(1) << log_n;
  const int tiles_per_row = int(n / kTile);
  const int row = blockIdx.x / tiles_per_row;
  const int64_t col0 = int64_t(blockIdx.x % tiles_per_row) * kTile;
  const int64_t in_poly0 = int64_t(row) * n + col0;  // row * N + first coefficient of the tile
  for (int i = threadIdx.x; i < entries * kTile; i += blockDim.x)
    sp[i] = pts[int64_t(i / kTile) * pt_stride + in_poly0 + (i % kTile)];
  __syncthreads();
  const PrimeInfo<T> p = tabs.prime[row_start + row];
  const int lane = threadIdx.x % kTile;
  const int64_t per = int64_t(rows) * n;
  for (int64_t poly = threadIdx.x / kTile; poly < polys; poly += blockDim.x / kTile) {
    const int64_t idx = poly * per + in_poly0 + lane;
    for (int g0 = 0; g0 < giants; g0 += kAcc) {
      T acc[kAcc];
#pragma unroll
      for (int j = 0; j < kAcc; ++j) acc[j] = 0;
      for (int b = 0; b < babies; ++b) {
        const T x = rot[b * rot_stride + idx];
#pragma unroll
        for (int j = 0; j < kAcc; ++j) {
          if (g0 + j >= giants) break;
          const int e = table[(g0 + j) * babies + b];
          if (e >= 0) acc[j] = csub(acc[j] + Word<T>::mont(x, sp[e * kTile + lane], p.q, p.neg_inv), p.twice_q);
        }
      }
#pragma unroll
      for (int j = 0; j < kAcc; ++j)
        if (g0 + j < giants) out[(g0 + j) * out_stride + idx] = acc[j];
    }
  }
}

// Throughput probe of the modular multiplication the kernels are built on:
// every thread runs 8 independent chains of `iters` Shoup products by a
// per-prime constant (the butterfly's product) on registers only and writes
// the results so nothing is optimised away.  Gives the attainable rate of
// 64-bit (32-bit) modular products on the integer pipes, the roof that the
// NTT-heavy kernels are measured against.
template <typename T>
__global__ void k_modmul_probe(T* __restrict__ out, int iters, ChainTables<T> tabs) {
  const PrimeInfo<T> p = tabs.prime[0];
  const TwPair<T> w = tabs.tw_fwd[1];
  T x[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) x[i] = T(threadIdx.x + i * 977 + blockIdx.x) % p.q;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < 8; ++i) x[i] = Word<T>::shoup(x[i], w.w, w.wp, p.q);
  }
  T acc = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) acc ^= x[i];
  out[blockIdx.x * int64_t(blockDim.x) + threadIdx.x] = acc;
}

// The same for the balanced FP64 product of the rows of primes below 2^42
// (Word<double>::shoup_bal on the FP64 tables' first prime): the
// attainable rate of the FP64 rows' modular products.
template <int CHAINS>
__global__ void k_modmul_probe_f64(double* __restrict__ out, int iters, ChainTables<double> tabs) {
  const PrimeInfo<double> p = tabs.prime[0];
  const TwPair<double> w = tabs.tw_fwd[1];
  double x[CHAINS];
#pragma unroll
  for (int i = 0; i < CHAINS; ++i) x[i] = double((threadIdx.x + i * 977 + blockIdx.x) % 65521u);
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < CHAINS; ++i) x[i] = Word<double>::shoup_bal(x[i], w.w, w.wp, p.q);
  }
  double acc = 0.0;
#pragma unroll
  for (int i = 0; i < CHAINS; ++i) acc += x[i];
  out[blockIdx.x * int64_t(blockDim.x) + threadIdx.x] = acc;
}

// Lift signed integer coefficients [batch, N] (int64) into every row:
// out[b, r, k] = x[b, k] mod q_r, canonical (fhelium_rns_ops.
// lift_centered_coefficients, csrc/ops/rns/cuda/rns_arithmetic_cuda.cu:211).
template <typename T>
__global__ void k_lift_signed(const int64_t* __restrict__ x, T* __restrict__ out, int64_t batch, int rows,
                              int row_start, int log_n, ChainTables<T> tabs) {
  const int64_t n = int64_t(1) << log_n;
  const int64_t total = batch * rows * n;
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < total;
       idx += int64_t(gridDim.x) * blockDim.x) {
    const int k = int(idx & (n - 1));
    const int64_t br = idx >> log_n;
    const int row = int(br % rows);
    const int64_t bi = br / rows;
    const PrimeInfo<T> p = tabs.prime[row_start + row];
    const int64_t v = x[bi * n + k];
    const uint64_t mag = v < 0 ? uint64_t(0) - uint64_t(v) : uint64_t(v);
    uint64_t m;
    if constexpr (sizeof(T) == 8) {
      m = csub(Word<uint64_t>::shoup(mag, 1, p.one_s, p.q), p.q);
    } else {
      m = mag % p.q;
    }
    out[idx] = T(v < 0 && m ? p.q - m : m);
  }
}

// Multiplication by the monomial X^k in Z[X]/(X^N + 1), coefficient domain:
// out[j] = in[j - k] for j >= k, -in[j - k + N] for j < k (0 <= k < 2N,
// k >= N negates once more).  Canonical output.
template <typename T>
__global__ void k_monomial(const T* __restrict__ in, T* __restrict__ out, int64_t batch, int rows, int row_start,
                           int log_n, int k, ChainTables<T> tabs) {
  const int64_t n = int64_t(1) << log_n;
  const int64_t total = batch * rows * n;
  const bool flip_all = k >= n;
  const int kk = int(k % n);
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < total;
       idx += int64_t(gridDim.x) * blockDim.x) {
    const int j = int(idx & (n - 1));
    const int64_t row = idx >> log_n;
    const PrimeInfo<T> p = tabs.prime[row_start + int(row % rows)];
    int src = j - kk;
    bool neg = flip_all;
    if (src < 0) {
      src += int(n);
      neg = !neg;
    }
    T x = csub(in[row * n + src], p.q);
    if (neg && x) x = p.q - x;
    out[idx] = x;
  }
}

// ModRaise: centred lift of coefficient/standard residues modulo the single
// prime `src_prime` to every row of [row_start, row_start + rows): the
// represented integer is taken in (-q/2, q/2] (fhelium/experimental/bootstrap/
// _modraise.py, centred basis extension).  in [batch, N], out [batch, rows, N].
template <typename T>
__global__ void k_modraise(const T* __restrict__ in, T* __restrict__ out, int64_t batch, int rows, int row_start,
                           int src_prime, int log_n, ChainTables<T> tabs) {
  const int64_t n = int64_t(1) << log_n;
  const int64_t total = batch * rows * n;
  const T qs = tabs.prime[src_prime].q;
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < total;
       idx += int64_t(gridDim.x) * blockDim.x) {
    const int k = int(idx & (n - 1));
    const int64_t br = idx >> log_n;
    const int row = int(br % rows);
    const int64_t bi = br / rows;
    const PrimeInfo<T> p = tabs.prime[row_start + row];
    const T v = csub(in[bi * n + k], qs);
    const bool negative = v > (qs >> 1);
    const T mag = negative ? qs - v : v;
    T r = reduce_any(mag, p);
    out[idx] = (negative && r) ? p.q - r : r;
  }
}

// Add a per-row constant (canonical residues c[row]) to coefficient 0
// (coefficient domain, `all_slots` = 0) or to every NTT slot (`all_slots` = 1).
template <typename T>
__global__ void k_add_constant(T* __restrict__ data, const T* __restrict__ c, int64_t batch, int rows, int row_start,
                               int log_n, int all_slots, ChainTables<T> tabs) {
  const int64_t n = int64_t(1) << log_n;
  const int64_t total = all_slots ? batch * rows * n : batch * rows;
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < total;
       idx += int64_t(gridDim.x) * blockDim.x) {
    const int64_t row = all_slots ? (idx >> log_n) : idx;
    const int r = int(row % rows);
    const PrimeInfo<T> p = tabs.prime[row_start + r];
    const int64_t at = all_slots ? idx : row * n;
    data[at] = csub(csub(data[at], p.q) + c[r], p.q);
  }
}

// Canonical addition (add / add_canonical): out = a + b mod q.
template <typename T>
__global__ void k_add_canonical(const T* __restrict__ a, const T* __restrict__ b, T* __restrict__ out,
                                int64_t polys, int limbs, int log_n, int level, int lazy, ChainTables<T> tabs) {
  const int64_t n = int64_t(1) << log_n;
  const int64_t total = polys * limbs * n;
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < total;
       idx += int64_t(gridDim.x) * blockDim.x) {
    const PrimeInfo<T> p = tabs.prime[level + int((idx >> log_n) % limbs)];
    if (lazy) {
      out[idx] = csub(a[idx] + b[idx], p.twice_q);
    } else {
      out[idx] = csub(csub(a[idx], p.q) + csub(b[idx], p.q), p.q);
    }
  }
}

// Bounded decryption of the reference's decryptor
// (fhelium/engine/ckks_decryptor.py:180-272): the centred class of the phase
// modulo the product D of the trailing one or two active Q primes, converted
// to float64 with the reference's float64 operations in its order, so the
// result is the same double.  Two primes q_a (row limbs - 2), q_b (row
// limbs - 1): mixed-radix digits d0 = x_a, d1 = (x_b - d0) q_a^{-1} mod q_b;
// if (d1, d0) is above floor(D / 2) (compared digit-wise, high digit first)
// the negated residues are decomposed instead and the value negated; the
// value is dbl(d1) * dbl(q_a) + dbl(d0), each operation rounded to nearest
// (no fused multiply-add).  One prime: x > q/2 ? x - q : x.
struct DecryptTail {
  uint64_t qa, qb;
  uint64_t inv, inv_s;   // q_a^{-1} mod q_b and its Shoup companion
  uint64_t qb_one_s;     // Shoup companion of 1 mod q_b (reduction of x_a)
  uint64_t h0, h1;       // mixed-radix digits of floor(q_a q_b / 2)
  int two;               // 1: two trailing primes, 0: one
};

__device__ __forceinline__ void tail_digits(uint64_t xa, uint64_t xb, const DecryptTail& t, uint64_t& d0,
                                            uint64_t& d1) {
  using W = Word<uint64_t>;
  const uint64_t a_b = csub(W::shoup(xa, 1, t.qb_one_s, t.qb), t.qb);
  d0 = xa;
  d1 = csub(W::shoup(csub(xb + t.qb - a_b, t.qb), t.inv, t.inv_s, t.qb), t.qb);
}

template <typename T>
__global__ void k_decrypt_tail(const T* __restrict__ phase, double* __restrict__ out, int64_t batch, int limbs,
                               int log_n, DecryptTail t) {
  const int64_t n = int64_t(1) << log_n;
  const int64_t total = batch * n;
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < total;
       idx += int64_t(gridDim.x) * blockDim.x) {
    const int64_t b = idx >> log_n;
    const int64_t k = idx & (n - 1);
    const T* row_b = phase + (b * limbs + limbs - 1) * n;
    uint64_t xb = csub(uint64_t(row_b[k]), t.qb);
    if (!t.two) {
      const int64_t c = xb > (t.qb >> 1) ? int64_t(xb) - int64_t(t.qb) : int64_t(xb);
      out[idx] = __ll2double_rn(c);
      continue;
    }
    uint64_t xa = csub(uint64_t(row_b[k - n]), t.qa);
    uint64_t d0, d1;
    tail_digits(xa, xb, t, d0, d1);
    const bool above = d1 > t.h1 || (d1 == t.h1 && d0 > t.h0);
    if (above) {
      xa = xa ? t.qa - xa : 0;
      xb = xb ? t.qb - xb : 0;
      tail_digits(xa, xb, t, d0, d1);
    }
    const double v = __dadd_rn(__dmul_rn(__ll2double_rn(int64_t(d1)), __ull2double_rn(t.qa)),
                               __ll2double_rn(int64_t(d0)));
    out[idx] = above ? -v : v;
  }
}

}  // namespace fhb
