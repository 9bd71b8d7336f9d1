// Negacyclic NTT core for one residue polynomial held by a thread-block
// cluster.
//
// Transform (same as the reference, csrc/ops/ntt/forward_ntt.cpp:15-21):
//   A[k] = sum_n a[n] psi^{(2 br(k) + 1) n}  (mod q), bit-reversed output,
// computed as radix-2 decimation in frequency where stage s, group g uses the
// twiddle psi^{br(2^s + g)}; the inverse runs Gentleman-Sande stages with
// psi^{-br(.)} in the mirrored order.  Any implementation of this linear map
// yields the same residues, so the kernels below are free to organise the
// butterflies for the hardware.
//
// Layout on the GPU: a polynomial of N = 2^LOGN residues is split across a
// cluster of C = 2^LOGC CTAs; CTA r owns the contiguous block
// [r*M, (r+1)*M), M = N / C, in its shared memory (padded every 2^PAD
// elements so that strided accesses spread over all banks).
//   * the first LOGC forward stages (half spans >= M) pair elements held by
//     different CTAs: each CTA reads the C inputs of 1/C of the columns
//     straight from their source (global memory), transforms them in
//     registers and pushes the results into the owning CTAs' shared memory
//     (st.shared::cluster);
//   * the remaining LOGM stages are CTA-local, done in register passes of
//     3 or 4 stages (radix-8/16 per thread, E = 8 or 16 residues per thread);
//   * the last forward pass leaves every thread with E consecutive outputs
//     in registers, which the caller's epilogue consumes (store, or fused
//     key multiply-accumulate).
// The inverse mirrors this: the first pass starts from E consecutive
// values per thread (from registers), the cross-CTA stages come last and
// read the other CTAs' blocks through distributed shared memory.
// Integer residues: forward butterflies keep Harvey's lazy range [0, 4q),
// inverse ones [0, 2q).  FP64 residues (T = double, primes below 2^42,
// N <= 2^16) run balanced: signed values, every twiddle product reduced
// with a quotient rounded to nearest to (-0.6 q, 0.6 q) and no conditional
// subtraction, so a forward value grows by at most 0.6 q per stage (inputs
// below 10 q leave the 16 stages below 20 q) and an inverse sum at most
// doubles per stage, with every value reduced to (-0.51 q, 0.51 q) when a
// pass stores it to shared memory (a pass of at most 4 stages from inputs
// below 2q keeps every product operand below 32 q).  Every product operand
// stays below 2^48 q / w.  For T = double the transforms' `twoq` argument
// carries 1 / q instead.
#pragma once
#include <cooperative_groups.h>

#include <type_traits>

#include "fhb_arith.cuh"

namespace fhb {
namespace cg = cooperative_groups;

constexpr int clamp_int(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// EPT = residues per thread (8 or 16; 0 = the default for the ring).
template <typename T, int LOGN, int EPT = 0>
struct NttGeom {
  static constexpr int kLogN = LOGN;
  static constexpr int kN = 1 << LOGN;
  static constexpr int kLogC = clamp_int(LOGN - 13, 0, 3);
  static constexpr int kC = 1 << kLogC;
  static constexpr int kLogM = LOGN - kLogC;
  static constexpr int kM = 1 << kLogM;
#ifndef FHB_NTT_E
#define FHB_NTT_E 8
#endif
  // Residues per thread.  8 (1024 threads for M = 8192) beats 16 (512
  // threads): the kernels are latency bound and twice the resident warps
  // hide more of it (key-switch core 33.9 vs 43.4 ms at L=35, batch 32).
  // (16 when 8 would need more than 1024 threads: N = 2^17, M = 16384.)
  static constexpr int kReqE = EPT ? EPT : FHB_NTT_E;
  static_assert(kReqE == 8 || kReqE == 16, "8 or 16 residues per thread");
  static constexpr int kE = (kM / kReqE > 1024) ? 16 : kReqE;
  static constexpr int kThreads = kM / kE;
  static constexpr int kPadShift = sizeof(T) == 8 ? 4 : 5;
  static constexpr int kSmemElems = kM + (kM >> kPadShift);
  // Register passes: radix-8/16 (3 or 4 stages) for 16 residues per thread,
  // radix-8 for 8; the last forward pass is always a full one, so its
  // outputs are thread-contiguous.
  static constexpr int kMaxK = kE == 16 ? 4 : 3;
  static constexpr int kPasses = kMaxK == 4 ? (kLogM + 3) / 4 : (kLogM + 2) / 3;
  static constexpr int kNum4 = kMaxK == 4 ? kLogM - 3 * kPasses : 0;
  static constexpr int pass_k(int j) {
    return kMaxK == 4 ? (j >= kPasses - kNum4 ? 4 : 3) : (j == 0 ? kLogM - 3 * (kPasses - 1) : 3);
  }
  static constexpr int pass_a(int j) { return j == 0 ? 0 : pass_a(j - 1) + pass_k(j - 1); }
  // inverse pass j is forward pass kPasses-1-j; its lowest half-span exponent
  static constexpr int inv_k(int j) { return pass_k(kPasses - 1 - j); }
  static constexpr int inv_l(int j) { return j == 0 ? 0 : inv_l(j - 1) + inv_k(j - 1); }
  __device__ __forceinline__ static int sidx(int n) { return n + (n >> kPadShift); }
};

template <typename T>
__device__ __forceinline__ TwPair<T> ldtw(const TwPair<T>* tw, int i) {
  if constexpr (std::is_same<T, double>::value) {
    const double2 v = __ldg(reinterpret_cast<const double2*>(tw + i));
    return TwPair<T>{v.x, v.y};
  } else if constexpr (sizeof(T) == 8) {
    const ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2*>(tw + i));
    return TwPair<T>{v.x, v.y};
  } else {
    const uint2 v = __ldg(reinterpret_cast<const uint2*>(tw + i));
    return TwPair<T>{v.x, v.y};
  }
}

// Twiddle accessors.  Forward stage st pairs use psi^{br(2^st + (ng >> (LOGN-st)))},
// inverse half-span exponent j uses psi^{-br((N >> (j+1)) + (ng >> (j+1)))}.
// TwGlobal reads the prime's row straight from global memory (L2).
template <typename T, int LOGN>
struct TwGlobal {
  static constexpr bool kQFromProduct = false;  // (w, floor(w 2^W / q)) pairs: Shoup products
  const TwPair<T>* g;
  __device__ __forceinline__ TwGlobal(const TwPair<T>* row) : g(row) {}
  __device__ __forceinline__ TwPair<T> fwd(int st, int ng) const { return ldtw(g, (1 << st) + (ng >> (LOGN - st))); }
  __device__ __forceinline__ TwPair<T> inv(int j, int ng) const {
    return ldtw(g, ((1 << LOGN) >> (j + 1)) + (ng >> (j + 1)));
  }
};

// TwShared serves the CTA-local stages from a copy in shared memory of just
// the twiddles this CTA's block [rank*M, (rank+1)*M) uses (M - 1 pairs), so a
// kernel that transforms several polynomials of the same prime loads them
// once.  Layout: forward local stage a at offset 2^a - 1 (2^a entries);
// inverse local exponent j at offset M - (M >> j) (M >> (j+1) entries).
// Cross-CTA stages (at most 7 distinct twiddles) still read global memory.
template <typename T, int LOGN>
struct TwShared {
  static constexpr bool kQFromProduct = false;
  using G = NttGeom<T, LOGN>;
  const TwPair<T>* g;
  const TwPair<T>* s;
  int base;
  __device__ __forceinline__ TwPair<T> fwd(int st, int ng) const {
    if (st < G::kLogC) return ldtw(g, (1 << st) + (ng >> (LOGN - st)));
    const int a = st - G::kLogC;
    return s[(1 << a) - 1 + ((ng - base) >> (G::kLogM - a))];
  }
  __device__ __forceinline__ TwPair<T> inv(int j, int ng) const {
    if (j >= G::kLogM) return ldtw(g, ((1 << LOGN) >> (j + 1)) + (ng >> (j + 1)));
    return s[(G::kM - (G::kM >> j)) + ((ng - base) >> (j + 1))];
  }
  // Copy this CTA's forward (inverse = false) or inverse twiddles from the
  // global row `row` into s_out (caller synchronises afterwards).
  __device__ __forceinline__ static void stage(TwPair<T>* s_out, const TwPair<T>* row, int rank, bool inverse) {
    for (int idx = threadIdx.x; idx < G::kM - 1; idx += blockDim.x) {
      int src;
      if (!inverse) {
        const int a = 31 - __clz(idx + 1);
        src = (1 << (G::kLogC + a)) + (rank << a) + (idx + 1 - (1 << a));
      } else {
        const int j = G::kLogM - 1 - (31 - __clz(G::kM - idx - 1));
        const int off = G::kM - (G::kM >> j);
        src = ((1 << LOGN) >> (j + 1)) + ((rank * G::kM) >> (j + 1)) + (idx - off);
      }
      s_out[idx] = ldtw(row, src);
    }
  }
};

// FP64 rows: the twiddle values alone from global memory (8 bytes each,
// half the load traffic of pairs).  The butterflies take the quotient from
// the product and 1/q (Word<double>::mul_qinv), which the accessor hands out
// in the pair's second slot.
template <int LOGN>
struct TwGlobalQ {
  static constexpr bool kQFromProduct = true;
  const double* g;
  double qinv;
  __device__ __forceinline__ TwPair<double> fwd(int st, int ng) const {
    return TwPair<double>{__ldg(g + (1 << st) + (ng >> (LOGN - st))), qinv};
  }
  __device__ __forceinline__ TwPair<double> inv(int j, int ng) const {
    return TwPair<double>{__ldg(g + ((1 << LOGN) >> (j + 1)) + (ng >> (j + 1))), qinv};
  }
};

template <typename T, int LOGN, class TW = TwGlobal<T, LOGN>, int EPT = 0>
struct Ntt {
  using G = NttGeom<T, LOGN, EPT>;
  using W = Word<T>;
  static constexpr int E = G::kE;

  // threadIdx.x behind an empty volatile asm: every transform recomputes its
  // per-thread addresses instead of the compiler hoisting all of them out of
  // the caller's digit loop (which used to exhaust the register budget).
  __device__ __forceinline__ static int tid() {
    int t = threadIdx.x;
    asm volatile("" : "+r"(t));
    return t;
  }

  static constexpr bool kBal = std::is_same<T, double>::value;

  // y w mod q: Shoup's product with the twiddle's companion, in [0, 2q); or
  // (FP64) balanced, with the companion or, for value-only twiddles, the
  // product's own quotient estimate (the accessor hands 1/q out in .wp)
  __device__ __forceinline__ static T tw_mul(T y, const TwPair<T>& w, T q) {
    if constexpr (kBal) {
      if constexpr (TW::kQFromProduct) {
        return W::mul_qinv_bal(y, w.w, q, w.wp);
      } else {
        return W::shoup_bal(y, w.w, w.wp, q);
      }
    } else {
      return W::shoup(y, w.w, w.wp, q);
    }
  }

  __device__ __forceinline__ static void fwd_bfly(T& x, T& y, const TwPair<T>& w, T q, T twoq) {
    if constexpr (kBal) {
      const T t = tw_mul(y, w, q);
      const T xx = x;
      x = xx + t;
      y = xx - t;
    } else {
      const T xx = csub(x, twoq);
      const T t = tw_mul(y, w, q);
      x = xx + t;
      y = xx - t + twoq;
    }
  }
  __device__ __forceinline__ static void inv_bfly(T& x, T& y, const TwPair<T>& w, T q, T twoq) {
    if constexpr (kBal) {
      const T s = x + y;
      const T d = x - y;
      x = s;
      y = tw_mul(d, w, q);
    } else {
      const T s = x + y;
      const T d = x - y + twoq;
      x = csub(s, twoq);
      y = tw_mul(d, w, q);
    }
  }

  // ---- forward -----------------------------------------------------------
  // Cross-CTA stages straight from the source: CTA `rank` owns the columns
  // m in [rank*M/C, (rank+1)*M/C) of the first log C stages; it reads the C
  // inputs of each column from `src` (global memory), runs the stages in
  // registers and pushes the results into the owning CTAs' shared memory
  // (remote stores, which do not stall the issuing thread).
  template <class Src>
  __device__ __forceinline__ static void fwd_cross_push(Src& src, T* s, const TW& tw, T q, T twoq, int rank) {
    cg::cluster_group cl = cg::this_cluster();
    constexpr int kCols = G::kM / G::kC;
    static_assert(kCols % G::kThreads == 0, "columns per CTA must be a multiple of the thread count");
#pragma unroll
    for (int u = 0; u < kCols / G::kThreads; ++u) {
      const int m = rank * kCols + u * G::kThreads + tid();
      const int sm = G::sidx(m);
      T x[G::kC];
      src.column(m, G::kM, x);
#pragma unroll
      for (int st = 0; st < G::kLogC; ++st) {
        const int h = G::kC >> (st + 1);
#pragma unroll
        for (int c = 0; c < G::kC; ++c)
          if (!(c & h)) fwd_bfly(x[c], x[c + h], tw.fwd(st, c * G::kM), q, twoq);
      }
#pragma unroll
      for (int c = 0; c < G::kC; ++c) *cl.map_shared_rank(s + sm, c) = x[c];
    }
  }

  template <int A, int K, bool LAST>
  __device__ __forceinline__ static void fwd_pass(T* s, const TW& tw, T q, T twoq, int rank,
                                                  T (&out)[E]) {
    constexpr int kLogHl = G::kLogM - A - K;
    constexpr int kHl = 1 << kLogHl;
    constexpr int kGs = 1 << K;
    constexpr int kNg = E >> K;
#pragma unroll
    for (int u = 0; u < kNg; ++u) {
      const int gid = LAST ? tid() * kNg + u : u * G::kThreads + tid();
      const int n0 = (gid & (kHl - 1)) | ((gid >> kLogHl) << (kLogHl + K));
      const int ng0 = rank * G::kM + n0;
      // All 2^K - 1 twiddles of the group are fetched before any butterfly so
      // their (L1/L2) latencies overlap; stage b uses 2^b of them, selected
      // by the top b bits of the element index within the group.
      TwPair<T> w[kGs - 1];
#pragma unroll
      for (int b = 0; b < K; ++b)
#pragma unroll
        for (int j = 0; j < (1 << b); ++j)
          w[(1 << b) - 1 + j] = tw.fwd(G::kLogC + A + b, ng0 + ((j << (K - b)) << kLogHl));
      T v[kGs];
#pragma unroll
      for (int i = 0; i < kGs; ++i) v[i] = s[G::sidx(n0 + i * kHl)];
#pragma unroll
      for (int b = 0; b < K; ++b) {
        const int h = kGs >> (b + 1);
#pragma unroll
        for (int i = 0; i < kGs; ++i)
          if (!(i & h)) fwd_bfly(v[i], v[i + h], w[(1 << b) - 1 + (i >> (K - b))], q, twoq);
      }
      if constexpr (LAST) {
#pragma unroll
        for (int i = 0; i < kGs; ++i) out[u * kGs + i] = v[i];
      } else {
#pragma unroll
        for (int i = 0; i < kGs; ++i) s[G::sidx(n0 + i * kHl)] = v[i];
      }
    }
  }

  template <int J>
  __device__ __forceinline__ static void fwd_local(T* s, const TW& tw, T q, T twoq, int rank,
                                                   T (&out)[E]) {
    constexpr int K = G::pass_k(J);
    constexpr int A = G::pass_a(J);
    if constexpr (J == G::kPasses - 1) {
      fwd_pass<A, K, true>(s, tw, q, twoq, rank, out);
    } else {
      fwd_pass<A, K, false>(s, tw, q, twoq, rank, out);
      __syncthreads();
      fwd_local<J + 1>(s, tw, q, twoq, rank, out);
    }
  }

  // Forward transform of one polynomial whose input residues (< 4q; FP64:
  // |x| < 10q) are
  // produced on demand: src.column(m, stride, x) fills x[c] with the input
  // at position c * stride + m of the polynomial (0 <= position < N).  On return out[e] holds the (lazy, < 4q)
  // output at local position tid() * E + e of CTA `rank`.  Starts with a
  // (cluster) barrier, so shared memory still being read by a previous
  // transform of this CTA or cluster is never overwritten.
  template <class Src>
  __device__ __forceinline__ static void forward_from(Src& src, T* s, const TW& tw, T q, T twoq, int rank,
                                                      T (&out)[E]) {
    if constexpr (G::kC > 1) {
      cg::cluster_group cl = cg::this_cluster();
      cl.sync();
      fwd_cross_push(src, s, tw, q, twoq, rank);
      cl.sync();
    } else {
      __syncthreads();
      for (int i = tid(); i < G::kM; i += G::kThreads) {
        T x[1];
        src.column(i, 0, x);
        s[G::sidx(i)] = x[0];
      }
      __syncthreads();
    }
    fwd_local<0>(s, tw, q, twoq, rank, out);
  }

  // ---- inverse -----------------------------------------------------------
  // Epilogue functor: epi(global_position, value in [0, 2q)).
  template <int L, int K, bool FIRST, bool STORE, class Epi>
  __device__ __forceinline__ static void inv_pass(T* s, const TW& tw, T q, T twoq, int rank,
                                                  const T (&in)[E], Epi& epi) {
    constexpr int kHl = 1 << L;
    constexpr int kGs = 1 << K;
    constexpr int kNg = E >> K;
#pragma unroll
    for (int u = 0; u < kNg; ++u) {
      const int gid = FIRST ? tid() * kNg + u : u * G::kThreads + tid();
      const int n0 = (gid & (kHl - 1)) | ((gid >> L) << (L + K));
      const int ng0 = rank * G::kM + n0;
      // Prefetch the group's 2^K - 1 twiddles: stage b (half span 2^(L+b))
      // has 2^(K-1-b) of them, selected by the element-index bits above b.
      TwPair<T> w[kGs - 1];
#pragma unroll
      for (int b = 0; b < K; ++b)
#pragma unroll
        for (int m = 0; m < (1 << (K - 1 - b)); ++m)
          w[kGs - (kGs >> b) + m] = tw.inv(L + b, ng0 + ((m << (b + 1)) << L));
      T v[kGs];
#pragma unroll
      for (int i = 0; i < kGs; ++i) v[i] = FIRST ? in[u * kGs + i] : s[G::sidx(n0 + i * kHl)];
#pragma unroll
      for (int b = 0; b < K; ++b) {
        const int h = 1 << b;
#pragma unroll
        for (int i = 0; i < kGs; ++i)
          if (!(i & h)) inv_bfly(v[i], v[i + h], w[kGs - (kGs >> b) + (i >> (b + 1))], q, twoq);
      }
      if constexpr (STORE) {
#pragma unroll
        for (int i = 0; i < kGs; ++i) epi(ng0 + i * kHl, v[i]);
      } else {
#pragma unroll
        for (int i = 0; i < kGs; ++i) {
          if constexpr (kBal) v[i] = W::reduce_bal(v[i], q, twoq);  // twoq holds 1/q here
          s[G::sidx(n0 + i * kHl)] = v[i];
        }
      }
    }
  }

  template <int J, class Epi>
  __device__ __forceinline__ static void inv_local(T* s, const TW& tw, T q, T twoq, int rank,
                                                   const T (&in)[E], Epi& epi) {
    constexpr int K = G::inv_k(J);
    constexpr int L = G::inv_l(J);
    constexpr bool kLast = J == G::kPasses - 1;
    constexpr bool kStore = kLast && G::kC == 1;
    inv_pass<L, K, J == 0, kStore>(s, tw, q, twoq, rank, in, epi);
    if constexpr (!kLast) {
      __syncthreads();
      inv_local<J + 1>(s, tw, q, twoq, rank, in, epi);
    }
  }

  // Cross-CTA inverse stages over the columns m in [rank*M/C, (rank+1)*M/C):
  // the C elements of a column are read from the C CTAs' shared memory
  // (ld.shared::cluster).  Pulling here measured faster than pushing them
  // from the last local pass (one more register array live across a
  // cluster barrier).
  template <class Epi>
  __device__ __forceinline__ static void inv_cross(T* s, const TW& tw, T q, T twoq, int rank,
                                                   Epi& epi) {
    if constexpr (G::kC > 1) {
      cg::cluster_group cl = cg::this_cluster();
      constexpr int kCols = G::kM / G::kC;
#pragma unroll
      for (int u = 0; u < kCols / G::kThreads; ++u) {
        const int m = rank * kCols + u * G::kThreads + tid();
        const int sm = G::sidx(m);
        T x[G::kC];
#pragma unroll
        for (int c = 0; c < G::kC; ++c) x[c] = *cl.map_shared_rank(s + sm, c);
#pragma unroll
        for (int b = 0; b < G::kLogC; ++b) {
          const int j = G::kLogM + b;
          const int h = 1 << b;
#pragma unroll
          for (int c = 0; c < G::kC; ++c)
            if (!(c & h)) {
              const int ng = c * G::kM + m;
              inv_bfly(x[c], x[c + h], tw.inv(j, ng), q, twoq);
            }
        }
#pragma unroll
        for (int c = 0; c < G::kC; ++c) epi(c * G::kM + m, x[c]);
      }
    }
  }

  // Inverse transform of the values `in` (thread-contiguous layout, as left
  // by `forward_from`, each < 2q; FP64: |x| < 2q, balanced).  Every output
  // is handed to epi(position, v) with v in [0, 2q) (FP64: |v| < 8q,
  // balanced); s is scratch.  Ends with a cluster
  // barrier so that shared memory may be reused (and so that peers never
  // outlive reads).
  template <class Epi>
  __device__ __forceinline__ static void inverse(T* s, const TW& tw, T q, T twoq, int rank,
                                                 const T (&in)[E], Epi& epi) {
    inv_local<0>(s, tw, q, twoq, rank, in, epi);
    if constexpr (G::kC > 1) {
      cg::cluster_group cl = cg::this_cluster();
      cl.sync();
      inv_cross(s, tw, q, twoq, rank, epi);
      cl.sync();
    } else {
      __syncthreads();
    }
  }
};

}  // namespace fhb
