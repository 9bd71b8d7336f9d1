// Residue arithmetic for the two buffer families on sm_100a.
//
// int64 family: primes q < 2^60, Montgomery radix R = 2^62 (4q < R).
// int32 family: primes q < 2^28, Montgomery radix R = 2^30.
// The radices match the reference's split-word Montgomery convention
// (csrc/ops/common/cuda/montgomery.cuh:10-59), so Montgomery-form tables and
// residues produced by either library are interchangeable.  Multiplications
// by per-prime constants (twiddles, basis-conversion factors, inverses) use
// Shoup's precomputed-quotient form instead: w' = floor(w 2^W / q) turns
// x*w mod q into one high multiply, two low multiplies and a subtraction.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace fhb {

template <typename T>
struct Word;

template <>
struct Word<uint64_t> {
  using T = uint64_t;
  static constexpr int kRadixBits = 62;
  static constexpr uint64_t kRadixMask = (uint64_t{1} << 62) - 1;
  // Shoup: x*w - floor(x*w'/2^64)*q in [0, 2q) for any 64-bit x, q < 2^63.
  __device__ __forceinline__ static T shoup(T x, T w, T wp, T q) {
    const T t = __umul64hi(x, wp);
    return x * w - t * q;
  }
  // Montgomery REDC(a*b) with R = 2^62, output in [0, 2q) when a*b < qR.
  __device__ __forceinline__ static T mont(T a, T b, T q, T neg_inv) {
    const T lo = a * b;
    const T hi = __umul64hi(a, b);
    const T m = (lo * neg_inv) & kRadixMask;
    const T mlo = m * q;
    const T mhi = __umul64hi(m, q);
    const T s = lo + mlo;
    const T h = hi + mhi + (s < lo ? 1 : 0);
    return (h << 2) | (s >> 62);
  }
};

template <>
struct Word<uint32_t> {
  using T = uint32_t;
  static constexpr int kRadixBits = 30;
  static constexpr uint32_t kRadixMask = (1u << 30) - 1;
  __device__ __forceinline__ static T shoup(T x, T w, T wp, T q) {
    const T t = __umulhi(x, wp);
    return x * w - t * q;
  }
  __device__ __forceinline__ static T mont(T a, T b, T q, T neg_inv) {
    const uint64_t p = static_cast<uint64_t>(a) * b;
    const uint32_t m = (static_cast<uint32_t>(p) * neg_inv) & kRadixMask;
    return static_cast<T>((p + static_cast<uint64_t>(m) * q) >> 30);
  }
};

// Residues of primes q < 2^42 held as exact integers in doubles (the
// key-switch core's FP64 form).  x w mod q for integers 0 <= x < 2^45,
// 0 <= w < 2^43 with x w / q < 2^47, given wc = w / q rounded to double:
//   h = fl(x w); l = fma(x, w, -h)    the rounding error of h, exact (an integer)
//   qt = floor(fl(x wc))              within one of floor(x w / q) (relative error < 2^-51)
//   r = fma(-qt, q, h) + l            = x w - qt q exactly (every intermediate is an integer < 2^53)
// so r lies in [-q, 2q) and one correction returns [0, 2q), as the integer
// Shoup product does.  The products run on the FP64 pipe, which on B200
// sustains about 1.5x the rate of the 64-bit integer Shoup butterflies.
template <>
struct Word<double> {
  using T = double;
  __device__ __forceinline__ static T shoup(T x, T w, T wc, T q) {
    const T h = x * w;
    const T l = fma(x, w, -h);
    const T qt = floor(x * wc);
    const T r = fma(-qt, q, h) + l;
    return r < 0.0 ? r + q : r;
  }
  // The same with the quotient taken from h and qinv = 1 / q rounded (for
  // products of two residues, and for twiddles stored without a companion):
  // h qinv carries a relative error below 2^-51, so for x w / q < 2^47 the
  // estimate is again within one of floor(x w / q).
  __device__ __forceinline__ static T mul_qinv(T x, T w, T q, T qinv) {
    const T h = x * w;
    const T l = fma(x, w, -h);
    const T qt = floor(h * qinv);
    const T r = fma(-qt, q, h) + l;
    return r < 0.0 ? r + q : r;
  }
  // Balanced forms for signed residues (the FP64 transforms): the quotient
  // estimate rounded to nearest.  Its relative error is below 2^-51, so for
  // |x w / q| < 2^48 it is within 0.1 of x w / q and the result x w - qt q
  // lies in (-0.6 q, 0.6 q) with no correction, exactly (every intermediate
  // is an integer below 2^53).
  __device__ __forceinline__ static T shoup_bal(T x, T w, T wc, T q) {
    const T h = x * w;
    const T l = fma(x, w, -h);
    const T qt = rint(x * wc);
    return fma(-qt, q, h) + l;
  }
  __device__ __forceinline__ static T mul_qinv_bal(T x, T w, T q, T qinv) {
    const T h = x * w;
    const T l = fma(x, w, -h);
    const T qt = rint(h * qinv);
    return fma(-qt, q, h) + l;
  }
  // x - rint(x / q) q for an integer |x| < 2^50: in (-0.51 q, 0.51 q), exact.
  __device__ __forceinline__ static T reduce_bal(T x, T q, T qinv) { return fma(-rint(x * qinv), q, x); }
  // A balanced value to the lazy unsigned range [0, 2q) (|x| < 2^50).
  __device__ __forceinline__ static T to_lazy(T x, T q, T qinv) {
    const T r = reduce_bal(x, q, qinv);
    return r < 0.0 ? r + q : r;
  }
};

template <typename T>
__device__ __forceinline__ T csub(T x, T m) {
  return x >= m ? x - m : x;
}

// Per-prime constants, one entry per row of the full level-zero [Q | P] chain.
template <typename T>
struct PrimeInfo {
  T q;
  T twice_q;
  T neg_inv;      // -q^{-1} mod R
  T r2;           // R^2 mod q
  T rmod, rmod_s;           // R mod q (standard -> Montgomery), Shoup companion
  T one_s;                  // floor(2^W / q): Shoup companion of w = 1
  T ninv, ninv_s;           // N^{-1} mod q
  T ninv_rinv, ninv_rinv_s; // N^{-1} R^{-1} mod q (Montgomery NTT -> standard)
  T rinv, rinv_s;           // R^{-1} mod q (Montgomery -> standard)
};

template <typename T>
struct alignas(2 * sizeof(T)) TwPair {
  T w;
  T wp;
};

// Reduce any word to [0, q) through Shoup with w = 1.
template <typename T>
__device__ __forceinline__ T reduce_any(T x, const PrimeInfo<T>& p) {
  return csub(Word<T>::shoup(x, T(1), p.one_s, p.q), p.q);
}

}  // namespace fhb
