// Operator-level kernels: the reference's custom-op kernels, one launch per op,
// taking the reference's own operands (the [8, limb] parameter rows, the
// mixed-radix and ModDown tables, index maps) instead of a context.
//
// These back the CUDA registrations of the reference's schemas
// (fhelium_b200/torch_ops.py) so that code written against
// torch.ops.fhelium_{rns,ckks}_ops runs unchanged on B200.  The fused entry
// points of fhb_capi.cu remain the fast path; here every op reads and writes
// HBM once and is bound by it.
//
// Representation of every output follows the reference's CPU kernels (the
// same integers; the reference's CUDA kernels return the same residues, lazy
// where noted):
//   montgomery_mul          canonical     csrc/ops/common/cpu/montgomery.h:124-143
//   add_lazy / sub_lazy     [0, 2q)       csrc/ops/common/cuda/montgomery.cuh:112-128
//   add/sub_canonical       [0, q)        csrc/ops/rns/cpu/rns_canonical_arithmetic_cpu.cpp:69-88
//   to/from_montgomery_     canonical     csrc/ops/rns/cpu/rns_arithmetic_cpu.cpp:181-184
//   canonicalize / center / shift_positive  csrc/ops/common/cpu/montgomery.h:197-214
//
// Operand addressing: every residue operand is [batch, rows, n] with rows n
// words apart and coefficients contiguous; its batch stride (in words) is
// passed separately, so limb slices of a larger tensor need no copy.
#include <cstdint>
#include <initializer_list>
#include <string>
#include <vector>

#include "fhb200.h"
#include "fhb_arith.cuh"
#include "fhb_context.h"

namespace fhb {
namespace {

constexpr int kOpThreads = 256;
constexpr int kMaxDecomposeRows = 8;
constexpr int kMaxModDownP = 16;

// Constants of parameter column j (csrc/ops/common/rns_parameters.h:6-16):
// rows {2q, q_lo, q_hi, -q^-1 lo, -q^-1 hi, R^2, Delta R^2, N^-1 R}, the
// split halves joined at bit W/2 - 1 (31 for int64 words, 15 for int32).
template <typename T>
struct ColumnPrime {
  T q, twice_q, neg_inv, r2;
};

template <typename T>
__device__ __forceinline__ ColumnPrime<T> column_prime(const T* params, int64_t ps, int64_t j) {
  constexpr int half = Word<T>::kRadixBits / 2;
  ColumnPrime<T> p;
  p.twice_q = params[j];
  p.q = params[ps + j] + (params[2 * ps + j] << half);
  p.neg_inv = params[3 * ps + j] + (params[4 * ps + j] << half);
  p.r2 = params[5 * ps + j];
  return p;
}

template <typename T>
__device__ __forceinline__ T mont_canonical(T a, T b, T q, T neg_inv) {
  return csub(Word<T>::mont(a, b, q, neg_inv), q);
}

// Representative of a signed value in [0, q).
template <typename T>
__device__ __forceinline__ T canon_signed(int64_t v, T q) {
  int64_t c = v % static_cast<int64_t>(q);
  if (c < 0) c += static_cast<int64_t>(q);
  return static_cast<T>(c);
}

template <typename T>
__device__ __forceinline__ T add_lazy2(T a, T b, T twice_q) {
  const T s = a + b;
  return s < twice_q ? s : s - twice_q;
}

template <typename T>
__device__ __forceinline__ T sub_lazy2(T a, T b, T twice_q) {
  const T d = a + twice_q - b;
  return d < twice_q ? d : d - twice_q;
}

template <typename T>
using S = typename std::conditional<sizeof(T) == 8, int64_t, int32_t>::type;

// Grid: x = coefficient blocks, y = row, z = batch (looped past 65535).
#define FHB_OP_INDEX                                                      \
  const int64_t k = int64_t(blockIdx.x) * kOpThreads + threadIdx.x;     \
  const int row = blockIdx.y;                                             \
  if (k >= n) return;

// Vectorised element-wise kernels: each thread owns V consecutive
// coefficients of one row (16-byte loads and stores when V > 1) and walks the
// batch items of its z-slice, so the row's constants and the index arithmetic
// are paid once per thread rather than once per element.
#define FHB_OP_VINDEX                                                         \
  const int64_t k = (int64_t(blockIdx.x) * kOpThreads + threadIdx.x) * V;   \
  const int row = blockIdx.y;                                                 \
  if (k >= n) return;

template <typename T, int V>
struct alignas(V * sizeof(T) >= 16 ? 16 : sizeof(T)) Vec {
  T v[V];
};

template <typename T, int V>
__device__ __forceinline__ Vec<T, V> ldv(const T* p) {
  Vec<T, V> r;
  if constexpr (V * sizeof(T) == 16) {
    *reinterpret_cast<uint4*>(r.v) = *reinterpret_cast<const uint4*>(p);
  } else {
#pragma unroll
    for (int i = 0; i < V; ++i) r.v[i] = p[i];
  }
  return r;
}

template <typename T, int V>
__device__ __forceinline__ void stv(T* p, const Vec<T, V>& r) {
  if constexpr (V * sizeof(T) == 16) {
    *reinterpret_cast<uint4*>(p) = *reinterpret_cast<const uint4*>(r.v);
  } else {
#pragma unroll
    for (int i = 0; i < V; ++i) p[i] = r.v[i];
  }
}

// Representative in [0, q) of a signed value; one or two corrections for the
// values that occur (|v| < 2q), the general remainder otherwise.
template <typename T>
__device__ __forceinline__ T canon_near(int64_t v, T q) {
  const int64_t qq = static_cast<int64_t>(q);
  if (v >= -2 * qq && v < 2 * qq) {
    if (v < 0) v += 2 * qq;
    if (v >= qq) v -= qq;
    return static_cast<T>(v);
  }
  return canon_signed<T>(v, q);
}

template <typename T, int OP>
__device__ __forceinline__ T binary_op(T x, T y, const ColumnPrime<T>& p) {
  if constexpr (OP == 0) return mont_canonical(x, y, p.q, p.neg_inv);
  if constexpr (OP == 1) return add_lazy2(x, y, p.twice_q);
  if constexpr (OP == 2) return sub_lazy2(x, y, p.twice_q);
  if constexpr (OP == 3) return csub(add_lazy2(x, y, p.twice_q), p.q);
  return csub(sub_lazy2(x, y, p.twice_q), p.q);
}

template <typename T, int OP, int V>
__global__ void k_op_binary(const T* __restrict__ a, int64_t as, const T* __restrict__ b, int64_t bs,
                            T* __restrict__ out, int64_t os, int64_t batch, int64_t n, const T* __restrict__ params,
                            int64_t ps) {
  FHB_OP_VINDEX
  const ColumnPrime<T> p = column_prime(params, ps, row);
  const int64_t off = row * n + k;
  for (int64_t bi = blockIdx.z; bi < batch; bi += gridDim.z) {
    const Vec<T, V> x = ldv<T, V>(a + bi * as + off);
    const Vec<T, V> y = ldv<T, V>(b + bi * bs + off);
    Vec<T, V> r;
#pragma unroll
    for (int i = 0; i < V; ++i) r.v[i] = binary_op<T, OP>(x.v[i], y.v[i], p);
    stv<T, V>(out + bi * os + off, r);
  }
}

template <typename T, int OP>
__device__ __forceinline__ T unary_op(T v, const ColumnPrime<T>& p) {
  if constexpr (OP == 0) return mont_canonical(v, p.r2, p.q, p.neg_inv);
  if constexpr (OP == 1) return mont_canonical(v, T(1), p.q, p.neg_inv);
  if constexpr (OP == 2) return v < p.q ? v : v - p.q;
  if constexpr (OP == 3) return static_cast<S<T>>(v) <= static_cast<S<T>>(p.q >> 1) ? v : T(v - p.q);
  return v + p.q;
}

template <typename T, int OP, int V>
__global__ void k_op_unary(T* __restrict__ x, int64_t xs, int64_t batch, int64_t n, const T* __restrict__ params,
                           int64_t ps) {
  FHB_OP_VINDEX
  const ColumnPrime<T> p = column_prime(params, ps, row);
  const int64_t off = row * n + k;
  for (int64_t bi = blockIdx.z; bi < batch; bi += gridDim.z) {
    Vec<T, V> r = ldv<T, V>(x + bi * xs + off);
#pragma unroll
    for (int i = 0; i < V; ++i) r.v[i] = unary_op<T, OP>(r.v[i], p);
    stv<T, V>(x + bi * xs + off, r);
  }
}

template <typename T>
__global__ void k_op_lift_centered(const T* __restrict__ coeffs, int64_t cs, T* __restrict__ out, int64_t os,
                                   int64_t batch, int64_t n, const T* __restrict__ twice_modulus) {
  FHB_OP_INDEX
  const T q = twice_modulus[row] >> 1;
  for (int64_t bi = blockIdx.z; bi < batch; bi += gridDim.z) out[bi * os + row * n + k] = coeffs[bi * cs + k] + q;
}

// Garner mixed-radix digits of one hybrid digit of `rows` primes
// (csrc/ops/rns/cpu/rns_arithmetic_cpu.cpp:482-615): digit 0 is the first
// residue, each next digit (x_r - partial_r) * normaliser_r, and each new
// digit is propagated into the partial sums of the rows after it.  Digits are
// canonical; partial sums are kept reduced modulo their row's prime (the
// digit depends only on x_r - partial_r mod q_r).
template <typename T>
__global__ void k_op_mixed_radix_decompose(const T* __restrict__ src, int64_t ss, T* __restrict__ out, int64_t os,
                                           int64_t batch, int rows, int64_t n, const T* __restrict__ normalizers,
                                           const T* __restrict__ propagation, int64_t prop_stride,
                                           const T* __restrict__ q_lo, const T* __restrict__ q_hi,
                                           const T* __restrict__ nq_lo, const T* __restrict__ nq_hi) {
  const int64_t k = int64_t(blockIdx.x) * kOpThreads + threadIdx.x;
  if (k >= n) return;
  constexpr int half = Word<T>::kRadixBits / 2;
  T q[kMaxDecomposeRows], ni[kMaxDecomposeRows];
  for (int r = 0; r < rows; ++r) {
    q[r] = q_lo[r] + (q_hi[r] << half);
    ni[r] = nq_lo[r] + (nq_hi[r] << half);
  }
  for (int64_t bi = blockIdx.z; bi < batch; bi += gridDim.z) {
    const T* s = src + bi * ss + k;
    int64_t digit[kMaxDecomposeRows];
    T first = s[0];
    if (first >= q[0]) first -= q[0];
    for (int r = 0; r < rows; ++r) digit[r] = static_cast<int64_t>(r == 0 ? first : canon_near<T>(first, q[r]));
    for (int step = 0; step + 1 < rows; ++step) {
      const int r = step + 1;
      const int64_t x = static_cast<int64_t>(static_cast<S<T>>(s[r * n]));
      const T d = mont_canonical(canon_near<T>(x - digit[r], q[r]),
                                 canon_near<T>(static_cast<S<T>>(normalizers[step]), q[r]), q[r], ni[r]);
      digit[r] = static_cast<int64_t>(d);
      // partial sums kept in [0, q_t): only their residue mod q_t is used
      for (int t = r + 1; t < rows; ++t)
        digit[t] = static_cast<int64_t>(csub(static_cast<T>(digit[t]) +
                                                 mont_canonical(d, propagation[step * prop_stride + t], q[t], ni[t]),
                                             q[t]));
    }
    T* o = out + bi * os + k;
    for (int r = 0; r < rows; ++r) o[r * n] = static_cast<T>(digit[r]);
  }
}

// Exact basis extension sum_r d_r (M_r mod p_j) into Montgomery form, lazy
// (csrc/ops/rns/cpu/rns_arithmetic_cpu.cpp:616-700): d_0 R^2 reduced, then
// each further digit's product added with one 2q correction.
template <typename T, int V>
__global__ void k_op_basis_extend(const T* __restrict__ digits, int64_t ds, int digit_rows, T* __restrict__ out,
                                  int64_t os, int64_t batch, int64_t n, const T* __restrict__ coeffs,
                                  int64_t coeff_stride, const T* __restrict__ params, int64_t ps) {
  FHB_OP_VINDEX
  const ColumnPrime<T> p = column_prime(params, ps, row);
  for (int64_t bi = blockIdx.z; bi < batch; bi += gridDim.z) {
    const T* d = digits + bi * ds + k;
    Vec<T, V> v = ldv<T, V>(d);
#pragma unroll
    for (int i = 0; i < V; ++i) v.v[i] = mont_canonical(v.v[i], p.r2, p.q, p.neg_inv);
    for (int r = 1; r < digit_rows; ++r) {
      const T c = coeffs[(r - 1) * coeff_stride + row];
      const Vec<T, V> x = ldv<T, V>(d + r * n);
#pragma unroll
      for (int i = 0; i < V; ++i) v.v[i] = add_lazy2(v.v[i], mont_canonical(x.v[i], c, p.q, p.neg_inv), p.twice_q);
    }
    stv<T, V>(out + bi * os + row * n + k, v);
  }
}

// acc_c += digit * key[c][key_row_start + row], c = 0, 1
// (csrc/ops/ckks/cpu/ckks_cpu.cpp:605-700).
template <typename T, int V>
__global__ void k_op_keyswitch_accumulate(T* __restrict__ acc0, int64_t a0s, T* __restrict__ acc1, int64_t a1s,
                                          const T* __restrict__ digit, int64_t ds, const T* __restrict__ key,
                                          int64_t key_component_stride, int64_t key_row_start, int64_t batch,
                                          int64_t n, const T* __restrict__ params, int64_t ps) {
  FHB_OP_VINDEX
  const ColumnPrime<T> p = column_prime(params, ps, row);
  const Vec<T, V> k0 = ldv<T, V>(key + (key_row_start + row) * n + k);
  const Vec<T, V> k1 = ldv<T, V>(key + key_component_stride + (key_row_start + row) * n + k);
  const int64_t off = row * n + k;
  for (int64_t bi = blockIdx.z; bi < batch; bi += gridDim.z) {
    const Vec<T, V> v = ldv<T, V>(digit + bi * ds + off);
    Vec<T, V> x0 = ldv<T, V>(acc0 + bi * a0s + off);
    Vec<T, V> x1 = ldv<T, V>(acc1 + bi * a1s + off);
#pragma unroll
    for (int i = 0; i < V; ++i) {
      x0.v[i] = add_lazy2(x0.v[i], mont_canonical(v.v[i], k0.v[i], p.q, p.neg_inv), p.twice_q);
      x1.v[i] = add_lazy2(x1.v[i], mont_canonical(v.v[i], k1.v[i], p.q, p.neg_inv), p.twice_q);
    }
    stv<T, V>(acc0 + bi * a0s + off, x0);
    stv<T, V>(acc1 + bi * a1s + off, x1);
  }
}

// ModDown Q P -> Q by sequential division by each special prime, canonical
// output (csrc/ops/ckks/cpu/ckks_cpu.cpp:474-601): the P residues are first
// turned into mixed-radix form over P (highest prime first), then each Q
// residue subtracts and divides by one P prime at a time.  `inverse` is the
// reference's [P, inv_stride] table of Montgomery-form inverses.
template <typename T>
__global__ void k_op_moddown(const T* __restrict__ qr, int64_t qs, const T* __restrict__ pr, int64_t prs,
                             T* __restrict__ out, int64_t os, int64_t batch, int qn, int pn, int64_t n,
                             const T* __restrict__ inverse, int64_t inv_stride, const T* __restrict__ params,
                             int64_t ps) {
  FHB_OP_INDEX
  (void)row;
  for (int64_t bi = blockIdx.z; bi < batch; bi += gridDim.z) {
    T chain[kMaxModDownP];
    for (int r = 0; r < pn; ++r) chain[r] = pr[bi * prs + r * n + k];
    for (int r = pn - 2; r >= 0; --r) {
      const ColumnPrime<T> p = column_prime(params, ps, qn + r);
      T v = chain[r];
      for (int lower = pn - 1; lower > r; --lower) {
        const T diff = sub_lazy2(v, chain[lower], p.twice_q);   // [0, 2q)
        const T inv = canon_near<T>(static_cast<S<T>>(inverse[(pn - lower - 1) * inv_stride + r + qn]), p.q);
        v = mont_canonical(csub(diff, p.q), inv, p.q, p.neg_inv);
      }
      chain[r] = v;
    }
    for (int i = 0; i < qn; ++i) {
      const ColumnPrime<T> p = column_prime(params, ps, i);
      T v = mont_canonical(qr[bi * qs + i * n + k], p.r2, p.q, p.neg_inv);
      for (int r = pn - 1; r >= 0; --r) {
        const T pm = mont_canonical(chain[r], p.r2, p.q, p.neg_inv);
        v = sub_lazy2(v, pm, p.twice_q);                            // [0, 2q)
        const T inv = canon_near<T>(static_cast<S<T>>(inverse[(pn - r - 1) * inv_stride + i]), p.q);
        v = mont_canonical(csub(v, p.q), inv, p.q, p.neg_inv);
      }
      v = mont_canonical(v, T(1), p.q, p.neg_inv);
      out[bi * os + i * n + k] = v < p.q ? v : v - p.q;
    }
  }
}

// Rescale by the dropped leading prime: (x_j - x_drop) * q_drop^-1, plus one
// when rounding to nearest and x_drop > floor(q_drop / 2)
// (csrc/ops/ckks/cpu/ckks_cpu.cpp:203-262).  Canonical output.
template <typename T, int V>
__global__ void k_op_rescale(const T* __restrict__ rem, int64_t rs, const T* __restrict__ dropped, int64_t ds,
                             T* __restrict__ out, int64_t os, int64_t batch, int64_t n,
                             const T* __restrict__ inverse_mont, const T* __restrict__ params, int64_t ps,
                             int64_t half_drop, int nearest) {
  FHB_OP_VINDEX
  const ColumnPrime<T> p = column_prime(params, ps, row);
  const T inv = canon_near<T>(static_cast<S<T>>(inverse_mont[row]), p.q);
  const int64_t off = row * n + k;
  for (int64_t bi = blockIdx.z; bi < batch; bi += gridDim.z) {
    const Vec<T, V> d = ldv<T, V>(dropped + bi * ds + k);
    const Vec<T, V> x = ldv<T, V>(rem + bi * rs + off);
    Vec<T, V> r;
#pragma unroll
    for (int i = 0; i < V; ++i) {
      const int64_t dv = static_cast<S<T>>(d.v[i]);
      T quo = mont_canonical(canon_near<T>(static_cast<int64_t>(static_cast<S<T>>(x.v[i])) - dv, p.q), inv, p.q,
                             p.neg_inv);
      if (nearest && dv > half_drop) quo += 1;
      r.v[i] = quo < p.q ? quo : quo - p.q;
    }
    stv<T, V>(out + bi * os + off, r);
  }
}

// Coefficient-domain Galois automorphism from the reference's index/sign maps
// (csrc/ops/ckks/cpu/ckks_cpu.cpp:287-380): out[k] = +-in[src[k]], canonical.
template <typename T>
__global__ void k_op_coefficient_automorphism(const T* __restrict__ in, int64_t is, T* __restrict__ out, int64_t os,
                                              int64_t batch, int64_t n, const int32_t* __restrict__ src,
                                              const int8_t* __restrict__ sign, const T* __restrict__ twice_moduli) {
  FHB_OP_INDEX
  const int64_t q = static_cast<int64_t>(twice_moduli[row] >> 1);
  const int32_t from = src[k];
  const bool negate = sign[k] == -1;
  for (int64_t bi = blockIdx.z; bi < batch; bi += gridDim.z) {
    int64_t v = static_cast<S<T>>(in[bi * is + row * n + from]);
    if (negate) v = -v;
    v += q;
    out[bi * os + row * n + k] = static_cast<T>(v < q ? v : v - q);
  }
}

// NTT-domain automorphism: a gather by the reference's index map
// (csrc/ops/ckks/cpu/ckks_cpu.cpp:382-472).
template <typename T>
__global__ void k_op_ntt_automorphism(const T* __restrict__ in, int64_t is, T* __restrict__ out, int64_t os,
                                      int64_t batch, int64_t n, const int32_t* __restrict__ src) {
  FHB_OP_INDEX
  const int32_t from = src[k];
  for (int64_t bi = blockIdx.z; bi < batch; bi += gridDim.z) out[bi * os + row * n + k] = in[bi * is + row * n + from];
}

// Index of the stored plaintext word for coefficient k: 0 dense, 1 cyclic
// repetition (k mod U), 2 contiguous repetition (k / (N / U)), 3 strided
// support (every (N / U)-th coefficient stored, the rest implicit)
// (csrc/ops/common/cuda/repetition.cuh:69-86, csrc/ops/ckks/cuda/plaintext_cuda.cu:93-114).
__device__ __forceinline__ int64_t plaintext_index(int layout, int64_t k, int64_t unique_mask, int shift) {
  switch (layout) {
    case 1: return k & unique_mask;
    case 2: return k >> shift;
    case 3: return (k & unique_mask) == 0 ? (k >> shift) : -1;
    default: return k;
  }
}

// out = lhs * rhs[index(k)] (Montgomery, canonical): montgomery_mul with a
// repeated (compressed) right operand.
template <typename T>
__global__ void k_op_mul_compressed(int layout, const T* __restrict__ a, int64_t as, const T* __restrict__ b,
                                    int64_t bs, int64_t unique, int64_t unique_mask, int shift, T* __restrict__ out,
                                    int64_t os, int64_t batch, int64_t n, const T* __restrict__ params, int64_t ps) {
  FHB_OP_INDEX
  const ColumnPrime<T> p = column_prime(params, ps, row);
  const int64_t idx = plaintext_index(layout, k, unique_mask, shift);
  for (int64_t bi = blockIdx.z; bi < batch; bi += gridDim.z)
    out[bi * os + row * n + k] =
        mont_canonical(a[bi * as + row * n + k], b[bi * bs + row * unique + idx], p.q, p.neg_inv);
}

// Plaintext addition to a standard-form ciphertext component: c + p R^-1,
// canonical, p a coefficient-domain Montgomery residue
// (csrc/ops/ckks/cuda/plaintext_cuda.cu:1-47).  Strided layout: coefficients
// off the support take implicit[b, row].
template <typename T>
__global__ void k_op_add_plaintext(int layout, const T* __restrict__ ct, int64_t cs, const T* __restrict__ pt,
                                   int64_t pbs, int64_t extent, int64_t unique_mask, int shift,
                                   const T* __restrict__ implicit, int64_t ibs, T* __restrict__ out, int64_t os,
                                   int64_t batch, int64_t n, const T* __restrict__ params, int64_t ps) {
  FHB_OP_INDEX
  const ColumnPrime<T> p = column_prime(params, ps, row);
  const int64_t idx = plaintext_index(layout, k, unique_mask, shift);
  for (int64_t bi = blockIdx.z; bi < batch; bi += gridDim.z) {
    const T pv = idx >= 0 ? pt[bi * pbs + row * extent + idx] : implicit[bi * ibs + row];
    T v = mont_canonical(ct[bi * cs + row * n + k], p.r2, p.q, p.neg_inv);
    v = add_lazy2(v, pv, p.twice_q);
    out[bi * os + row * n + k] = mont_canonical(v, T(1), p.q, p.neg_inv);
  }
}

// out = x * scalars[row] (Montgomery, canonical)
// (csrc/ops/rns/cuda/rns_arithmetic_cuda.cu:175-191).
template <typename T>
__global__ void k_op_mul_row_scalars(const T* __restrict__ x, int64_t xs, T* __restrict__ out, int64_t os,
                                     int64_t batch, int64_t n, const T* __restrict__ scalars,
                                     const T* __restrict__ params, int64_t ps) {
  FHB_OP_INDEX
  const ColumnPrime<T> p = column_prime(params, ps, row);
  const T s = scalars[row];
  for (int64_t bi = blockIdx.z; bi < batch; bi += gridDim.z)
    out[bi * os + row * n + k] = mont_canonical(x[bi * xs + row * n + k], s, p.q, p.neg_inv);
}

int log2_exact(int64_t v) {
  int s = 0;
  while ((int64_t{1} << s) < v) ++s;
  return (int64_t{1} << s) == v ? s : -1;
}

// Vector kernels: V coefficients per thread; z-slices of the batch only as
// many as needed for about 16 blocks per SM.
dim3 op_grid_v(int64_t n, int v, int64_t rows, int64_t batch) {
  const int64_t xb = (n / v + kOpThreads - 1) / kOpThreads;
  int64_t z = (148 * 16 + xb * rows - 1) / (xb * rows);
  if (z > batch) z = batch;
  if (z > 65535) z = 65535;
  if (z < 1) z = 1;
  return dim3(static_cast<unsigned>(xb), static_cast<unsigned>(rows), static_cast<unsigned>(z));
}

// 16-byte vectors are used when every operand start and batch stride, and n,
// are whole vectors.
template <typename T>
bool vec_ok(int64_t n, std::initializer_list<const void*> ptrs, std::initializer_list<int64_t> strides) {
  constexpr int64_t V = 16 / sizeof(T);
  if (n % V) return false;
  for (const void* p : ptrs)
    if (reinterpret_cast<uintptr_t>(p) % 16) return false;
  for (int64_t st : strides)
    if (st % V) return false;
  return true;
}

dim3 op_grid(int64_t n, int64_t rows, int64_t batch) {
  const int64_t z = batch < 65535 ? batch : 65535;
  return dim3(static_cast<unsigned>((n + kOpThreads - 1) / kOpThreads), static_cast<unsigned>(rows),
              static_cast<unsigned>(z > 0 ? z : 1));
}

int launch_status() {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(1000 + int(e), std::string("kernel launch: ") + cudaGetErrorString(e));
  return 0;
}

int check_shape(int bits, int64_t batch, int64_t rows, int64_t n) {
  if (bits != 64 && bits != 32) return fail(-2, "residue_bits must be 64 or 32");
  if (batch < 0 || rows < 0 || n < 0) return fail(-4, "negative size");
  if (rows > 65535) return fail(-4, "more than 65535 rows");
  if (n > (int64_t{1} << 17)) return fail(-4, "ring degree above 2^17");
  return 0;
}

bool empty(int64_t batch, int64_t rows, int64_t n) { return batch == 0 || rows == 0 || n == 0; }

#define FHB_NONNULL(p) \
  if (!(p)) return fail(-1, #p " is NULL");

#define FHB_DISPATCH(bits, ...)       \
  if ((bits) == 64) {                 \
    using T = uint64_t;               \
    __VA_ARGS__;                      \
  } else {                            \
    using T = uint32_t;               \
    __VA_ARGS__;                      \
  }

}  // namespace
}  // namespace fhb

using fhb::fail;

// Launch of one compile-time op at vector width VW or 1 (names of the calling entry point).
#define FHB_BIN(OPN)                                                                                            \
  case OPN:                                                                                                    \
    if (vec)                                                                                                   \
      fhb::k_op_binary<T, OPN, VW><<<g, fhb::kOpThreads, 0, st>>>((const T*)lhs, lhs_batch_stride, (const T*)rhs, \
                                                                  rhs_batch_stride, (T*)out, out_batch_stride,  \
                                                                  batch, n, (const T*)params, param_row_stride); \
    else                                                                                                       \
      fhb::k_op_binary<T, OPN, 1><<<g, fhb::kOpThreads, 0, st>>>((const T*)lhs, lhs_batch_stride, (const T*)rhs,  \
                                                                 rhs_batch_stride, (T*)out, out_batch_stride,   \
                                                                 batch, n, (const T*)params, param_row_stride); \
    break;

#define FHB_UN(OPN)                                                                                             \
  case OPN:                                                                                                    \
    if (vec)                                                                                                   \
      fhb::k_op_unary<T, OPN, VW><<<g, fhb::kOpThreads, 0, st>>>((T*)residues, batch_stride, batch, n,           \
                                                                 (const T*)params, param_row_stride);           \
    else                                                                                                       \
      fhb::k_op_unary<T, OPN, 1><<<g, fhb::kOpThreads, 0, st>>>((T*)residues, batch_stride, batch, n,            \
                                                                (const T*)params, param_row_stride);            \
    break;


extern "C" {

int fhb_op_rns_binary(int residue_bits, int op, const void* lhs, int64_t lhs_batch_stride, const void* rhs,
                      int64_t rhs_batch_stride, void* out, int64_t out_batch_stride, int64_t batch, int rows,
                      int64_t n, const void* params, int64_t param_row_stride, fhb_stream stream) {
  if (int rc = fhb::check_shape(residue_bits, batch, rows, n)) return rc;
  if (op < 0 || op > 4) return fail(-2, "unknown binary op");
  if (fhb::empty(batch, rows, n)) return 0;
  FHB_NONNULL(lhs) FHB_NONNULL(rhs) FHB_NONNULL(out) FHB_NONNULL(params)
  FHB_DISPATCH(residue_bits, {
    const bool vec = fhb::vec_ok<T>(n, {lhs, rhs, out}, {lhs_batch_stride, rhs_batch_stride, out_batch_stride});
    constexpr int VW = 16 / sizeof(T);
    const dim3 g = fhb::op_grid_v(n, vec ? VW : 1, rows, batch);
    cudaStream_t st = (cudaStream_t)stream;
    switch (op) { FHB_BIN(0) FHB_BIN(1) FHB_BIN(2) FHB_BIN(3) FHB_BIN(4) }
  })
  return fhb::launch_status();
}

int fhb_op_rns_unary(int residue_bits, int op, void* residues, int64_t batch_stride, int64_t batch, int rows,
                     int64_t n, const void* params, int64_t param_row_stride, fhb_stream stream) {
  if (int rc = fhb::check_shape(residue_bits, batch, rows, n)) return rc;
  if (op < 0 || op > 4) return fail(-2, "unknown unary op");
  if (fhb::empty(batch, rows, n)) return 0;
  FHB_NONNULL(residues) FHB_NONNULL(params)
  FHB_DISPATCH(residue_bits, {
    const bool vec = fhb::vec_ok<T>(n, {residues}, {batch_stride});
    constexpr int VW = 16 / sizeof(T);
    const dim3 g = fhb::op_grid_v(n, vec ? VW : 1, rows, batch);
    cudaStream_t st = (cudaStream_t)stream;
    switch (op) { FHB_UN(0) FHB_UN(1) FHB_UN(2) FHB_UN(3) FHB_UN(4) }
  })
  return fhb::launch_status();
}

int fhb_op_lift_centered(int residue_bits, const void* coefficients, int64_t coefficient_batch_stride, void* out,
                         int64_t out_batch_stride, int64_t batch, int rows, int64_t n, const void* twice_modulus,
                         fhb_stream stream) {
  if (int rc = fhb::check_shape(residue_bits, batch, rows, n)) return rc;
  if (fhb::empty(batch, rows, n)) return 0;
  FHB_NONNULL(coefficients) FHB_NONNULL(out) FHB_NONNULL(twice_modulus)
  FHB_DISPATCH(residue_bits,
               fhb::k_op_lift_centered<T><<<fhb::op_grid(n, rows, batch), fhb::kOpThreads, 0,
                                            (cudaStream_t)stream>>>(
                   (const T*)coefficients, coefficient_batch_stride, (T*)out, out_batch_stride, batch, n,
                   (const T*)twice_modulus))
  return fhb::launch_status();
}

int fhb_op_mixed_radix_decompose(int residue_bits, const void* source, int64_t source_batch_stride, void* out,
                                 int64_t out_batch_stride, int64_t batch, int rows, int64_t n,
                                 const void* normalizers, const void* propagation, int64_t propagation_row_stride,
                                 const void* modulus_lo, const void* modulus_hi, const void* neg_inv_modulus_lo,
                                 const void* neg_inv_modulus_hi, fhb_stream stream) {
  if (int rc = fhb::check_shape(residue_bits, batch, rows, n)) return rc;
  if (rows > fhb::kMaxDecomposeRows) return fail(-4, "a mixed-radix digit has at most 8 rows");
  if (fhb::empty(batch, rows, n)) return 0;
  FHB_NONNULL(source) FHB_NONNULL(out) FHB_NONNULL(modulus_lo) FHB_NONNULL(modulus_hi)
  FHB_NONNULL(neg_inv_modulus_lo) FHB_NONNULL(neg_inv_modulus_hi)
  if (rows > 1 && (!normalizers || !propagation)) return fail(-1, "normalizers/propagation are NULL");
  FHB_DISPATCH(residue_bits,
               fhb::k_op_mixed_radix_decompose<T><<<fhb::op_grid(n, 1, batch), fhb::kOpThreads, 0,
                                                    (cudaStream_t)stream>>>(
                   (const T*)source, source_batch_stride, (T*)out, out_batch_stride, batch, rows, n,
                   (const T*)normalizers, (const T*)propagation, propagation_row_stride, (const T*)modulus_lo,
                   (const T*)modulus_hi, (const T*)neg_inv_modulus_lo, (const T*)neg_inv_modulus_hi))
  return fhb::launch_status();
}

int fhb_op_basis_extend(int residue_bits, const void* digits, int64_t digits_batch_stride, int digit_rows,
                        void* out, int64_t out_batch_stride, int64_t batch, int destination_rows, int64_t n,
                        const void* coefficients, int64_t coefficient_row_stride, const void* params,
                        int64_t param_row_stride, fhb_stream stream) {
  if (int rc = fhb::check_shape(residue_bits, batch, destination_rows, n)) return rc;
  if (digit_rows < 1) return fail(-4, "need at least one digit row");
  if (fhb::empty(batch, destination_rows, n)) return 0;
  FHB_NONNULL(digits) FHB_NONNULL(out) FHB_NONNULL(params)
  if (digit_rows > 1 && !coefficients) return fail(-1, "coefficients is NULL");
  FHB_DISPATCH(residue_bits, {
    const bool vec = fhb::vec_ok<T>(n, {digits, out}, {digits_batch_stride, out_batch_stride});
    constexpr int VW = 16 / sizeof(T);
    const dim3 g = fhb::op_grid_v(n, vec ? VW : 1, destination_rows, batch);
    if (vec)
      fhb::k_op_basis_extend<T, VW><<<g, fhb::kOpThreads, 0, (cudaStream_t)stream>>>(
          (const T*)digits, digits_batch_stride, digit_rows, (T*)out, out_batch_stride, batch, n,
          (const T*)coefficients, coefficient_row_stride, (const T*)params, param_row_stride);
    else
      fhb::k_op_basis_extend<T, 1><<<g, fhb::kOpThreads, 0, (cudaStream_t)stream>>>(
          (const T*)digits, digits_batch_stride, digit_rows, (T*)out, out_batch_stride, batch, n,
          (const T*)coefficients, coefficient_row_stride, (const T*)params, param_row_stride);
  })
  return fhb::launch_status();
}

int fhb_op_keyswitch_accumulate(int residue_bits, void* acc0, int64_t acc0_batch_stride, void* acc1,
                                int64_t acc1_batch_stride, const void* digit, int64_t digit_batch_stride,
                                const void* key_digit, int64_t key_component_stride, int64_t key_row_start,
                                int64_t batch, int rows, int64_t n, const void* params, int64_t param_row_stride,
                                fhb_stream stream) {
  if (int rc = fhb::check_shape(residue_bits, batch, rows, n)) return rc;
  if (key_row_start < 0) return fail(-4, "negative key row start");
  if (fhb::empty(batch, rows, n)) return 0;
  FHB_NONNULL(acc0) FHB_NONNULL(acc1) FHB_NONNULL(digit) FHB_NONNULL(key_digit) FHB_NONNULL(params)
  FHB_DISPATCH(residue_bits, {
    const bool vec = fhb::vec_ok<T>(n, {acc0, acc1, digit, key_digit},
                                    {acc0_batch_stride, acc1_batch_stride, digit_batch_stride, key_component_stride});
    constexpr int VW = 16 / sizeof(T);
    const dim3 g = fhb::op_grid_v(n, vec ? VW : 1, rows, batch);
    if (vec)
      fhb::k_op_keyswitch_accumulate<T, VW><<<g, fhb::kOpThreads, 0, (cudaStream_t)stream>>>(
          (T*)acc0, acc0_batch_stride, (T*)acc1, acc1_batch_stride, (const T*)digit, digit_batch_stride,
          (const T*)key_digit, key_component_stride, key_row_start, batch, n, (const T*)params, param_row_stride);
    else
      fhb::k_op_keyswitch_accumulate<T, 1><<<g, fhb::kOpThreads, 0, (cudaStream_t)stream>>>(
          (T*)acc0, acc0_batch_stride, (T*)acc1, acc1_batch_stride, (const T*)digit, digit_batch_stride,
          (const T*)key_digit, key_component_stride, key_row_start, batch, n, (const T*)params, param_row_stride);
  })
  return fhb::launch_status();
}

int fhb_op_moddown(int residue_bits, const void* q_residues, int64_t q_batch_stride, const void* p_residues,
                   int64_t p_batch_stride, void* out, int64_t out_batch_stride, int64_t batch, int q_rows,
                   int p_rows, int64_t n, const void* inverses, int64_t inverse_row_stride, const void* params,
                   int64_t param_row_stride, fhb_stream stream) {
  if (int rc = fhb::check_shape(residue_bits, batch, q_rows, n)) return rc;
  if (p_rows < 1 || p_rows > fhb::kMaxModDownP) return fail(-4, "need 1..16 special primes");
  if (fhb::empty(batch, q_rows, n)) return 0;
  FHB_NONNULL(q_residues) FHB_NONNULL(p_residues) FHB_NONNULL(out) FHB_NONNULL(inverses) FHB_NONNULL(params)
  FHB_DISPATCH(residue_bits,
               fhb::k_op_moddown<T><<<fhb::op_grid(n, 1, batch), fhb::kOpThreads, 0, (cudaStream_t)stream>>>(
                   (const T*)q_residues, q_batch_stride, (const T*)p_residues, p_batch_stride, (T*)out,
                   out_batch_stride, batch, q_rows, p_rows, n, (const T*)inverses, inverse_row_stride,
                   (const T*)params, param_row_stride))
  return fhb::launch_status();
}

int fhb_op_rescale(int residue_bits, const void* remaining, int64_t remaining_batch_stride, const void* dropped,
                   int64_t dropped_batch_stride, void* out, int64_t out_batch_stride, int64_t batch, int rows,
                   int64_t n, const void* inverse_montgomery, const void* params, int64_t param_row_stride,
                   int64_t half_drop_prime, int nearest, fhb_stream stream) {
  if (int rc = fhb::check_shape(residue_bits, batch, rows, n)) return rc;
  if (fhb::empty(batch, rows, n)) return 0;
  FHB_NONNULL(remaining) FHB_NONNULL(dropped) FHB_NONNULL(out) FHB_NONNULL(inverse_montgomery) FHB_NONNULL(params)
  FHB_DISPATCH(residue_bits, {
    const bool vec = fhb::vec_ok<T>(n, {remaining, dropped, out},
                                    {remaining_batch_stride, dropped_batch_stride, out_batch_stride});
    constexpr int VW = 16 / sizeof(T);
    const dim3 g = fhb::op_grid_v(n, vec ? VW : 1, rows, batch);
    if (vec)
      fhb::k_op_rescale<T, VW><<<g, fhb::kOpThreads, 0, (cudaStream_t)stream>>>(
          (const T*)remaining, remaining_batch_stride, (const T*)dropped, dropped_batch_stride, (T*)out,
          out_batch_stride, batch, n, (const T*)inverse_montgomery, (const T*)params, param_row_stride,
          half_drop_prime, nearest);
    else
      fhb::k_op_rescale<T, 1><<<g, fhb::kOpThreads, 0, (cudaStream_t)stream>>>(
          (const T*)remaining, remaining_batch_stride, (const T*)dropped, dropped_batch_stride, (T*)out,
          out_batch_stride, batch, n, (const T*)inverse_montgomery, (const T*)params, param_row_stride,
          half_drop_prime, nearest);
  })
  return fhb::launch_status();
}

int fhb_op_coefficient_automorphism(int residue_bits, const void* in, int64_t in_batch_stride, void* out,
                                    int64_t out_batch_stride, int64_t batch, int rows, int64_t n,
                                    const int32_t* source_indices, const int8_t* source_sign,
                                    const void* twice_moduli, fhb_stream stream) {
  if (int rc = fhb::check_shape(residue_bits, batch, rows, n)) return rc;
  if (fhb::empty(batch, rows, n)) return 0;
  FHB_NONNULL(in) FHB_NONNULL(out) FHB_NONNULL(source_indices) FHB_NONNULL(source_sign) FHB_NONNULL(twice_moduli)
  FHB_DISPATCH(residue_bits,
               fhb::k_op_coefficient_automorphism<T><<<fhb::op_grid(n, rows, batch), fhb::kOpThreads, 0,
                                                       (cudaStream_t)stream>>>(
                   (const T*)in, in_batch_stride, (T*)out, out_batch_stride, batch, n, source_indices, source_sign,
                   (const T*)twice_moduli))
  return fhb::launch_status();
}

int fhb_op_ntt_automorphism(int residue_bits, const void* in, int64_t in_batch_stride, void* out,
                            int64_t out_batch_stride, int64_t batch, int rows, int64_t n,
                            const int32_t* source_indices, fhb_stream stream) {
  if (int rc = fhb::check_shape(residue_bits, batch, rows, n)) return rc;
  if (fhb::empty(batch, rows, n)) return 0;
  FHB_NONNULL(in) FHB_NONNULL(out) FHB_NONNULL(source_indices)
  FHB_DISPATCH(residue_bits,
               fhb::k_op_ntt_automorphism<T><<<fhb::op_grid(n, rows, batch), fhb::kOpThreads, 0,
                                               (cudaStream_t)stream>>>(
                   (const T*)in, in_batch_stride, (T*)out, out_batch_stride, batch, n, source_indices))
  return fhb::launch_status();
}

int fhb_op_mul_compressed(int residue_bits, int layout, const void* lhs, int64_t lhs_batch_stride,
                          const void* compressed_rhs, int64_t rhs_batch_stride, int64_t unique, void* out,
                          int64_t out_batch_stride, int64_t batch, int rows, int64_t n, const void* params,
                          int64_t param_row_stride, fhb_stream stream) {
  if (int rc = fhb::check_shape(residue_bits, batch, rows, n)) return rc;
  if (layout != 1 && layout != 2) return fail(-2, "layout must be 1 (cyclic) or 2 (contiguous)");
  const int un = fhb::log2_exact(unique), nn = fhb::log2_exact(n);
  if (un < 0 || nn < 0 || unique >= n) return fail(-4, "unique count must be a power of two below the ring dimension");
  if (fhb::empty(batch, rows, n)) return 0;
  FHB_NONNULL(lhs) FHB_NONNULL(compressed_rhs) FHB_NONNULL(out) FHB_NONNULL(params)
  FHB_DISPATCH(residue_bits,
               fhb::k_op_mul_compressed<T><<<fhb::op_grid(n, rows, batch), fhb::kOpThreads, 0,
                                             (cudaStream_t)stream>>>(
                   layout, (const T*)lhs, lhs_batch_stride, (const T*)compressed_rhs, rhs_batch_stride, unique,
                   unique - 1, nn - un, (T*)out, out_batch_stride, batch, n, (const T*)params, param_row_stride))
  return fhb::launch_status();
}

int fhb_op_add_plaintext(int residue_bits, int layout, const void* ciphertext, int64_t ciphertext_batch_stride,
                         const void* plaintext, int64_t plaintext_batch_stride, int64_t plaintext_extent,
                         const void* implicit_plaintext, int64_t implicit_batch_stride, void* out,
                         int64_t out_batch_stride, int64_t batch, int rows, int64_t n, const void* params,
                         int64_t param_row_stride, fhb_stream stream) {
  if (int rc = fhb::check_shape(residue_bits, batch, rows, n)) return rc;
  if (layout < 0 || layout > 3) return fail(-2, "layout must be 0 (dense), 1 (cyclic), 2 (contiguous) or 3 (strided)");
  const int un = fhb::log2_exact(plaintext_extent), nn = fhb::log2_exact(n);
  if (layout == 0 && plaintext_extent != n) return fail(-4, "a dense plaintext has N coefficients per row");
  if (layout != 0 && (un < 0 || nn < 0 || plaintext_extent > n || (layout != 3 && plaintext_extent == n)))
    return fail(-4, "plaintext extent must be a power of two below the ring dimension");
  if (layout == 3 && !implicit_plaintext) return fail(-1, "implicit_plaintext is NULL");
  if (fhb::empty(batch, rows, n)) return 0;
  FHB_NONNULL(ciphertext) FHB_NONNULL(plaintext) FHB_NONNULL(out) FHB_NONNULL(params)
  // cyclic: k mod U; contiguous: k >> log2(N/U); strided: support mask N/U - 1, shift log2(N/U)
  const int64_t mask = layout == 1 ? plaintext_extent - 1 : layout == 3 ? (n / plaintext_extent) - 1 : 0;
  const int shift = layout >= 2 ? nn - un : 0;
  FHB_DISPATCH(residue_bits,
               fhb::k_op_add_plaintext<T><<<fhb::op_grid(n, rows, batch), fhb::kOpThreads, 0,
                                            (cudaStream_t)stream>>>(
                   layout, (const T*)ciphertext, ciphertext_batch_stride, (const T*)plaintext,
                   plaintext_batch_stride, plaintext_extent, mask, shift, (const T*)implicit_plaintext,
                   implicit_batch_stride, (T*)out, out_batch_stride, batch, n, (const T*)params, param_row_stride))
  return fhb::launch_status();
}

int fhb_op_mul_row_scalars(int residue_bits, const void* residues, int64_t residues_batch_stride, void* out,
                           int64_t out_batch_stride, int64_t batch, int rows, int64_t n, const void* row_scalars,
                           const void* params, int64_t param_row_stride, fhb_stream stream) {
  if (int rc = fhb::check_shape(residue_bits, batch, rows, n)) return rc;
  if (fhb::empty(batch, rows, n)) return 0;
  FHB_NONNULL(residues) FHB_NONNULL(out) FHB_NONNULL(row_scalars) FHB_NONNULL(params)
  FHB_DISPATCH(residue_bits,
               fhb::k_op_mul_row_scalars<T><<<fhb::op_grid(n, rows, batch), fhb::kOpThreads, 0,
                                              (cudaStream_t)stream>>>(
                   (const T*)residues, residues_batch_stride, (T*)out, out_batch_stride, batch, n,
                   (const T*)row_scalars, (const T*)params, param_row_stride))
  return fhb::launch_status();
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Transform contexts: the NTT schemas take a parameter-row slice, not a chain.
namespace {

using u128 = unsigned __int128;

uint64_t mulmod64(uint64_t a, uint64_t b, uint64_t m) { return static_cast<uint64_t>((u128)a * b % m); }

uint64_t powmod64(uint64_t b, uint64_t e, uint64_t m) {
  uint64_t r = 1 % m;
  b %= m;
  for (; e; e >>= 1) {
    if (e & 1) r = mulmod64(r, b, m);
    b = mulmod64(b, b, m);
  }
  return r;
}

// Deterministic Miller-Rabin for 64-bit integers (the first twelve prime
// bases suffice below 3.3e24).
bool is_prime64(uint64_t n) {
  if (n < 2) return false;
  static const uint64_t bases[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
  for (uint64_t p : bases)
    if (n % p == 0) return n == p;
  uint64_t d = n - 1;
  int s = 0;
  while (!(d & 1)) d >>= 1, ++s;
  for (uint64_t a : bases) {
    uint64_t x = powmod64(a, d, n);
    if (x == 1 || x == n - 1) continue;
    bool composite = true;
    for (int i = 1; i < s && composite; ++i) {
      x = mulmod64(x, x, n);
      if (x == n - 1) composite = false;
    }
    if (composite) return false;
  }
  return true;
}

}  // namespace

extern "C" int fhb_context_create_transform(int residue_bits, int log_n, const uint64_t* moduli, int count,
                                            int device, fhb_context** out) {
  if (!moduli || !out) return fail(-1, "NULL argument");
  if (count < 1) return fail(-2, "need at least one prime");
  if (residue_bits != 64 && residue_bits != 32) return fail(-2, "residue_bits must be 64 or 32");
  if (log_n < 1 || log_n > 20) return fail(-7, "log_n outside the supported 12..17");
  // One auxiliary special prime completes the chain: the largest NTT prime
  // below the word bound that is not among the given ones.
  const uint64_t step = uint64_t{2} << log_n;
  const uint64_t bound = residue_bits == 64 ? (uint64_t{1} << 60) : (uint64_t{1} << 28);
  uint64_t aux = 0;
  for (uint64_t q = (bound - 1) / step * step + 1; q > step; q -= step) {
    bool taken = false;
    for (int i = 0; i < count; ++i) taken |= moduli[i] == q;
    if (!taken && is_prime64(q)) {
      aux = q;
      break;
    }
  }
  if (!aux) return fail(-2, "no auxiliary NTT prime below the word bound");
  std::vector<uint64_t> chain(moduli, moduli + count);
  chain.push_back(aux);
  return fhb_context_create(residue_bits, log_n, chain.data(), count, 1, device, out);
}
