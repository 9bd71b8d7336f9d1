/*
 * CPU restatement of the reference's CKKS evaluation-path kernels.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the fhelium_b200 package links,
 * loads or calls this file: it is the checker that the CUDA path is
 * compared against (tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg).
 *
 * Every routine restates the arithmetic of one CPU kernel of the reference
 * (visualDust/fhelium 0.10.0) and cites it.  Residues are held as int64 for
 * both buffer widths; `radix_bits` is 62 for the int64 family and 30 for the
 * int32 family (Montgomery R = 2^radix_bits), matching
 * csrc/ops/common/cpu/montgomery.h:124-143.  Outputs follow the reference CPU
 * representation (canonical where the reference CPU kernel is canonical,
 * lazy [0, 2q) where it is lazy).
 *
 * Tables passed in use the reference layouts:
 *   params  [8, limb]  rows {2q, q_lo, q_hi, -q^-1 lo, -q^-1 hi, R^2, dR^2,
 *                            N^-1 R}   (csrc/ops/common/rns_parameters.h:6-16)
 *   twiddles [limb, N] bit-reversed psi powers in Montgomery form
 *                      (fhelium/engine/ntt/plans/twiddles.py:45-84)
 * Parallelism: plain loops; the caller may split rows across processes.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

typedef struct {
  uint64_t q;
  uint64_t twice_q;
  uint64_t neg_inv; /* -q^{-1} mod R */
  uint64_t r2;      /* R^2 mod q */
  uint64_t n_inv_mont; /* N^{-1} R mod q */
  int radix_bits;
} orc_prime;

/* Rebuild one prime's constants from the split-word parameter column
 * (csrc/ops/common/cpu/montgomery.h:106-122). */
static orc_prime load_prime(const int64_t* params, int64_t limbs, int64_t j,
                            int radix_bits) {
  orc_prime p;
  const int half = radix_bits / 2;
  p.twice_q = (uint64_t)params[0 * limbs + j];
  p.q = (uint64_t)params[1 * limbs + j] + ((uint64_t)params[2 * limbs + j] << half);
  p.neg_inv = (uint64_t)params[3 * limbs + j] + ((uint64_t)params[4 * limbs + j] << half);
  p.r2 = (uint64_t)params[5 * limbs + j];
  p.n_inv_mont = (uint64_t)params[7 * limbs + j];
  p.radix_bits = radix_bits;
  return p;
}

/* REDC(a*b) with canonical output (csrc/ops/common/cpu/montgomery.h:124-143). */
static inline uint64_t mont_mul(uint64_t a, uint64_t b, const orc_prime* p) {
  const u128 product = (u128)a * b;
  const uint64_t mask = (p->radix_bits == 64) ? ~0ull : ((1ull << p->radix_bits) - 1);
  const uint64_t m = (uint64_t)(((u128)(uint64_t)product * p->neg_inv)) & mask;
  const u128 reduced = (product + (u128)m * p->q) >> p->radix_bits;
  const uint64_t r = (uint64_t)reduced;
  return r < p->q ? r : r - p->q;
}

/* Signed operand canonicalisation before multiply
 * (csrc/ops/common/cpu/montgomery.h:147-153,164-170). */
static inline uint64_t canon_signed(int64_t v, const orc_prime* p) {
  int64_t c = v % (int64_t)p->q;
  if (c < 0) c += (int64_t)p->q;
  return (uint64_t)c;
}
static inline uint64_t mont_mul_split(int64_t a, int64_t b, const orc_prime* p) {
  return mont_mul(canon_signed(a, p), canon_signed(b, p), p);
}
static inline uint64_t add_lazy(uint64_t a, uint64_t b, uint64_t twice_q) {
  const uint64_t s = a + b;
  return s < twice_q ? s : s - twice_q;
}
static inline uint64_t sub_lazy(uint64_t a, uint64_t b, uint64_t twice_q) {
  const uint64_t d = a + twice_q - b;
  return d < twice_q ? d : d - twice_q;
}
static inline uint64_t canon_lazy(uint64_t v, uint64_t twice_q) {
  const uint64_t q = twice_q >> 1;
  return v < q ? v : v - q;
}

/* ---------------------------------------------------------------------- */
/* Pointwise RNS ops (csrc/ops/rns/cpu/rns_arithmetic_cpu.cpp, binary_cpu). */

void orc_montgomery_mul(int64_t* out, const int64_t* a, const int64_t* b,
                        int64_t batch, int64_t limbs, int64_t n,
                        const int64_t* params, int radix_bits) {
  for (int64_t bi = 0; bi < batch; ++bi)
    for (int64_t j = 0; j < limbs; ++j) {
      const orc_prime p = load_prime(params, limbs, j, radix_bits);
      const int64_t base = (bi * limbs + j) * n;
      for (int64_t k = 0; k < n; ++k)
        out[base + k] = (int64_t)mont_mul((uint64_t)a[base + k], (uint64_t)b[base + k], &p);
    }
}

void orc_add_lazy(int64_t* out, const int64_t* a, const int64_t* b,
                  int64_t batch, int64_t limbs, int64_t n, const int64_t* params) {
  for (int64_t bi = 0; bi < batch; ++bi)
    for (int64_t j = 0; j < limbs; ++j) {
      const uint64_t tq = (uint64_t)params[j];
      const int64_t base = (bi * limbs + j) * n;
      for (int64_t k = 0; k < n; ++k)
        out[base + k] = (int64_t)add_lazy((uint64_t)a[base + k], (uint64_t)b[base + k], tq);
    }
}

/* Canonical add: (a + b) mod q with canonical inputs
 * (csrc/ops/rns/cpu/rns_canonical_arithmetic_cpu.cpp). */
void orc_add_canonical(int64_t* out, const int64_t* a, const int64_t* b,
                       int64_t batch, int64_t limbs, int64_t n,
                       const int64_t* moduli) {
  for (int64_t bi = 0; bi < batch; ++bi)
    for (int64_t j = 0; j < limbs; ++j) {
      const uint64_t q = (uint64_t)moduli[j];
      const int64_t base = (bi * limbs + j) * n;
      for (int64_t k = 0; k < n; ++k) {
        uint64_t s = (uint64_t)a[base + k] % q + (uint64_t)b[base + k] % q;
        out[base + k] = (int64_t)(s >= q ? s - q : s);
      }
    }
}

/* ---------------------------------------------------------------------- */
/* Negacyclic NTT, radix-2 DIF with bit-reversed output
 * (csrc/ops/ntt/cpu/indexed_ntt_cpu.cpp:35-170; to_montgomery selects the
 *  kStandard input (x R^2 first) or kMontgomery input; schedule
 *  fhelium/engine/ntt/plans/indexed_radix2.py: stage s, group g uses
 *  twiddle index 2^s + g, butterfly (u + w v, u - w v)). */
void orc_forward_ntt(int64_t* data, int64_t batch, int64_t limbs,
                     int log_n, const int64_t* twiddles,
                     const int64_t* params, int radix_bits, int to_montgomery) {
  const int64_t n = (int64_t)1 << log_n;
  for (int64_t bi = 0; bi < batch; ++bi)
    for (int64_t j = 0; j < limbs; ++j) {
      const orc_prime p = load_prime(params, limbs, j, radix_bits);
      uint64_t* x = (uint64_t*)data + (bi * limbs + j) * n;
      const int64_t* tw = twiddles + j * n;
      if (to_montgomery)
        for (int64_t k = 0; k < n; ++k) x[k] = mont_mul(x[k], p.r2, &p);
      int64_t half = n;
      for (int s = 0; s < log_n; ++s) {
        const int64_t groups = (int64_t)1 << s;
        half >>= 1;
        for (int64_t g = 0; g < groups; ++g) {
          const uint64_t w = (uint64_t)tw[groups + g];
          const int64_t first = 2 * g * half;
          for (int64_t e = first; e < first + half; ++e) {
            const uint64_t u = x[e];
            const uint64_t v = mont_mul(w, x[e + half], &p);
            x[e] = add_lazy(u, v, p.twice_q);
            x[e + half] = sub_lazy(u, v, p.twice_q);
          }
        }
      }
    }
}

/* Inverse: Gentleman-Sande stages with half span 1, 2, 4, ..., twiddle index
 * group_count + g, then x N^{-1} R, REDC and canonicalise
 * (csrc/ops/ntt/cpu/indexed_ntt_cpu.cpp:200-300, output kStandard). */
void orc_inverse_ntt_to_standard(int64_t* data, int64_t batch, int64_t limbs,
                                 int log_n, const int64_t* inv_twiddles,
                                 const int64_t* params, int radix_bits) {
  const int64_t n = (int64_t)1 << log_n;
  for (int64_t bi = 0; bi < batch; ++bi)
    for (int64_t j = 0; j < limbs; ++j) {
      const orc_prime p = load_prime(params, limbs, j, radix_bits);
      uint64_t* x = (uint64_t*)data + (bi * limbs + j) * n;
      const int64_t* tw = inv_twiddles + j * n;
      int64_t half = 1;
      for (int rem = log_n; rem > 0; --rem) {
        const int64_t groups = (int64_t)1 << (rem - 1);
        int64_t first = 0;
        for (int64_t g = 0; g < groups; ++g) {
          const uint64_t w = (uint64_t)tw[groups + g];
          for (int64_t e = first; e < first + half; ++e) {
            const uint64_t u = x[e];
            const uint64_t v = x[e + half];
            x[e] = add_lazy(u, v, p.twice_q);
            x[e + half] = mont_mul(w, sub_lazy(u, v, p.twice_q), &p);
          }
          first += 2 * half;
        }
        half <<= 1;
      }
      for (int64_t k = 0; k < n; ++k) {
        uint64_t v = mont_mul(x[k], p.n_inv_mont, &p);
        v = mont_mul(v, 1, &p);
        x[k] = canon_lazy(v, p.twice_q);
      }
    }
}

/* ---------------------------------------------------------------------- */
/* Garner mixed-radix digits of one hybrid digit
 * (csrc/ops/rns/cpu/rns_arithmetic_cpu.cpp:482-615).  src/out [batch, rows, n];
 * moduli_params is [8, rows] for the digit's own primes. */
void orc_mixed_radix_decompose(int64_t* out, const int64_t* src, int64_t batch,
                               int64_t rows, int64_t n, const int64_t* normalizers,
                               const int64_t* propagation, const int64_t* params,
                               int radix_bits) {
  orc_prime pr[8];
  for (int64_t r = 0; r < rows; ++r) pr[r] = load_prime(params, rows, r, radix_bits);
  int64_t digits[8];
  for (int64_t bi = 0; bi < batch; ++bi)
    for (int64_t k = 0; k < n; ++k) {
      const int64_t* s = src + bi * rows * n + k;
      uint64_t first = (uint64_t)s[0];
      if (first >= pr[0].q) first -= pr[0].q;
      for (int64_t r = 0; r < rows; ++r) digits[r] = (int64_t)first;
      for (int64_t step = 0; step < rows - 1; ++step) {
        const int64_t row = step + 1;
        const int64_t d = (int64_t)mont_mul_split(s[row * n] - digits[row],
                                                  normalizers[step], &pr[row]);
        digits[row] = d;
        for (int64_t t = row + 1; t < rows; ++t)
          digits[t] += (int64_t)mont_mul((uint64_t)d,
                                         (uint64_t)propagation[step * rows + t], &pr[t]);
      }
      for (int64_t r = 0; r < rows; ++r) out[bi * rows * n + r * n + k] = digits[r];
    }
}

/* Exact basis extension sum_r d_r M_r into Montgomery/lazy rows
 * (csrc/ops/rns/cpu/rns_arithmetic_cpu.cpp:616-700).  coeffs [digits-1, dst]. */
void orc_basis_extend_to_montgomery(int64_t* out, const int64_t* digits_in,
                                    int64_t batch, int64_t digits, int64_t n,
                                    const int64_t* coeffs, int64_t coeff_stride,
                                    const int64_t* params, int64_t dst_rows,
                                    int radix_bits) {
  for (int64_t bi = 0; bi < batch; ++bi)
    for (int64_t j = 0; j < dst_rows; ++j) {
      const orc_prime p = load_prime(params, dst_rows, j, radix_bits);
      for (int64_t k = 0; k < n; ++k) {
        const int64_t* d = digits_in + bi * digits * n + k;
        uint64_t v = mont_mul((uint64_t)d[0], p.r2, &p);
        for (int64_t r = 1; r < digits; ++r)
          v = add_lazy(v, mont_mul((uint64_t)d[r * n], (uint64_t)coeffs[(r - 1) * coeff_stride + j], &p),
                       p.twice_q);
        out[(bi * dst_rows + j) * n + k] = (int64_t)v;
      }
    }
}

/* acc_k += digit * key[k][key_row_start + row]  (k = 0, 1)
 * (csrc/ops/ckks/cpu/ckks_cpu.cpp:605-700).  key [2, key_rows, n]. */
void orc_keyswitch_accumulate(int64_t* acc0, int64_t* acc1, const int64_t* digit,
                              const int64_t* key, int64_t key_rows,
                              int64_t key_row_start, int64_t batch, int64_t rows,
                              int64_t n, const int64_t* params, int radix_bits) {
  for (int64_t bi = 0; bi < batch; ++bi)
    for (int64_t j = 0; j < rows; ++j) {
      const orc_prime p = load_prime(params, rows, j, radix_bits);
      const int64_t* k0 = key + (key_row_start + j) * n;
      const int64_t* k1 = key + (key_rows + key_row_start + j) * n;
      const int64_t base = (bi * rows + j) * n;
      for (int64_t k = 0; k < n; ++k) {
        const uint64_t v = (uint64_t)digit[base + k];
        acc0[base + k] = (int64_t)add_lazy((uint64_t)acc0[base + k], mont_mul(v, (uint64_t)k0[k], &p), p.twice_q);
        acc1[base + k] = (int64_t)add_lazy((uint64_t)acc1[base + k], mont_mul(v, (uint64_t)k1[k], &p), p.twice_q);
      }
    }
}

/* Sequential divide-by-P ModDown with canonical Q output
 * (csrc/ops/ckks/cpu/ckks_cpu.cpp:474-601).  q_res [batch, qn, n],
 * p_res [batch, pn, n], inverse [pn, inv_stride], params [8, qn+pn]. */
void orc_keyswitch_moddown(int64_t* out, const int64_t* q_res, const int64_t* p_res,
                           int64_t batch, int64_t qn, int64_t pn, int64_t n,
                           const int64_t* inverse, int64_t inv_stride,
                           const int64_t* params, int radix_bits) {
  const int64_t rows = qn + pn;
  int64_t chain[16];
  for (int64_t bi = 0; bi < batch; ++bi)
    for (int64_t k = 0; k < n; ++k) {
      for (int64_t r = 0; r < pn; ++r) chain[r] = p_res[(bi * pn + r) * n + k];
      for (int64_t r = pn - 2; r >= 0; --r) {
        const orc_prime p = load_prime(params, rows, qn + r, radix_bits);
        int64_t v = chain[r];
        for (int64_t lower = pn - 1; lower > r; --lower) {
          const uint64_t diff = sub_lazy((uint64_t)v, (uint64_t)chain[lower], p.twice_q);
          v = (int64_t)mont_mul_split((int64_t)diff,
                                      inverse[(pn - lower - 1) * inv_stride + (r + qn)], &p);
        }
        chain[r] = v;
      }
      for (int64_t i = 0; i < qn; ++i) {
        const orc_prime p = load_prime(params, rows, i, radix_bits);
        uint64_t v = mont_mul((uint64_t)q_res[(bi * qn + i) * n + k], p.r2, &p);
        for (int64_t pr = pn - 1; pr >= 0; --pr) {
          const uint64_t pm = mont_mul((uint64_t)chain[pr], p.r2, &p);
          v = sub_lazy(v, pm, p.twice_q);
          v = mont_mul_split((int64_t)v, inverse[(pn - pr - 1) * inv_stride + i], &p);
        }
        v = mont_mul(v, 1, &p);
        out[(bi * qn + i) * n + k] = (int64_t)canon_lazy(v, p.twice_q);
      }
    }
}

/* Rescale by the leading prime, nearest or truncating
 * (csrc/ops/ckks/cpu/ckks_cpu.cpp:203-262).  remaining [batch, rows, n],
 * dropped [batch, n]. */
void orc_rescale_drop_leading(int64_t* out, const int64_t* remaining,
                              const int64_t* dropped, int64_t batch, int64_t rows,
                              int64_t n, const int64_t* inverse_mont,
                              const int64_t* params, int64_t half_drop, int nearest,
                              int radix_bits) {
  for (int64_t bi = 0; bi < batch; ++bi)
    for (int64_t j = 0; j < rows; ++j) {
      const orc_prime p = load_prime(params, rows, j, radix_bits);
      for (int64_t k = 0; k < n; ++k) {
        const int64_t dv = dropped[bi * n + k];
        uint64_t quo = mont_mul_split(remaining[(bi * rows + j) * n + k] - dv,
                                      inverse_mont[j], &p);
        if (nearest && dv > half_drop) quo += 1;
        out[(bi * rows + j) * n + k] = (int64_t)canon_lazy(quo, p.twice_q);
      }
    }
}

/* Coefficient-domain Galois automorphism with sign and canonical output
 * (csrc/ops/ckks/cpu/ckks_cpu.cpp:287-380). */
void orc_coefficient_automorphism(int64_t* out, const int64_t* in, int64_t batch,
                                  int64_t limbs, int64_t n, const int32_t* src,
                                  const int8_t* sign, const int64_t* twice_moduli) {
  for (int64_t bi = 0; bi < batch; ++bi)
    for (int64_t j = 0; j < limbs; ++j) {
      const int64_t tq = twice_moduli[j];
      const int64_t q = tq >> 1;
      const int64_t base = (bi * limbs + j) * n;
      for (int64_t k = 0; k < n; ++k) {
        int64_t v = in[base + src[k]];
        if (sign[k] == -1) v = -v;
        v += q;
        out[base + k] = v < q ? v : v - q;
      }
    }
}

/* NTT-domain automorphism is a pure gather (csrc/ops/ckks/cpu/ckks_cpu.cpp:382-472). */
void orc_ntt_automorphism(int64_t* out, const int64_t* in, int64_t batch,
                          int64_t limbs, int64_t n, const int32_t* src) {
  for (int64_t row = 0; row < batch * limbs; ++row)
    for (int64_t k = 0; k < n; ++k) out[row * n + k] = in[row * n + src[k]];
}

/* Bit-reversed psi^{br(k)} R and psi^{-br(k)} R mod q tables for one prime
 * (fhelium/engine/ntt/plans/twiddles.py:45-84 followed by the Montgomery
 * conversion of fhelium/engine/rns/runtime.py:201-203). */
static uint64_t mulmod_u(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)((u128)a * b % q); }
void orc_twiddles(uint64_t q, uint64_t psi, uint64_t psi_inv, int log_n, int radix_bits,
                  int64_t* fwd, int64_t* inv) {
  const int64_t n = (int64_t)1 << log_n;
  const uint64_t r = (uint64_t)(((u128)1 << radix_bits) % q);
  uint64_t pw = 1, pwi = 1;
  for (int64_t i = 0; i < n; ++i) {
    int64_t br = 0;
    for (int b = 0; b < log_n; ++b) br |= ((i >> b) & 1) << (log_n - 1 - b);
    fwd[br] = (int64_t)mulmod_u(pw, r, q);
    inv[br] = (int64_t)mulmod_u(pwi, r, q);
    pw = mulmod_u(pw, psi, q);
    pwi = mulmod_u(pwi, psi_inv, q);
  }
}
