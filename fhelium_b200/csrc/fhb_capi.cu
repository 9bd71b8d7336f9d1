// extern "C" entry points of libfhb200.so (declared in include/fhb200.h).
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/fhb200.h"
#include "fhb_kernels.cuh"
#include "fhb_runners.h"

struct fhb_context {
  fhb::Context* impl;
};

namespace fhb {
Context* build_context(int bits, int log_n, const uint64_t* moduli, int num_q, int num_p, int device,
                       int* status);
void destroy_context(Context* c);
const char* last_error();

namespace {

constexpr int kMinLogN = 12;
constexpr int kMaxLogN = 17;

class DeviceGuard {
 public:
  explicit DeviceGuard(int device) {
    cudaGetDevice(&prev_);
    if (prev_ != device) cudaSetDevice(device);
    dev_ = device;
  }
  ~DeviceGuard() {
    if (prev_ != dev_) cudaSetDevice(prev_);
  }

 private:
  int prev_ = 0, dev_ = 0;
};

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

int check_ptr(const void* p, const char* name) {
  if (!p) return fail(-2, std::string(name) + " is NULL");
  if (!aligned16(p)) return fail(-2, std::string(name) + " is not 16-byte aligned");
  return 0;
}

int check_level(const Context& c, int level) {
  if (level < 0 || level >= c.num_q) return fail(-4, "level out of range [0, num_q)");
  return 0;
}

uint32_t galois_inverse(uint32_t g, int log_n) {
  // inverse of odd g modulo 2^(log_n + 1) by Newton iteration
  uint64_t x = 1;
  for (int i = 0; i < 6; ++i) x *= 2 - uint64_t(g) * x;
  return uint32_t(x & ((uint64_t{2} << log_n) - 1));
}

int check_galois(const Context& c, uint32_t g) {
  if (!(g & 1) || g >= (2u << c.log_n)) return fail(-5, "galois element must be odd and < 2N");
  return 0;
}

// Grid of the element-wise row kernels: V coefficients per thread, rows on y,
// z-slices of the batch for about 16 blocks per SM.
dim3 row_grid(int64_t n, int v, int64_t rows, int64_t batch) {
  const int64_t xb = (n / v + kEwThreads - 1) / kEwThreads;
  int64_t z = (148 * 16 + xb * rows - 1) / (xb * rows);
  if (z > batch) z = batch;
  if (z > 65535) z = 65535;
  if (z < 1) z = 1;
  return dim3(unsigned(xb), unsigned(rows), unsigned(z));
}

int elementwise_grid(int64_t total) {
  int64_t blocks = (total + 255) / 256;
  const int64_t cap = 148 * 32;
  return int(blocks < 1 ? 1 : (blocks > cap ? cap : blocks));
}

#define FHB_LOGN_SWITCH(T, FN, ...)                                   \
  switch (c.log_n) {                                                  \
    case 12: return FN<T, 12>(__VA_ARGS__);                           \
    case 13: return FN<T, 13>(__VA_ARGS__);                           \
    case 14: return FN<T, 14>(__VA_ARGS__);                           \
    case 15: return FN<T, 15>(__VA_ARGS__);                           \
    case 16: return FN<T, 16>(__VA_ARGS__);                           \
    case 17: return FN<T, 17>(__VA_ARGS__);                           \
    default: return fail(-7, "log_n outside the supported 12..17"); \
  }

#define FHB_DISPATCH(FN, ...)                 \
  if (c.bits == 64) {                         \
    FHB_LOGN_SWITCH(uint64_t, FN, __VA_ARGS__) \
  } else {                                    \
    FHB_LOGN_SWITCH(uint32_t, FN, __VA_ARGS__) \
  }

int forward(const Context& c, const void* in, void* out, int64_t polys, int rows, int row_start, bool mont,
            cudaStream_t st) {
  FHB_DISPATCH(run_forward, c, in, out, polys, rows, row_start, mont, st);
}
int inverse(const Context& c, const void* in, void* out, int64_t polys, int rows, int row_start, int kind,
            cudaStream_t st) {
  FHB_DISPATCH(run_inverse, c, in, out, polys, rows, row_start, kind, st);
}
int mul_coef(const Context& c, const void* a, const void* b, void* out, int64_t batch, int level,
             cudaStream_t st) {
  FHB_DISPATCH(run_mul_coef, c, a, b, out, batch, level, st);
}
int ks_core(const Context& c, const void* digits, const void* key, void* acc0, void* acc1, int64_t batch,
            int level, cudaStream_t st, const uint64_t* item_keys = nullptr, const void* ct3 = nullptr,
            bool pre = false, int64_t ct3_pitch = 0) {
  FHB_DISPATCH(run_ks_core, c, digits, key, acc0, acc1, batch, level, st, item_keys, ct3, pre, ct3_pitch);
}
int ks_sum(const Context& c, const void* digits, const uint64_t* key_ptrs, void* acc0, void* acc1, int giants,
           int64_t batch, int level, cudaStream_t st, bool pre = false) {
  FHB_DISPATCH(run_ks_sum, c, digits, key_ptrs, acc0, acc1, giants, batch, level, st, pre);
}
int prepare(const Context& c, const void* digits, void* prepared, int64_t batch, int level, cudaStream_t st) {
  FHB_DISPATCH(run_prepare, c, digits, prepared, batch, level, st);
}
int apply_prepared(const Context& c, const void* prepared, const void* key, void* acc0, void* acc1,
                   int64_t batch, int level, uint32_t galois, cudaStream_t st) {
  FHB_DISPATCH(run_apply_prepared, c, prepared, key, acc0, acc1, batch, level, galois, st);
}

template <typename T>
int modup(const Context& c, const void* comp, void* digits, int64_t batch, int level, uint32_t galois,
          cudaStream_t st, const uint32_t* item_galois = nullptr) {
  const int limbs = c.num_q - level;
  const uint32_t ginv = galois == 1 ? 0u : galois_inverse(galois, c.log_n);
  const LevelTables<T> lt = level_tables<T>(c, level);
  if (batch == 0 || lt.num_digits == 0) return 0;
  constexpr int V = 16 / sizeof(T);
  const bool vec = aligned16(comp) && aligned16(digits);
  const dim3 g = row_grid(c.n(), vec ? V : 1, lt.num_digits, batch);
  if (vec)
    k_modup_digits<T, V><<<g, kEwThreads, 0, st>>>((const T*)comp, (T*)digits, batch, limbs, c.log_n, level, ginv,
                                                  item_galois, tables<T>(c), lt);
  else
    k_modup_digits<T, 1><<<g, kEwThreads, 0, st>>>((const T*)comp, (T*)digits, batch, limbs, c.log_n, level, ginv,
                                                  item_galois, tables<T>(c), lt);
  return cuda_status(cudaGetLastError(), "k_modup_digits");
}

// out_pitch: words between the output's components (0: batch * out rows * N).
template <typename T>
int moddown(const Context& c, const void* t0, const void* t1, const void* a0, const void* a1, void* out,
            int64_t batch, int level, uint32_t add0_galois, int rescale, cudaStream_t st,
            const uint32_t* item_galois = nullptr, int64_t out_pitch = 0) {
  const uint32_t ginv = add0_galois == 1 ? 0u : galois_inverse(add0_galois, c.log_n);
  if constexpr (sizeof(T) == 8) {
    if (c.basis_tc && c.tc_moddown)  // P -> Q conversion on the int8 tensor cores
      return tc_moddown(const_cast<Context&>(c), t0, t1, a0, a1, out, batch, level, ginv, item_galois, rescale, st);
  }
  if (out_pitch <= 0) out_pitch = batch * (c.num_q - level - (rescale ? 1 : 0)) * c.n();
  k_moddown<T><<<elementwise_grid(batch << c.log_n), 256, 0, st>>>(
      (const T*)t0, (const T*)t1, (const T*)a0, (const T*)a1, (T*)out, batch, c.log_n, level, c.num_q, c.num_p,
      ginv, item_galois, rescale, tables<T>(c), level_tables<T>(c, level), out_pitch);
  return cuda_status(cudaGetLastError(), "k_moddown");
}

template <typename T>
int rescale(const Context& c, const void* in, void* out, int64_t polys, int level, int nearest, cudaStream_t st) {
  const int limbs = c.num_q - level;
  k_rescale<T><<<elementwise_grid(polys * (limbs - 1) << c.log_n), 256, 0, st>>>(
      (const T*)in, (T*)out, polys, limbs, c.log_n, level, nearest, tables<T>(c), level_tables<T>(c, level));
  return cuda_status(cudaGetLastError(), "k_rescale");
}

template <typename T>
int automorphism(const Context& c, const void* in, void* out, int64_t batch, int rows, int row_start,
                 uint32_t galois, cudaStream_t st) {
  k_automorphism<T><<<elementwise_grid(batch * rows << c.log_n), 256, 0, st>>>(
      (const T*)in, (T*)out, batch, rows, row_start, c.log_n, galois_inverse(galois, c.log_n), tables<T>(c));
  return cuda_status(cudaGetLastError(), "k_automorphism");
}

template <typename T>
int add(const Context& c, const void* a, const void* b, void* out, int64_t polys, int level, int lazy,
        cudaStream_t st) {
  const int limbs = c.num_q - level;
  k_add_canonical<T><<<elementwise_grid(polys * limbs << c.log_n), 256, 0, st>>>(
      (const T*)a, (const T*)b, (T*)out, polys, limbs, c.log_n, level, lazy, tables<T>(c));
  return cuda_status(cudaGetLastError(), "k_add_canonical");
}

// in_pitch: words between the input components (0: batch * rows * N); the
// output [3, batch, rows, N] is contiguous.
template <typename T>
int mul_ntt(const Context& c, const void* a, const void* b, void* out, int64_t batch, int level,
            cudaStream_t st, int64_t in_pitch = 0) {
  const int limbs = c.num_q - level;
  constexpr int V = 16 / sizeof(T);
  const int64_t out_pitch = batch * limbs * c.n();
  if (in_pitch <= 0) in_pitch = out_pitch;
  if (aligned16(a) && aligned16(b) && aligned16(out) && in_pitch % V == 0)
    k_mul_ntt<T, V><<<row_grid(c.n(), V, limbs, batch), kEwThreads, 0, st>>>(
        (const T*)a, (const T*)b, (T*)out, batch, limbs, c.log_n, level, tables<T>(c), in_pitch, out_pitch);
  else
    k_mul_ntt<T, 1><<<row_grid(c.n(), 1, limbs, batch), kEwThreads, 0, st>>>(
        (const T*)a, (const T*)b, (T*)out, batch, limbs, c.log_n, level, tables<T>(c), in_pitch, out_pitch);
  return cuda_status(cudaGetLastError(), "k_mul_ntt");
}

template <typename T>
int rns_binary(const Context& c, const void* a, const void* b, void* out, int64_t batch, int rows, int row_start,
               int op, int b_mode, cudaStream_t st) {
  constexpr int V = 16 / sizeof(T);
  if (aligned16(a) && (b == nullptr || b_mode == 2 || aligned16(b)) && aligned16(out))
    k_rns_binary<T, V><<<row_grid(c.n(), V, rows, batch), kEwThreads, 0, st>>>(
        (const T*)a, (const T*)b, (T*)out, batch, rows, row_start, c.log_n, op, b_mode, tables<T>(c));
  else
    k_rns_binary<T, 1><<<row_grid(c.n(), 1, rows, batch), kEwThreads, 0, st>>>(
        (const T*)a, (const T*)b, (T*)out, batch, rows, row_start, c.log_n, op, b_mode, tables<T>(c));
  return cuda_status(cudaGetLastError(), "k_rns_binary");
}

template <typename T>
int bsgs_inner(const Context& c, const void* rot, int64_t rot_stride, const void* pts, int64_t pt_stride,
               int entries, const int* table, int giants, int babies, void* out, int64_t out_stride, int64_t polys,
               int rows, int row_start, cudaStream_t st) {
  const size_t staged = size_t(entries) * 32 * sizeof(T);
  // staging pays once a plaintext slice is shared by a warp's worth of
  // polynomials per block (8 warps); below that the direct kernel is faster
  if (entries > 0 && staged <= 96 * 1024 && polys >= 8) {
    const int rc = ensure_dynamic_smem(reinterpret_cast<const void*>(k_bsgs_inner_staged<T>), int(staged));
    if (rc != 0) return rc;
    const int64_t blocks = (int64_t(rows) << c.log_n) / 32;
    k_bsgs_inner_staged<T><<<unsigned(blocks), 256, staged, st>>>(
        (const T*)rot, rot_stride, (const T*)pts, pt_stride, entries, table, giants, babies, (T*)out, out_stride,
        polys, rows, row_start, c.log_n, tables<T>(c));
    return cuda_status(cudaGetLastError(), "k_bsgs_inner_staged");
  }
  k_bsgs_inner<T><<<elementwise_grid(polys * rows << c.log_n), 256, 0, st>>>(
      (const T*)rot, rot_stride, (const T*)pts, pt_stride, table, giants, babies, (T*)out, out_stride, polys, rows,
      row_start, c.log_n, tables<T>(c));
  return cuda_status(cudaGetLastError(), "k_bsgs_inner");
}

template <typename T>
int lift_signed(const Context& c, const void* x, void* out, int64_t batch, int rows, int row_start,
                cudaStream_t st) {
  k_lift_signed<T><<<elementwise_grid(batch * rows << c.log_n), 256, 0, st>>>(
      (const int64_t*)x, (T*)out, batch, rows, row_start, c.log_n, tables<T>(c));
  return cuda_status(cudaGetLastError(), "k_lift_signed");
}

template <typename T>
int monomial(const Context& c, const void* in, void* out, int64_t batch, int rows, int row_start, int k,
             cudaStream_t st) {
  k_monomial<T><<<elementwise_grid(batch * rows << c.log_n), 256, 0, st>>>(
      (const T*)in, (T*)out, batch, rows, row_start, c.log_n, k, tables<T>(c));
  return cuda_status(cudaGetLastError(), "k_monomial");
}

template <typename T>
int modraise(const Context& c, const void* in, void* out, int64_t batch, int rows, int row_start, int src_prime,
             cudaStream_t st) {
  k_modraise<T><<<elementwise_grid(batch * rows << c.log_n), 256, 0, st>>>(
      (const T*)in, (T*)out, batch, rows, row_start, src_prime, c.log_n, tables<T>(c));
  return cuda_status(cudaGetLastError(), "k_modraise");
}

template <typename T>
int add_constant(const Context& c, void* data, const void* constants, int64_t batch, int rows, int row_start,
                 int all_slots, cudaStream_t st) {
  const int64_t total = all_slots ? (batch * rows << c.log_n) : batch * rows;
  k_add_constant<T><<<elementwise_grid(total), 256, 0, st>>>((T*)data, (const T*)constants, batch, rows, row_start,
                                                             c.log_n, all_slots, tables<T>(c));
  return cuda_status(cudaGetLastError(), "k_add_constant");
}

#define FHB_WORD(FN, ...) (c.bits == 64 ? FN<uint64_t>(__VA_ARGS__) : FN<uint32_t>(__VA_ARGS__))

int64_t word_bytes(const Context& c) { return c.bits / 8; }

struct Scratch {
  char* coef;    // [3, B, L, N]
  char* digits;  // [B, L, N]
  char* t0;      // [B, L+P, N]
  char* t1;      // [B, L+P, N]
  char* ext;     // tensor-core form only: [D_l, B, L+P, N] digit extensions
};

Scratch carve(const Context& c, void* base, int64_t batch, int level) {
  const int64_t w = word_bytes(c), n = c.n(), l = c.num_q - level, lp = l + c.num_p;
  char* p = static_cast<char*>(base);
  Scratch s;
  s.coef = p;
  s.digits = s.coef + 3 * batch * l * n * w;
  s.t0 = s.digits + batch * l * n * w;
  s.t1 = s.t0 + batch * lp * n * w;
  s.ext = s.t1 + batch * lp * n * w;
  return s;
}

}  // namespace
}  // namespace fhb

using fhb::Context;
using fhb::fail;

#define CTX_OR_FAIL()                                              \
  if (!ctx || !ctx->impl) return fail(-1, "context is NULL");      \
  const Context& c = *ctx->impl;                                   \
  fhb::DeviceGuard guard_(c.device);                               \
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream)

#define TRY(expr)                 \
  do {                            \
    int rc_ = (expr);             \
    if (rc_ != 0) return rc_;     \
  } while (0)

extern "C" {

int fhb_version(void) { return 1; }

int fhb_modmul_probe(const fhb_context* ctx, void* out, int blocks, int iters, fhb_stream stream) {
  CTX_OR_FAIL();
  TRY(fhb::check_ptr(out, "out"));
  if (blocks < 1 || iters < 1) return fail(-2, "need blocks >= 1 and iters >= 1");
  if (c.bits == 64)
    fhb::k_modmul_probe<uint64_t><<<blocks, 256, 0, st>>>((uint64_t*)out, iters, fhb::tables<uint64_t>(c));
  else
    fhb::k_modmul_probe<uint32_t><<<blocks, 256, 0, st>>>((uint32_t*)out, iters, fhb::tables<uint32_t>(c));
  return fhb::cuda_status(cudaGetLastError(), "k_modmul_probe");
}

int fhb_modmul_probe_f64(const fhb_context* ctx, void* out, int blocks, int iters, fhb_stream stream) {
  CTX_OR_FAIL();
  TRY(fhb::check_ptr(out, "out"));
  if (blocks < 1 || iters < 1) return fail(-2, "need blocks >= 1 and iters >= 1");
  if (!c.f64_tables_ok) return fail(-7, "the chain has no rows of primes below 2^42 (no FP64 tables)");
  fhb::k_modmul_probe_f64<8><<<blocks, 256, 0, st>>>(static_cast<double*>(out), iters, c.t64f);
  return fhb::cuda_status(cudaGetLastError(), "k_modmul_probe_f64");
}

const char* fhb_last_error(void) { return fhb::last_error(); }

int fhb_context_create(int residue_bits, int log_n, const uint64_t* moduli, int num_q, int num_p, int device,
                       fhb_context** out) {
  if (!out || !moduli) return fail(-2, "NULL argument");
  if (residue_bits != 64 && residue_bits != 32) return fail(-2, "residue_bits must be 64 or 32");
  if (log_n < fhb::kMinLogN || log_n > fhb::kMaxLogN) return fail(-7, "log_n outside the supported 12..17");
  if (num_q < 1 || num_p < 1 || num_p > fhb::kMaxDigitWidth) return fail(-2, "need num_q >= 1 and 1 <= num_p <= 8");
  const uint64_t bound = residue_bits == 64 ? (uint64_t{1} << 60) : (uint64_t{1} << 28);
  for (int i = 0; i < num_q + num_p; ++i) {
    const uint64_t q = moduli[i];
    if (q < 3 || q >= bound || !(q & 1) || (q - 1) % (uint64_t{2} << log_n) != 0)
      return fail(-2, "modulus " + std::to_string(i) + " is not an odd NTT prime below the word bound");
  }
  fhb::DeviceGuard guard(device);
  int status = 0;
  fhb::Context* c = fhb::build_context(residue_bits, log_n, moduli, num_q, num_p, device, &status);
  if (!c) return status ? status : fail(-3, "context construction failed");
  *out = new fhb_context{c};
  return 0;
}

int fhb_context_destroy(fhb_context* ctx) {
  if (!ctx) return 0;
  fhb::destroy_context(ctx->impl);
  delete ctx;
  return 0;
}

int fhb_context_root(const fhb_context* ctx, int prime_id, uint64_t* psi) {
  if (!ctx || !ctx->impl || !psi) return fail(-1, "NULL argument");
  if (prime_id < 0 || prime_id >= ctx->impl->qp()) return fail(-4, "prime id out of range");
  *psi = ctx->impl->roots[prime_id];
  return 0;
}

int fhb_context_set_tuning(fhb_context* ctx, int param, int value) {
  if (!ctx || !ctx->impl) return fail(-1, "context is NULL");
  switch (param) {
    case FHB_TUNE_KS_ORDER:
      if (value < 0 || value > 2) return fail(-2, "key-switch work order must be 0, 1 or 2");
      ctx->impl->ks_order = value;
      return 0;
    case FHB_TUNE_NTT_FORWARD_EPT:
    case FHB_TUNE_NTT_INVERSE_EPT:
      if (value != 0 && value != 8 && value != 16) return fail(-2, "residues per thread must be 0, 8 or 16");
      (param == FHB_TUNE_NTT_FORWARD_EPT ? ctx->impl->ntt_ept_fwd : ctx->impl->ntt_ept_inv) = value;
      return 0;
    case FHB_TUNE_BASIS_CONVERSION:
      if (value != 0 && value != 1) return fail(-2, "basis conversion must be 0 (CUDA cores) or 1 (tensor cores)");
      if (value == 1) {
        fhb::DeviceGuard guard(ctx->impl->device);
        TRY(fhb::tc_basis_prepare(*ctx->impl));
      }
      ctx->impl->basis_tc = value;
      return 0;
    case FHB_TUNE_TC_WAIT_US:
      if (value < 0) return fail(-2, "wait limit must be >= 0 microseconds");
      ctx->impl->tc_wait_ns = uint64_t(value) * 1000u;
      return 0;
    case FHB_TUNE_TC_TEST_STALL:
      if (value != 0 && value != 1) return fail(-2, "stall must be 0 or 1");
      ctx->impl->tc_test_stall = value;
      return 0;
    case FHB_TUNE_TC_MODDOWN:
      if (value != 0 && value != 1) return fail(-2, "value must be 0 or 1");
      ctx->impl->tc_moddown = value;
      return 0;
    case FHB_TUNE_TC_NTT_FUSED:
      if (value != 0 && value != 1) return fail(-2, "value must be 0 or 1");
      ctx->impl->tc_ntt_fused = value;
      return 0;
    case FHB_TUNE_F64_CORE:
      if (value != 0 && value != 1) return fail(-2, "value must be 0 or 1");
      ctx->impl->f64_core = value;
      return 0;
    case FHB_TUNE_OVERLAP_CHUNKS:
      if (value < 1 || value > fhb::kMaxOverlapChunks) return fail(-2, "value must be in 1..8");
      ctx->impl->overlap_chunks = value;
      return 0;
    default:
      return fail(-2, "unknown tuning parameter");
  }
}

int fhb_context_get_tuning(const fhb_context* ctx, int param, int* value) {
  if (!ctx || !ctx->impl || !value) return fail(-1, "NULL argument");
  switch (param) {
    case FHB_TUNE_KS_ORDER: *value = ctx->impl->ks_order; return 0;
    case FHB_TUNE_NTT_FORWARD_EPT: *value = ctx->impl->ntt_ept_fwd; return 0;
    case FHB_TUNE_NTT_INVERSE_EPT: *value = ctx->impl->ntt_ept_inv; return 0;
    case FHB_TUNE_BASIS_CONVERSION: *value = ctx->impl->basis_tc; return 0;
    case FHB_TUNE_TC_WAIT_US: *value = int(ctx->impl->tc_wait_ns / 1000u); return 0;
    case FHB_TUNE_TC_TEST_STALL: *value = ctx->impl->tc_test_stall; return 0;
    case FHB_TUNE_TC_MODDOWN: *value = ctx->impl->tc_moddown; return 0;
    case FHB_TUNE_TC_NTT_FUSED: *value = ctx->impl->tc_ntt_fused; return 0;
    case FHB_TUNE_F64_CORE: *value = ctx->impl->f64_core && ctx->impl->f64_tables_ok; return 0;
    case FHB_TUNE_OVERLAP_CHUNKS: *value = ctx->impl->overlap_chunks; return 0;
    default: return fail(-2, "unknown tuning parameter");
  }
}

int fhb_forward_ntt(const fhb_context* ctx, const void* in, void* out, int64_t batch, int rows, int row_start,
                    int input_montgomery, fhb_stream stream) {
  CTX_OR_FAIL();
  TRY(fhb::check_ptr(in, "in"));
  TRY(fhb::check_ptr(out, "out"));
  if (batch < 0 || rows < 1 || row_start < 0 || row_start + rows > c.qp()) return fail(-4, "row interval out of range");
  return fhb::forward(c, in, out, batch * rows, rows, row_start, input_montgomery != 0, st);
}

int fhb_inverse_ntt(const fhb_context* ctx, const void* in, void* out, int64_t batch, int rows, int row_start,
                    int output_kind, fhb_stream stream) {
  CTX_OR_FAIL();
  TRY(fhb::check_ptr(in, "in"));
  TRY(fhb::check_ptr(out, "out"));
  if (batch < 0 || rows < 1 || row_start < 0 || row_start + rows > c.qp()) return fail(-4, "row interval out of range");
  if (output_kind < 0 || output_kind > 3) return fail(-2, "unknown inverse output kind");
  return fhb::inverse(c, in, out, batch * rows, rows, row_start, output_kind, st);
}

int fhb_tc_ntt_prepare(const fhb_context* ctx) {
  fhb_stream stream = nullptr;
  CTX_OR_FAIL();
  (void)st;
  (void)c;
  return fhb::tc_ntt_prepare(*ctx->impl);
}

static int tc_transform(const fhb_context* ctx, const void* in, void* out, int64_t batch, int rows, int row_start,
                        bool inverse, fhb_stream stream) {
  CTX_OR_FAIL();
  TRY(fhb::check_ptr(in, "in"));
  TRY(fhb::check_ptr(out, "out"));
  if (batch < 0 || rows < 1 || row_start < 0 || row_start + rows > c.qp()) return fail(-4, "row interval out of range");
  return fhb::tc_ntt(*ctx->impl, in, out, batch * rows, rows, row_start, inverse, st);
}

int fhb_tc_forward_ntt(const fhb_context* ctx, const void* in, void* out, int64_t batch, int rows, int row_start,
                       fhb_stream stream) {
  return tc_transform(ctx, in, out, batch, rows, row_start, false, stream);
}

int fhb_tc_inverse_ntt(const fhb_context* ctx, const void* in, void* out, int64_t batch, int rows, int row_start,
                       fhb_stream stream) {
  return tc_transform(ctx, in, out, batch, rows, row_start, true, stream);
}

int fhb_tc_ntt_status(const fhb_context* ctx, int* flag) {
  fhb_stream stream = nullptr;
  CTX_OR_FAIL();
  (void)st;
  (void)c;
  if (!flag) return fail(-2, "flag is NULL");
  return fhb::tc_ntt_status(*ctx->impl, flag);
}

int fhb_tc_basis_extend(const fhb_context* ctx, const void* digits, void* ext, int64_t batch, int level,
                        fhb_stream stream) {
  CTX_OR_FAIL();
  TRY(fhb::check_ptr(digits, "digits"));
  TRY(fhb::check_ptr(ext, "ext"));
  TRY(fhb::check_level(c, level));
  if (batch < 0) return fail(-2, "batch must be >= 0");
  return fhb::tc_extend(*ctx->impl, digits, ext, batch, level, false, st);
}

int64_t fhb_tc_basis_extend_words(const fhb_context* ctx, int64_t batch, int level) {
  if (!ctx || !ctx->impl || batch < 0 || level < 0 || level >= ctx->impl->num_q) return -1;
  return fhb::tc_ext_words(*ctx->impl, batch, level);
}

int fhb_tc_basis_status(const fhb_context* ctx, int* flag) {
  fhb_stream stream = nullptr;
  CTX_OR_FAIL();
  (void)st;
  (void)c;
  if (!flag) return fail(-2, "flag is NULL");
  return fhb::tc_basis_status(*ctx->impl, flag);
}

int fhb_tc_ntt_tables_host(uint64_t q, uint64_t psi, int pass, uint8_t* bmat, uint32_t* post) {
  if (!bmat) return fail(-2, "bmat is NULL");
  if (pass < 0 || pass > 5) return fail(-2, "pass must be 0..5");
  if (q < 3 || q >= (uint64_t{1} << 28) || !(q & 1) || (q - 1) % (uint64_t{2} << 16) != 0)
    return fail(-2, "q must be an odd NTT prime below 2^28 for N = 2^16");
  if (psi == 0 || psi >= q) return fail(-2, "psi out of range");
  fhb::tc_ntt_tables_host(q, psi, pass, bmat, post);
  return 0;
}

int fhb_ckks_multiply(const fhb_context* ctx, const void* a, const void* b, void* out, int64_t batch, int level,
                      fhb_stream stream) {
  CTX_OR_FAIL();
  TRY(fhb::check_ptr(a, "a"));
  TRY(fhb::check_ptr(b, "b"));
  TRY(fhb::check_ptr(out, "out"));
  TRY(fhb::check_level(c, level));
  return FHB_WORD(fhb::mul_ntt, c, a, b, out, batch, level, st);
}

int fhb_ckks_multiply_to_coefficient(const fhb_context* ctx, const void* a, const void* b, void* out,
                                     int64_t batch, int level, fhb_stream stream) {
  CTX_OR_FAIL();
  TRY(fhb::check_ptr(a, "a"));
  TRY(fhb::check_ptr(b, "b"));
  TRY(fhb::check_ptr(out, "out"));
  TRY(fhb::check_level(c, level));
  return fhb::mul_coef(c, a, b, out, batch, level, st);
}

int fhb_ckks_modup_digits(const fhb_context* ctx, const void* comp, void* digits, int64_t batch, int level,
                          uint32_t galois, fhb_stream stream) {
  CTX_OR_FAIL();
  TRY(fhb::check_ptr(comp, "comp"));
  TRY(fhb::check_ptr(digits, "digits"));
  TRY(fhb::check_level(c, level));
  TRY(fhb::check_galois(c, galois));
  return FHB_WORD(fhb::modup, c, comp, digits, batch, level, galois, st);
}

int fhb_ckks_keyswitch_core(const fhb_context* ctx, const void* digits, const void* key, void* acc0, void* acc1,
                            int64_t batch, int level, fhb_stream stream) {
  CTX_OR_FAIL();
  TRY(fhb::check_ptr(digits, "digits"));
  TRY(fhb::check_ptr(key, "key"));
  TRY(fhb::check_ptr(acc0, "acc0"));
  TRY(fhb::check_ptr(acc1, "acc1"));
  TRY(fhb::check_level(c, level));
  return fhb::ks_core(c, digits, key, acc0, acc1, batch, level, st);
}

int fhb_ckks_keyswitch_core_extended(const fhb_context* ctx, const void* ext, const void* key, void* acc0,
                                     void* acc1, int64_t batch, int level, fhb_stream stream) {
  CTX_OR_FAIL();
  TRY(fhb::check_ptr(ext, "ext"));
  TRY(fhb::check_ptr(key, "key"));
  TRY(fhb::check_ptr(acc0, "acc0"));
  TRY(fhb::check_ptr(acc1, "acc1"));
  TRY(fhb::check_level(c, level));
  if (batch < 0) return fail(-2, "batch must be >= 0");
  return fhb::ks_core(c, ext, key, acc0, acc1, batch, level, st, nullptr, nullptr, true);
}

int fhb_ckks_moddown(const fhb_context* ctx, const void* t0, const void* t1, const void* add0, const void* add1,
                     void* out, int64_t batch, int level, uint32_t add0_galois, int rescale, fhb_stream stream) {
  CTX_OR_FAIL();
  TRY(fhb::check_ptr(t0, "t0"));
  TRY(fhb::check_ptr(t1, "t1"));
  TRY(fhb::check_ptr(out, "out"));
  TRY(fhb::check_level(c, level));
  TRY(fhb::check_galois(c, add0_galois));
  if (rescale && level + 1 >= c.num_q) return fail(-4, "cannot rescale at the last level");
  return FHB_WORD(fhb::moddown, c, t0, t1, add0, add1, out, batch, level, add0_galois, rescale, st);
}

int fhb_ckks_prepare_rotation(const fhb_context* ctx, const void* digits, void* prepared, int64_t batch, int level,
                              fhb_stream stream) {
  CTX_OR_FAIL();
  TRY(fhb::check_ptr(digits, "digits"));
  TRY(fhb::check_ptr(prepared, "prepared"));
  TRY(fhb::check_level(c, level));
  if (batch < 0) return fail(-2, "batch must be >= 0");
  if (c.basis_tc) {
    // tensor-core form: extensions straight into the prepared layout
    // [D_l, B, QP_l, N], then their forward NTT in place (no x R)
    const int qpl = c.qp() - level;
    TRY(fhb::tc_extend(*ctx->impl, digits, prepared, batch, level, false, st));
    const int64_t polys = fhb::tc_ext_words(c, batch, level) / c.n();
    return fhb::forward(c, prepared, prepared, polys, qpl, level, true, st);
  }
  return fhb::prepare(c, digits, prepared, batch, level, st);
}

int fhb_ckks_apply_prepared_rotation(const fhb_context* ctx, const void* prepared, const void* key, void* acc0,
                                     void* acc1, int64_t batch, int level, uint32_t galois, fhb_stream stream) {
  CTX_OR_FAIL();
  TRY(fhb::check_ptr(prepared, "prepared"));
  TRY(fhb::check_ptr(key, "key"));
  TRY(fhb::check_ptr(acc0, "acc0"));
  TRY(fhb::check_ptr(acc1, "acc1"));
  TRY(fhb::check_level(c, level));
  TRY(fhb::check_galois(c, galois));
  return fhb::apply_prepared(c, prepared, key, acc0, acc1, batch, level, galois, st);
}

int fhb_ckks_rescale(const fhb_context* ctx, const void* in, void* out, int64_t polys, int level, int nearest,
                     fhb_stream stream) {
  CTX_OR_FAIL();
  TRY(fhb::check_ptr(in, "in"));
  TRY(fhb::check_ptr(out, "out"));
  TRY(fhb::check_level(c, level));
  if (level + 1 >= c.num_q) return fail(-4, "cannot rescale at the last level");
  return FHB_WORD(fhb::rescale, c, in, out, polys, level, nearest, st);
}

int fhb_ckks_automorphism(const fhb_context* ctx, const void* in, void* out, int64_t batch, int rows, int row_start,
                          uint32_t galois, fhb_stream stream) {
  CTX_OR_FAIL();
  TRY(fhb::check_ptr(in, "in"));
  TRY(fhb::check_ptr(out, "out"));
  TRY(fhb::check_galois(c, galois));
  if (batch < 0 || rows < 1 || row_start < 0 || row_start + rows > c.qp()) return fail(-4, "row interval out of range");
  if (in == out) return fail(-2, "automorphism cannot run in place");
  return FHB_WORD(fhb::automorphism, c, in, out, batch, rows, row_start, galois, st);
}

int fhb_ckks_add(const fhb_context* ctx, const void* a, const void* b, void* out, int64_t polys, int level,
                 int lazy, fhb_stream stream) {
  CTX_OR_FAIL();
  TRY(fhb::check_ptr(a, "a"));
  TRY(fhb::check_ptr(b, "b"));
  TRY(fhb::check_ptr(out, "out"));
  TRY(fhb::check_level(c, level));
  return FHB_WORD(fhb::add, c, a, b, out, polys, level, lazy, st);
}

int fhb_rns_binary(const fhb_context* ctx, int op, const void* a, const void* b, void* out, int64_t batch, int rows,
                   int row_start, int b_mode, fhb_stream stream) {
  CTX_OR_FAIL();
  TRY(fhb::check_ptr(a, "a"));
  TRY(fhb::check_ptr(out, "out"));
  if (op != fhb::kOpNegCanon) TRY(fhb::check_ptr(b, "b"));
  if (op < 0 || op > fhb::kOpNegCanon) return fail(-2, "unknown RNS op");
  if (b_mode < 0 || b_mode > 2) return fail(-2, "unknown operand broadcast mode");
  if (batch < 0 || rows < 1 || row_start < 0 || row_start + rows > c.qp()) return fail(-4, "row interval out of range");
  return FHB_WORD(fhb::rns_binary, c, a, b, out, batch, rows, row_start, op, b_mode, st);
}

int fhb_rns_lift_signed(const fhb_context* ctx, const int64_t* coefficients, void* out, int64_t batch, int rows,
                        int row_start, fhb_stream stream) {
  CTX_OR_FAIL();
  TRY(fhb::check_ptr(coefficients, "coefficients"));
  TRY(fhb::check_ptr(out, "out"));
  if (batch < 0 || rows < 1 || row_start < 0 || row_start + rows > c.qp()) return fail(-4, "row interval out of range");
  return FHB_WORD(fhb::lift_signed, c, coefficients, out, batch, rows, row_start, st);
}

int fhb_ckks_monomial(const fhb_context* ctx, const void* in, void* out, int64_t batch, int rows, int row_start, int k,
                      fhb_stream stream) {
  CTX_OR_FAIL();
  TRY(fhb::check_ptr(in, "in"));
  TRY(fhb::check_ptr(out, "out"));
  if (in == out) return fail(-2, "monomial multiplication cannot run in place");
  if (k < 0 || k >= 2 * c.n()) return fail(-2, "monomial exponent must be in [0, 2N)");
  if (batch < 0 || rows < 1 || row_start < 0 || row_start + rows > c.qp()) return fail(-4, "row interval out of range");
  return FHB_WORD(fhb::monomial, c, in, out, batch, rows, row_start, k, st);
}

int fhb_ckks_modraise(const fhb_context* ctx, const void* in, void* out, int64_t batch, int src_prime, int rows,
                      int row_start, fhb_stream stream) {
  CTX_OR_FAIL();
  TRY(fhb::check_ptr(in, "in"));
  TRY(fhb::check_ptr(out, "out"));
  if (src_prime < 0 || src_prime >= c.qp()) return fail(-4, "source prime out of range");
  if (batch < 0 || rows < 1 || row_start < 0 || row_start + rows > c.qp()) return fail(-4, "row interval out of range");
  return FHB_WORD(fhb::modraise, c, in, out, batch, rows, row_start, src_prime, st);
}

int fhb_rns_add_constant(const fhb_context* ctx, void* data, const void* constants, int64_t batch, int rows,
                         int row_start, int all_slots, fhb_stream stream) {
  CTX_OR_FAIL();
  TRY(fhb::check_ptr(data, "data"));
  if (!constants) return fail(-2, "constants is NULL");
  if (batch < 0 || rows < 1 || row_start < 0 || row_start + rows > c.qp()) return fail(-4, "row interval out of range");
  return FHB_WORD(fhb::add_constant, c, data, constants, batch, rows, row_start, all_slots ? 1 : 0, st);
}

int64_t fhb_ckks_keyswitch_scratch_bytes(const fhb_context* ctx, int64_t batch, int level) {
  if (!ctx || !ctx->impl) return -1;
  const Context& c = *ctx->impl;
  if (level < 0 || level >= c.num_q || batch < 0) return -1;
  const int64_t l = c.num_q - level, lp = l + c.num_p;
  int64_t per_ct = (3 * l + l + 2 * lp) * c.n() * fhb::word_bytes(c);
  // tensor-core form: the extensions of every digit to every row
  if (c.basis_tc) per_ct += fhb::tc_ext_words(c, 1, level) * fhb::word_bytes(c);
  if (batch > INT64_MAX / per_ct) return -1;  // the size does not fit in 64 bits
  return per_ct * batch;
}

// Scratch check shared by the entry points that take a caller scratch buffer:
// a negative batch, an invalid level or a size that overflows is an invalid
// argument, not a small buffer.
static int check_scratch(const fhb_context* ctx, int64_t batch, int level, int64_t scratch_bytes) {
  if (batch < 0) return fail(-2, "batch must be >= 0");
  const int64_t need = fhb_ckks_keyswitch_scratch_bytes(ctx, batch, level);
  if (need < 0) return fail(-4, "invalid level, or the scratch size of this batch overflows 64 bits");
  if (scratch_bytes < need) return fail(-8, "scratch too small");
  return 0;
}

// Key-switch core on the ModUp digits in s.digits: with the tensor-core
// basis conversion the extensions are materialised first (own-digit rows
// skipped when the core reuses c2 there) and the core only transforms.
static int ks_core_from_digits(const Context& c, const fhb::Scratch& s, const void* key, int64_t batch, int level,
                               cudaStream_t st, const uint64_t* item_keys = nullptr, const void* ct3 = nullptr) {
  if (!c.basis_tc) return fhb::ks_core(c, s.digits, key, s.t0, s.t1, batch, level, st, item_keys, ct3);
  TRY(fhb::tc_extend(const_cast<Context&>(c), s.digits, s.ext, batch, level, ct3 != nullptr, st));
  return fhb::ks_core(c, s.ext, key, s.t0, s.t1, batch, level, st, item_keys, ct3, true);
}

static int keyswitch_tail(const Context& c, const fhb::Scratch& s, const void* key, const void* add0,
                          const void* add1, uint32_t add0_galois, void* out, int64_t batch, int level, int rescale,
                          cudaStream_t st) {
  TRY(ks_core_from_digits(c, s, key, batch, level, st));
  return FHB_WORD(fhb::moddown, c, s.t0, s.t1, add0, add1, out, batch, level, add0_galois, rescale, st);
}

// Relinearisation of an NTT-domain ct3 (coefficient-domain c2 already in
// s.t0): ModUp of c2, the key-switch core with c0, c1 folded in as P c_k
// (NTT domain) and c2's own-digit rows reused, ModDown (+ rescale).
static int relinearize_tail(const Context& c, const fhb::Scratch& s, const void* key, const void* ct3, void* out,
                            int64_t batch, int level, int rescale, cudaStream_t st) {
  TRY(FHB_WORD(fhb::modup, c, s.t0, s.digits, batch, level, 1u, st));
  TRY(ks_core_from_digits(c, s, key, batch, level, st, nullptr, ct3));
  return FHB_WORD(fhb::moddown, c, s.t0, s.t1, nullptr, nullptr, out, batch, level, 1u, rescale, st);
}

int fhb_ckks_relinearize(const fhb_context* ctx, const void* ct3, const void* key, void* out, void* scratch,
                         int64_t scratch_bytes, int64_t batch, int level, int rescale, fhb_stream stream) {
  CTX_OR_FAIL();
  TRY(fhb::check_ptr(ct3, "ct3"));
  TRY(fhb::check_ptr(key, "key"));
  TRY(fhb::check_ptr(out, "out"));
  TRY(fhb::check_ptr(scratch, "scratch"));
  TRY(fhb::check_level(c, level));
  TRY(check_scratch(ctx, batch, level, scratch_bytes));
  if (rescale && level + 1 >= c.num_q) return fail(-4, "cannot rescale at the last level");
  const int limbs = c.num_q - level;
  const fhb::Scratch s = fhb::carve(c, scratch, batch, level);
  const int64_t comp = batch * limbs * c.n() * fhb::word_bytes(c);
  TRY(fhb::inverse(c, static_cast<const char*>(ct3) + 2 * comp, s.t0, batch * limbs, limbs, level,
                   fhb::kInvStandard, st));
  return relinearize_tail(c, s, key, ct3, out, batch, level, rescale, st);
}

// True when the byte ranges [a, a + na) and [b, b + nb) share a byte.
static bool ranges_overlap(const void* a, int64_t na, const void* b, int64_t nb) {
  const auto x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
  return x < y + uintptr_t(nb) && y < x + uintptr_t(na);
}

// Streams (priorities: [0] highest, [1] and [2] lowest) and events of the
// chunked fused HMult, created once per context.
static int overlap_resources(Context& c) {
  if (c.ov_streams[2]) return 0;
  int least = 0, greatest = 0;
  TRY(fhb::cuda_status(cudaDeviceGetStreamPriorityRange(&least, &greatest), "stream priorities"));
  c.ov_events.assign(4 * fhb::kMaxOverlapChunks + 4, nullptr);
  for (cudaEvent_t& ev : c.ov_events)
    TRY(fhb::cuda_status(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "overlap event"));
  const int prio[3] = {greatest, least, least};
  for (int i = 0; i < 3; ++i)
    TRY(fhb::cuda_status(cudaStreamCreateWithPriority(&c.ov_streams[i], cudaStreamNonBlocking, prio[i]),
                         "overlap stream"));
  return 0;
}

// HMult + relinearise (+ rescale) of a batch cut into k chunks.  The key-
// switch core runs in 8-CTA clusters, which leave SMs idle (15 clusters
// resident on 148 SMs at N = 2^16); the element-wise stages of the other
// chunks fill them.  Streams: [0] (highest priority) the inverse NTTs of d2
// and the cores, [1] the tensor products and ModUp digits, [2] the ModDowns:
//   [1]: tp0 tp1 | mu0 tp2 | mu1 tp3 | mu2 ...   ([1] waits for inv_i before mu_i)
//   [0]: inv0 inv1 | core0 inv2 | core1 inv3 | core2 ...
//   [2]: md0 | md1 | ...                          (md_i after core_i)
// so chunk i+1's ModUp and chunk i-1's ModDown run beside chunk i's core.
// Every wait is enqueued after the record it waits for.  Results are those
// of the one-pass call; the chunks' scratch regions are disjoint slices.
static int multiply_relinearize_chunked(const fhb_context* ctx, const char* a, const char* b, const void* key,
                                        char* out, char* scratch, int64_t batch, int level, int rescale,
                                        cudaStream_t st, int k) {
  const Context& c = *ctx->impl;
  Context& cm = const_cast<Context&>(c);
  std::lock_guard<std::mutex> lock(cm.ov_mutex);
  TRY(overlap_resources(cm));
  const int limbs = c.num_q - level, out_limbs = limbs - (rescale ? 1 : 0);
  const int64_t wb = fhb::word_bytes(c), n = c.n();
  const int64_t in_pitch = batch * limbs * n, out_pitch = batch * out_limbs * n;  // words
  const int64_t per_ct = fhb_ckks_keyswitch_scratch_bytes(ctx, 1, level);
  int64_t b0[fhb::kMaxOverlapChunks + 1];
  const int64_t base = std::max<int64_t>(4, batch / k / 4 * 4);  // whole key-switch groups of four
  for (int i = 0; i < k; ++i) b0[i] = std::min<int64_t>(batch, i * base);
  b0[k] = batch;
  cudaStream_t hi = cm.ov_streams[0], pre = cm.ov_streams[1], post = cm.ov_streams[2];
  const cudaEvent_t* ev = cm.ov_events.data();
  enum { kTp = 0, kInv = 1, kMu = 2, kCore = 3 };
  auto E = [&](int kind, int i) { return ev[4 + 4 * i + kind]; };
  auto rec = [&](cudaEvent_t e, cudaStream_t s) { return fhb::cuda_status(cudaEventRecord(e, s), "overlap record"); };
  auto wait = [&](cudaStream_t s, cudaEvent_t e) {
    return fhb::cuda_status(cudaStreamWaitEvent(s, e, 0), "overlap wait");
  };
  auto bc = [&](int i) { return b0[i + 1] - b0[i]; };
  auto scr = [&](int i) { return fhb::carve(c, scratch + per_ct * b0[i], bc(i), level); };
  auto tp = [&](int i) -> int {
    const int64_t off = b0[i] * limbs * n * wb;
    TRY(FHB_WORD(fhb::mul_ntt, c, a + off, b + off, scr(i).coef, bc(i), level, pre, in_pitch));
    return rec(E(kTp, i), pre);
  };
  auto inv = [&](int i) -> int {
    const fhb::Scratch s = scr(i);
    TRY(wait(hi, E(kTp, i)));
    TRY(fhb::inverse(c, s.coef + 2 * bc(i) * limbs * n * wb, s.t0, bc(i) * limbs, limbs, level, fhb::kInvStandard,
                     hi));
    return rec(E(kInv, i), hi);
  };
  auto mu = [&](int i) -> int {
    const fhb::Scratch s = scr(i);
    TRY(wait(pre, E(kInv, i)));
    TRY(FHB_WORD(fhb::modup, c, s.t0, s.digits, bc(i), level, 1u, pre));
    return rec(E(kMu, i), pre);
  };
  auto core = [&](int i) -> int {
    const fhb::Scratch s = scr(i);
    TRY(wait(hi, E(kMu, i)));
    TRY(ks_core_from_digits(c, s, key, bc(i), level, hi, nullptr, s.coef));
    return rec(E(kCore, i), hi);
  };
  auto md = [&](int i) -> int {
    const fhb::Scratch s = scr(i);
    TRY(wait(post, E(kCore, i)));
    return FHB_WORD(fhb::moddown, c, s.t0, s.t1, nullptr, nullptr, out + b0[i] * out_limbs * n * wb, bc(i), level,
                    1u, rescale, post, nullptr, out_pitch);
  };
  TRY(rec(ev[0], st));
  for (cudaStream_t s : {hi, pre, post}) TRY(wait(s, ev[0]));
  TRY(tp(0));
  if (k > 1) TRY(tp(1));
  TRY(inv(0));
  if (k > 1) TRY(inv(1));
  TRY(mu(0));
  if (k > 2) TRY(tp(2));
  for (int i = 0; i < k; ++i) {
    TRY(core(i));
    TRY(md(i));
    if (i + 1 < k) {
      TRY(mu(i + 1));
      if (i + 3 < k) TRY(tp(i + 3));
    }
    if (i + 2 < k) TRY(inv(i + 2));
  }
  for (int j = 0; j < 3; ++j) TRY(rec(ev[1 + j], cm.ov_streams[j]));
  for (int j = 0; j < 3; ++j) TRY(wait(st, ev[1 + j]));
  return 0;
}

int fhb_ckks_multiply_relinearize(const fhb_context* ctx, const void* a, const void* b, const void* key, void* out,
                                  void* scratch, int64_t scratch_bytes, int64_t batch, int level, int rescale,
                                  fhb_stream stream) {
  CTX_OR_FAIL();
  TRY(fhb::check_ptr(a, "a"));
  TRY(fhb::check_ptr(b, "b"));
  TRY(fhb::check_ptr(key, "key"));
  TRY(fhb::check_ptr(out, "out"));
  TRY(fhb::check_ptr(scratch, "scratch"));
  TRY(fhb::check_level(c, level));
  TRY(check_scratch(ctx, batch, level, scratch_bytes));
  if (rescale && level + 1 >= c.num_q) return fail(-4, "cannot rescale at the last level");
  const int limbs = c.num_q - level;
  // a batch of at least two chunks of 8: chunks overlapped (not under stream
  // capture, and not with ModDown on the tensor cores, which writes whole
  // batches)
  const int k = int(std::min<int64_t>(c.overlap_chunks, batch / 8));
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  TRY(fhb::cuda_status(cudaStreamIsCapturing(st, &cap), "capture status"));
  // a chunk's ModDown must not overwrite input a later chunk still reads
  const int64_t in_bytes = 2 * batch * limbs * c.n() * fhb::word_bytes(c);
  const int64_t out_bytes = 2 * batch * (limbs - (rescale ? 1 : 0)) * c.n() * fhb::word_bytes(c);
  const bool alias = ranges_overlap(out, out_bytes, a, in_bytes) || ranges_overlap(out, out_bytes, b, in_bytes);
  if (k > 1 && cap == cudaStreamCaptureStatusNone && !(c.basis_tc && c.tc_moddown) && !alias)
    return multiply_relinearize_chunked(ctx, static_cast<const char*>(a), static_cast<const char*>(b), key,
                                        static_cast<char*>(out), static_cast<char*>(scratch), batch, level, rescale,
                                        st, k);
  const fhb::Scratch s = fhb::carve(c, scratch, batch, level);
  const int64_t comp = batch * limbs * c.n() * fhb::word_bytes(c);
  // ct3 = a x b into the scratch (elementwise, every SM), then the
  // relinearisation of an NTT-domain ct3
  TRY(FHB_WORD(fhb::mul_ntt, c, a, b, s.coef, batch, level, st));
  TRY(fhb::inverse(c, s.coef + 2 * comp, s.t0, batch * limbs, limbs, level, fhb::kInvStandard, st));
  return relinearize_tail(c, s, key, s.coef, out, batch, level, rescale, st);
}

int fhb_ckks_keyswitch_sum(const fhb_context* ctx, const void* digits, const uint64_t* key_ptrs, void* acc0,
                           void* acc1, int giants, int64_t batch, int level, fhb_stream stream) {
  CTX_OR_FAIL();
  TRY(fhb::check_ptr(digits, "digits"));
  TRY(fhb::check_ptr(acc0, "acc0"));
  TRY(fhb::check_ptr(acc1, "acc1"));
  if (!key_ptrs) return fail(-2, "key_ptrs is NULL");
  if (giants < 1 || batch < 0) return fail(-2, "need giants >= 1 and batch >= 0");
  TRY(fhb::check_level(c, level));
  return fhb::ks_sum(c, digits, key_ptrs, acc0, acc1, giants, batch, level, st);
}

int fhb_ckks_decrypt_tail(const fhb_context* ctx, const void* phase, double* out, int64_t batch, int level,
                          fhb_stream stream) {
  CTX_OR_FAIL();
  TRY(fhb::check_ptr(phase, "phase"));
  if (!out) return fail(-2, "out is NULL");
  TRY(fhb::check_level(c, level));
  if (batch < 0) return fail(-2, "batch must be >= 0");
  if (batch == 0) return 0;
  using u128 = unsigned __int128;
  const int limbs = c.num_q - level;
  fhb::DecryptTail t{};
  t.two = limbs >= 2;
  t.qb = c.moduli[c.num_q - 1];
  t.qb_one_s = uint64_t((u128(1) << 64) / t.qb);
  if (t.two) {
    t.qa = c.moduli[c.num_q - 2];
    uint64_t inv = 1, base = t.qa % t.qb, e = t.qb - 2;  // q_a^{-1} mod q_b (q_b prime)
    for (; e; e >>= 1, base = uint64_t(u128(base) * base % t.qb))
      if (e & 1) inv = uint64_t(u128(inv) * base % t.qb);
    t.inv = inv;
    t.inv_s = uint64_t((u128(inv) << 64) / t.qb);
    const u128 half = u128(t.qa) * t.qb / 2;
    t.h0 = uint64_t(half % t.qa);
    t.h1 = uint64_t(half / t.qa);
  }
  const int grid = fhb::elementwise_grid(batch << c.log_n);
  if (c.bits == 64)
    fhb::k_decrypt_tail<uint64_t><<<grid, 256, 0, st>>>(static_cast<const uint64_t*>(phase), out, batch, limbs,
                                                         c.log_n, t);
  else
    fhb::k_decrypt_tail<uint32_t><<<grid, 256, 0, st>>>(static_cast<const uint32_t*>(phase), out, batch, limbs,
                                                         c.log_n, t);
  return fhb::cuda_status(cudaGetLastError(), "k_decrypt_tail");
}

int fhb_ckks_keyswitch_sum_extended(const fhb_context* ctx, const void* ext, const uint64_t* key_ptrs, void* acc0,
                                    void* acc1, int giants, int64_t batch, int level, fhb_stream stream) {
  CTX_OR_FAIL();
  TRY(fhb::check_ptr(ext, "ext"));
  TRY(fhb::check_ptr(acc0, "acc0"));
  TRY(fhb::check_ptr(acc1, "acc1"));
  if (!key_ptrs) return fail(-2, "key_ptrs is NULL");
  if (giants < 1 || batch < 0) return fail(-2, "need giants >= 1 and batch >= 0");
  TRY(fhb::check_level(c, level));
  return fhb::ks_sum(c, ext, key_ptrs, acc0, acc1, giants, batch, level, st, true);
}

int fhb_ckks_bsgs_inner_product(const fhb_context* ctx, const void* rot, int64_t rot_stride, const void* pts,
                                int64_t pt_stride, int entries, const int32_t* table, int giants, int babies,
                                void* out, int64_t out_stride, int64_t polys, int rows, int row_start,
                                fhb_stream stream) {
  CTX_OR_FAIL();
  TRY(fhb::check_ptr(rot, "rot"));
  TRY(fhb::check_ptr(pts, "pts"));
  TRY(fhb::check_ptr(out, "out"));
  if (!table) return fail(-2, "table is NULL");
  if (giants < 1 || babies < 1 || polys < 0 || entries < 1)
    return fail(-2, "need giants >= 1, babies >= 1, entries >= 1, polys >= 0");
  if (rows < 1 || row_start < 0 || row_start + rows > c.qp()) return fail(-4, "row interval out of range");
  const int64_t per = int64_t(rows) << c.log_n;
  if (rot_stride < polys * per || out_stride < polys * per || pt_stride < per)
    return fail(-2, "strides smaller than one baby / giant / plaintext");
  return FHB_WORD(fhb::bsgs_inner, c, rot, rot_stride, pts, pt_stride, entries, table, giants, babies, out,
                  out_stride, polys, rows, row_start, st);
}

int fhb_ckks_rotate_multi(const fhb_context* ctx, const void* ct, const uint64_t* key_ptrs, const uint32_t* galois,
                          void* out, void* scratch, int64_t scratch_bytes, int64_t batch, int level,
                          fhb_stream stream) {
  CTX_OR_FAIL();
  TRY(fhb::check_ptr(ct, "ct"));
  TRY(fhb::check_ptr(out, "out"));
  TRY(fhb::check_ptr(scratch, "scratch"));
  if (!key_ptrs || !galois) return fail(-2, "key_ptrs and galois must be device arrays of batch entries");
  TRY(fhb::check_level(c, level));
  TRY(check_scratch(ctx, batch, level, scratch_bytes));
  const int limbs = c.num_q - level;
  const fhb::Scratch s = fhb::carve(c, scratch, batch, level);
  const int64_t comp = batch * limbs * c.n() * fhb::word_bytes(c);
  TRY(FHB_WORD(fhb::modup, c, static_cast<const char*>(ct) + comp, s.digits, batch, level, 1u, st, galois));
  TRY(ks_core_from_digits(c, s, nullptr, batch, level, st, key_ptrs));
  return FHB_WORD(fhb::moddown, c, s.t0, s.t1, ct, nullptr, out, batch, level, 1u, 0, st, galois);
}

// Rotation of a batch cut into k chunks, overlapped like the fused HMult:
// the ModUp digits (through sigma_g) of every chunk on stream [1] up front,
// the cores on stream [0] (highest priority), the ModDowns (+ sigma_g(c0)) on
// stream [2], so the element-wise stages run on the SMs the cores' clusters
// leave idle.  Results are those of the one-pass call.
static int rotate_chunked(const fhb_context* ctx, const char* ct, const void* key, char* out, char* scratch,
                          int64_t batch, int level, uint32_t galois, cudaStream_t st, int k) {
  const Context& c = *ctx->impl;
  Context& cm = const_cast<Context&>(c);
  std::lock_guard<std::mutex> lock(cm.ov_mutex);
  TRY(overlap_resources(cm));
  const int limbs = c.num_q - level;
  const int64_t wb = fhb::word_bytes(c), n = c.n();
  const int64_t pitch = batch * limbs * n;  // words between the components of ct and out
  const int64_t per_ct = fhb_ckks_keyswitch_scratch_bytes(ctx, 1, level);
  int64_t b0[fhb::kMaxOverlapChunks + 1];
  const int64_t base = std::max<int64_t>(4, batch / k / 4 * 4);
  for (int i = 0; i < k; ++i) b0[i] = std::min<int64_t>(batch, i * base);
  b0[k] = batch;
  cudaStream_t hi = cm.ov_streams[0], pre = cm.ov_streams[1], post = cm.ov_streams[2];
  const cudaEvent_t* ev = cm.ov_events.data();
  auto E = [&](int kind, int i) { return ev[4 + 4 * i + kind]; };  // 0: ModUp done, 1: core done
  auto bc = [&](int i) { return b0[i + 1] - b0[i]; };
  auto scr = [&](int i) { return fhb::carve(c, scratch + per_ct * b0[i], bc(i), level); };
  auto rec = [&](cudaEvent_t e, cudaStream_t s) { return fhb::cuda_status(cudaEventRecord(e, s), "overlap record"); };
  auto wait = [&](cudaStream_t s, cudaEvent_t e) {
    return fhb::cuda_status(cudaStreamWaitEvent(s, e, 0), "overlap wait");
  };
  TRY(rec(ev[0], st));
  for (cudaStream_t s : {hi, pre, post}) TRY(wait(s, ev[0]));
  for (int i = 0; i < k; ++i) {
    TRY(FHB_WORD(fhb::modup, c, ct + (pitch + b0[i] * limbs * n) * wb, scr(i).digits, bc(i), level, galois, pre));
    TRY(rec(E(0, i), pre));
  }
  for (int i = 0; i < k; ++i) {
    const fhb::Scratch s = scr(i);
    TRY(wait(hi, E(0, i)));
    TRY(ks_core_from_digits(c, s, key, bc(i), level, hi));
    TRY(rec(E(1, i), hi));
    TRY(wait(post, E(1, i)));
    const int64_t off = b0[i] * limbs * n * wb;
    TRY(FHB_WORD(fhb::moddown, c, s.t0, s.t1, ct + off, nullptr, out + off, bc(i), level, galois, 0, post, nullptr,
                 pitch));
  }
  for (int j = 0; j < 3; ++j) TRY(rec(ev[1 + j], cm.ov_streams[j]));
  for (int j = 0; j < 3; ++j) TRY(wait(st, ev[1 + j]));
  return 0;
}

int fhb_ckks_rotate(const fhb_context* ctx, const void* ct, const void* key, void* out, void* scratch,
                    int64_t scratch_bytes, int64_t batch, int level, uint32_t galois, fhb_stream stream) {
  CTX_OR_FAIL();
  TRY(fhb::check_ptr(ct, "ct"));
  TRY(fhb::check_ptr(key, "key"));
  TRY(fhb::check_ptr(out, "out"));
  TRY(fhb::check_ptr(scratch, "scratch"));
  TRY(fhb::check_level(c, level));
  TRY(fhb::check_galois(c, galois));
  TRY(check_scratch(ctx, batch, level, scratch_bytes));
  const int limbs = c.num_q - level;
  // chunks overlapped as in fhb_ckks_multiply_relinearize (not when out
  // overlaps ct: a chunk's ModDown must not overwrite input another chunk
  // still reads)
  const int k = int(std::min<int64_t>(c.overlap_chunks, batch / 8));
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  TRY(fhb::cuda_status(cudaStreamIsCapturing(st, &cap), "capture status"));
  const int64_t ct_bytes = 2 * batch * limbs * c.n() * fhb::word_bytes(c);
  if (k > 1 && cap == cudaStreamCaptureStatusNone && !(c.basis_tc && c.tc_moddown) &&
      !ranges_overlap(out, ct_bytes, ct, ct_bytes))
    return rotate_chunked(ctx, static_cast<const char*>(ct), key, static_cast<char*>(out),
                          static_cast<char*>(scratch), batch, level, galois, st, k);
  const fhb::Scratch s = fhb::carve(c, scratch, batch, level);
  const int64_t comp = batch * limbs * c.n() * fhb::word_bytes(c);
  TRY(FHB_WORD(fhb::modup, c, static_cast<const char*>(ct) + comp, s.digits, batch, level, galois, st));
  return keyswitch_tail(c, s, key, ct, nullptr, galois, out, batch, level, 0, st);
}

}  // extern "C"
