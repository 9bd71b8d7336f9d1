// Device-resident tables for one CKKS modulus chain (host-side definition).
#pragma once
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "fhb_arith.cuh"

namespace fhb {

constexpr int kMaxDigitWidth = 8;  // hybrid digit width bound (= P count)
constexpr int kMaxOverlapChunks = 8;  // chunks of the overlapped fused HMult

// One active hybrid digit at one level.
struct DigitDesc {
  int32_t prime0;     // first prime id of the digit (component-local row = prime0 - level)
  int32_t alpha;      // number of primes in the digit
  int32_t key_digit;  // stable level-zero key digit index
  int32_t pad;
};

// Word-size dependent device tables.  All TwPair entries are (w, Shoup(w)).
template <typename T>
struct ChainTables {
  PrimeInfo<T>* prime = nullptr;  // [QP]
  TwPair<T>* tw_fwd = nullptr;    // [QP][N]  psi^{br(k)}
  TwPair<T>* tw_inv = nullptr;    // [QP][N]  psi^{-br(k)}
  // ModDown by P (level independent): Garner constants of the P part and, per
  // prime id, Mp_k mod q and P^{-1} mod q.
  TwPair<T>* p_garner = nullptr;  // [8][8]
  TwPair<T>* p_mix = nullptr;     // [8][QP]
  TwPair<T>* p_inv = nullptr;     // [QP]
  // P R^{-1} mod q for the Q primes: Shoup(x, .) of a Montgomery-form NTT
  // value x = y R gives P y, the form in which an addend d enters the key-
  // switch accumulators before ModDown ((t + P d - [t]_P) / P = (t - [t]_P) / P + d).
  TwPair<T>* p_rinv = nullptr;    // [QP]
  // FP64 tables only: the twiddle values alone, [QP][N] in the order of
  // tw_fwd / tw_inv, for the standalone transforms, whose butterflies take
  // the quotient from the product and 1/q (prime.one_s).
  T* twv_fwd = nullptr;
  T* twv_inv = nullptr;
};

// Per-level key-switch / rescale tables (device).
template <typename T>
struct LevelTables {
  int num_digits = 0;
  DigitDesc* digits = nullptr;    // [nd]
  TwPair<T>* garner = nullptr;    // [nd][8][8]: [k][i<k] = M_i mod b_k, [k][k] = M_k^{-1} mod b_k
  TwPair<T>* ext = nullptr;       // [nd][8][QP]: M_r mod p  (M_0 = 1)
  TwPair<T>* rescale_inv = nullptr;  // [QP]: q_level^{-1} mod p (rows > level)
};

// Tables of the exact int8 tensor-core NTT (int32 residues, N = 2^16), built
// on first use.  All device arrays are owned through Context::allocations.
struct TcNttTables {
  uint8_t* bmat[6] = {};              // per pass: [QP][byte matrix of the pass] (64 KiB or 4 KiB per prime)
  uint32_t* post[6] = {};             // per pass with a twiddle: [QP][N] t 2^32 mod q in output order, else null
  uint32_t* qinfo = nullptr;          // [QP][2]: q, -q^{-1} mod 2^32
  int* err = nullptr;                 // device flag: a bounded wait gave up
};

// Tables of the exact int8 tensor-core basis conversion (int64 residues),
// built on first use.  All device arrays are owned through
// Context::allocations.
struct TcBasisTables {
  std::vector<uint8_t*> bmat;     // per level: [digit][16-row chunk][128 x 32 ks] byte matrices
  std::vector<uint8_t*> md_bmat;  // per level: [16-row chunk of Q_l][128 x 32 ks] ModDown byte matrices
  uint64_t* pinfo = nullptr;      // [QP][2]: p, -p^{-1} mod 2^64
  int ks = 1;                     // K-steps of 32 bytes (digits of up to 4 or 8 primes)
  int sms = 0;                    // multiprocessors of the context's device (one CTA each)
  int* err = nullptr;             // device flag: a bounded wait gave up
};

struct Context {
  int bits = 0;        // 64 or 32
  int log_n = 0;
  int num_q = 0;
  int num_p = 0;
  int device = 0;
  std::vector<uint64_t> moduli;
  std::vector<uint64_t> roots;  // primitive 2N-th roots psi
  ChainTables<uint64_t> t64;
  ChainTables<uint32_t> t32;
  std::vector<LevelTables<uint64_t>> lv64;
  std::vector<LevelTables<uint32_t>> lv32;
  // the same per-level tables as a device array [num_q] (kernels over
  // ciphertexts of several levels index it by each item's level)
  LevelTables<uint64_t>* lv64_dev = nullptr;
  LevelTables<uint32_t>* lv32_dev = nullptr;
  std::vector<void*> allocations;
  int ks_order = 2;  // tuning: work order of the key-switch clusters (see ks_work)
  int ntt_ept_fwd = 0;  // tuning: residues per thread of the standalone forward NTT (0 = default)
  int ntt_ept_inv = 0;  // tuning: same for the inverse NTT and the fused HMult -> inverse NTT
  TcNttTables* tc = nullptr;  // tensor-core NTT tables (null until prepared)
  std::mutex tc_mutex;
  // tuning: basis conversion of the key switch on the CUDA cores (0) or the
  // int8 tensor cores (1, int64 contexts)
  int basis_tc = 0;
  // tuning, with basis_tc: ModDown's P -> Q conversion on the tensor cores
  // (1) or on the CUDA cores (0, default: faster on B200)
  int tc_moddown = 0;
  // FP64 tables for the tensor-core form's key-switch core (int64 chains whose
  // Q primes are below 2^42): per-prime constants and twiddles as (c, c / q)
  // double pairs; p_rinv holds P mod q (the FP64 core's accumulators carry R)
  ChainTables<double> t64f;
  // FP64 extension constants of every level's digits for the FP64 rows:
  // [level][digit][r][2][QP] pairs, [.][0] = (M_r mod p) 2^30 mod p (for the
  // 30-bit halves of digits that hold a wider prime), [.][1] = M_r mod p
  TwPair<double>* ext64f = nullptr;
  int ext64f_digits = 0;  // digits per level in that layout (those of level 0)
  bool f64_tables_ok = false;
  int f64_prime_end = 0;  // Q primes [0, f64_prime_end) are below 2^42 (FP64 rows)
  // tuning: the rows of primes below 2^42 run in FP64 arithmetic (1, default
  // when the tables exist: the NTTs and the key-switch kernels) or on the
  // integer pipe (0)
  int f64_core = 1;
  // tuning: chunks of the fused HMult + relinearise (+ rescale) call whose
  // element-wise stages run beside the other chunks' key-switch cores (1 =
  // one pass over the batch); streams and events created on first use and
  // guarded by ov_mutex: [0] the cores and transforms (highest priority),
  // [1] tensor products and ModUp digits, [2] ModDown (lowest priority)
  int overlap_chunks = 4;
  cudaStream_t ov_streams[3] = {};
  std::vector<cudaEvent_t> ov_events;
  std::mutex ov_mutex;
  // tuning: the tensor-core NTT's 16-point pass fused with the adjacent
  // 64-point pass (1) or three separate passes (0, default: faster on B200)
  int tc_ntt_fused = 0;
  // limit of the tensor-core kernels' pipeline waits in ns (0 = the default
  // second); their drain waits always keep the default
  unsigned long long tc_wait_ns = 0;
  // test only: tensor-core kernels first wait on a barrier nothing completes
  // (so their pipeline limit runs out and they report it)
  int tc_test_stall = 0;
  TcBasisTables* tcb = nullptr;  // tensor-core basis conversion tables (null until prepared)
  std::mutex tcb_mutex;
  std::vector<std::vector<DigitDesc>> level_digits;  // host copy of each level's active digits
  int qp() const { return num_q + num_p; }
  int n() const { return 1 << log_n; }
};

template <typename T>
inline const ChainTables<T>& tables(const Context& c);
template <>
inline const ChainTables<uint64_t>& tables<uint64_t>(const Context& c) { return c.t64; }
template <>
inline const ChainTables<uint32_t>& tables<uint32_t>(const Context& c) { return c.t32; }
template <typename T>
inline const LevelTables<T>& level_tables(const Context& c, int level);
template <>
inline const LevelTables<uint64_t>& level_tables<uint64_t>(const Context& c, int level) { return c.lv64[level]; }
template <>
inline const LevelTables<uint32_t>& level_tables<uint32_t>(const Context& c, int level) { return c.lv32[level]; }
template <typename T>
inline const LevelTables<T>* level_tables_dev(const Context& c);
template <>
inline const LevelTables<uint64_t>* level_tables_dev<uint64_t>(const Context& c) { return c.lv64_dev; }
template <>
inline const LevelTables<uint32_t>* level_tables_dev<uint32_t>(const Context& c) { return c.lv32_dev; }

// Exact int8 tensor-core NTT (fhb_tc_ntt.cu).  tc_ntt_prepare builds the
// tables once (blocking); tc_ntt runs both passes of one direction;
// tc_ntt_status reads and clears the device error flag (synchronising);
// tc_ntt_tables_host fills one pass's tables for one prime on the host.
int tc_ntt_prepare(Context& c);
int tc_ntt(Context& c, const void* in, void* out, int64_t polys, int rows, int row_start, bool inverse,
           cudaStream_t st);
int tc_ntt_status(Context& c, int* flag);
size_t tc_ntt_table_bytes(int pass);
void tc_ntt_tables_host(uint64_t q, uint64_t psi, int pass, uint8_t* bmat, uint32_t* post);

// Exact int8 tensor-core basis conversion (fhb_tc_basis.cu).  tc_extend
// writes the extensions of every active digit of `level` to every row of
// Q_l P: ext [digits][batch][QP_l][N] in [0, 2p) (tc_ext_words words), from
// the Garner digits [batch][L][N]; skip_own leaves a digit's own rows
// unwritten.  tc_basis_status reads and clears the device error flag.
int tc_basis_prepare(Context& c);
int64_t tc_ext_words(const Context& c, int64_t batch, int level);
int tc_extend(Context& c, const void* digits, void* ext, int64_t batch, int level, bool skip_own, cudaStream_t st);
int tc_basis_status(Context& c, int* flag);
// ModDown by P (+ addends, + rescale) with the P -> Q conversion on the
// tensor cores; same arguments and result as the CUDA-core ModDown.
int tc_moddown(Context& c, const void* t0, const void* t1, const void* add0, const void* add1, void* out,
               int64_t batch, int level, uint32_t add0_ginv, const uint32_t* item_galois, int rescale,
               cudaStream_t st);
void tc_basis_tables_host(const Context& c, int level, int ks, std::vector<uint8_t>& out);

// Host-side status plumbing shared by the C ABI.
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_status(cudaError_t e, const char* where);
// Opt `kernel` into `bytes` of dynamic shared memory on the current device,
// once per (device, kernel): later launches (also those recorded into CUDA
// graphs) make no further runtime calls.
int ensure_dynamic_smem(const void* kernel, int bytes);

}  // namespace fhb
