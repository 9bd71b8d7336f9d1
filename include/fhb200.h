/*
 * fhelium_b200 C ABI: B200 (sm_100a) kernels for the CKKS evaluation path of
 * visualDust/fhelium.
 *
 * Conventions shared by every entry point
 * ----------------------------------------
 *  - Residue buffers are device pointers to contiguous little-endian words,
 *    uint64 for the int64 family (62-bit buffer, primes < 2^60) and uint32
 *    for the int32 family (30-bit buffer, primes < 2^28), laid out exactly
 *    like the reference's tensors: [*batch, limb, N] with limb j holding the
 *    residue modulo prime id (level + j) of the level-zero chain
 *    [scale q..., base q, p...]  (reference fhelium/core/ciphertext.py:26-67,
 *    fhelium/engine/rns/chain.py).  Ciphertexts are [component, *batch, limb, N].
 *  - Residue states follow the reference: NTT domain = Montgomery form
 *    (x * 2^62 or x * 2^30 mod q), lazy in [0, 2q); coefficient domain =
 *    standard form, canonical in [0, q).
 *  - Every call is asynchronous on `stream` (a cudaStream_t, NULL = legacy
 *    default stream), allocates nothing, and returns 0 on success, a
 *    negative value for an invalid argument and 1000 + cudaError_t for a CUDA
 *    failure; fhb_last_error() gives the message of the calling thread's last
 *    failure.  Buffers must be 16-byte aligned and must not overlap unless an
 *    entry point says so.
 *  - Each entry point names the reference interface it replaces
 *    (file:line in the reference project).
 */
#ifndef FHB200_H
#define FHB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fhb_context fhb_context;
typedef void* fhb_stream; /* cudaStream_t */

enum fhb_inverse_output {
  FHB_INV_MONTGOMERY = 0,    /* coefficient/Montgomery lazy [0, 2q) */
  FHB_INV_STANDARD_LAZY = 1, /* coefficient/standard lazy [0, 2q) */
  FHB_INV_STANDARD = 2,      /* coefficient/standard canonical [0, q) */
  FHB_INV_CENTERED = 3       /* coefficient/standard centred (signed) */
};

int fhb_version(void);

/* Diagnostic: blocks x 256 threads each run 8 independent chains of `iters`
 * Shoup modular products (the butterfly product) on registers and write one
 * word per thread to out (blocks * 256 words): blocks * 256 * 8 * iters
 * products, the attainable modular-multiplication rate the NTT-based
 * kernels are measured against.  No counterpart in the reference. */
int fhb_modmul_probe(const fhb_context* ctx, void* out, int blocks, int iters, fhb_stream stream);
/* Diagnostic: the same for the balanced FP64 product of the rows of primes
 * below 2^42 (out: blocks * 256 doubles); -7 when the chain has none. */
int fhb_modmul_probe_f64(const fhb_context* ctx, void* out, int blocks, int iters, fhb_stream stream);
const char* fhb_last_error(void);

/* Build the device tables (twiddles with Shoup companions, Montgomery
 * constants, hybrid-digit Garner/extension constants for every level, ModDown
 * and rescale constants) of one modulus chain on `device`.  moduli =
 * num_q + num_p primes in reference order.  residue_bits is 64 or 32.
 * Replaces the table construction of RnsRuntime / CkksEngine.__init__
 * (fhelium/engine/rns/runtime.py:136-216, fhelium/engine/ckks_engine.py:
 * 2952-3068).  This is set-up: it allocates and copies synchronously. */
int fhb_context_create(int residue_bits, int log_n, const uint64_t* moduli, int num_q, int num_p,
                       int device, fhb_context** out);
int fhb_context_destroy(fhb_context* ctx);
/* The primitive 2N-th root psi used for prime `prime_id` (same choice as
 * fhelium/engine/ntt/plans/twiddles.py:10-20). */
int fhb_context_root(const fhb_context* ctx, int prime_id, uint64_t* psi);

/* Launch tuning of a context (set by the autotuner, fhelium_b200/autotune.py).
 * FHB_TUNE_KS_ORDER: work order of the key-switch clusters, 0 = the rows of
 * one ciphertext back to back, 1 = one row across the batch back to back,
 * 2 = one row across a group of four ciphertexts, group by group (default).
 * FHB_TUNE_NTT_FORWARD_EPT / FHB_TUNE_NTT_INVERSE_EPT: residues per thread of
 * the standalone forward / inverse NTT (and of the fused HMult -> inverse
 * NTT): 8 = radix-8 register passes, 16 = radix-16 passes over half the
 * threads, 0 = the ring's default.
 * FHB_TUNE_BASIS_CONVERSION: 0 = the key switch's exact basis extension on
 * the CUDA cores, fused into the key-switch core (the context's default; the
 * Python engine's "auto" keeps it on chains with FP64 rows and sets 1 on
 * other int64 chains); 1 = on the int8
 * tensor cores (int64 contexts; fhb_tc_basis_extend), the core then reads the
 * materialised extensions (key-switch scratch grows by
 * fhb_tc_basis_extend_words x 8 bytes).  Setting 1 builds its tables
 * (blocking).
 * FHB_TUNE_TC_WAIT_US: limit of the tensor-core kernels' pipeline waits in
 * microseconds (0 = the default second); a wait that runs out makes the
 * kernel return early and raise its status flag (fhb_tc_basis_status,
 * fhb_tc_ntt_status).  Their drain waits keep the default.  For tests.
 * FHB_TUNE_TC_TEST_STALL: 1 = every tensor-core launch first waits on a
 * barrier that nothing completes, so its pipeline limit runs out and the
 * abort path (drain, TMEM release, status flag) runs; outputs are then
 * invalid.  For tests of that path only.
 * FHB_TUNE_TC_MODDOWN (with the tensor-core form): 1 = ModDown's P -> Q
 * conversion on the tensor cores too, 0 = on the CUDA cores (default: faster
 * on B200).
 * FHB_TUNE_TC_NTT_FUSED: fhb_tc_forward_ntt / fhb_tc_inverse_ntt in two
 * launches, the 16-point pass fused with the adjacent 64-point pass over each
 * 8192-word span (1), or in three (0, default: faster on B200).
 * FHB_TUNE_F64_CORE (int64 chains): 1 = the rows of primes below 2^42 run in
 * exact FP64 arithmetic (integers held in doubles, balanced residues,
 * products on the FP64 pipe; default) in the forward / inverse NTTs and, for
 * N <= 2^16, in the key-switch core (both basis-conversion forms), the
 * hoisted-rotation kernels and the mixed-level items stages; 0 = on the
 * integer pipe.  Reads back 0 where the chain has no such primes.
 * FHB_TUNE_OVERLAP_CHUNKS (1..8, default 4): fhb_ckks_multiply_relinearize
 * and fhb_ckks_rotate cut a batch of at least 16 ciphertexts into at most
 * this many chunks and run one chunk's element-wise stages (tensor product,
 * ModUp digits, ModDown) on low-priority streams beside another chunk's
 * key-switch core, whose 8-CTA clusters leave SMs idle; 1 = one pass over
 * the batch.  The streams belong to the context and are forked from and
 * joined back into the caller's stream.  Under stream capture, or when the
 * output overlaps an input, the call runs in one pass.
 * Results do not depend on any of these (stall aside).  No counterpart in the reference
 * (its launch shapes and arithmetic units are fixed). */
enum fhb_tuning_param {
  FHB_TUNE_KS_ORDER = 0,
  FHB_TUNE_NTT_FORWARD_EPT = 1,
  FHB_TUNE_NTT_INVERSE_EPT = 2,
  FHB_TUNE_BASIS_CONVERSION = 3,
  FHB_TUNE_TC_WAIT_US = 4,
  FHB_TUNE_TC_TEST_STALL = 5,
  FHB_TUNE_TC_MODDOWN = 6,
  FHB_TUNE_TC_NTT_FUSED = 7,
  FHB_TUNE_F64_CORE = 8,
  FHB_TUNE_OVERLAP_CHUNKS = 9
};
int fhb_context_set_tuning(fhb_context* ctx, int param, int value);
int fhb_context_get_tuning(const fhb_context* ctx, int param, int* value);

/* Forward negacyclic NTT of `batch` x `rows` polynomials whose rows are prime
 * ids [row_start, row_start + rows).  input_montgomery = 0: standard input,
 * output x R (forward_ntt_to_montgomery_*); = 1: Montgomery input
 * (forward_ntt_montgomery_*).  Output lazy [0, 2q).  in == out allowed.
 * Replaces fhelium_ntt_ops.forward_ntt_{to_montgomery,montgomery}_compact_
 * grouped_smem_ (csrc/ops/ntt/forward_ntt.cpp:25-67,
 * csrc/ops/ntt/cuda/forward_ntt_cuda.cpp:77-90). */
int fhb_forward_ntt(const fhb_context* ctx, const void* in, void* out, int64_t batch, int rows,
                    int row_start, int input_montgomery, fhb_stream stream);

/* Exact int8 tensor-core forms of the two transforms above (tcgen05.mma
 * kind::i8, int32 accumulation in tensor memory): a 64 x 64 x 16 three-pass
 * NTT whose passes run over the residues' four bytes and byte-split constant
 * matrices held in shared memory, reduced exactly in the epilogue.  int32
 * contexts with log_n = 16 only (else -7).
 *   fhb_tc_forward_ntt: standard input -> NTT/Montgomery output, canonical
 *     [0, q): equal mod q to fhb_forward_ntt(input_montgomery = 0), whose
 *     output is lazy [0, 2q) (forward_ntt_to_montgomery_compact_grouped_smem_,
 *     csrc/ops/ntt/forward_ntt.cpp:25-67).
 *   fhb_tc_inverse_ntt: NTT/Montgomery input (any word value) -> standard
 *     canonical, bit-identical to fhb_inverse_ntt(output_kind = 2)
 *     (inverse_ntt_to_standard_compact_grouped_smem_, csrc/ops/ntt/
 *     inverse_ntt.cpp:23-73).
 * in == out allowed; no scratch.  The first call builds the constants
 * (byte matrices and twiddles, about 2 MiB per prime, blocking) unless
 * fhb_tc_ntt_prepare ran.  fhb_tc_ntt_status synchronises, returns in *flag
 * whether a bounded wait inside the kernels gave up since the last call
 * (outputs then invalid), and clears the flag.  fhb_tc_ntt_tables_host (host
 * only, no device) fills, for a prime q < 2^28 with primitive 2N-th root psi
 * at N = 2^16, the byte matrix of one pass (passes 0-2 forward, 3-5 inverse;
 * 64 KiB for passes 0, 1, 4, 5 and 4 KiB for passes 2, 3, in the kernels'
 * shared-memory layout) and, for the twiddled passes 0, 1, 3, 4 when post is
 * not NULL, the N twiddles t as t 2^32 mod q (uint32) in output order. */
int fhb_tc_ntt_prepare(const fhb_context* ctx);
int fhb_tc_forward_ntt(const fhb_context* ctx, const void* in, void* out, int64_t batch, int rows,
                       int row_start, fhb_stream stream);
int fhb_tc_inverse_ntt(const fhb_context* ctx, const void* in, void* out, int64_t batch, int rows,
                       int row_start, fhb_stream stream);
int fhb_tc_ntt_status(const fhb_context* ctx, int* flag);

/* Exact int8 tensor-core basis extension (int64 contexts): from the Garner
 * digits [batch, L, N] of fhb_ckks_modup_digits, ext [D_l, batch, L+P, N]
 * receives, for every active hybrid digit, its exact extension
 * sum_r d_r (M_r mod p) to every row of Q_l P, in [0, 2p)
 * (fhb_tc_basis_extend_words words).  Equals, modulo p, the reference's
 * mixed_radix_basis_extend_to_montgomery without the Montgomery factor
 * (csrc/ops/rns/cuda/mixed_radix_cuda.cu:146-182).  fhb_tc_basis_status
 * synchronises, returns in *flag whether a bounded wait of the kernel gave
 * up since the last call (outputs then invalid), and clears the flag. */
int fhb_tc_basis_extend(const fhb_context* ctx, const void* digits, void* ext, int64_t batch, int level,
                        fhb_stream stream);
int64_t fhb_tc_basis_extend_words(const fhb_context* ctx, int64_t batch, int level);
int fhb_tc_basis_status(const fhb_context* ctx, int* flag);
int fhb_tc_ntt_tables_host(uint64_t q, uint64_t psi, int pass, uint8_t* bmat, uint32_t* post);

/* Inverse NTT from NTT/Montgomery lazy input, output per fhb_inverse_output.
 * in == out allowed.  Replaces fhelium_ntt_ops.inverse_ntt_{montgomery,
 * to_standard_lazy,to_standard,to_centered}_compact_grouped_smem_
 * (csrc/ops/ntt/inverse_ntt.cpp:23-73). */
int fhb_inverse_ntt(const fhb_context* ctx, const void* in, void* out, int64_t batch, int rows,
                    int row_start, int output_kind, fhb_stream stream);

/* NTT-domain tensor product of two level-`level` ciphertexts a, b
 * [2, batch, L, N] -> out [3, batch, L, N] (Montgomery lazy).  Replaces
 * CkksEngine.multiply (fhelium/engine/ckks_engine.py:1530-1606: four
 * fhelium_rns_ops.montgomery_mul + one add_lazy). */
int fhb_ckks_multiply(const fhb_context* ctx, const void* a, const void* b, void* out, int64_t batch,
                      int level, fhb_stream stream);

/* Tensor product fused with the inverse NTT of all three products:
 * out [3, batch, L, N] coefficient/standard canonical.  Equals multiply
 * followed by the three inverse_to_standard_ calls that open
 * CkksEngine.relinearize (fhelium/engine/ckks_engine.py:1655-1660). */
int fhb_ckks_multiply_to_coefficient(const fhb_context* ctx, const void* a, const void* b, void* out,
                                     int64_t batch, int level, fhb_stream stream);

/* ModUp stage 1: Garner mixed-radix digits of every active hybrid digit of a
 * coefficient/standard component comp [batch, L, N] -> digits [batch, L, N].
 * galois != 1 first applies sigma_g (X -> X^g) to comp.  Replaces the
 * per-digit fhelium_rns_ops.mixed_radix_decompose calls
 * (fhelium/engine/hybrid_keyswitch.py:95-170,
 * csrc/ops/rns/cuda/mixed_radix_cuda.cu:31-79) and, for rotations, the
 * coefficient automorphism of c1 (csrc/ops/ckks/cuda/automorphism_cuda.cu:15-31). */
int fhb_ckks_modup_digits(const fhb_context* ctx, const void* comp, void* digits, int64_t batch,
                          int level, uint32_t galois, fhb_stream stream);

/* Fused ModUp stage 2 + forward NTT + key inner product + inverse NTT.
 * digits [batch, L, N] (from fhb_ckks_modup_digits); key [D, 2, QP0, N]
 * NTT/Montgomery (reference KeySwitchKey layout, key_generator.py:243-262);
 * acc0, acc1 [batch, L + P, N] receive coefficient/standard canonical rows.
 * Replaces, per digit, mixed_radix_basis_extend_to_montgomery + the forward
 * NTT + keyswitch_accumulate_digit_products_ and the two inverse NTTs of
 * _moddown_switch_accumulators (fhelium/engine/hybrid_keyswitch.py:321-371,
 * 530-546; csrc/ops/ckks/cuda/keyswitch_cuda.cu:198-292). */
int fhb_ckks_keyswitch_core(const fhb_context* ctx, const void* digits, const void* key, void* acc0,
                            void* acc1, int64_t batch, int level, fhb_stream stream);

/* The key-switch core of the tensor-core form: as fhb_ckks_keyswitch_core,
 * but from the digit extensions of fhb_tc_basis_extend ([D_l, batch, L+P, N],
 * int64 contexts) instead of the Garner digits, so the core only transforms,
 * multiplies by the key and accumulates.  Same result. */
int fhb_ckks_keyswitch_core_extended(const fhb_context* ctx, const void* ext, const void* key, void* acc0,
                                     void* acc1, int64_t batch, int level, fhb_stream stream);

/* ModDown by P, fused with the final addition and optionally the rescale.
 * t0, t1 [batch, L + P, N] canonical; add0, add1 [batch, L, N] canonical or
 * NULL; add0 is read through sigma_g when add0_galois != 1.
 * out [2, batch, L - (rescale ? 1 : 0), N] canonical.  Replaces
 * fhelium_ckks_ops.keyswitch_moddown_qp_to_q (csrc/ops/ckks/ckks.cpp:82-84),
 * the d + correction / add_canonical that follows it
 * (fhelium/engine/ckks_engine.py:1664-1667, :3334-3350) and
 * rescale_drop_leading_prime_nearest (csrc/ops/ckks/ckks.cpp:61-64). */
int fhb_ckks_moddown(const fhb_context* ctx, const void* t0, const void* t1, const void* add0,
                     const void* add1, void* out, int64_t batch, int level, uint32_t add0_galois,
                     int rescale, fhb_stream stream);

/* Hoisting: NTT-domain extended digits of one ModUp, prepared
 * [D_l, batch, L + P, N].  Replaces HybridKeySwitcher.prepare_rotation_digits
 * (fhelium/engine/hybrid_keyswitch.py:373-417). */
int fhb_ckks_prepare_rotation(const fhb_context* ctx, const void* digits, void* prepared, int64_t batch,
                              int level, fhb_stream stream);

/* Hoisting: per step, NTT-domain sigma_g of the prepared digits, key inner
 * product and inverse NTT into acc0/acc1 [batch, L + P, N].  Replaces
 * _apply_prepared_rotation (fhelium/engine/hybrid_keyswitch.py:419-469). */
int fhb_ckks_apply_prepared_rotation(const fhb_context* ctx, const void* prepared, const void* key,
                                     void* acc0, void* acc1, int64_t batch, int level, uint32_t galois,
                                     fhb_stream stream);

/* Rescale `polys` coefficient/standard polynomials [polys, L, N] ->
 * [polys, L - 1, N] by the leading prime (nearest or truncating).  Replaces
 * fhelium_ckks_ops.rescale_drop_leading_prime_{nearest,truncate}
 * (csrc/ops/ckks/ckks.cpp:57-72, csrc/ops/ckks/cuda/rescale_cuda.cu:22-92). */
int fhb_ckks_rescale(const fhb_context* ctx, const void* in, void* out, int64_t polys, int level,
                     int nearest, fhb_stream stream);

/* Coefficient-domain Galois automorphism sigma_g of [batch, rows, N] (rows =
 * prime ids [row_start, row_start + rows)), canonical output, in != out.
 * Replaces fhelium_ckks_ops.apply_coefficient_galois_automorphism
 * (csrc/ops/ckks/ckks.cpp:73-76). */
int fhb_ckks_automorphism(const fhb_context* ctx, const void* in, void* out, int64_t batch, int rows, int row_start,
                          uint32_t galois, fhb_stream stream);

/* out = a + b (mod q) over [polys, L, N]; lazy = 1 keeps [0, 2q)
 * (fhelium_rns_ops.add_lazy), lazy = 0 gives canonical output
 * (fhelium_rns_ops.add_canonical, csrc/ops/rns/rns_canonical_arithmetic.cpp:15-23). */
int fhb_ckks_add(const fhb_context* ctx, const void* a, const void* b, void* out, int64_t polys,
                 int level, int lazy, fhb_stream stream);

enum fhb_rns_op {
  FHB_OP_MONTGOMERY_MUL = 0, /* REDC(a b): fhelium_rns_ops.montgomery_mul */
  FHB_OP_ADD_LAZY = 1,       /* fhelium_rns_ops.add_lazy */
  FHB_OP_SUB_LAZY = 2,       /* fhelium_rns_ops.sub_lazy */
  FHB_OP_ADD_CANONICAL = 3,  /* fhelium_rns_ops.add_canonical */
  FHB_OP_SUB_CANONICAL = 4,  /* fhelium_rns_ops.sub_canonical */
  FHB_OP_NEGATE = 5          /* canonical negation (b unused) */
};

/* Pointwise RNS arithmetic on [batch, rows, N] (rows = prime ids
 * [row_start, row_start + rows)).  b_mode 0: b has a's shape; 1: b is
 * [rows, N] shared by the batch; 2: b is [rows] row scalars
 * (montgomery_mul_row_scalars_).  out may alias a.  Replaces
 * csrc/ops/rns/rns_arithmetic.cpp:30-72 and
 * csrc/ops/rns/rns_canonical_arithmetic.cpp:15-23. */
int fhb_rns_binary(const fhb_context* ctx, int op, const void* a, const void* b, void* out, int64_t batch, int rows,
                   int row_start, int b_mode, fhb_stream stream);

/* Lift signed int64 coefficients [batch, N] into canonical residues
 * [batch, rows, N].  Replaces fhelium_rns_ops.lift_centered_coefficients
 * (csrc/ops/rns/rns_arithmetic.cpp:30-72). */
int fhb_rns_lift_signed(const fhb_context* ctx, const int64_t* coefficients, void* out, int64_t batch, int rows,
                        int row_start, fhb_stream stream);

/* Multiply [batch, rows, N] coefficient/standard polynomials by X^k
 * (0 <= k < 2N) in Z[X]/(X^N + 1); in != out.  Replaces the bootstrap's
 * monomial multiplication (fhelium/experimental/bootstrap/_full_slot.py:
 * _multiply_by_monomial). */
int fhb_ckks_monomial(const fhb_context* ctx, const void* in, void* out, int64_t batch, int rows, int row_start, int k,
                      fhb_stream stream);

/* ModRaise: centred lift of [batch, N] coefficient/standard residues modulo
 * prime `src_prime` to [batch, rows, N] over prime ids [row_start,
 * row_start + rows).  Replaces the bootstrap's modulus raise
 * (fhelium/experimental/bootstrap/_modraise.py:338). */
int fhb_ckks_modraise(const fhb_context* ctx, const void* in, void* out, int64_t batch, int src_prime, int rows,
                      int row_start, fhb_stream stream);

/* data[b, r, 0] += constants[r] (coefficient domain, all_slots = 0) or
 * data[b, r, :] += constants[r] (NTT domain, all_slots = 1), canonical
 * constants; in place.  Replaces the constant additions of the bootstrap's
 * polynomial evaluators (fhelium/experimental/bootstrap/_polynomial.py). */
int fhb_rns_add_constant(const fhb_context* ctx, void* data, const void* constants, int64_t batch, int rows,
                         int row_start, int all_slots, fhb_stream stream);

/* Scratch bytes needed by fhb_ckks_relinearize / fhb_ckks_rotate. */
int64_t fhb_ckks_keyswitch_scratch_bytes(const fhb_context* ctx, int64_t batch, int level);

/* HMult-result relinearisation (optionally fused with the rescale):
 * ct3 [3, batch, L, N] NTT/Montgomery -> out [2, batch, L (- 1), N]
 * coefficient/standard canonical.  Replaces CkksEngine.relinearize
 * (+ rescale_to_next_level) (fhelium/engine/ckks_engine.py:1608-1675,
 * fhelium/engine/ckks_rescale.py:339-377).  scratch: device buffer of at
 * least fhb_ckks_keyswitch_scratch_bytes(ctx, batch, level) bytes. */
int fhb_ckks_relinearize(const fhb_context* ctx, const void* ct3, const void* key, void* out,
                         void* scratch, int64_t scratch_bytes, int64_t batch, int level, int rescale,
                         fhb_stream stream);

/* fhb_ckks_relinearize for callers that cannot allocate device memory.  No
 * counterpart in the reference.  Same arguments and result as
 * fhb_ckks_relinearize minus the scratch buffer: the scratch is a fixed
 * 32 MiB array inside the library (fhb_ckks_relinearize_noalloc_max_scratch_bytes),
 * held by every GPU that loads it until the process exits.  Meant for code
 * that is handed only its input and output buffers, e.g. a plugin inside a
 * host framework whose memory pool owns all device memory, or a serving loop
 * that must not allocate.  Batches needing more than the fixed size
 * (fhb_ckks_keyswitch_scratch_bytes) are rejected with an error, and so are a
 * negative batch and an invalid level.  Usable range: the largest batch is
 * 32 MiB / fhb_ckks_keyswitch_scratch_bytes(ctx, 1, level), e.g. 5 at level 0
 * of slots8192_scale40_levels7_int64, 1 at level 0 of
 * slots16384_scale40_levels16_int64, none below level 26 of
 * slots32768_scale40_levels34_int64 (1 from level 26 on).  The first call on
 * a device looks the array's address up (cudaGetSymbolAddress) and should
 * come before any stream capture; the address is kept for the life of the
 * process, so do not use this entry point across a cudaDeviceReset.  All
 * calls share the array: calls that can overlap on the GPU (other streams,
 * other host threads) race. */
int fhb_ckks_relinearize_noalloc(const fhb_context* ctx, const void* ct3, const void* key, void* out, int64_t batch,
                                 int level, int rescale, fhb_stream stream);
int64_t fhb_ckks_relinearize_noalloc_max_scratch_bytes(void);

/* HMult + relinearise (+ rescale) in one call: a, b [2, batch, L, N]
 * NTT/Montgomery -> out [2, batch, L (- 1), N] coefficient/standard. */
int fhb_ckks_multiply_relinearize(const fhb_context* ctx, const void* a, const void* b, const void* key,
                                  void* out, void* scratch, int64_t scratch_bytes, int64_t batch, int level,
                                  int rescale, fhb_stream stream);

/* Rotation with a direct key: ct [2, batch, L, N] coefficient/standard ->
 * out [2, batch, L, N].  galois = Galois element g of the step.  Replaces
 * CkksEngine._apply_rotation_key (fhelium/engine/ckks_engine.py:3822-3897). */
int fhb_ckks_rotate(const fhb_context* ctx, const void* ct, const void* key, void* out, void* scratch,
                    int64_t scratch_bytes, int64_t batch, int level, uint32_t galois, fhb_stream stream);

/* Key switches of `giants` ciphertexts with their own keys, summed before
 * the inverse NTT ("lazy ModDown"): digits [giants, batch, L, N] from
 * fhb_ckks_modup_digits (sigma_g applied per giant), key_ptrs a DEVICE array
 * of `giants` key addresses ([D, 2, QP0, N] each); acc0, acc1 [batch, L+P, N]
 * receive coefficient/standard rows for one fhb_ckks_moddown.  The result is
 * within `giants` units of the sum of separately rounded key switches.
 * Replaces the rotate-and-add of every giant step of the reference's BSGS
 * linear transforms (fhelium/experimental/bootstrap/_linear.py:235-393). */
int fhb_ckks_keyswitch_sum(const fhb_context* ctx, const void* digits, const uint64_t* key_ptrs, void* acc0,
                           void* acc1, int giants, int64_t batch, int level, fhb_stream stream);

/* fhb_ckks_keyswitch_sum of the tensor-core form (int64 contexts): from the
 * extensions of the giants' digits, i.e. fhb_tc_basis_extend of the digits
 * [giants, batch, L, N] taken as one batch of giants x batch ciphertexts
 * (ext [D_l, giants x batch, L+P, N]).  Same result. */
int fhb_ckks_keyswitch_sum_extended(const fhb_context* ctx, const void* ext, const uint64_t* key_ptrs, void* acc0,
                                    void* acc1, int giants, int64_t batch, int level, fhb_stream stream);

/* ---- mixed-level batches: one launch per stage over every item ----------
 * One item is one ciphertext (batch 1) with its own operation and level:
 * HMult + relinearise + rescale of a and b (kind 0), or a rotation of a by
 * its own Galois element with its own key (kind 1).  fhb_ckks_items_plan_info
 * (host only) validates the items and returns the plan and scratch sizes;
 * fhb_ckks_items_plan writes the device plan (item descriptors with their
 * scratch regions resolved, and the work lists of the cluster stages) into
 * `plan` with a blocking copy, binding it to `scratch`; fhb_ckks_items_run
 * then issues six launches over all items - forward NTT of the HMult
 * operands, tensor product, inverse NTT of d2, ModUp digits, key-switch
 * core, ModDown with the rescale or with sigma_g(c0) - with no host call, so
 * it can be captured in a CUDA graph and replayed (the plan, scratch, inputs
 * and outputs must stay allocated).  Results are integer-equal to the
 * per-level calls (fhb_ckks_multiply_relinearize with rescale after a
 * forward NTT of the operands, fhb_ckks_rotate).  Replaces the reference's
 * one engine call sequence per ciphertext (fhelium/engine/ckks_engine.py:
 * 1530-1675, 2183-2300), which has no batched counterpart. */
enum fhb_item_kind { FHB_ITEM_HMULT_RELIN_RESCALE = 0, FHB_ITEM_ROTATE = 1 };
typedef struct fhb_ks_item {
  int32_t kind;       /* fhb_item_kind */
  int32_t level;
  uint32_t galois;    /* rotation: Galois element of the step (odd, < 2N); ignored for HMult */
  int32_t reserved;   /* 0 */
  const void* a;      /* [2, L, N] coefficient/standard: HMult lhs, or the ciphertext to rotate */
  const void* b;      /* HMult rhs [2, L, N] coefficient/standard; NULL for a rotation */
  const void* key;    /* relinearisation or rotation key [D, 2, QP0, N] NTT/Montgomery */
  void* out;          /* HMult [2, L - 1, N], rotation [2, L, N]: coefficient/standard canonical */
} fhb_ks_item;
typedef struct fhb_items_plan_info {
  int64_t plan_bytes;     /* device bytes of the plan */
  int64_t scratch_bytes;  /* device scratch bytes of the items */
  int32_t items, hmult_items, forward_units, inverse_units, core_units, max_limbs, max_digits;
  int32_t core_f64_units; /* key-switch units whose rows' primes are below 2^42 (run in FP64 arithmetic) */
} fhb_items_plan_info;
int fhb_ckks_items_plan_info(const fhb_context* ctx, const fhb_ks_item* items, int count, fhb_items_plan_info* info);
int fhb_ckks_items_plan(const fhb_context* ctx, const fhb_ks_item* items, int count, void* plan, void* scratch,
                        const fhb_items_plan_info* info);
int fhb_ckks_items_run(const fhb_context* ctx, const void* plan, const fhb_items_plan_info* info, fhb_stream stream);
/* Status word of the runs of a plan since the last read: 0, or the first
 * error a kernel raised (1: a work list names an item outside the plan; 2: a
 * device descriptor no longer matches the check word the planner stored
 * with it; 3: a work-list row outside its item's rows; 4: the HMult list
 * names a rotation).  Every kernel verifies the item it is about to use, so
 * a plan changed in device memory after planning makes the affected items
 * skip their work instead of addressing memory through it.  Reads with a
 * blocking copy (call after the runs have completed) and resets the word. */
int fhb_ckks_items_status(const fhb_context* ctx, void* plan, const fhb_items_plan_info* info, int* status);

/* Bounded decryption to float64 coefficients: phase [batch, L, N]
 * coefficient/standard canonical (c0 + c1 s) -> out [batch, N] float64 (a
 * DEVICE pointer), the centred representative modulo the product of the
 * trailing one or two active Q primes, computed with the reference's float64
 * operations in its order so the doubles are equal.  Replaces
 * CkksDecryptor._reconstruct_tail_q_coefficients_float64
 * (fhelium/engine/ckks_decryptor.py:180-272). */
int fhb_ckks_decrypt_tail(const fhb_context* ctx, const void* phase, double* out, int64_t batch, int level,
                          fhb_stream stream);

/* Baby-step/giant-step inner products of a diagonal linear transform
 * (bootstrapping's CoeffsToSlots / SlotsToCoeffs):
 *   out[k] = sum_b rot[b] (.) pts[table[k * babies + b]]
 * for k < giants, skipping table entries < 0.  rot: babies blocks of `polys`
 * NTT/Montgomery polynomials [polys, rows, N] (block pitch rot_stride
 * words); pts: `entries` plaintexts [rows, N] (pitch pt_stride words),
 * shared by every polynomial; out: giants blocks (pitch out_stride words),
 * lazy Montgomery products.  table is a DEVICE int32 array whose entries
 * are < entries.  Replaces the per-diagonal plaintext product and addition
 * of the reference's BSGS evaluation
 * (fhelium/experimental/bootstrap/_linear.py:235-393). */
int fhb_ckks_bsgs_inner_product(const fhb_context* ctx, const void* rot, int64_t rot_stride, const void* pts,
                                int64_t pt_stride, int entries, const int32_t* table, int giants, int babies,
                                void* out, int64_t out_stride, int64_t polys, int rows, int row_start,
                                fhb_stream stream);

/* Mixed-step rotation of one level: item b of ct [2, batch, L, N]
 * (coefficient/standard) is rotated by its own Galois element galois[b]
 * with the key at key_ptrs[b] (a device address of a [digits, 2, QP, N]
 * key).  key_ptrs and galois are DEVICE arrays of batch entries.  Replaces
 * a loop of CkksEngine._apply_rotation_key calls, one per ciphertext
 * (fhelium/engine/ckks_engine.py:3822-3897), with one launch sequence.
 * The reference has no batched mixed-step counterpart. */
int fhb_ckks_rotate_multi(const fhb_context* ctx, const void* ct, const uint64_t* key_ptrs, const uint32_t* galois,
                          void* out, void* scratch, int64_t scratch_bytes, int64_t batch, int level,
                          fhb_stream stream);

/* ------------------------------------------------------------------------
 * Operator-level entry points: one kernel per custom op of the reference,
 * taking the reference's own operands, so that its operator schemas
 * (torch.ops.fhelium_{rns,ntt,ckks}_ops) can be served on B200 without a
 * chain context (fhelium_b200/torch_ops.py registers them).
 *
 * residue_bits selects the word (64: int64 family, 32: int32 family); every
 * table has that word type.  A residue operand is [batch, rows, n] with rows
 * n words apart and coefficients contiguous; *_batch_stride is its distance
 * between batch items in words (0 broadcasts a single item).  `params` is the
 * reference's [8, limb] parameter tensor (rows {2q, q_lo, q_hi, -q^-1 lo,
 * -q^-1 hi, R^2, Delta R^2, N^-1 R}, csrc/ops/common/rns_parameters.h:6-16)
 * sliced to the operand's limbs: column j describes row j, rows
 * param_row_stride words apart.  Outputs carry the integers the reference's
 * CPU kernels return.  In-place entry points update their operand; outputs
 * of the others must not overlap their inputs. */

/* op 0 montgomery_mul (canonical), 1 add_lazy, 2 sub_lazy ([0, 2q)),
 * 3 add_canonical, 4 sub_canonical; rhs_batch_stride 0 = singleton rhs batch.
 * Ops 1 and 2 read only parameter row 0 (2q): a twice-modulus vector with
 * param_row_stride 0 serves add_lazy_with_twice_modulus
 * (csrc/ops/rns/rns_arithmetic.cpp:47-49).
 * Replaces fhelium_rns_ops.{montgomery_mul, add_lazy, sub_lazy,
 * add_canonical(_), sub_canonical(_)} (csrc/ops/rns/rns_arithmetic.cpp:31,46,50,
 * csrc/ops/rns/rns_canonical_arithmetic.cpp:16-21). */
int fhb_op_rns_binary(int residue_bits, int op, const void* lhs, int64_t lhs_batch_stride, const void* rhs,
                      int64_t rhs_batch_stride, void* out, int64_t out_batch_stride, int64_t batch, int rows,
                      int64_t n, const void* params, int64_t param_row_stride, fhb_stream stream);
/* In place: op 0 to_montgomery_, 1 from_montgomery_ (canonical),
 * 2 canonicalize_residues_, 3 center_residues_, 4 shift_residues_positive_
 * (csrc/ops/rns/rns_arithmetic.cpp:41-59). */
int fhb_op_rns_unary(int residue_bits, int op, void* residues, int64_t batch_stride, int64_t batch, int rows,
                     int64_t n, const void* params, int64_t param_row_stride, fhb_stream stream);
/* out[b, j, k] = coefficients[b, k] + q_j (q_j = twice_modulus[j] / 2).
 * Replaces fhelium_rns_ops.lift_centered_coefficients
 * (csrc/ops/rns/rns_arithmetic.cpp:60-62). */
int fhb_op_lift_centered(int residue_bits, const void* coefficients, int64_t coefficient_batch_stride, void* out,
                         int64_t out_batch_stride, int64_t batch, int rows, int64_t n, const void* twice_modulus,
                         fhb_stream stream);
/* Garner mixed-radix digits of one hybrid digit (rows <= 8); normalizers
 * [rows - 1], propagation [rows - 1, propagation_row_stride], the four
 * split-word vectors [rows].  Replaces fhelium_rns_ops.mixed_radix_decompose
 * (csrc/ops/rns/rns_arithmetic.cpp:63-68). */
int fhb_op_mixed_radix_decompose(int residue_bits, const void* source, int64_t source_batch_stride, void* out,
                                 int64_t out_batch_stride, int64_t batch, int rows, int64_t n,
                                 const void* normalizers, const void* propagation, int64_t propagation_row_stride,
                                 const void* modulus_lo, const void* modulus_hi, const void* neg_inv_modulus_lo,
                                 const void* neg_inv_modulus_hi, fhb_stream stream);
/* Exact basis extension of digit_rows mixed-radix digits into
 * destination_rows Montgomery/lazy rows; coefficients [digit_rows - 1,
 * coefficient_row_stride] (column j for destination row j).  Replaces
 * fhelium_rns_ops.mixed_radix_basis_extend_to_montgomery
 * (csrc/ops/rns/rns_arithmetic.cpp:69-72). */
int fhb_op_basis_extend(int residue_bits, const void* digits, int64_t digits_batch_stride, int digit_rows,
                        void* out, int64_t out_batch_stride, int64_t batch, int destination_rows, int64_t n,
                        const void* coefficients, int64_t coefficient_row_stride, const void* params,
                        int64_t param_row_stride, fhb_stream stream);
/* In place: acc_c[b, j] += digit[b, j] * key[c, key_row_start + j] (c = 0, 1;
 * key component c at key_digit + c * key_component_stride words).  Replaces
 * fhelium_ckks_ops.keyswitch_accumulate_digit_products_
 * (csrc/ops/ckks/ckks.cpp:85-88, csrc/ops/ckks/cuda/keyswitch_cuda.cu:198-292). */
int fhb_op_keyswitch_accumulate(int residue_bits, void* acc0, int64_t acc0_batch_stride, void* acc1,
                                int64_t acc1_batch_stride, const void* digit, int64_t digit_batch_stride,
                                const void* key_digit, int64_t key_component_stride, int64_t key_row_start,
                                int64_t batch, int rows, int64_t n, const void* params, int64_t param_row_stride,
                                fhb_stream stream);
/* ModDown of coefficient/standard Q and P rows (p_rows <= 16) to canonical Q
 * rows; inverses [p_rows, inverse_row_stride]; params covers q_rows + p_rows
 * columns.  Replaces fhelium_ckks_ops.keyswitch_moddown_qp_to_q
 * (csrc/ops/ckks/ckks.cpp:82-84, csrc/ops/ckks/cuda/keyswitch_cuda.cu:55-196). */
int fhb_op_moddown(int residue_bits, const void* q_residues, int64_t q_batch_stride, const void* p_residues,
                   int64_t p_batch_stride, void* out, int64_t out_batch_stride, int64_t batch, int q_rows,
                   int p_rows, int64_t n, const void* inverses, int64_t inverse_row_stride, const void* params,
                   int64_t param_row_stride, fhb_stream stream);
/* Drop the leading prime: remaining [batch, rows, n], dropped [batch, n],
 * inverse_montgomery [rows]; nearest = 1 rounds (half_drop_prime =
 * floor(q_drop / 2)), 0 truncates.  Canonical output; out may equal
 * remaining.  Replaces fhelium_ckks_ops.rescale_drop_leading_prime_{nearest,
 * truncate}(_) (csrc/ops/ckks/ckks.cpp:60-75, csrc/ops/ckks/cuda/
 * rescale_cuda.cu:22-54). */
int fhb_op_rescale(int residue_bits, const void* remaining, int64_t remaining_batch_stride, const void* dropped,
                   int64_t dropped_batch_stride, void* out, int64_t out_batch_stride, int64_t batch, int rows,
                   int64_t n, const void* inverse_montgomery, const void* params, int64_t param_row_stride,
                   int64_t half_drop_prime, int nearest, fhb_stream stream);
/* Coefficient-domain automorphism from the reference's maps: out[k] =
 * sign[k] * in[source_indices[k]], canonical.  Replaces
 * fhelium_ckks_ops.apply_coefficient_galois_automorphism
 * (csrc/ops/ckks/ckks.cpp:76-78, csrc/ops/ckks/cuda/automorphism_cuda.cu:15-31). */
int fhb_op_coefficient_automorphism(int residue_bits, const void* in, int64_t in_batch_stride, void* out,
                                    int64_t out_batch_stride, int64_t batch, int rows, int64_t n,
                                    const int32_t* source_indices, const int8_t* source_sign,
                                    const void* twice_moduli, fhb_stream stream);
/* NTT-domain automorphism: out[k] = in[source_indices[k]].  Replaces
 * fhelium_ckks_ops.apply_ntt_galois_automorphism (csrc/ops/ckks/ckks.cpp:79-81,
 * csrc/ops/ckks/cuda/automorphism_cuda.cu:33-44). */
int fhb_op_ntt_automorphism(int residue_bits, const void* in, int64_t in_batch_stride, void* out,
                            int64_t out_batch_stride, int64_t batch, int rows, int64_t n,
                            const int32_t* source_indices, fhb_stream stream);
/* out = lhs * rhs[i(k)] (Montgomery, canonical) with a compressed right
 * operand of `unique` words per row (a power of two below n): layout 1 cyclic
 * (i = k mod unique), 2 contiguous (i = k / (n / unique)).  Replaces
 * fhelium_rns_ops.montgomery_mul_{cyclic,contiguous}_compressed
 * (csrc/ops/rns/rns_arithmetic.cpp:32-37, csrc/ops/rns/cuda/rns_arithmetic_cuda.cu:55-78). */
int fhb_op_mul_compressed(int residue_bits, int layout, const void* lhs, int64_t lhs_batch_stride,
                          const void* compressed_rhs, int64_t rhs_batch_stride, int64_t unique, void* out,
                          int64_t out_batch_stride, int64_t batch, int rows, int64_t n, const void* params,
                          int64_t param_row_stride, fhb_stream stream);
/* Plaintext addition to a coefficient/standard ciphertext component:
 * out = c + p R^-1 mod q, canonical, p a coefficient/Montgomery plaintext word
 * of plaintext_extent words per row.  layout 0 dense (extent n), 1 cyclic,
 * 2 contiguous repetition (extent a power of two below n), 3 strided
 * (coefficients k with k mod (n / extent) = 0 stored at k / (n / extent), the
 * rest take implicit_plaintext[b, row], batch stride implicit_batch_stride).
 * out may equal ciphertext.  Replaces fhelium_ckks_ops.add_{prepared,
 * cyclic_compressed,contiguous_compressed,strided}_plaintext_component(_)
 * (csrc/ops/ckks/ckks.cpp:30-59, csrc/ops/ckks/cuda/plaintext_cuda.cu:1-114). */
int fhb_op_add_plaintext(int residue_bits, int layout, const void* ciphertext, int64_t ciphertext_batch_stride,
                         const void* plaintext, int64_t plaintext_batch_stride, int64_t plaintext_extent,
                         const void* implicit_plaintext, int64_t implicit_batch_stride, void* out,
                         int64_t out_batch_stride, int64_t batch, int rows, int64_t n, const void* params,
                         int64_t param_row_stride, fhb_stream stream);
/* out = residues * row_scalars[row] (Montgomery, canonical); out may equal
 * residues.  Replaces fhelium_rns_ops.montgomery_mul_row_scalars_ and
 * montgomery_mul_row_scalars_canonical (csrc/ops/rns/rns_arithmetic.cpp:38-40,
 * csrc/ops/rns/rns_canonical_arithmetic.cpp:20-22). */
int fhb_op_mul_row_scalars(int residue_bits, const void* residues, int64_t residues_batch_stride, void* out,
                           int64_t out_batch_stride, int64_t batch, int rows, int64_t n, const void* row_scalars,
                           const void* params, int64_t param_row_stride, fhb_stream stream);
/* A context whose prime ids 0..count-1 are exactly `moduli` (plus one
 * auxiliary special prime of the library's choosing at id `count`), for the
 * transforms (fhb_forward_ntt, fhb_inverse_ntt, tensor-core forms) and the
 * element-wise entry points of a parameter-row slice.  Used to serve the
 * reference's NTT schemas, whose operands carry a slice of rows rather than a
 * chain (csrc/ops/ntt/forward_ntt.cpp:25-67, inverse_ntt.cpp:23-73).  Set-up:
 * allocates and copies synchronously. */
int fhb_context_create_transform(int residue_bits, int log_n, const uint64_t* moduli, int count, int device,
                                 fhb_context** out);

#ifdef __cplusplus
}
#endif

#endif /* FHB200_H */
