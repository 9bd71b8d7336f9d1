// Exact integer tensor-core NTT for int32 residues (q < 2^28) at N = 2^16 on
// the 5th-generation tensor cores: tcgen05.mma kind::i8 with int32
// accumulators in tensor memory (TMEM), operands in shared memory.
//
// Three-pass form, N = 64 x 64 x 16.  Write the input index as
// n = 1024 i1 + 16 i2 + i3 and the output position (bit-reversed order, as
// the CUDA-core form and the reference: out[p] = sum_n x[n] psi^{(2 br16(p) +
// 1) n}, csrc/ops/ntt/forward_ntt.cpp:15-21) as p = 1024 P1 + 16 P2 + P3, so
// br16(p) = m1 + 64 m2 + 4096 m3 with m1 = br6(P1), m2 = br6(P2), m3 = br4(P3).
// Expanding (2 br16(p) + 1) n modulo 2N and dropping the multiples of 2N:
//
//   pass 1: Y1[P1][i2][i3] = R psi^{16 i2 (2 m1 + 1)} sum_i1 x[i1][i2][i3] psi^{1024 i1 (2 m1 + 1)}
//   pass 2: Y2[P1][P2][i3] = psi^{(2 m1 + 1) i3 + 128 m2 i3} sum_i2 Y1[P1][i2][i3] psi^{2048 m2 i2}
//   pass 3: out[P1][P2][P3] = sum_i3 Y2[P1][P2][i3] psi^{8192 m3 i3}
//
// (R = 2^30: Montgomery output).  The inverse runs the passes in the opposite
// order with psi^{-1}; its first pass carries N^{-1} R^{-1}.
//
// Every pass is a batch of independent length-n products
// D[m][n] = sum_k A[m][k] W[k][n] mod q over "instances" m (n = 64 or 16
// outputs per instance); an instance's k-th input and n-th output sit at
// f(m) + k S and f(m) + n S in the polynomial, with f and S fixed per pass
// (pass 1: f(m) = m, S = 1024; pass 2: f(m) = (m / 16) 1024 + m % 16,
// S = 16; pass 3: f(m) = 16 m, S = 1).  The product is exact with unsigned
// 8-bit digits: the residues split into their four bytes A = sum_d 2^{8d} A_d,
// the constant matrix is pre-scaled per data byte, W^(d) = 2^{8d} 2^{32} W mod
// q, and split into bytes W^(d) = sum_e 2^{8e} W^(d)_e.  Tensor-core
// accumulator e collects sum_{d,k} A_d W^(d)_e (K = 4 n byte products,
// < 2^24), the epilogue forms S = sum_e 2^{8e} acc_e < 2^49 and one
// Montgomery reduction by 2^32 returns (A W mod q) in [0, 2q); the optional
// elementwise twiddle t is stored as t 2^32 mod q and applied by a second
// reduction by 2^32 (exact for inputs < 2q < 2^32 / q), and the result is made
// canonical.
//
// The constant matrix of a pass is small enough to stay in shared memory (64
// KiB for n = 64, 4 KiB for n = 16), so a persistent CTA loads it once per
// prime and then streams units of 128 instances of that prime through a
// double-buffered pipeline:
//   producer (warp 12, lane 0): bulk copies of a unit's raw words into a raw
//       buffer (one copy for contiguous units, one per k row otherwise);
//   transposers (warps 8-11): raw words -> the four byte planes of the A tile
//       (K-major canonical layout, K = 4 n bytes: [A_0 | A_1 | A_2 | A_3]);
//   MMA issuer (warp 13, lane 0): n / 8 MMAs of M = 128, N = 4 n (twiddle
//       bytes e x n outputs), K = 32 into one of two TMEM accumulator sets;
//   epilogue (warps 0-7; warp w reads TMEM lane quarter w % 4 and the
//       outputs of half w / 4): recombination, twiddle, store.
// Raw buffers rotate over three slots, A tiles and accumulator sets over two,
// so the copies of units i + 1 and i + 2, the transposition and MMAs of unit i
// and the epilogue of unit i - 1 overlap; each epilogue warp requests all its
// twiddles of a unit before it waits for the unit's accumulators.  Every mbarrier wait is bounded (about one
// second of the global timer); a wait that gives up sets a CTA abort flag that
// releases every other wait and raises the device error flag, and the CTA
// drains its own bulk copies and MMAs (again with bounded waits) before it
// frees TMEM and exits.
#include <cstring>
#include <vector>

#include "fhb_context.h"
#include "fhb_tc_common.cuh"

namespace fhb {
namespace tcntt {
using namespace fhb::tc;

constexpr int kLogN = 16;
constexpr int kPolyWords = 1 << kLogN;
constexpr int kUnit = 128;                // instances per unit (MMA M)
constexpr int kThreads = 448;             // 14 warps
constexpr int kEpilogueWarps = 8;         // warps 0..7
constexpr int kTransposeWarp0 = 8;        // warps 8..11
constexpr int kTransposeWarps = 4;
constexpr int kProducerWarp = 12;
constexpr int kMmaWarp = 13;

// Pass geometry: NK = outputs (and inputs) per instance.
template <int NK>
struct Geom {
  static constexpr int kKBytes = 4 * NK;                 // K of the concatenated digit planes
  static constexpr int kNmma = 4 * NK;                   // MMA N: 4 twiddle bytes x NK outputs
  static constexpr int kSteps = kKBytes / 32;            // MMAs per unit
  static constexpr int kSbo = kKBytes / 16 * 128;        // 8-row group stride (A and B)
  static constexpr int kBBytes = kNmma * kKBytes;        // constant byte matrix
  static constexpr int kABytes = kUnit * kKBytes;        // one A tile
  static constexpr int kRawBytes = kUnit * NK * 4;       // one unit's raw words
  static constexpr int kUnitsPerPoly = (kPolyWords / NK) / kUnit;
  // pipeline depth: raw copy slots, A tiles, TMEM accumulator sets (n = 16
  // units are small, so it affords deeper rings)
  static constexpr int kRawSlots = NK == 64 ? 3 : 8;
  static constexpr int kASlots = NK == 64 ? 2 : 4;
  static constexpr int kAccSlots = NK == 64 ? 2 : 4;
  static constexpr int kTmemCols = kAccSlots * kNmma;
  // n = 16: two CTAs per SM (their shared memory, TMEM and registers fit)
  static constexpr int kCtasPerSm = NK == 64 ? 1 : 2;
};

constexpr int kBarrierBytes = 512;
// smem: [B | raw slots | A slots | barriers]
template <int NK>
constexpr int smem_bytes() {
  return 1024 + Geom<NK>::kBBytes + Geom<NK>::kRawSlots * Geom<NK>::kRawBytes +
         Geom<NK>::kASlots * Geom<NK>::kABytes + kBarrierBytes;
}
template <int NK>
constexpr int num_barriers() {
  return 3 + 2 * (Geom<NK>::kRawSlots + Geom<NK>::kASlots + Geom<NK>::kAccSlots);
}
static_assert(8 * num_barriers<16>() + 8 <= kBarrierBytes && 8 * num_barriers<64>() + 8 <= kBarrierBytes,
              "barrier area");
static_assert(smem_bytes<64>() <= 232448, "shared memory per CTA");

constexpr uint32_t instr_desc(uint32_t n) { return tc::instr_desc_u8(n); }

// ---------------------------------------------------------------- device ---
// Byte transpose of four words: out[d] = byte d of v0 | byte d of v1 << 8 |
// byte d of v2 << 16 | byte d of v3 << 24.
__device__ __forceinline__ void byte_transpose(uint32_t v0, uint32_t v1, uint32_t v2, uint32_t v3,
                                               uint32_t& o0, uint32_t& o1, uint32_t& o2, uint32_t& o3) {
  const uint32_t a = __byte_perm(v0, v1, 0x5140), b = __byte_perm(v0, v1, 0x7362);
  const uint32_t c = __byte_perm(v2, v3, 0x5140), e = __byte_perm(v2, v3, 0x7362);
  o0 = __byte_perm(a, c, 0x5410);
  o1 = __byte_perm(a, c, 0x7632);
  o2 = __byte_perm(b, e, 0x5410);
  o3 = __byte_perm(b, e, 0x7632);
}

// Instance map of a pass kind (1: f(m) = m, S = 1024; 2: f(m) = (m / 16)
// 1024 + m % 16, S = 16; 3: f(m) = 16 m, S = 1): offset of instance m within
// a polynomial, and the stride between its successive inputs / outputs.
template <int KIND>
__device__ __forceinline__ int inst_offset(int m) {
  if (KIND == 1) return m;
  if (KIND == 2) return (m >> 4) * 1024 + (m & 15);
  return m * 16;
}
template <int KIND>
constexpr int inst_stride() {
  return KIND == 1 ? 1024 : (KIND == 2 ? 16 : 1);
}

// Word index of input k of local instance ml in a unit's raw buffer:
// kind 1 keeps one 128-word row per k, kinds 2 and 3 copy the unit's
// contiguous span as it lies in the polynomial.
template <int KIND, int NK>
__device__ __forceinline__ int raw_index(int ml, int k) {
  if (KIND == 1) return k * kUnit + ml;
  if (KIND == 2) return (ml >> 4) * 1024 + k * 16 + (ml & 15);
  return ml * NK + k;
}

// Byte planes of one 128-instance tile: instance ml's input k is raw word
// raw_index<KIND, NK>(ml, k); byte d of it goes to K position d NK + k of row
// ml of the K-major canonical A tile.  Transposer warp tw of kTransposeWarps
// takes every kTransposeWarps-th (8-instance group, 16-k group); a thread
// handles (instance, 4 consecutive k), so a warp's 32 four-byte stores fall
// in 32 distinct banks.
template <int KIND, int NK>
__device__ __forceinline__ void transpose_tile(const uint32_t* raw, uint8_t* at, int tw, int lane) {
  using G = Geom<NK>;
  const int r8 = lane >> 2, q4 = lane & 3;
  constexpr int kWarpUnits = (kUnit / 8) * (NK / 16);
  for (int wu = tw; wu < kWarpUnits; wu += kTransposeWarps) {
    const int ml = (wu % (kUnit / 8)) * 8 + r8;
    const int k = (wu / (kUnit / 8)) * 16 + q4 * 4;
    uint32_t v0, v1, v2, v3;
    if (KIND == 3) {
      const uint4 v = *reinterpret_cast<const uint4*>(raw + raw_index<KIND, NK>(ml, k));
      v0 = v.x;
      v1 = v.y;
      v2 = v.z;
      v3 = v.w;
    } else {
      v0 = raw[raw_index<KIND, NK>(ml, k)];
      v1 = raw[raw_index<KIND, NK>(ml, k + 1)];
      v2 = raw[raw_index<KIND, NK>(ml, k + 2)];
      v3 = raw[raw_index<KIND, NK>(ml, k + 3)];
    }
    uint32_t w[4];
    byte_transpose(v0, v1, v2, v3, w[0], w[1], w[2], w[3]);
    const uint32_t rowoff = uint32_t((ml & 7) * 16 + (ml >> 3) * G::kSbo);
#pragma unroll
    for (int d = 0; d < 4; ++d) {
      const int kap = d * NK + k;
      *reinterpret_cast<uint32_t*>(at + rowoff + (kap >> 4) * 128 + (kap & 15)) = w[d];
    }
  }
}

// kChunk outputs [c0, c0 + kChunk) of this lane's instance from the four
// byte accumulators at TMEM address taddr + e NK (taddr = lane quarter +
// accumulator set + c0): S = sum_e 2^{8e} acc_e < 2^49, one Montgomery
// reduction by 2^32 (A W mod q in [0, 2q)), the twiddle tws[j] = t 2^32 mod q
// by a second one when POST, then the canonical residue.
template <int NK, int kChunk, bool POST>
__device__ __forceinline__ void reduce_chunk(uint32_t taddr, const uint32_t* tws, uint32_t q, uint32_t qneg,
                                             uint32_t (&res)[16]) {
  uint32_t acc[4][16];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    if (kChunk == 16)
      tmem_ld16(taddr + uint32_t(e * NK), acc[e]);
    else
      tmem_ld8(taddr + uint32_t(e * NK), acc[e]);
  }
  tmem_wait_ld();
#pragma unroll
  for (int j = 0; j < kChunk; ++j) {
    const uint64_t sum = uint64_t(acc[0][j]) + (uint64_t(acc[1][j]) << 8) + (uint64_t(acc[2][j]) << 16) +
                         (uint64_t(acc[3][j]) << 24);
    const uint32_t mm = uint32_t(sum) * qneg;
    uint32_t r = uint32_t((sum + uint64_t(mm) * q) >> 32);  // S 2^-32 mod q, in [0, 2q)
    if (POST) {
      const uint64_t pr = uint64_t(r) * tws[j];  // < 2 q^2 < q 2^32
      const uint32_t m2 = uint32_t(pr) * qneg;
      r = uint32_t((pr + uint64_t(m2) * q) >> 32);  // r t mod q, in [0, 2q)
    }
    res[j] = r >= q ? r - q : r;
  }
}

struct PassArgs {
  const uint32_t* in;
  uint32_t* out;
  const uint8_t* bmat;                // [QP][byte matrix]
  const uint32_t* post;               // [QP][N] twiddles t 2^32 mod q in output order, or null
  const uint32_t* qinfo;              // [QP][2]
  int64_t batch;                      // polynomials per row (polys = batch x rows)
  int rows;
  int row_start;
  int ctas_per_row;
  int* err;
  unsigned long long wait_ns;         // limit of the pipeline waits (drain waits keep kWaitNs)
  int stall;                          // test only: the epilogue first waits on a barrier nothing completes
};

// in == out is allowed: a unit's outputs occupy exactly the words its raw
// copy read, and a unit's output is written only after its raw copy landed.
template <int KIND, int NK, bool POST>
__global__ void __launch_bounds__(kThreads, Geom<NK>::kCtasPerSm) k_tc_ntt_pass(PassArgs args) {
  using G = Geom<NK>;
  constexpr int S = inst_stride<KIND>();
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw0 = smem_addr(smem_raw);
  const uint32_t base = (raw0 + 1023u) & ~1023u;
  uint8_t* const gbase = smem_raw + (base - raw0);
  const uint32_t b_addr = base;
  const uint32_t rawbuf_addr = base + G::kBBytes;
  const uint32_t* const rawbuf = reinterpret_cast<const uint32_t*>(gbase + G::kBBytes);
  constexpr int kRawSlots = G::kRawSlots, kASlots = G::kASlots, kAccSlots = G::kAccSlots;
  const uint32_t a_addr = base + G::kBBytes + kRawSlots * G::kRawBytes;
  uint8_t* const a_tile = gbase + G::kBBytes + kRawSlots * G::kRawBytes;
  uint64_t* const bars =
      reinterpret_cast<uint64_t*>(gbase + G::kBBytes + kRawSlots * G::kRawBytes + kASlots * G::kABytes);
  const uint32_t bar0 = smem_addr(bars);
  // barriers: b_full, raw_full/empty[kRawSlots], a_full/empty[kASlots], acc_full/empty[kAccSlots], drain
  const uint32_t bfull_bar = bar0;
  auto rawf_bar = [&](int r) { return bar0 + 8u * (1 + r); };
  auto rawe_bar = [&](int r) { return bar0 + 8u * (1 + kRawSlots + r); };
  auto af_bar = [&](int b) { return bar0 + 8u * (1 + 2 * kRawSlots + b); };
  auto ae_bar = [&](int b) { return bar0 + 8u * (1 + 2 * kRawSlots + kASlots + b); };
  auto accf_bar = [&](int b) { return bar0 + 8u * (1 + 2 * kRawSlots + 2 * kASlots + b); };
  auto acce_bar = [&](int b) { return bar0 + 8u * (1 + 2 * kRawSlots + 2 * kASlots + kAccSlots + b); };
  const uint32_t drain_bar = bar0 + 8u * (num_barriers<NK>() - 1);
  const uint32_t never_bar = bar0 + 8u * (num_barriers<NK>() - 2);  // nothing arrives on it
  uint32_t* const tmem_slot = reinterpret_cast<uint32_t*>(bars + num_barriers<NK>());
  volatile int* const abort = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  constexpr int kChunk = NK / 2 < 16 ? NK / 2 : 16;  // epilogue columns per TMEM load
  // CTA -> (prime row, contiguous range of its units); a unit = (polynomial
  // of the row, block of 128 instances)
  const int row = blockIdx.x / args.ctas_per_row, part = blockIdx.x % args.ctas_per_row;
  const int64_t units = args.batch * G::kUnitsPerPoly;
  const int64_t u_begin = units * part / args.ctas_per_row, u_end = units * (part + 1) / args.ctas_per_row;
  const int nu = int(u_end - u_begin);
  const int prime = args.row_start + row;
  auto unit_poly = [&](int i) { return ((u_begin + i) / G::kUnitsPerPoly) * args.rows + row; };
  auto unit_m0 = [&](int i) { return int((u_begin + i) % G::kUnitsPerPoly) * kUnit; };

  if (tid == 0) {
    mbar_init(bfull_bar, 1);
    for (int r = 0; r < kRawSlots; ++r) {
      mbar_init(rawf_bar(r), 1);
      mbar_init(rawe_bar(r), kTransposeWarps);
    }
    for (int b = 0; b < kASlots; ++b) {
      mbar_init(af_bar(b), kTransposeWarps);
      mbar_init(ae_bar(b), 1);
    }
    for (int b = 0; b < kAccSlots; ++b) {
      mbar_init(accf_bar(b), 1);
      mbar_init(acce_bar(b), kEpilogueWarps);
    }
    mbar_init(drain_bar, 1);
    mbar_init(never_bar, 1);
    *abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == kMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                 "r"(G::kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == kProducerWarp && lane == 0) {
    // constants once, then each unit's raw words
    const uint8_t* bsrc = args.bmat + size_t(prime) * G::kBBytes;
    constexpr int kPiece = G::kBBytes < 16384 ? G::kBBytes : 16384;
    mbar_expect_tx(bfull_bar, G::kBBytes);
    for (int o = 0; o < G::kBBytes; o += kPiece) bulk_load(b_addr + o, bsrc + o, kPiece, bfull_bar);
    int i = 0;
    for (; i < nu; ++i) {
      const int r = i % kRawSlots, use = i / kRawSlots;
      if (i >= kRawSlots && !mbar_wait(rawe_bar(r), (use & 1) ^ 1, abort, args.err, args.wait_ns)) break;
      const uint32_t* src = args.in + unit_poly(i) * int64_t(kPolyWords) + inst_offset<KIND>(unit_m0(i));
      const uint32_t dst = rawbuf_addr + r * G::kRawBytes;
      mbar_expect_tx(rawf_bar(r), G::kRawBytes);
      if (KIND == 1) {
        for (int k = 0; k < NK; ++k) bulk_load(dst + k * kUnit * 4, src + k * 1024, kUnit * 4, rawf_bar(r));
      } else {
        constexpr int kRawPiece = G::kRawBytes < 8192 ? G::kRawBytes : 8192;
        for (int o = 0; o < G::kRawBytes; o += kRawPiece)
          bulk_load(dst + o, reinterpret_cast<const uint8_t*>(src) + o, kRawPiece, rawf_bar(r));
      }
    }
    // after an abort, wait (bounded) for the copies still in flight
    if (*abort) {
      mbar_wait(bfull_bar, 0, nullptr, args.err, kWaitNs);
      for (int t = i - kRawSlots < 0 ? 0 : i - kRawSlots; t < i; ++t)
        mbar_wait(rawf_bar(t % kRawSlots), (t / kRawSlots) & 1, nullptr, args.err, kWaitNs);
    }
  } else if (warp >= kTransposeWarp0 && warp < kTransposeWarp0 + kTransposeWarps) {
    // raw words -> byte planes
    const int tw = warp - kTransposeWarp0;
    for (int i = 0; i < nu; ++i) {
      const int b = i % kASlots, r = i % kRawSlots;
      if (!warp_wait(rawf_bar(r), (i / kRawSlots) & 1, abort, args.err, lane, args.wait_ns)) break;
      if (i >= kASlots && !warp_wait(ae_bar(b), ((i / kASlots) & 1) ^ 1, abort, args.err, lane, args.wait_ns))
        break;
      transpose_tile<KIND, NK>(rawbuf + r * (G::kRawBytes / 4), a_tile + b * G::kABytes, tw, lane);
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(rawe_bar(r));
        mbar_arrive(af_bar(b));
      }
    }
  } else if (warp == kMmaWarp && lane == 0) {
    constexpr uint32_t kIdesc = instr_desc(G::kNmma);
    bool ok = mbar_wait(bfull_bar, 0, abort, args.err, args.wait_ns);
    for (int i = 0; i < nu && ok; ++i) {
      const int b = i % kASlots, c = i % kAccSlots;
      if (!mbar_wait(af_bar(b), (i / kASlots) & 1, abort, args.err, args.wait_ns) ||
          (i >= kAccSlots &&
           !mbar_wait(acce_bar(c), ((i / kAccSlots) & 1) ^ 1, abort, args.err, args.wait_ns))) {
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t d_tmem = tmem + uint32_t(c * G::kNmma);
      const uint32_t a_base = a_addr + b * G::kABytes;
#pragma unroll
      for (int st = 0; st < G::kSteps; ++st)
        mma_i8(d_tmem, smem_desc(a_base + st * 256, 128, G::kSbo), smem_desc(b_addr + st * 256, 128, G::kSbo),
               kIdesc, st > 0 ? 1u : 0u);
      mma_commit(ae_bar(b));
      mma_commit(accf_bar(c));
    }
  } else if (warp < kEpilogueWarps) {
    const uint32_t q = args.qinfo[2 * prime], qneg = args.qinfo[2 * prime + 1];
    const uint32_t* post = POST ? args.post + (size_t(prime) << kLogN) : nullptr;
    const int quarter = warp & 3, half = warp >> 2;
    const int ml = quarter * 32 + lane;
    const uint32_t lane_addr = uint32_t(quarter * 32) << 16;
    constexpr int kHalf = NK / 2;  // outputs of this warp: [half * kHalf, half * kHalf + kHalf)
    // a warp's kHalf twiddles of a unit: 16-byte vector loads where they are
    // contiguous (stride 1), else one coalesced load per output column
    auto load_tw = [&](const uint32_t* t, uint32_t (&v)[kHalf]) {
      if (S == 1) {
#pragma unroll
        for (int j = 0; j < kHalf / 4; ++j) {
          const uint4 x = *reinterpret_cast<const uint4*>(t + half * kHalf + 4 * j);
          v[4 * j] = x.x;
          v[4 * j + 1] = x.y;
          v[4 * j + 2] = x.z;
          v[4 * j + 3] = x.w;
        }
      } else {
#pragma unroll
        for (int j = 0; j < kHalf; ++j) v[j] = t[(half * kHalf + j) * S];
      }
    };
    // twiddles of the next unit are requested one unit ahead when they fit in
    // registers (n = 16); otherwise all of a unit's are requested before its wait
    constexpr bool kAhead = kHalf <= 8;
    uint32_t tws_next[kHalf];
    if (POST && kAhead && nu > 0) load_tw(post + inst_offset<KIND>(unit_m0(0) + ml), tws_next);
    // test only: a wait that must run out (its limit is the pipeline's)
    const bool stalled = args.stall && !warp_wait(never_bar, 0, abort, args.err, lane, args.wait_ns);
    for (int i = 0; i < nu && !stalled; ++i) {
      const int b = i % kAccSlots;
      const int off = inst_offset<KIND>(unit_m0(i) + ml);
      uint32_t* dst = args.out + unit_poly(i) * int64_t(kPolyWords) + off;
      uint32_t tws[kHalf];
      if (POST) {
        if (kAhead) {
#pragma unroll
          for (int j = 0; j < kHalf; ++j) tws[j] = tws_next[j];
          if (i + 1 < nu) load_tw(post + inst_offset<KIND>(unit_m0(i + 1) + ml), tws_next);
        } else {
          load_tw(post + off, tws);
        }
      }
      if (!warp_wait(accf_bar(b), (i / kAccSlots) & 1, abort, args.err, lane, args.wait_ns)) break;
      tc_fence_after();
#pragma unroll
      for (int cc = 0; cc < kHalf / kChunk; ++cc) {
        const int c0 = half * kHalf + cc * kChunk;
        uint32_t res[16];
        reduce_chunk<NK, kChunk, POST>(tmem + lane_addr + uint32_t(b * G::kNmma + c0), tws + cc * kChunk, q, qneg,
                                       res);
        if (S == 1) {
          uint4* o = reinterpret_cast<uint4*>(dst + c0);
#pragma unroll
          for (int j = 0; j < kChunk / 4; ++j)
            o[j] = make_uint4(res[4 * j], res[4 * j + 1], res[4 * j + 2], res[4 * j + 3]);
        } else {
#pragma unroll
          for (int j = 0; j < kChunk; ++j) dst[(c0 + j) * S] = res[j];
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acce_bar(b));
    }
  }

  __syncthreads();
  // Drain the MMAs (and the arrivals they signal) before TMEM is freed.
  if (warp == kMmaWarp && lane == 0) {
    mma_commit(drain_bar);
    mbar_wait(drain_bar, 0, nullptr, args.err, kWaitNs);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kMmaWarp) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(G::kTmemCols));
  }
}

// ------------------------------------------------ fused passes 2 and 3 ---
// The 64-point pass over i2 (kind 2) and the 16-point pass over i3 (kind 3)
// of the 8 consecutive 1024-word blocks 1024 P1 .. 1024 (P1 + 8) - 1 of a
// polynomial read and write exactly those 8192 words: the kind-2 instances
// 128 u .. 128 u + 127 and the kind-3 instances 512 u .. 512 u + 511 of unit
// u.  So one CTA runs both passes on a unit with one HBM read and one write:
// forward = pass 2 (kind 2, twiddled) then pass 3 (kind 3), inverse = inverse
// pass 1 (kind 3, twiddled) then inverse pass 2 (kind 2, twiddled).  The
// first stage's canonical outputs are written back over the unit's raw words
// in shared memory (each output sits where its input was), and the second
// stage transposes them from there like a raw copy.
//
// Roles as in k_tc_ntt_pass; per unit i (r = i % 2 raw slot):
//   producer     copy(i) into raw slot r                    [rawf(r)]
//   transposers  A tile of stage 1 from raw r               [af1]  (needs ae1)
//                A tiles of stage 2 from raw r (stage-1 out) [af2, rawe(r)] (needs stg(r), ae2)
//   MMA          stage 1 -> TMEM columns [0, 256)            [ae1, accf1] (needs af1, acce1)
//                stage 2 -> TMEM columns [256, 512)          [ae2, accf2] (needs af2, acce2)
//   epilogue     stage 1: reduce, twiddle -> raw r           [acce1, stg(r)] (needs accf1)
//                stage 2: reduce (, twiddle) -> global        [acce2] (needs accf2)
// Each role runs unit i + 1's first stage before unit i's second one, so
// the copy of unit i + 1 and both stages overlap; single A tiles and TMEM
// regions per stage (the two stages take all 512 columns), two raw slots.
// Measured on B200 (64 x 36 limbs): exact, but the serial two-stage chain per
// unit with one CTA per SM makes it slower than the two passes it replaces
// (0.76 against 0.60 ms), so it is selected by FHB_TUNE_TC_NTT_FUSED only.
constexpr int kFWords = 8 * 1024;                  // words of a unit
constexpr int kFRawBytes = kFWords * 4;            // 32 KiB
constexpr int kFUnitsPerPoly = kPolyWords / kFWords;
constexpr int kFTiles16 = kFWords / 16 / kUnit;    // 128-instance tiles of the 16-point stage
constexpr int kFCols = 256;                        // TMEM columns of one stage
static_assert(Geom<64>::kABytes == kFTiles16 * Geom<16>::kABytes && Geom<64>::kNmma == kFCols &&
                  kFTiles16 * Geom<16>::kNmma == kFCols,
              "both stages fill one 32 KiB A area and 256 TMEM columns");
constexpr int kFNumBarriers = 19;
// smem: [B64 | B16 | raw 0 | raw 1 | A64 | A16 x 4 | barriers]
constexpr int kFSmem = 1024 + Geom<64>::kBBytes + Geom<16>::kBBytes + 2 * kFRawBytes + 2 * Geom<64>::kABytes +
                       kBarrierBytes;
static_assert(kFSmem <= 232448 && 8 * kFNumBarriers + 8 <= kBarrierBytes, "fused pass shared memory");

struct FusedArgs {
  const uint32_t* in;
  uint32_t* out;
  const uint8_t* bmat64;    // [QP][64-point byte matrix] of the kind-2 stage
  const uint8_t* bmat16;    // [QP][16-point byte matrix] of the kind-3 stage
  const uint32_t* post1;    // [QP][N] twiddles of stage 1
  const uint32_t* post2;    // [QP][N] twiddles of stage 2, or null
  const uint32_t* qinfo;
  int64_t batch;
  int rows;
  int row_start;
  int ctas_per_row;
  int* err;
  unsigned long long wait_ns;
  int stall;
};

// Span offset of output / input n of local instance ml of a kind-2 tile, or
// of tile t of the kind-3 stage.
__device__ __forceinline__ int span2(int ml, int n) { return (ml >> 4) * 1024 + n * 16 + (ml & 15); }
__device__ __forceinline__ int span3(int t, int ml, int n) { return (t * kUnit + ml) * 16 + n; }

template <bool INV>
__global__ void __launch_bounds__(kThreads, 1) k_tc_ntt_fused(FusedArgs args) {
  // stage 1 / stage 2 shapes: forward (kind 2, 64) then (kind 3, 16); inverse the reverse
  constexpr int NK1 = INV ? 16 : 64, NK2 = INV ? 64 : 16;
  constexpr bool POST2 = INV;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw0 = smem_addr(smem_raw);
  const uint32_t base = (raw0 + 1023u) & ~1023u;
  uint8_t* const gbase = smem_raw + (base - raw0);
  const uint32_t b64_addr = base, b16_addr = base + Geom<64>::kBBytes;
  const uint32_t rawbuf_addr = b16_addr + Geom<16>::kBBytes;
  uint32_t* const rawbuf = reinterpret_cast<uint32_t*>(gbase + (rawbuf_addr - base));
  const uint32_t a64_addr = rawbuf_addr + 2 * kFRawBytes, a16_addr = a64_addr + Geom<64>::kABytes;
  uint8_t* const a64 = gbase + (a64_addr - base);
  uint8_t* const a16 = gbase + (a16_addr - base);
  uint64_t* const bars = reinterpret_cast<uint64_t*>(gbase + (a16_addr - base) + Geom<64>::kABytes);
  const uint32_t bar0 = smem_addr(bars);
  // barriers: b_full, rawf[2], rawe[2], stg[2], af1, ae1, af2, ae2, accf1, acce1, accf2, acce2, never, drain
  const uint32_t bfull_bar = bar0;
  auto rawf_bar = [&](int r) { return bar0 + 8u * (1 + r); };
  auto rawe_bar = [&](int r) { return bar0 + 8u * (3 + r); };
  auto stg_bar = [&](int r) { return bar0 + 8u * (5 + r); };
  const uint32_t af1 = bar0 + 8u * 7, ae1 = bar0 + 8u * 8, af2 = bar0 + 8u * 9, ae2 = bar0 + 8u * 10;
  const uint32_t accf1 = bar0 + 8u * 11, acce1 = bar0 + 8u * 12, accf2 = bar0 + 8u * 13, acce2 = bar0 + 8u * 14;
  const uint32_t never_bar = bar0 + 8u * 15, drain_bar = bar0 + 8u * 16;
  uint32_t* const tmem_slot = reinterpret_cast<uint32_t*>(bars + kFNumBarriers);
  volatile int* const abort = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int row = blockIdx.x / args.ctas_per_row, part = blockIdx.x % args.ctas_per_row;
  const int64_t units = args.batch * kFUnitsPerPoly;
  const int64_t u_begin = units * part / args.ctas_per_row, u_end = units * (part + 1) / args.ctas_per_row;
  const int nu = int(u_end - u_begin);
  const int prime = args.row_start + row;
  // unit i: words [unit_word(i), unit_word(i) + 8192) of the buffer
  auto unit_word = [&](int i) {
    const int64_t u = u_begin + i;
    return ((u / kFUnitsPerPoly) * args.rows + row) * int64_t(kPolyWords) + (u % kFUnitsPerPoly) * kFWords;
  };
  auto unit_span = [&](int i) { return int((u_begin + i) % kFUnitsPerPoly) * kFWords; };  // within the polynomial

  if (tid == 0) {
    mbar_init(bfull_bar, 1);
    for (int r = 0; r < 2; ++r) {
      mbar_init(rawf_bar(r), 1);
      mbar_init(rawe_bar(r), kTransposeWarps);
      mbar_init(stg_bar(r), kEpilogueWarps);
    }
    mbar_init(af1, kTransposeWarps);
    mbar_init(ae1, 1);
    mbar_init(af2, kTransposeWarps);
    mbar_init(ae2, 1);
    mbar_init(accf1, 1);
    mbar_init(acce1, kEpilogueWarps);
    mbar_init(accf2, 1);
    mbar_init(acce2, kEpilogueWarps);
    mbar_init(never_bar, 1);
    mbar_init(drain_bar, 1);
    *abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == kMmaWarp) tmem_alloc(smem_addr(tmem_slot), 2 * kFCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == kProducerWarp && lane == 0) {
    mbar_expect_tx(bfull_bar, Geom<64>::kBBytes + Geom<16>::kBBytes);
    const uint8_t* b64src = args.bmat64 + size_t(prime) * Geom<64>::kBBytes;
    for (int o = 0; o < Geom<64>::kBBytes; o += 16384) bulk_load(b64_addr + o, b64src + o, 16384, bfull_bar);
    bulk_load(b16_addr, args.bmat16 + size_t(prime) * Geom<16>::kBBytes, Geom<16>::kBBytes, bfull_bar);
    int i = 0;
    for (; i < nu; ++i) {
      const int r = i & 1;
      if (i >= 2 && !mbar_wait(rawe_bar(r), ((i >> 1) & 1) ^ 1, abort, args.err, args.wait_ns)) break;
      const uint8_t* src = reinterpret_cast<const uint8_t*>(args.in + unit_word(i));
      const uint32_t dst = rawbuf_addr + r * kFRawBytes;
      mbar_expect_tx(rawf_bar(r), kFRawBytes);
      for (int o = 0; o < kFRawBytes; o += 8192) bulk_load(dst + o, src + o, 8192, rawf_bar(r));
    }
    if (*abort) {
      mbar_wait(bfull_bar, 0, nullptr, args.err, kWaitNs);
      for (int t = i - 2 < 0 ? 0 : i - 2; t < i; ++t)
        mbar_wait(rawf_bar(t & 1), (t >> 1) & 1, nullptr, args.err, kWaitNs);
    }
  } else if (warp >= kTransposeWarp0 && warp < kTransposeWarp0 + kTransposeWarps) {
    const int tw = warp - kTransposeWarp0;
    // stage 1 of unit i from its raw copy
    auto stage1 = [&](int i) {
      const int r = i & 1;
      if (!warp_wait(rawf_bar(r), (i >> 1) & 1, abort, args.err, lane, args.wait_ns)) return false;
      if (i >= 1 && !warp_wait(ae1, (i & 1) ^ 1, abort, args.err, lane, args.wait_ns)) return false;
      const uint32_t* raw = rawbuf + r * kFWords;
      if (INV) {
#pragma unroll 1
        for (int t = 0; t < kFTiles16; ++t)
          transpose_tile<3, 16>(raw + t * kUnit * 16, a16 + t * Geom<16>::kABytes, tw, lane);
      } else {
        transpose_tile<2, 64>(raw, a64, tw, lane);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(af1);
      return true;
    };
    // stage 2 of unit i from stage 1's outputs, then the raw slot is free
    auto stage2 = [&](int i) {
      const int r = i & 1;
      if (!warp_wait(stg_bar(r), (i >> 1) & 1, abort, args.err, lane, args.wait_ns)) return false;
      if (i >= 1 && !warp_wait(ae2, (i & 1) ^ 1, abort, args.err, lane, args.wait_ns)) return false;
      const uint32_t* raw = rawbuf + r * kFWords;
      if (INV) {
        transpose_tile<2, 64>(raw, a64, tw, lane);
      } else {
#pragma unroll 1
        for (int t = 0; t < kFTiles16; ++t)
          transpose_tile<3, 16>(raw + t * kUnit * 16, a16 + t * Geom<16>::kABytes, tw, lane);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(af2);
        mbar_arrive(rawe_bar(r));
      }
      return true;
    };
    bool ok = nu == 0 || stage1(0);
    for (int i = 0; i < nu && ok; ++i) {
      if (i + 1 < nu && !stage1(i + 1)) break;
      ok = stage2(i);
    }
  } else if (warp == kMmaWarp && lane == 0) {
    // one 64-point tile: 8 MMAs of N = 256; four 16-point tiles: 2 MMAs of N = 64 each
    auto issue64 = [&](uint32_t d_tmem) {
#pragma unroll
      for (int st = 0; st < Geom<64>::kSteps; ++st)
        mma_i8(d_tmem, smem_desc(a64_addr + st * 256, 128, Geom<64>::kSbo),
               smem_desc(b64_addr + st * 256, 128, Geom<64>::kSbo), instr_desc(Geom<64>::kNmma), st > 0 ? 1u : 0u);
    };
    auto issue16 = [&](uint32_t d_tmem) {
#pragma unroll
      for (int t = 0; t < kFTiles16; ++t)
#pragma unroll
        for (int st = 0; st < Geom<16>::kSteps; ++st)
          mma_i8(d_tmem + uint32_t(t * Geom<16>::kNmma),
                 smem_desc(a16_addr + t * Geom<16>::kABytes + st * 256, 128, Geom<16>::kSbo),
                 smem_desc(b16_addr + st * 256, 128, Geom<16>::kSbo), instr_desc(Geom<16>::kNmma),
                 st > 0 ? 1u : 0u);
    };
    auto mma1 = [&](int i) {
      if (!mbar_wait(af1, i & 1, abort, args.err, args.wait_ns) ||
          (i >= 1 && !mbar_wait(acce1, (i & 1) ^ 1, abort, args.err, args.wait_ns)))
        return false;
      tc_fence_after();
      if (INV)
        issue16(tmem);
      else
        issue64(tmem);
      mma_commit(ae1);
      mma_commit(accf1);
      return true;
    };
    auto mma2 = [&](int i) {
      if (!mbar_wait(af2, i & 1, abort, args.err, args.wait_ns) ||
          (i >= 1 && !mbar_wait(acce2, (i & 1) ^ 1, abort, args.err, args.wait_ns)))
        return false;
      tc_fence_after();
      if (INV)
        issue64(tmem + kFCols);
      else
        issue16(tmem + kFCols);
      mma_commit(ae2);
      mma_commit(accf2);
      return true;
    };
    bool ok = mbar_wait(bfull_bar, 0, abort, args.err, args.wait_ns) && (nu == 0 || mma1(0));
    for (int i = 0; i < nu && ok; ++i) {
      if (i + 1 < nu && !mma1(i + 1)) break;
      ok = mma2(i);
    }
  } else if (warp < kEpilogueWarps) {
    const uint32_t q = args.qinfo[2 * prime], qneg = args.qinfo[2 * prime + 1];
    const uint32_t* post1 = args.post1 + (size_t(prime) << kLogN);
    const uint32_t* post2 = POST2 ? args.post2 + (size_t(prime) << kLogN) : nullptr;
    const int quarter = warp & 3, half = warp >> 2;
    const int ml = quarter * 32 + lane;
    const uint32_t lane_addr = uint32_t(quarter * 32) << 16;
    // this thread's 32 outputs of a stage: kind 2 -> outputs [32 half, 32 half + 32)
    // of instance ml; kind 3 -> outputs [8 half, 8 half + 8) of instance ml of each tile
    auto load_tw2 = [&](const uint32_t* t, int span, uint32_t (&v)[32]) {
#pragma unroll
      for (int j = 0; j < 32; ++j) v[j] = t[span + span2(ml, half * 32 + j)];
    };
    auto load_tw3 = [&](const uint32_t* t, int span, uint32_t (&v)[32]) {
#pragma unroll
      for (int tt = 0; tt < kFTiles16; ++tt) {
        const uint4* p = reinterpret_cast<const uint4*>(t + span + span3(tt, ml, half * 8));
        const uint4 x = p[0], y = p[1];
        v[8 * tt] = x.x, v[8 * tt + 1] = x.y, v[8 * tt + 2] = x.z, v[8 * tt + 3] = x.w;
        v[8 * tt + 4] = y.x, v[8 * tt + 5] = y.y, v[8 * tt + 6] = y.z, v[8 * tt + 7] = y.w;
      }
    };
    auto epi1 = [&](int i) {
      const int r = i & 1;
      uint32_t tws[32];
      if (INV)
        load_tw3(post1, unit_span(i), tws);
      else
        load_tw2(post1, unit_span(i), tws);
      if (!warp_wait(accf1, i & 1, abort, args.err, lane, args.wait_ns)) return false;
      tc_fence_after();
      uint32_t* stage = rawbuf + r * kFWords;  // outputs over the unit's raw words
      if (INV) {
#pragma unroll
        for (int tt = 0; tt < kFTiles16; ++tt) {
          uint32_t res[16];
          reduce_chunk<16, 8, true>(tmem + lane_addr + uint32_t(tt * Geom<16>::kNmma + half * 8), tws + 8 * tt, q,
                                    qneg, res);
          uint4* o = reinterpret_cast<uint4*>(stage + span3(tt, ml, half * 8));
          o[0] = make_uint4(res[0], res[1], res[2], res[3]);
          o[1] = make_uint4(res[4], res[5], res[6], res[7]);
        }
      } else {
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
          const int c0 = half * 32 + cc * 16;
          uint32_t res[16];
          reduce_chunk<64, 16, true>(tmem + lane_addr + uint32_t(c0), tws + 16 * cc, q, qneg, res);
#pragma unroll
          for (int j = 0; j < 16; ++j) stage[span2(ml, c0 + j)] = res[j];
        }
      }
      // the slot is overwritten by a bulk copy (async proxy) once stage 2 has read it
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      tc_fence_before();
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(acce1);
        mbar_arrive(stg_bar(r));
      }
      return true;
    };
    auto epi2 = [&](int i) {
      uint32_t tws[32];
      if (POST2) load_tw2(post2, unit_span(i), tws);
      if (!warp_wait(accf2, i & 1, abort, args.err, lane, args.wait_ns)) return false;
      tc_fence_after();
      uint32_t* dst = args.out + unit_word(i);
      if (INV) {
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
          const int c0 = half * 32 + cc * 16;
          uint32_t res[16];
          reduce_chunk<64, 16, POST2>(tmem + kFCols + lane_addr + uint32_t(c0), tws + 16 * cc, q, qneg, res);
#pragma unroll
          for (int j = 0; j < 16; ++j) dst[span2(ml, c0 + j)] = res[j];
        }
      } else {
#pragma unroll
        for (int tt = 0; tt < kFTiles16; ++tt) {
          uint32_t res[16];
          reduce_chunk<16, 8, false>(tmem + kFCols + lane_addr + uint32_t(tt * Geom<16>::kNmma + half * 8), tws, q,
                                     qneg, res);
          uint4* o = reinterpret_cast<uint4*>(dst + span3(tt, ml, half * 8));
          o[0] = make_uint4(res[0], res[1], res[2], res[3]);
          o[1] = make_uint4(res[4], res[5], res[6], res[7]);
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acce2);
      return true;
    };
    // test only: a wait that must run out (its limit is the pipeline's)
    const bool stalled = args.stall && !warp_wait(never_bar, 0, abort, args.err, lane, args.wait_ns);
    bool ok = !stalled && (nu == 0 || epi1(0));
    for (int i = 0; i < nu && ok; ++i) {
      if (i + 1 < nu && !epi1(i + 1)) break;
      ok = epi2(i);
    }
  }

  __syncthreads();
  if (warp == kMmaWarp && lane == 0) {
    mma_commit(drain_bar);
    mbar_wait(drain_bar, 0, nullptr, args.err, kWaitNs);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kMmaWarp) {
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, 2 * kFCols);
  }
}

// ------------------------------------------------------------------ host ---
using u128 = unsigned __int128;

uint64_t mulmod64(uint64_t a, uint64_t b, uint64_t q) { return uint64_t((u128)a * b % q); }

uint64_t powmod64(uint64_t b, uint64_t e, uint64_t q) {
  uint64_t r = 1 % q;
  b %= q;
  for (; e; e >>= 1) {
    if (e & 1) r = mulmod64(r, b, q);
    b = mulmod64(b, b, q);
  }
  return r;
}

uint32_t brev(uint32_t v, int bits) {
  uint32_t r = 0;
  for (int i = 0; i < bits; ++i, v >>= 1) r = (r << 1) | (v & 1);
  return r;
}

// Pass table: 0, 1, 2 = forward passes 1, 2, 3; 3, 4, 5 = inverse passes
// over the instance maps of passes 3, 2, 1 (the inverse runs backwards).
constexpr int kPassNk[6] = {64, 64, 16, 16, 64, 64};
constexpr bool kPassPost[6] = {true, true, false, true, true, false};

// Exponent of psi (mod 2N) of the constant matrix W[k][n] of a pass.
uint32_t pass_exponent(int pass, uint32_t k, uint32_t n) {
  const uint32_t mask = (2u << kLogN) - 1;
  switch (pass) {
    case 0: return (1024u * k * (2u * brev(n, 6) + 1u)) & mask;          // k = i1, n = P1
    case 1: return (2048u * brev(n, 6) * k) & mask;                      // k = i2, n = P2
    case 2: return (8192u * brev(n, 4) * k) & mask;                      // k = i3, n = P3
    case 3: return (0u - 8192u * brev(k, 4) * n) & mask;                 // k = P3, n = i3
    case 4: return (0u - 2048u * brev(k, 6) * n) & mask;                 // k = P2, n = i2
    default: return (0u - 1024u * n * (2u * brev(k, 6) + 1u)) & mask;   // k = P1, n = i1
  }
}

}  // namespace tcntt

size_t tc_ntt_table_bytes(int pass) {
  if (pass < 0 || pass > 5) return 0;
  const int nk = tcntt::kPassNk[pass];
  return size_t(4 * nk) * size_t(4 * nk);
}

// Fill the byte matrix of one pass for one prime (tc_ntt_table_bytes(pass)
// bytes at `bmat`, the kernel's shared-memory layout: row e * NK + n, byte
// d * NK + k of a K-major canonical tile with 8-row groups NK * 32 bytes
// apart) and, for passes with a twiddle, the N twiddles t as t 2^32 mod q in
// output order at `post`.
void tc_ntt_tables_host(uint64_t q, uint64_t psi, int pass, uint8_t* bmat, uint32_t* post) {
  using namespace tcntt;
  const uint32_t two_n = 2u << kLogN;
  std::vector<uint32_t> pw(two_n);
  pw[0] = 1;
  for (uint32_t i = 1; i < two_n; ++i) pw[i] = uint32_t(uint64_t(pw[i - 1]) * psi % q);  // q < 2^28
  const uint32_t nk = uint32_t(kPassNk[pass]);
  const uint32_t sbo = nk * 32;
  uint64_t scale[4];
  for (int d = 0; d < 4; ++d) scale[d] = powmod64(2, 8 * d + 32, q);
  for (uint32_t k = 0; k < nk; ++k) {
    for (uint32_t n = 0; n < nk; ++n) {
      const uint64_t w = pw[pass_exponent(pass, k, n)];
      for (uint32_t d = 0; d < 4; ++d) {
        const uint32_t wd = uint32_t(w * scale[d] % q);
        const uint32_t kap = d * nk + k;
        for (uint32_t e = 0; e < 4; ++e) {
          const uint32_t r = e * nk + n;
          bmat[(r & 7) * 16 + (r >> 3) * sbo + (kap >> 4) * 128 + (kap & 15)] = uint8_t(wd >> (8 * e));
        }
      }
    }
  }
  if (!post || !kPassPost[pass]) return;
  const uint64_t R = powmod64(2, 30, q);
  const uint64_t ninv_rinv = mulmod64(powmod64(R, q - 2, q), powmod64((uint64_t(1) << kLogN) % q, q - 2, q), q);
  for (uint32_t p1 = 0; p1 < 64; ++p1) {
    const uint32_t odd1 = 2u * brev(p1, 6) + 1u;
    for (uint32_t a = 0; a < 64; ++a) {
      for (uint32_t i3 = 0; i3 < 16; ++i3) {
        // output address 1024 p1 + 16 a + i3 in every twiddled pass
        uint32_t ex;
        uint64_t c = 1;
        if (pass == 0) {  // a = i2: R psi^{16 i2 (2 m1 + 1)}
          ex = (16u * a * odd1) & (two_n - 1);
          c = R;
        } else if (pass == 1 || pass == 3) {  // a = P2: psi^{+-((2 m1 + 1) i3 + 128 m2 i3)}
          ex = (odd1 * i3 + 128u * brev(a, 6) * i3) & (two_n - 1);
          if (pass == 3) {
            ex = (two_n - ex) & (two_n - 1);
            c = ninv_rinv;
          }
        } else {  // pass 4, a = i2: psi^{-16 i2 (2 m1 + 1)}
          ex = (two_n - ((16u * a * odd1) & (two_n - 1))) & (two_n - 1);
        }
        const uint64_t w = mulmod64(pw[ex], c, q);
        post[1024 * p1 + 16 * a + i3] = uint32_t((w << 32) % q);
      }
    }
  }
}

int tc_ntt_prepare(Context& c) {
  using namespace tcntt;
  std::lock_guard<std::mutex> lock(c.tc_mutex);
  if (c.tc) return 0;
  if (c.bits != 32 || c.log_n != kLogN) return fail(-7, "the tensor-core NTT needs an int32 context with log_n = 16");
  const int qp = c.qp();
  auto* t = new TcNttTables();
  std::vector<void*> mine;
  auto dev_alloc = [&](size_t bytes) -> void* {
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
    mine.push_back(p);
    return p;
  };
  auto give_up = [&](const char* where) {
    cudaError_t e = cudaGetLastError();
    for (void* p : mine) cudaFree(p);
    delete t;
    return e != cudaSuccess ? cuda_status(e, where) : fail(-6, std::string("out of memory: ") + where);
  };
  const size_t n = size_t(1) << kLogN;
  std::vector<uint32_t> post(size_t(qp) * n);
  for (int pass = 0; pass < 6; ++pass) {
    const size_t tb = tc_ntt_table_bytes(pass);
    std::vector<uint8_t> bm(size_t(qp) * tb);
    for (int j = 0; j < qp; ++j)
      tc_ntt_tables_host(c.moduli[j], c.roots[j], pass, bm.data() + size_t(j) * tb,
                         kPassPost[pass] ? post.data() + size_t(j) * n : nullptr);
    t->bmat[pass] = static_cast<uint8_t*>(dev_alloc(bm.size()));
    if (!t->bmat[pass] || cudaMemcpy(t->bmat[pass], bm.data(), bm.size(), cudaMemcpyHostToDevice) != cudaSuccess)
      return give_up("tensor-core NTT byte matrices");
    if (kPassPost[pass]) {
      auto*& dst = t->post[pass];
      dst = static_cast<uint32_t*>(dev_alloc(post.size() * sizeof(post[0])));
      if (!dst || cudaMemcpy(dst, post.data(), post.size() * sizeof(post[0]), cudaMemcpyHostToDevice) != cudaSuccess)
        return give_up("tensor-core NTT twiddles");
    }
  }
  std::vector<uint32_t> qi(2 * size_t(qp));
  for (int j = 0; j < qp; ++j) {
    const uint32_t q = uint32_t(c.moduli[j]);
    uint32_t x = 1;  // q^{-1} mod 2^32 by Newton iteration
    for (int i = 0; i < 5; ++i) x *= 2u - q * x;
    qi[2 * j] = q;
    qi[2 * j + 1] = 0u - x;
  }
  t->qinfo = static_cast<uint32_t*>(dev_alloc(qi.size() * 4));
  t->err = static_cast<int*>(dev_alloc(sizeof(int)));
  if (!t->qinfo || !t->err || cudaMemcpy(t->qinfo, qi.data(), qi.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(t->err, 0, sizeof(int)) != cudaSuccess)
    return give_up("tensor-core NTT constants");
  for (void* p : mine) c.allocations.push_back(p);
  c.tc = t;
  return 0;
}

namespace {
template <int KIND, int NK, bool POST>
int launch_pass(const Context& c, const uint32_t* in, uint32_t* out, int pass, int64_t polys, int rows,
                int row_start, cudaStream_t st) {
  using namespace tcntt;
  auto kern = k_tc_ntt_pass<KIND, NK, POST>;
  const int smem = smem_bytes<NK>();
  if (int rc = ensure_dynamic_smem(reinterpret_cast<const void*>(kern), smem)) return rc;
  // persistent CTAs: as many as are resident at once (148 SMs), each
  // streaming units of one prime
  const int64_t batch = polys / rows;
  const int64_t units = batch * Geom<NK>::kUnitsPerPoly;
  int64_t per_row = 148 * Geom<NK>::kCtasPerSm / rows;
  if (per_row > units) per_row = units;
  if (per_row < 1) per_row = 1;
  PassArgs a{in, out, c.tc->bmat[pass], POST ? c.tc->post[pass] : nullptr, c.tc->qinfo, batch, rows,
             row_start, int(per_row), c.tc->err, c.tc_wait_ns ? c.tc_wait_ns : kWaitNs, c.tc_test_stall};
  kern<<<dim3(unsigned(rows * per_row)), kThreads, smem, st>>>(a);
  return cuda_status(cudaGetLastError(), "k_tc_ntt_pass");
}

template <bool INV>
int launch_fused(const Context& c, const uint32_t* in, uint32_t* out, int64_t polys, int rows, int row_start,
                 cudaStream_t st) {
  using namespace tcntt;
  auto kern = k_tc_ntt_fused<INV>;
  if (int rc = ensure_dynamic_smem(reinterpret_cast<const void*>(kern), kFSmem)) return rc;
  // persistent CTAs, one per SM (all of its TMEM), each streaming units of one prime
  const int64_t batch = polys / rows;
  const int64_t units = batch * kFUnitsPerPoly;
  int64_t per_row = 148 / rows;
  if (per_row > units) per_row = units;
  if (per_row < 1) per_row = 1;
  // forward: pass 2 (table 1, twiddled) + pass 3 (table 2); inverse: table 3 (twiddled) + table 4 (twiddled)
  const int p64 = INV ? 4 : 1, p16 = INV ? 3 : 2;
  FusedArgs a{in, out, c.tc->bmat[p64], c.tc->bmat[p16], c.tc->post[INV ? 3 : 1], INV ? c.tc->post[4] : nullptr,
              c.tc->qinfo, batch, rows, row_start, int(per_row), c.tc->err, c.tc_wait_ns ? c.tc_wait_ns : kWaitNs,
              c.tc_test_stall};
  kern<<<dim3(unsigned(rows * per_row)), kThreads, kFSmem, st>>>(a);
  return cuda_status(cudaGetLastError(), "k_tc_ntt_fused");
}
}  // namespace

// The passes of a direction; passes after the first run in place on `out`
// (every unit writes exactly the words its raw copy read, after the copy
// landed), so in == out is allowed and no scratch is needed.
int tc_ntt(Context& c, const void* in, void* out, int64_t polys, int rows, int row_start, bool inverse,
           cudaStream_t st) {
  if (int rc = tc_ntt_prepare(c)) return rc;
  if (polys == 0) return 0;
  const auto* x = static_cast<const uint32_t*>(in);
  auto* y = static_cast<uint32_t*>(out);
  if (c.tc_ntt_fused) {
    if (!inverse) {
      if (int rc = launch_pass<1, 64, true>(c, x, y, 0, polys, rows, row_start, st)) return rc;
      return launch_fused<false>(c, y, y, polys, rows, row_start, st);
    }
    if (int rc = launch_fused<true>(c, x, y, polys, rows, row_start, st)) return rc;
    return launch_pass<1, 64, false>(c, y, y, 5, polys, rows, row_start, st);
  }
  if (!inverse) {
    if (int rc = launch_pass<1, 64, true>(c, x, y, 0, polys, rows, row_start, st)) return rc;
    if (int rc = launch_pass<2, 64, true>(c, y, y, 1, polys, rows, row_start, st)) return rc;
    return launch_pass<3, 16, false>(c, y, y, 2, polys, rows, row_start, st);
  }
  if (int rc = launch_pass<3, 16, true>(c, x, y, 3, polys, rows, row_start, st)) return rc;
  if (int rc = launch_pass<2, 64, true>(c, y, y, 4, polys, rows, row_start, st)) return rc;
  return launch_pass<1, 64, false>(c, y, y, 5, polys, rows, row_start, st);
}

int tc_ntt_status(Context& c, int* flag) {
  std::lock_guard<std::mutex> lock(c.tc_mutex);
  *flag = 0;
  if (!c.tc) return 0;
  if (cudaError_t e = cudaMemcpy(flag, c.tc->err, sizeof(int), cudaMemcpyDeviceToHost)) return cuda_status(e, "flag");
  return cuda_status(cudaMemset(c.tc->err, 0, sizeof(int)), "flag reset");
}

}  // namespace fhb
