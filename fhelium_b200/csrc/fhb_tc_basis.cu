// Exact integer tensor-core basis extension (ModUp stage 2) for int64
// residues (primes < 2^60) on the 5th-generation tensor cores:
// tcgen05.mma kind::i8 with int32 accumulators in tensor memory.
//
// What it computes (the reference's mixed_radix_basis_extend_to_montgomery,
// csrc/ops/rns/cuda/mixed_radix_cuda.cu:146-182, restated as a matrix
// product): for every active hybrid digit a of a level, every ciphertext b,
// every destination row j of Q_l P (prime p = p_{level + j}) and every
// coefficient k,
//   ext[a][b][j][k] = sum_{r < alpha_a} d_r[k] (M_r mod p)   (mod p), in [0, 2p),
// where d_r are the digit's Garner mixed-radix digits (canonical, < 2^60) and
// M_r the product of the digit's first r primes.  This is the value the
// CUDA-core key-switch core computes on the fly as the source of each
// forward NTT; the tensor-core form materialises it once so the core only
// transforms.
//
// Exact byte form.  Split d_r = sum_u 2^{8u} d_{r,u} (u < 8) and pre-scale the
// constants per data byte and by 2^64: C'_{r,u} = 2^{8u} 2^64 (M_r mod p) mod p,
// itself split into bytes C'_{r,u} = sum_e 2^{8e} c_{r,u,e}.  One MMA of
//   M = 128 coefficients, K = 32 (8 data bytes x 4 digit rows), N = 8 bytes e
//   x up to 16 destination rows
// gives acc[k][(j, e)] = sum_{r,u} d_{r,u}[k] c_{r,u,e}(j) < 32 * 255^2 < 2^21
// (K = 64 and < 2^22 for digits of 5..8 primes), so the sum is exact in int32.
// The epilogue forms S = sum_e 2^{8e} acc_e < 2^78 = 2^64 (sum_r d_r M_r mod p)
// (mod p) and one Montgomery reduction by 2^64 returns the extension in
// [0, 2p) (S < p 2^64 for p > 2^14).  The A operand needs no byte shuffle:
// in the K-major canonical layout the 8 bytes of a little-endian residue word
// are 8 consecutive K positions, so the A tile is the digit words themselves,
// placed two rows to a 16-byte core-matrix row.
//
// Kernel: persistent CTAs, one per SM (the 512 TMEM columns are the SM's),
// each streaming a contiguous range of units (digit, ciphertext, 128
// coefficients), digit-major, through a warp-specialised pipeline:
//   loaders (warps 16-17): the digit words of a unit into one of 4 A tiles;
//       lane 0 of warp 16 also bulk-copies the byte matrix of each new digit
//       into one of two B buffers;
//   MMA issuer (warp 18, lane 0): per unit one MMA per 16-row chunk of
//       destination rows (K-steps of 32) into a ring of 4 TMEM slots of 128
//       columns;
//   epilogue (warps 0-15; warp w reads TMEM lane quarter w % 4 and the four
//       rows 4 (w / 4) .. + 3 of a chunk): recombination, reduction, store.
// Every mbarrier wait is bounded; a wait that gives up raises a CTA abort
// flag that releases every other wait and sets the device error flag, and
// the CTA drains its bulk copies and MMAs (bounded) before it frees TMEM.
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "fhb_context.h"
#include "fhb_kernels.cuh"
#include "fhb_tc_common.cuh"

namespace fhb {
namespace tcb {
using namespace fhb::tc;

constexpr int kUnit = 128;             // coefficients per unit (MMA M)
constexpr int kChunkRows = 16;         // destination rows per MMA: N = 8 x 16 = 128 at most
constexpr int kAccCols = 128;          // TMEM columns per accumulator slot
constexpr int kAccSlots = 4;
constexpr int kASlots = 4;
constexpr int kTmemCols = kAccSlots * kAccCols;  // 512: the whole SM
constexpr int kEpilogueWarps = 16;     // warps 0..15
constexpr int kPermuteWarp0 = 16;      // warps 16, 17
constexpr int kPermuteWarps = 2;
constexpr int kProducerWarp = 18;
constexpr int kMmaWarp = 19;
constexpr int kThreads = 32 * 20;
constexpr int kRowBytes = kUnit * 8;   // one digit row of a unit, 1 KiB
// raw staging slots (one unit's digit rows each): deep enough that the
// bulk copies of several units are in flight behind the one being permuted
template <int KS>
constexpr int raw_slots() { return KS == 1 ? 8 : 6; }
constexpr int kMaxRawSlots = 8;
constexpr int kPinfoBytes = 2048;      // the level's (p, -p^{-1} mod 2^64) pairs, up to 128 rows
constexpr int kNumBarriers = 2 + 2 + 2 * kMaxRawSlots + 2 * kASlots + 2 * kAccSlots + 2;  // ... drain, never
constexpr int kBarrierBytes = 384;
// Requested even when the tables are smaller, so that no second CTA (which
// would wait for TMEM) is ever resident beside the first.
constexpr int kMinSmem = 120 * 1024;
static_assert(8 * kNumBarriers + 8 <= kBarrierBytes, "barrier area");

struct ExtendArgs {
  const uint64_t* digits;    // [batch][q_limbs][N]: Garner digits, canonical; row r = prime level + r
  uint64_t* ext;             // [nd][batch][qp_limbs][N]: extensions, [0, 2p)
  const uint8_t* bmat;       // [nd][nchunks][128 * K]: byte matrices of this level's digits
  const uint64_t* pinfo;     // [QP0][2]: p, -p^{-1} mod 2^64
  const DigitDesc* digit;    // [nd] active digits of this level
  int64_t batch;
  int level, q_limbs, qp_limbs, nd, nchunks, log_n;
  int skip_own;              // 1: leave a digit's own rows unwritten (relinearisation reuses c2 there)
  int* err;
  unsigned long long wait_ns;  // limit of the pipeline waits (drain waits keep kWaitNs)
  int stall;                   // test only: the epilogue first waits on a barrier nothing completes
};

// Position of a CTA's current unit in its contiguous range of the unit list
// (outer, ciphertext, coefficient block), advanced by counting instead of
// dividing: a 64-bit division per unit and thread costs as much as the
// epilogue's arithmetic.
struct UnitIter {
  int outer;      // digit (basis extension) or component (ModDown)
  int64_t b;      // ciphertext
  int64_t blk;    // block of kUnit coefficients
  int64_t batch, nblk;
  __device__ __forceinline__ UnitIter(int64_t u, int64_t batch_, int64_t nblk_) : batch(batch_), nblk(nblk_) {
    const int64_t per_outer = batch_ * nblk_;
    outer = int(u / per_outer);
    const int64_t r = u - int64_t(outer) * per_outer;
    b = r / nblk_;
    blk = r - b * nblk_;
  }
  __device__ __forceinline__ void next() {
    if (++blk == nblk) {
      blk = 0;
      if (++b == batch) {
        b = 0;
        ++outer;
      }
    }
  }
};

// Extension value from the eight byte accumulators of one output:
// S = sum_e 2^{8e} acc_e (< 2^78) and its Montgomery reduction by 2^64.
// Accumulators are < 2^22, so byte-adjacent pairs combine in 32 bits
// (acc_e + 2^8 acc_{e+1} < 2^31) and the pairs in two 48-bit halves.
__device__ __forceinline__ uint64_t recombine_redc(const uint32_t* acc, uint64_t p, uint64_t pneg) {
  const uint32_t p01 = acc[0] + (acc[1] << 8), p23 = acc[2] + (acc[3] << 8);
  const uint32_t p45 = acc[4] + (acc[5] << 8), p67 = acc[6] + (acc[7] << 8);
  const uint64_t lo = uint64_t(p01) + (uint64_t(p23) << 16);  // S mod 2^32 part, < 2^48
  const uint64_t hi = uint64_t(p45) + (uint64_t(p67) << 16);  // coefficient of 2^32, < 2^48
  const uint64_t slo = lo + (hi << 32);
  const uint64_t shi = (hi >> 32) + (slo < lo ? 1u : 0u);
  const uint64_t m = slo * pneg;  // S + m p = 0 mod 2^64
  return shi + __umul64hi(m, p) + (slo != 0 ? 1u : 0u);
}

template <int KS>
__global__ void __launch_bounds__(kThreads, 1) k_tc_extend(ExtendArgs args) {
  constexpr int K = 32 * KS;           // bytes of one A / B row
  constexpr int kSbo = K / 16 * 128;   // byte distance between 8-row groups
  constexpr int kATile = kUnit * K;
  constexpr int kBTile = 128 * K;      // byte matrix of one 16-row chunk (128 MMA N rows)
  constexpr int kRawSlots = raw_slots<KS>();
  constexpr int kRawSlotBytes = 4 * KS * kRowBytes;  // up to 4 KS digit rows
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw0 = smem_addr(smem_raw);
  const uint32_t base = (raw0 + 1023u) & ~1023u;
  uint8_t* const gbase = smem_raw + (base - raw0);
  const int bbytes = args.nchunks * kBTile;
  // [B buffers 2 x bbytes | raw slots | A tiles | pinfo | barriers]
  const uint32_t b_addr0 = base;
  const uint32_t rawbuf_addr = base + 2u * uint32_t(bbytes);
  const uint64_t* const rawbuf = reinterpret_cast<const uint64_t*>(gbase + 2 * bbytes);
  const uint32_t a_addr0 = rawbuf_addr + uint32_t(kRawSlots * kRawSlotBytes);
  uint8_t* const a_tile0 = gbase + 2 * bbytes + kRawSlots * kRawSlotBytes;
  ulonglong2* const spinfo = reinterpret_cast<ulonglong2*>(a_tile0 + kASlots * kATile);
  uint64_t* const bars = reinterpret_cast<uint64_t*>(a_tile0 + kASlots * kATile + kPinfoBytes);
  const uint32_t bar0 = smem_addr(bars);
  auto bfull = [&](int x) { return bar0 + 8u * x; };
  auto bempty = [&](int x) { return bar0 + 8u * (2 + x); };
  auto rawfull = [&](int r) { return bar0 + 8u * (4 + r); };
  auto rawempty = [&](int r) { return bar0 + 8u * (4 + kMaxRawSlots + r); };
  auto afull = [&](int s) { return bar0 + 8u * (4 + 2 * kMaxRawSlots + s); };
  auto aempty = [&](int s) { return bar0 + 8u * (4 + 2 * kMaxRawSlots + kASlots + s); };
  auto accfull = [&](int s) { return bar0 + 8u * (4 + 2 * kMaxRawSlots + 2 * kASlots + s); };
  auto accempty = [&](int s) { return bar0 + 8u * (4 + 2 * kMaxRawSlots + 2 * kASlots + kAccSlots + s); };
  const uint32_t drain_bar = bar0 + 8u * (kNumBarriers - 2);
  const uint32_t never_bar = bar0 + 8u * (kNumBarriers - 1);  // nothing arrives on it
  uint32_t* const tmem_slot = reinterpret_cast<uint32_t*>(bars + kNumBarriers);
  volatile int* const abort = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t n = int64_t(1) << args.log_n;
  const int64_t nblk = n / kUnit;
  const int64_t per_digit = args.batch * nblk;
  const int64_t units = int64_t(args.nd) * per_digit;
  const int64_t u_begin = units * blockIdx.x / gridDim.x, u_end = units * (blockIdx.x + 1) / gridDim.x;
  const int nu = int(u_end - u_begin);
  const unsigned long long lim = args.wait_ns;

  for (int j = tid; j < args.qp_limbs; j += kThreads)
    spinfo[j] = reinterpret_cast<const ulonglong2*>(args.pinfo)[args.level + j];
  if (tid == 0) {
    for (int x = 0; x < 2; ++x) {
      mbar_init(bfull(x), 1);
      mbar_init(bempty(x), 1);
    }
    for (int r = 0; r < kRawSlots; ++r) {
      mbar_init(rawfull(r), 1);
      mbar_init(rawempty(r), kPermuteWarps);
    }
    for (int s = 0; s < kASlots; ++s) {
      mbar_init(afull(s), kPermuteWarps);
      mbar_init(aempty(s), 1);
    }
    for (int s = 0; s < kAccSlots; ++s) {
      mbar_init(accfull(s), 1);
      mbar_init(accempty(s), kEpilogueWarps);
    }
    mbar_init(drain_bar, 1);
    mbar_init(never_bar, 1);
    *abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == kMmaWarp) tmem_alloc(smem_addr(tmem_slot), kTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == kProducerWarp && lane == 0) {
    // the byte matrices of each new digit into one of two B buffers, and the
    // digit rows of each unit (alpha contiguous 1 KiB rows) into a raw slot
    int cur = -1, dseq = -1, i = 0;
    int issued[2] = {0, 0};
    UnitIter it(u_begin, args.batch, nblk);
    for (; i < nu; ++i, it.next()) {
      const int a = it.outer;
      const int64_t b = it.b, blk = it.blk;
      if (a != cur) {
        cur = a;
        ++dseq;
        const int x = dseq & 1;
        if (dseq >= 2 && !mbar_wait(bempty(x), ((dseq >> 1) - 1) & 1, abort, args.err, lim)) break;
        mbar_expect_tx(bfull(x), uint32_t(bbytes));
        const uint8_t* src = args.bmat + size_t(a) * size_t(bbytes);
        for (int o = 0; o < bbytes; o += 16384)
          bulk_load(b_addr0 + uint32_t(x * bbytes + o), src + o, uint32_t(min(16384, bbytes - o)), bfull(x));
        ++issued[x];
      }
      const int r = i % kRawSlots;
      if (i >= kRawSlots && !mbar_wait(rawempty(r), ((i / kRawSlots) & 1) ^ 1, abort, args.err, lim)) break;
      const DigitDesc d = args.digit[a];
      const uint64_t* src = args.digits + (b * args.q_limbs + (d.prime0 - args.level)) * n + blk * kUnit;
      mbar_expect_tx(rawfull(r), uint32_t(d.alpha * kRowBytes));
      for (int rr = 0; rr < d.alpha; ++rr)
        bulk_load(rawbuf_addr + uint32_t(r * kRawSlotBytes + rr * kRowBytes), src + int64_t(rr) * n, kRowBytes,
                  rawfull(r));
    }
    // after an abort, wait (bounded, default limit) for the copies still in flight
    if (*abort) {
      for (int x = 0; x < 2; ++x)
        if (issued[x] > 0) mbar_wait(bfull(x), (issued[x] - 1) & 1, nullptr, args.err, kWaitNs);
      for (int t = i - kRawSlots < 0 ? 0 : i - kRawSlots; t < i; ++t)
        mbar_wait(rawfull(t % kRawSlots), (t / kRawSlots) & 1, nullptr, args.err, kWaitNs);
    }
  } else if (warp >= kPermuteWarp0 && warp < kPermuteWarp0 + kPermuteWarps) {
    // raw rows -> A tile: word (coefficient m, digit row r) at byte
    // (m / 8) sbo + (r / 2) 128 + (m % 8) 16 + (r % 2) 8, i.e. its 8 bytes are
    // K positions 8 r .. 8 r + 7; rows r >= alpha are zero.
    const int lt = tid - kPermuteWarp0 * 32;
    UnitIter it(u_begin, args.batch, nblk);
    for (int i = 0; i < nu; ++i, it.next()) {
      const int a = it.outer;
      const int r = i % kRawSlots, s = i % kASlots;
      if (!warp_wait(rawfull(r), (i / kRawSlots) & 1, abort, args.err, lane, lim)) break;
      if (i >= kASlots && !warp_wait(aempty(s), ((i / kASlots) & 1) ^ 1, abort, args.err, lane, lim)) break;
      const int alpha = args.digit[a].alpha;
      const uint64_t* raw = rawbuf + r * (kRawSlotBytes / 8);
      uint8_t* at = a_tile0 + s * kATile;
#pragma unroll
      for (int it = 0; it < kUnit * 2 * KS / (32 * kPermuteWarps); ++it) {
        const int idx = lt + it * 32 * kPermuteWarps;
        const int m = idx & (kUnit - 1), r2 = idx >> 7;
        const uint64_t w0 = 2 * r2 < alpha ? raw[(2 * r2) * kUnit + m] : 0;
        const uint64_t w1 = 2 * r2 + 1 < alpha ? raw[(2 * r2 + 1) * kUnit + m] : 0;
        *reinterpret_cast<ulonglong2*>(at + (m >> 3) * kSbo + r2 * 128 + (m & 7) * 16) = make_ulonglong2(w0, w1);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(rawempty(r));
        mbar_arrive(afull(s));
      }
    }
  } else if (warp == kMmaWarp && lane == 0) {
    int cur = -1, dseq = -1, t = 0;
    bool ok = true;
    UnitIter it(u_begin, args.batch, nblk);
    for (int i = 0; i < nu && ok; ++i, it.next()) {
      const int a = it.outer;
      if (a != cur) {
        if (dseq >= 0) mma_commit(bempty(dseq & 1));  // the previous digit's byte matrix may be overwritten
        cur = a;
        ++dseq;
        if (!mbar_wait(bfull(dseq & 1), (dseq >> 1) & 1, abort, args.err, lim)) break;
      }
      const int s = i % kASlots;
      if (!mbar_wait(afull(s), (i / kASlots) & 1, abort, args.err, lim)) break;
      tc_fence_after();
      const uint32_t a_base = a_addr0 + uint32_t(s * kATile);
      const uint32_t b_base = b_addr0 + uint32_t((dseq & 1) * bbytes);
      for (int c = 0; c < args.nchunks; ++c, ++t) {
        const int slot = t % kAccSlots;
        if (t >= kAccSlots && !mbar_wait(accempty(slot), ((t / kAccSlots) & 1) ^ 1, abort, args.err, lim)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const int rows = min(kChunkRows, args.qp_limbs - c * kChunkRows);
        const uint32_t idesc = instr_desc_u8(uint32_t((rows * 8 + 15) & ~15));
#pragma unroll
        for (int ks = 0; ks < KS; ++ks)
          mma_i8(tmem + uint32_t(slot * kAccCols), smem_desc(a_base + ks * 256, 128, kSbo),
                 smem_desc(b_base + uint32_t(c * kBTile + ks * 256), 128, kSbo), idesc, ks > 0 ? 1u : 0u);
        mma_commit(accfull(slot));
      }
      if (ok) mma_commit(aempty(s));
    }
  } else if (warp < kEpilogueWarps) {
    const int quarter = warp & 3, grp = warp >> 2;
    const int m = quarter * 32 + lane;
    const uint32_t lane_addr = uint32_t(quarter * 32) << 16;
    int t = 0;
    // test only: a wait that must run out (its limit is the pipeline's)
    bool ok = !args.stall || warp_wait(never_bar, 0, abort, args.err, lane, lim);
    UnitIter it(u_begin, args.batch, nblk);
    for (int i = 0; i < nu && ok; ++i, it.next()) {
      const int a = it.outer;
      const int64_t b = it.b, blk = it.blk;
      const DigitDesc d = args.digit[a];
      const int own0 = args.skip_own ? d.prime0 - args.level : 0, own1 = args.skip_own ? own0 + d.alpha : 0;
      uint64_t* dst = args.ext + (int64_t(a) * args.batch + b) * args.qp_limbs * n + blk * kUnit + m;
      for (int c = 0; c < args.nchunks; ++c, ++t) {
        const int slot = t % kAccSlots;
        if (!warp_wait(accfull(slot), (t / kAccSlots) & 1, abort, args.err, lane, lim)) {
          ok = false;
          break;
        }
        tc_fence_after();
        uint32_t acc[32];
        tmem_ld32(tmem + lane_addr + uint32_t(slot * kAccCols + grp * 32), acc);
        tmem_wait_ld();
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(accempty(slot));
        // four independent outputs computed unconditionally (the rows past
        // the level read a valid pinfo row and are not stored), so their
        // multiply chains interleave
        const int j0 = c * kChunkRows + grp * 4;
        uint64_t res[4];
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
          const ulonglong2 pi = spinfo[min(j0 + jj, args.qp_limbs - 1)];
          res[jj] = recombine_redc(acc + 8 * jj, pi.x, pi.y);
        }
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
          const int j = j0 + jj;
          if (j < args.qp_limbs && (j < own0 || j >= own1)) dst[int64_t(j) * n] = res[jj];
        }
      }
    }
  }

  __syncthreads();
  // Drain the MMAs (and the arrivals they signal) before TMEM is freed; the
  // drain keeps the default limit whatever the pipeline's.
  if (warp == kMmaWarp && lane == 0) {
    mma_commit(drain_bar);
    mbar_wait(drain_bar, 0, nullptr, args.err, kWaitNs);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kMmaWarp) {
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, kTmemCols);
  }
}

// ---------------------------------------------------------------------------
// ModDown by P on the tensor cores (int64): for every Q row i of the level
// and coefficient k of the key-switch accumulators t (canonical coefficient
// rows [B][Q_l + P][N], component c = 0, 1),
//   v_i = (t_i - [t]_P mod q_i) P^{-1} + add_i          (mod q_i)
// where [t]_P = sum_r e_r (M_r mod q_i) is the exact extension of the P part
// from its Garner digits e_r, M_r the product of the first r special primes
// (csrc/ops/ckks/cpu/ckks_cpu.cpp:474-601 computes the same (t - [t]_P) / P
// by sequential division).  The extension is one int8 MMA per 16-row chunk of
// Q rows (A = the digits' bytes, B = the bytes of 2^{8u} 2^64 (M_r mod q_i)
// mod q_i, exactly as in k_tc_extend); the epilogue reduces it by 2^64 and
// finishes v_i, optionally rescaling by the leading prime in place
// (csrc/ops/ckks/cpu/ckks_cpu.cpp:203-262): out_{i-1} = (v_i - v_0) q_0^{-1} +
// [v_0 > q_0 / 2].  The loaders compute the Garner digits and v_0 of each
// coefficient on the CUDA cores (v_0 is needed by every row's rescale).
// Same result as k_moddown, word for word.
constexpr int kMdEpilogueWarps = 16;
constexpr int kMdLoaderWarp0 = 16;
constexpr int kMdLoaderWarps = 2;   // two coefficients per loader thread
constexpr int kMdMmaWarp = 18;
constexpr int kMdProducerWarp = 19;
constexpr int kMdThreads = 32 * 20;
constexpr int kMdV0Slots = 8;
constexpr int kMdRawSlots = 6;      // one unit's P rows and row 0 each (bulk copies in flight)
constexpr int kMdRawSlotBytes = (kMaxDigitWidth + 1) * kRowBytes;
constexpr int kMdNumBarriers = 1 + 2 * kMdRawSlots + 2 * kASlots + 2 * kAccSlots + 2 * kMdV0Slots + 2;
constexpr int kMdBarrierBytes = 384;
static_assert(8 * kMdNumBarriers + 8 <= kMdBarrierBytes, "barrier area");
static_assert(64 * kMdLoaderWarps == kUnit, "two coefficients of a unit per loader thread");

struct ModDownArgs {
  const uint64_t* t0;          // [B][qp_limbs][N] canonical
  const uint64_t* t1;
  const uint64_t* add0;        // nullable [B][q_limbs][N] canonical (read through sigma_g for a rotation)
  const uint64_t* add1;        // nullable
  uint64_t* out;               // [2][B][out_limbs][N]
  const uint8_t* bmat;         // [nchunks][128 K]: P part -> Q_l rows of this level
  const uint64_t* pinfo;       // [QP0][2]: p, -p^{-1} mod 2^64
  ChainTables<uint64_t> tabs;  // primes, P Garner / mix / inverse constants
  const TwPair<uint64_t>* rescale_inv;  // [QP0] of this level
  const uint32_t* item_galois;          // nullable: per-item Galois element of add0
  uint32_t add0_ginv;                   // else one inverse Galois element (0: none)
  int64_t batch;
  int level, num_q, num_p, q_limbs, out_limbs, nchunks, log_n, rescale;
  int* err;
  unsigned long long wait_ns;
  int stall;
};

template <int KS>
__global__ void __launch_bounds__(kMdThreads, 1) k_tc_moddown(ModDownArgs args) {
  using W = Word<uint64_t>;
  constexpr int K = 32 * KS;
  constexpr int kSbo = K / 16 * 128;
  constexpr int kATile = kUnit * K;
  constexpr int kBTile = 128 * K;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw0 = smem_addr(smem_raw);
  const uint32_t base = (raw0 + 1023u) & ~1023u;
  uint8_t* const gbase = smem_raw + (base - raw0);
  const int bbytes = args.nchunks * kBTile;
  // [B tiles | raw slots | A tiles | v0 slots | barriers]
  const uint32_t b_addr = base;
  const uint32_t rawbuf_addr = base + uint32_t(bbytes);
  const uint64_t* const rawbuf = reinterpret_cast<const uint64_t*>(gbase + bbytes);
  const uint32_t a_addr0 = rawbuf_addr + uint32_t(kMdRawSlots * kMdRawSlotBytes);
  uint8_t* const a_tile0 = gbase + bbytes + kMdRawSlots * kMdRawSlotBytes;
  uint64_t* const v0s = reinterpret_cast<uint64_t*>(a_tile0 + kASlots * kATile);
  uint64_t* const bars = v0s + kMdV0Slots * kUnit;
  const uint32_t bar0 = smem_addr(bars);
  const uint32_t bfull = bar0;
  auto rawfull = [&](int r) { return bar0 + 8u * (1 + r); };
  auto rawempty = [&](int r) { return bar0 + 8u * (1 + kMdRawSlots + r); };
  constexpr int kA0 = 1 + 2 * kMdRawSlots;
  auto afull = [&](int s) { return bar0 + 8u * (kA0 + s); };
  auto aempty = [&](int s) { return bar0 + 8u * (kA0 + kASlots + s); };
  auto accfull = [&](int s) { return bar0 + 8u * (kA0 + 2 * kASlots + s); };
  auto accempty = [&](int s) { return bar0 + 8u * (kA0 + 2 * kASlots + kAccSlots + s); };
  auto v0full = [&](int s) { return bar0 + 8u * (kA0 + 2 * kASlots + 2 * kAccSlots + s); };
  auto v0empty = [&](int s) { return bar0 + 8u * (kA0 + 2 * kASlots + 2 * kAccSlots + kMdV0Slots + s); };
  const uint32_t drain_bar = bar0 + 8u * (kMdNumBarriers - 2);
  const uint32_t never_bar = bar0 + 8u * (kMdNumBarriers - 1);  // nothing arrives on it
  uint32_t* const tmem_slot = reinterpret_cast<uint32_t*>(bars + kMdNumBarriers);
  volatile int* const abort = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t n = int64_t(1) << args.log_n;
  const int64_t nblk = n / kUnit;
  const int64_t per_comp = args.batch * nblk;
  const int64_t units = 2 * per_comp;
  const int64_t u_begin = units * blockIdx.x / gridDim.x, u_end = units * (blockIdx.x + 1) / gridDim.x;
  const int nu = int(u_end - u_begin);
  const unsigned long long lim = args.wait_ns;
  const int qp_limbs = args.q_limbs + args.num_p;
  // where the addend of component c, ciphertext b, coefficient k is read:
  // add0 through sigma_g for a rotation (source index and sign), add1 as is
  auto addend_source = [&](int c, int64_t b, int k, int& kk, bool& neg) {
    kk = k;
    neg = false;
    if (c == 0) {
      const uint32_t gi = args.item_galois
                              ? (args.item_galois[b] == 1 ? 0u : galois_inverse_dev(args.item_galois[b], args.log_n))
                              : args.add0_ginv;
      if (gi) kk = galois_source(k, args.log_n, gi, neg);
    }
  };
  auto addend = [&](int c, int64_t b, int i, int kk, bool neg, uint64_t q) -> uint64_t {
    const uint64_t* ad = c == 0 ? args.add0 : args.add1;
    if (!ad) return 0;
    uint64_t x = csub(ad[(b * args.q_limbs + i) * n + kk], q);
    return (neg && x) ? q - x : x;
  };

  if (tid == 0) {
    mbar_init(bfull, 1);
    for (int r = 0; r < kMdRawSlots; ++r) {
      mbar_init(rawfull(r), 1);
      mbar_init(rawempty(r), kMdLoaderWarps);
    }
    for (int s = 0; s < kASlots; ++s) {
      mbar_init(afull(s), kMdLoaderWarps);
      mbar_init(aempty(s), 1);
    }
    for (int s = 0; s < kAccSlots; ++s) {
      mbar_init(accfull(s), 1);
      mbar_init(accempty(s), kMdEpilogueWarps);
    }
    for (int s = 0; s < kMdV0Slots; ++s) {
      mbar_init(v0full(s), kMdLoaderWarps);
      mbar_init(v0empty(s), kMdEpilogueWarps);
    }
    mbar_init(drain_bar, 1);
    mbar_init(never_bar, 1);
    *abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == kMdMmaWarp) tmem_alloc(smem_addr(tmem_slot), kTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == kMdProducerWarp && lane == 0) {
    // the level's byte matrices once, then per unit the P rows (and row 0,
    // for the rescale) of its 128 coefficients into a raw slot
    mbar_expect_tx(bfull, uint32_t(bbytes));
    for (int o = 0; o < bbytes; o += 16384)
      bulk_load(b_addr + uint32_t(o), args.bmat + o, uint32_t(min(16384, bbytes - o)), bfull);
    const int rows = args.num_p + (args.rescale ? 1 : 0);
    int i = 0;
    UnitIter it(u_begin, args.batch, nblk);
    for (; i < nu; ++i, it.next()) {
      const int c = it.outer;
      const int64_t b = it.b, blk = it.blk;
      const int r = i % kMdRawSlots;
      if (i >= kMdRawSlots && !mbar_wait(rawempty(r), ((i / kMdRawSlots) & 1) ^ 1, abort, args.err, lim)) break;
      const uint64_t* t = (c == 0 ? args.t0 : args.t1) + b * qp_limbs * n + blk * kUnit;
      mbar_expect_tx(rawfull(r), uint32_t(rows * kRowBytes));
      for (int rr = 0; rr < args.num_p; ++rr)
        bulk_load(rawbuf_addr + uint32_t(r * kMdRawSlotBytes + rr * kRowBytes), t + int64_t(args.q_limbs + rr) * n,
                  kRowBytes, rawfull(r));
      if (args.rescale)
        bulk_load(rawbuf_addr + uint32_t(r * kMdRawSlotBytes + args.num_p * kRowBytes), t, kRowBytes, rawfull(r));
    }
    // after an abort, wait (bounded, default limit) for the copies still in flight
    if (*abort) {
      mbar_wait(bfull, 0, nullptr, args.err, kWaitNs);
      for (int u = i - kMdRawSlots < 0 ? 0 : i - kMdRawSlots; u < i; ++u)
        mbar_wait(rawfull(u % kMdRawSlots), (u / kMdRawSlots) & 1, nullptr, args.err, kWaitNs);
    }
  } else if (warp >= kMdLoaderWarp0 && warp < kMdLoaderWarp0 + kMdLoaderWarps) {
    // Garner digits e_r of the P part of one coefficient -> the A tile (word
    // (m, r) at (m / 8) sbo + (r / 2) 128 + (m % 8) 16 + (r % 2) 8; rows r >= P
    // zero); with rescale also v_0 of the coefficient -> its v0 slot
    const int lt = tid - kMdLoaderWarp0 * 32;
    const PrimeInfo<uint64_t> p0 = args.tabs.prime[args.level];
    UnitIter it(u_begin, args.batch, nblk);
    for (int i = 0; i < nu; ++i, it.next()) {
      const int c = it.outer;
      const int64_t b = it.b, blk = it.blk;
      const int r = i % kMdRawSlots, s = i % kASlots, vs = i % kMdV0Slots;
      if (!warp_wait(rawfull(r), (i / kMdRawSlots) & 1, abort, args.err, lane, lim)) break;
      if (i >= kASlots && !warp_wait(aempty(s), ((i / kASlots) & 1) ^ 1, abort, args.err, lane, lim)) break;
      if (args.rescale && i >= kMdV0Slots &&
          !warp_wait(v0empty(vs), ((i / kMdV0Slots) & 1) ^ 1, abort, args.err, lane, lim))
        break;
      const uint64_t* raw = rawbuf + r * (kMdRawSlotBytes / 8);
      uint64_t e2[2][kMaxDigitWidth], t0v[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int m = lt + 64 * h;
#pragma unroll
        for (int rr = 0; rr < kMaxDigitWidth; ++rr) e2[h][rr] = rr < args.num_p ? raw[rr * kUnit + m] : 0;
        t0v[h] = args.rescale ? raw[args.num_p * kUnit + m] : 0;
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(rawempty(r));
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int m = lt + 64 * h;
        const int k = int(blk * kUnit) + m;
        uint64_t* e = e2[h];
        for (int rr = 0; rr < args.num_p; ++rr) {
          const PrimeInfo<uint64_t> p = args.tabs.prime[args.num_q + rr];
          uint64_t x = csub(e[rr], p.q);
          if (rr > 0) {
            uint64_t acc = 0;
            for (int j = 0; j < rr; ++j) {
              const TwPair<uint64_t> g = args.tabs.p_garner[rr * kMaxDigitWidth + j];
              acc = csub(acc + csub(W::shoup(e[j], g.w, g.wp, p.q), p.q), p.q);
            }
            const TwPair<uint64_t> inv = args.tabs.p_garner[rr * kMaxDigitWidth + rr];
            x = csub(W::shoup(csub(x + p.q - acc, p.q), inv.w, inv.wp, p.q), p.q);
          }
          e[rr] = x;
        }
        uint8_t* at = a_tile0 + s * kATile + (m >> 3) * kSbo + (m & 7) * 16;
#pragma unroll
        for (int r2 = 0; r2 < 2 * KS; ++r2)
          *reinterpret_cast<ulonglong2*>(at + r2 * 128) = make_ulonglong2(
              2 * r2 < kMaxDigitWidth ? e[2 * r2] : 0, 2 * r2 + 1 < kMaxDigitWidth ? e[2 * r2 + 1] : 0);
        if (args.rescale) {
          uint64_t sub = 0;
          for (int rr = 0; rr < args.num_p; ++rr) {
            const TwPair<uint64_t> mx = args.tabs.p_mix[int64_t(rr) * (args.num_q + args.num_p) + args.level];
            sub = csub(sub + csub(W::shoup(e[rr], mx.w, mx.wp, p0.q), p0.q), p0.q);
          }
          const TwPair<uint64_t> pinv = args.tabs.p_inv[args.level];
          uint64_t v = csub(csub(t0v[h], p0.q) + p0.q - sub, p0.q);
          v = csub(W::shoup(v, pinv.w, pinv.wp, p0.q), p0.q);
          int kk;
          bool neg;
          addend_source(c, b, k, kk, neg);
          v0s[vs * kUnit + m] = csub(v + addend(c, b, 0, kk, neg, p0.q), p0.q);
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(afull(s));
        if (args.rescale) mbar_arrive(v0full(vs));
      }
    }
  } else if (warp == kMdMmaWarp && lane == 0) {
    bool ok = mbar_wait(bfull, 0, abort, args.err, lim);
    int t = 0;
    for (int i = 0; i < nu && ok; ++i) {
      const int s = i % kASlots;
      if (!mbar_wait(afull(s), (i / kASlots) & 1, abort, args.err, lim)) break;
      tc_fence_after();
      const uint32_t a_base = a_addr0 + uint32_t(s * kATile);
      for (int ch = 0; ch < args.nchunks; ++ch, ++t) {
        const int slot = t % kAccSlots;
        if (t >= kAccSlots && !mbar_wait(accempty(slot), ((t / kAccSlots) & 1) ^ 1, abort, args.err, lim)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const int rows = min(kChunkRows, args.q_limbs - ch * kChunkRows);
        const uint32_t idesc = instr_desc_u8(uint32_t((rows * 8 + 15) & ~15));
#pragma unroll
        for (int ks = 0; ks < KS; ++ks)
          mma_i8(tmem + uint32_t(slot * kAccCols), smem_desc(a_base + ks * 256, 128, kSbo),
                 smem_desc(b_addr + uint32_t(ch * kBTile + ks * 256), 128, kSbo), idesc, ks > 0 ? 1u : 0u);
        mma_commit(accfull(slot));
      }
      if (ok) mma_commit(aempty(s));
    }
  } else if (warp < kMdEpilogueWarps) {
    const int quarter = warp & 3, grp = warp >> 2;
    const int m = quarter * 32 + lane;
    const uint32_t lane_addr = uint32_t(quarter * 32) << 16;
    const uint64_t half0 = args.tabs.prime[args.level].q >> 1;
    int t = 0;
    // test only: a wait that must run out (its limit is the pipeline's)
    bool ok = !args.stall || warp_wait(never_bar, 0, abort, args.err, lane, lim);
    UnitIter it(u_begin, args.batch, nblk);
    for (int i = 0; i < nu && ok; ++i, it.next()) {
      const int c = it.outer;
      const int64_t b = it.b, blk = it.blk;
      const int k = int(blk * kUnit) + m;
      int kk;
      bool neg;
      addend_source(c, b, k, kk, neg);
      const uint64_t* tt = (c == 0 ? args.t0 : args.t1) + b * qp_limbs * n + k;
      uint64_t* o = args.out + (int64_t(c) * args.batch + b) * args.out_limbs * n + k;
      const int vs = i % kMdV0Slots;
      uint64_t v0 = 0;
      if (args.rescale) {
        if (!warp_wait(v0full(vs), (i / kMdV0Slots) & 1, abort, args.err, lane, lim)) break;
        v0 = v0s[vs * kUnit + m];
      }
      for (int ch = 0; ch < args.nchunks; ++ch, ++t) {
        const int slot = t % kAccSlots;
        // this item's accumulator rows and addends are requested before the
        // wait, so their latency overlaps it
        uint64_t tv[4], av[4];
        bool valid[4];
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
          const int row = ch * kChunkRows + grp * 4 + jj;
          valid[jj] = row < args.q_limbs && !(args.rescale && row == 0);
          tv[jj] = valid[jj] ? tt[int64_t(row) * n] : 0;
          av[jj] = valid[jj] ? addend(c, b, row, kk, neg, args.tabs.prime[args.level + row].q) : 0;
        }
        if (!warp_wait(accfull(slot), (t / kAccSlots) & 1, abort, args.err, lane, lim)) {
          ok = false;
          break;
        }
        tc_fence_after();
        uint32_t acc[32];
        tmem_ld32(tmem + lane_addr + uint32_t(slot * kAccCols + grp * 32), acc);
        tmem_wait_ld();
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(accempty(slot));
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
          // computed for every row (past the level on the last prime's
          // constants) and stored only where valid, so the four chains interleave
          const int row = min(ch * kChunkRows + grp * 4 + jj, args.q_limbs - 1);
          const int pid = args.level + row;
          const ulonglong2 pi = __ldg(reinterpret_cast<const ulonglong2*>(args.pinfo) + pid);
          const uint64_t q = pi.x;
          const uint64_t sub = csub(recombine_redc(acc + 8 * jj, q, pi.y), q);
          const TwPair<uint64_t> pinv = args.tabs.p_inv[pid];
          uint64_t v = csub(csub(tv[jj], q) + q - sub, q);
          v = csub(W::shoup(v, pinv.w, pinv.wp, q), q);
          v = csub(v + av[jj], q);
          if (!args.rescale) {
            if (valid[jj]) o[int64_t(row) * n] = v;
          } else {
            const PrimeInfo<uint64_t> p = args.tabs.prime[pid];
            const uint64_t x0 = reduce_any(v0, p);
            const TwPair<uint64_t> inv = args.rescale_inv[pid];
            uint64_t r = csub(W::shoup(csub(v + q - x0, q), inv.w, inv.wp, q), q);
            r += v0 > half0 ? 1u : 0u;
            if (valid[jj]) o[int64_t(row - 1) * n] = csub(r, q);
          }
        }
      }
      if (args.rescale && ok) {
        __syncwarp();
        if (lane == 0) mbar_arrive(v0empty(vs));
      }
    }
  }

  __syncthreads();
  if (warp == kMdMmaWarp && lane == 0) {
    mma_commit(drain_bar);
    mbar_wait(drain_bar, 0, nullptr, args.err, kWaitNs);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kMdMmaWarp) {
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, kTmemCols);
  }
}

}  // namespace tcb

// ------------------------------------------------------------------ host ---
namespace {
using u128 = unsigned __int128;

// K-steps of 32 bytes for digits of up to `alpha` primes.
int ksteps_for(int alpha) { return alpha <= 4 ? 1 : 2; }

int chunks_for(int qp_limbs) { return (qp_limbs + tcb::kChunkRows - 1) / tcb::kChunkRows; }

int smem_for(int nchunks, int ks) {
  const int k = 32 * ks;
  const int raw = (ks == 1 ? tcb::raw_slots<1>() : tcb::raw_slots<2>()) * 4 * ks * tcb::kRowBytes;
  const int need = 1024 + 2 * nchunks * 128 * k + raw + tcb::kASlots * tcb::kUnit * k + tcb::kPinfoBytes +
                   tcb::kBarrierBytes;
  return need > tcb::kMinSmem ? need : tcb::kMinSmem;
}
}  // namespace

// Byte matrices of one level (host): for each active digit, chunk c and
// destination row j = 16 c + jl, MMA row n = 8 jl + e, K position
// kap = 8 r + u holds byte e of 2^{8u} 2^64 (M_r mod p_{level+j}) mod p.
// Layout per chunk: K-major canonical tile of 128 rows x K bytes.
void tc_basis_tables_host(const Context& c, int level, int ks, std::vector<uint8_t>& out) {
  const int k = 32 * ks, sbo = k / 16 * 128, tile = 128 * k;
  const int qpl = c.qp() - level, nch = chunks_for(qpl);
  const std::vector<DigitDesc>& dd = c.level_digits[level];
  out.assign(dd.size() * size_t(nch) * tile, 0);
  for (size_t a = 0; a < dd.size(); ++a) {
    for (int j = 0; j < qpl; ++j) {
      const uint64_t p = c.moduli[level + j];
      uint8_t* t = out.data() + (a * nch + j / tcb::kChunkRows) * size_t(tile);
      const int jl = j % tcb::kChunkRows;
      uint64_t mr = 1 % p;  // M_r mod p, r = 0, 1, ...
      for (int r = 0; r < dd[a].alpha; ++r) {
        if (r > 0) mr = uint64_t((u128)mr * (c.moduli[dd[a].prime0 + r - 1] % p) % p);
        for (int u = 0; u < 8; ++u) {
          const uint64_t scaled = uint64_t((u128(uint64_t((u128(mr) << (8 * u)) % p)) << 64) % p);
          const int kap = 8 * r + u;
          for (int e = 0; e < 8; ++e) t[jl * sbo + (kap >> 4) * 128 + e * 16 + (kap & 15)] = uint8_t(scaled >> (8 * e));
        }
      }
    }
  }
}

// ModDown byte matrices of one level (host): chunk c, Q row i = 16 c + il,
// MMA row n = 8 il + e, K position kap = 8 r + u holds byte e of
// 2^{8u} 2^64 (M_r mod q_{level+i}) mod q, M_r the product of the first r
// special primes.
void tc_moddown_tables_host(const Context& c, int level, int ks, std::vector<uint8_t>& out) {
  const int k = 32 * ks, sbo = k / 16 * 128, tile = 128 * k;
  const int ql = c.num_q - level;
  out.assign(size_t(chunks_for(ql)) * tile, 0);
  for (int i = 0; i < ql; ++i) {
    const uint64_t q = c.moduli[level + i];
    uint8_t* t = out.data() + size_t(i / tcb::kChunkRows) * tile;
    const int il = i % tcb::kChunkRows;
    uint64_t mr = 1 % q;
    for (int r = 0; r < c.num_p; ++r) {
      if (r > 0) mr = uint64_t((u128)mr * (c.moduli[c.num_q + r - 1] % q) % q);
      for (int u = 0; u < 8; ++u) {
        const uint64_t scaled = uint64_t((u128(uint64_t((u128(mr) << (8 * u)) % q)) << 64) % q);
        const int kap = 8 * r + u;
        for (int e = 0; e < 8; ++e) t[il * sbo + (kap >> 4) * 128 + e * 16 + (kap & 15)] = uint8_t(scaled >> (8 * e));
      }
    }
  }
}

int tc_basis_prepare(Context& c) {
  std::lock_guard<std::mutex> lock(c.tcb_mutex);
  if (c.tcb) return 0;
  if (c.bits != 64) return fail(-7, "the tensor-core basis conversion needs an int64 context");
  if (c.log_n < 7) return fail(-7, "ring too small for the tensor-core basis conversion");
  const int ks = ksteps_for(c.num_p);
  if (c.qp() > tcb::kPinfoBytes / 16) return fail(-7, "the chain is too long for the tensor-core basis conversion");
  if (smem_for(chunks_for(c.qp()), ks) > 227 * 1024 ||
      1024 + chunks_for(c.num_q) * 128 * 32 * ks + tcb::kMdRawSlots * tcb::kMdRawSlotBytes +
              tcb::kASlots * tcb::kUnit * 32 * ks + tcb::kMdV0Slots * tcb::kUnit * 8 + tcb::kMdBarrierBytes >
          227 * 1024)
    return fail(-7, "the chain is too long for the tensor-core basis conversion's shared-memory tables");
  auto* t = new TcBasisTables();
  t->ks = ks;
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
  std::vector<uint8_t> host;
  t->bmat.assign(c.num_q, nullptr);
  t->md_bmat.assign(c.num_q, nullptr);
  for (int level = 0; level < c.num_q; ++level) {
    tc_basis_tables_host(c, level, ks, host);
    t->bmat[level] = static_cast<uint8_t*>(dev_alloc(host.size()));
    if (!t->bmat[level] || cudaMemcpy(t->bmat[level], host.data(), host.size(), cudaMemcpyHostToDevice) != cudaSuccess)
      return give_up("tensor-core basis conversion byte matrices");
    tc_moddown_tables_host(c, level, ks, host);
    t->md_bmat[level] = static_cast<uint8_t*>(dev_alloc(host.size()));
    if (!t->md_bmat[level] ||
        cudaMemcpy(t->md_bmat[level], host.data(), host.size(), cudaMemcpyHostToDevice) != cudaSuccess)
      return give_up("tensor-core ModDown byte matrices");
  }
  std::vector<uint64_t> pinfo(2 * size_t(c.qp()));
  for (int j = 0; j < c.qp(); ++j) {
    const uint64_t p = c.moduli[j];
    uint64_t x = 1;  // p^{-1} mod 2^64 by Newton iteration
    for (int i = 0; i < 6; ++i) x *= 2 - p * x;
    pinfo[2 * j] = p;
    pinfo[2 * j + 1] = 0 - x;
  }
  t->pinfo = static_cast<uint64_t*>(dev_alloc(pinfo.size() * 8));
  t->err = static_cast<int*>(dev_alloc(sizeof(int)));
  if (!t->pinfo || !t->err ||
      cudaMemcpy(t->pinfo, pinfo.data(), pinfo.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(t->err, 0, sizeof(int)) != cudaSuccess)
    return give_up("tensor-core basis conversion constants");
  if (cudaDeviceGetAttribute(&t->sms, cudaDevAttrMultiProcessorCount, c.device) != cudaSuccess || t->sms < 1)
    return give_up("multiprocessor count");
  for (void* p : mine) c.allocations.push_back(p);
  c.tcb = t;
  return 0;
}

int64_t tc_ext_words(const Context& c, int64_t batch, int level) {
  return int64_t(c.level_digits[level].size()) * batch * (c.qp() - level) * c.n();
}

int tc_extend(Context& c, const void* digits, void* ext, int64_t batch, int level, bool skip_own, cudaStream_t st) {
  if (int rc = tc_basis_prepare(c)) return rc;
  const TcBasisTables& t = *c.tcb;
  const int nd = int(c.level_digits[level].size());
  if (batch == 0 || nd == 0) return 0;
  const int qpl = c.qp() - level, nch = chunks_for(qpl);
  const int smem = smem_for(nch, t.ks);
  auto kern = t.ks == 1 ? tcb::k_tc_extend<1> : tcb::k_tc_extend<2>;
  if (int rc = ensure_dynamic_smem(reinterpret_cast<const void*>(kern), smem)) return rc;
  const int64_t units = int64_t(nd) * batch * (c.n() / tcb::kUnit);
  const int grid = int(units < t.sms ? units : t.sms);
  tcb::ExtendArgs a{static_cast<const uint64_t*>(digits), static_cast<uint64_t*>(ext), t.bmat[level], t.pinfo,
                    c.lv64[level].digits, batch, level, c.num_q - level, qpl, nd, nch, c.log_n,
                    skip_own ? 1 : 0, t.err, c.tc_wait_ns ? c.tc_wait_ns : tc::kWaitNs, c.tc_test_stall};
  kern<<<grid, tcb::kThreads, smem, st>>>(a);
  return cuda_status(cudaGetLastError(), "k_tc_extend");
}

int tc_moddown(Context& c, const void* t0, const void* t1, const void* add0, const void* add1, void* out,
               int64_t batch, int level, uint32_t add0_ginv, const uint32_t* item_galois, int rescale,
               cudaStream_t st) {
  if (int rc = tc_basis_prepare(c)) return rc;
  const TcBasisTables& t = *c.tcb;
  if (batch == 0) return 0;
  const int ql = c.num_q - level, nch = chunks_for(ql);
  const int k = 32 * t.ks;
  int smem = 1024 + nch * 128 * k + tcb::kMdRawSlots * tcb::kMdRawSlotBytes + tcb::kASlots * tcb::kUnit * k +
             tcb::kMdV0Slots * tcb::kUnit * 8 +
             tcb::kMdBarrierBytes;
  if (smem < tcb::kMinSmem) smem = tcb::kMinSmem;
  auto kern = t.ks == 1 ? tcb::k_tc_moddown<1> : tcb::k_tc_moddown<2>;
  if (int rc = ensure_dynamic_smem(reinterpret_cast<const void*>(kern), smem)) return rc;
  const int64_t units = 2 * batch * (c.n() / tcb::kUnit);
  const int grid = int(units < t.sms ? units : t.sms);
  tcb::ModDownArgs a{static_cast<const uint64_t*>(t0), static_cast<const uint64_t*>(t1),
                     static_cast<const uint64_t*>(add0), static_cast<const uint64_t*>(add1),
                     static_cast<uint64_t*>(out), t.md_bmat[level], t.pinfo, c.t64, c.lv64[level].rescale_inv,
                     item_galois, add0_ginv, batch, level, c.num_q, c.num_p, ql, ql - (rescale ? 1 : 0), nch,
                     c.log_n, rescale, t.err, c.tc_wait_ns ? c.tc_wait_ns : tc::kWaitNs, c.tc_test_stall};
  kern<<<grid, tcb::kMdThreads, smem, st>>>(a);
  return cuda_status(cudaGetLastError(), "k_tc_moddown");
}

int tc_basis_status(Context& c, int* flag) {
  std::lock_guard<std::mutex> lock(c.tcb_mutex);
  *flag = 0;
  if (!c.tcb) return 0;
  if (cudaError_t e = cudaMemcpy(flag, c.tcb->err, sizeof(int), cudaMemcpyDeviceToHost)) return cuda_status(e, "flag");
  return cuda_status(cudaMemset(c.tcb->err, 0, sizeof(int)), "flag reset");
}

}  // namespace fhb
