// Exact integer tensor-core NTT for int32 residues (q < 2^28) at N = 2^16 on
// the 5th-generation tensor cores: tcgen05.mma kind::i8 with int32
// accumulators in tensor memory (TMEM), operands staged in shared memory.
//
// Four-step form with N = 256 x 256.  Write the polynomial as the row-major
// matrix X[i1][i2] = x[256 i1 + i2] and the output (bit-reversed order, as
// the CUDA-core form and the reference: out[k] = sum_n x[n] psi^{(2 br16(k)
// + 1) n}, csrc/ops/ntt/forward_ntt.cpp:15-21) as O[r][c] = out[256 r + c].
// With br16(256 r + c) = br8(r) + 256 br8(c) and psi^{2N} = 1,
//
//   Y[r][i2] = T1[r][i2] sum_i1 W1[r][i1] X[i1][i2]     (forward pass 1)
//   O[r][c]  = sum_i2 Y[r][i2] W2[i2][c]                (forward pass 2)
//
//   W1[r][i1] = psi^{256 i1 (2 br8(r) + 1)},  T1[r][i2] = R psi^{i2 (2 br8(r) + 1)},
//   W2[i2][c] = psi^{512 i2 br8(c)}           (R = 2^30: Montgomery output).
//
// The inverse runs the two passes backwards with psi^{-1}; its first pass
// carries N^{-1} R^{-1} (Montgomery input, standard output):
//
//   E[r][i2]  = T1'[r][i2] sum_c O[r][c] W2'[c][i2],    W2'[c][i2] = psi^{-512 br8(c) i2}
//   x[i1][i2] = sum_r W1'[i1][r] E[r][i2],              W1'[i1][r] = psi^{-256 i1 (2 br8(r) + 1)}
//   T1'[r][i2] = N^{-1} R^{-1} psi^{-i2 (2 br8(r) + 1)}.
//
// Every pass is one GEMM D[m][n] = sum_k A[m][k] B[k][n] mod q with the data
// as A (rows m) and the constant matrix as B; a pass whose data index k runs
// along memory rows reads A transposed ("column" passes: forward 1, inverse
// 2), the others read it row-wise; D is stored in the orientation the next
// pass reads.  The product is exact with unsigned 8-bit digits: the data
// splits into its four bytes A = sum_d 2^{8d} A_d, the constant side is
// pre-scaled per data digit, B^(d) = 2^{8d} 2^{32} B mod q, and split into
// bytes B^(d) = sum_e 2^{8e} B^(d)_e.  Tensor-core accumulator e collects
// sum_d A_d B^(d)_e (4 x 256 products of bytes: < 2^26, exact in int32), the
// epilogue forms S = sum_e 2^{8e} acc_e < 2^51 and one Montgomery reduction
// by 2^32 returns S 2^{-32} = (A B mod q) in [0, 2q); the optional
// elementwise twiddle is a Shoup product and the result is made canonical.
//
// CTA = 128 rows (m) of one polynomial x all 256 output columns, in four
// tiles of 64 columns.  One MMA is M = 128, N = 256 (the 4 twiddle bytes e
// x 64 columns), K = 32 bytes; a tile is 32 MMAs (8 K-chunks x 4 data
// digits).  The A tile (128 rows x 256 x 4 digit planes = 128 KB) is written
// once into shared memory by all threads; the B chunks (8 KB each, laid out
// on the host in the tensor cores' canonical K-major layout) stream through
// a 12-stage ring by bulk copies; two TMEM accumulator sets of 256 columns
// let the epilogue of tile j overlap the MMAs of tile j + 1.
//
// Roles (256 threads): warps 0-3 epilogue (TMEM lanes 32 w .. 32 w + 31),
// warp 4 lane 0 bulk-copy producer, warp 5 TMEM owner and lane 0 MMA issuer.
// Every mbarrier wait is bounded (about one second of the global timer); a
// wait that gives up sets a CTA abort flag that releases every other wait,
// raises the device error flag, and the CTA drains its own bulk copies and
// MMAs (again with bounded waits) before it frees TMEM and exits.
#include <cstring>
#include <vector>

#include "fhb_context.h"

namespace fhb {
namespace tcntt {

constexpr int kLogN = 16;
constexpr int kSide = 256;
constexpr int kRowsPerCta = 128;
constexpr int kTiles = 4;                // 64-column output tiles per CTA
constexpr int kTileCols = 64;
constexpr int kChunksPerTile = 32;       // 8 K-chunks x 4 data digits
constexpr int kChunkBytes = 8192;        // B chunk: 256 (e, column) rows x 32 bytes of K
constexpr int kStages = 12;
constexpr int kPlaneBytes = kRowsPerCta * kSide;  // one data digit plane of the A tile
constexpr int kABytes = 4 * kPlaneBytes;
constexpr int kBBytes = kStages * kChunkBytes;
constexpr int kBarrierBytes = 512;  // 2 x 12 + 5 mbarriers, TMEM slot, abort flag
constexpr int kSmemBytes = 1024 + kABytes + kBBytes + kBarrierBytes;
static_assert(8 * (2 * kStages + 5) + 8 <= kBarrierBytes, "barrier area too small");
static_assert(kSmemBytes <= 232448, "shared memory per CTA");
constexpr int kThreads = 256;
constexpr int kTmemCols = 512;
constexpr size_t kPassBytesPerPrime = size_t(kTiles) * kChunksPerTile * kChunkBytes;  // 1 MiB
constexpr unsigned long long kWaitNs = 1000000000ull;

// tcgen05 instruction descriptor: D int32 (c_format 2 at bit 4), A and B
// unsigned 8-bit (formats 0), both K-major, N = 256 (N >> 3 at bit 17),
// M = 128 (M >> 4 at bit 24).
constexpr uint32_t kInstrDesc = (2u << 4) | ((256u >> 3) << 17) | ((128u >> 4) << 24);

// ---------------------------------------------------------------- device ---
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the phase of `parity` to complete.  Returns false when
// the CTA aborted (abort != nullptr) or about one second passed; the latter
// raises the abort flag and the device error flag.  The global timer is read
// only every 1024 polls: the common case is a barrier that completes within
// a few polls.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort, int* err) {
  if (mbar_test(bar, parity)) return true;
  unsigned long long t0 = 0;
  for (uint32_t it = 1;; ++it) {
    if (mbar_test(bar, parity)) return true;
    if (abort && *abort) return false;
    if ((it & 1023) == 0) {
      const unsigned long long t = global_ns();
      if (t0 == 0) {
        t0 = t;
      } else if (t - t0 > kWaitNs) {
        if (abort) *abort = 1;
        atomicExch(err, 1);
        return false;
      }
    }
  }
}

__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

// Shared-memory matrix descriptor, no swizzle, K-major canonical layout:
// core matrices of 8 rows x 16 bytes (128 contiguous bytes); `lbo` = byte
// distance between the two K-adjacent core matrices of an MMA, `sbo` = byte
// distance between 8-row groups.  Version 1 (bit 46) for sm_100.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return uint64_t((addr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
         (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);
}

__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t accumulate) {
  const uint32_t mask = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}"
      ::"r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(kInstrDesc), "r"(accumulate), "r"(mask));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

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

// Offset of byte (row, k) of one digit plane of the A tile (rows 0..127,
// k 0..255): core matrix (row / 8, k / 16) at (row / 8) * 2048 + (k / 16) * 128.
__device__ __forceinline__ uint32_t a_offset(int row, int k) {
  return uint32_t((row & 7) * 16 + (row >> 3) * 2048 + (k >> 4) * 128 + (k & 15));
}

struct PassArgs {
  const uint32_t* in;
  uint32_t* out;
  const uint8_t* bmat;                // [QP][4][32][8192]
  const TwPair<uint32_t>* post;       // [QP][N] or null
  const uint32_t* qinfo;              // [QP][2]
  int64_t batch;                      // polynomials per row (polys = batch x rows)
  int rows;
  int row_start;
  int* err;
};

// COLUMN: A[m][k] = in[k * 256 + m] and D[m][n] -> out[n * 256 + m];
// otherwise A[m][k] = in[m * 256 + k] and D[m][n] -> out[m * 256 + n].
// in == out is allowed (plain loads: a CTA reads its slab before it writes it).
template <bool COLUMN, bool POST>
__global__ void __launch_bounds__(kThreads, 1) k_tc_ntt_pass(PassArgs args) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_addr(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t* const gbase = smem_raw + (base - raw);
  uint8_t* const a_tile = gbase;
  const uint32_t a_addr = base;
  const uint32_t b_addr = base + kABytes;
  uint64_t* const bars = reinterpret_cast<uint64_t*>(gbase + kABytes + kBBytes);
  // barrier slots: full[kStages] empty[kStages] acc_full[2] acc_empty[2] drain[1]
  const uint32_t bar0 = smem_addr(bars);
  auto full_bar = [&](int s) { return bar0 + 8u * s; };
  auto empty_bar = [&](int s) { return bar0 + 8u * (kStages + s); };
  auto accf_bar = [&](int b) { return bar0 + 8u * (2 * kStages + b); };
  auto acce_bar = [&](int b) { return bar0 + 8u * (2 * kStages + 2 + b); };
  const uint32_t drain_bar = bar0 + 8u * (2 * kStages + 4);
  uint32_t* const tmem_slot = reinterpret_cast<uint32_t*>(gbase + kABytes + kBBytes + 8 * (2 * kStages + 5));
  volatile int* const abort = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // prime-major order: consecutive CTAs share a prime, so its constant
  // matrices stay in L2 while they are streamed
  const int64_t pair = blockIdx.x >> 1;
  const int row = int(pair / args.batch);
  const int64_t poly = (pair - int64_t(row) * args.batch) * args.rows + row;
  const int m0 = (blockIdx.x & 1) * kRowsPerCta;
  const int prime = args.row_start + row;
  const uint32_t* src = args.in + poly * (int64_t(1) << kLogN);
  uint32_t* dst = args.out + poly * (int64_t(1) << kLogN);
  const uint8_t* bsrc = args.bmat + size_t(prime) * kPassBytesPerPrime;

  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(full_bar(s), 1);
      mbar_init(empty_bar(s), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(accf_bar(b), 1);
      mbar_init(acce_bar(b), 4);
    }
    mbar_init(drain_bar, 1);
    *abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 5) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  // The producer starts the B ring before the A tile is staged.
  int issued = 0;
  const bool producer = warp == 4 && lane == 0;
  if (producer) {
    for (; issued < kStages; ++issued) {
      mbar_expect_tx(full_bar(issued), kChunkBytes);
      bulk_load(b_addr + issued * kChunkBytes, bsrc + size_t(issued) * kChunkBytes, kChunkBytes, full_bar(issued));
    }
  }

  // Stage the A tile: four byte planes of rows m0 .. m0 + 127.
  if (COLUMN) {
    // unit = (row, 16 consecutive k); a warp covers 32 consecutive rows so
    // every load is one 128-byte line and every 16-byte store is conflict-free.
    // Two units per step keep 32 loads per thread in flight.
    for (int u0 = tid; u0 < kRowsPerCta * 16; u0 += 2 * kThreads) {
      uint32_t v[2][16];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int u = u0 + h * kThreads, r = u & (kRowsPerCta - 1), k16 = u >> 7;
#pragma unroll
        for (int t = 0; t < 16; ++t) v[h][t] = src[(k16 * 16 + t) * kSide + m0 + r];
      }
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int u = u0 + h * kThreads, r = u & (kRowsPerCta - 1), k16 = u >> 7;
        uint32_t w[4][4];
#pragma unroll
        for (int g = 0; g < 4; ++g)
          byte_transpose(v[h][4 * g], v[h][4 * g + 1], v[h][4 * g + 2], v[h][4 * g + 3], w[0][g], w[1][g], w[2][g],
                         w[3][g]);
        const uint32_t off = a_offset(r, k16 * 16);
#pragma unroll
        for (int d = 0; d < 4; ++d)
          *reinterpret_cast<uint4*>(a_tile + d * kPlaneBytes + off) = make_uint4(w[d][0], w[d][1], w[d][2], w[d][3]);
      }
    }
  } else {
    // unit = (row, 4 consecutive k); lane = 8 rows x 4 k-quads, so the
    // 32 four-byte stores of a warp fall in 32 distinct banks.  Eight units
    // per step keep eight 16-byte loads per thread in flight.
    const int r8 = lane >> 2, q4 = lane & 3;
    for (int wu0 = warp; wu0 < 16 * 16; wu0 += 8 * (kThreads / 32)) {
      uint4 v[8];
#pragma unroll
      for (int h = 0; h < 8; ++h) {
        const int wu = wu0 + h * (kThreads / 32);
        const int r = (wu >> 4) * 8 + r8, k = ((wu & 15) * 4 + q4) * 4;
        v[h] = *reinterpret_cast<const uint4*>(src + (m0 + r) * kSide + k);
      }
#pragma unroll
      for (int h = 0; h < 8; ++h) {
        const int wu = wu0 + h * (kThreads / 32);
        const int r = (wu >> 4) * 8 + r8, k = ((wu & 15) * 4 + q4) * 4;
        uint32_t w0, w1, w2, w3;
        byte_transpose(v[h].x, v[h].y, v[h].z, v[h].w, w0, w1, w2, w3);
        const uint32_t off = a_offset(r, k);
        *reinterpret_cast<uint32_t*>(a_tile + 0 * kPlaneBytes + off) = w0;
        *reinterpret_cast<uint32_t*>(a_tile + 1 * kPlaneBytes + off) = w1;
        *reinterpret_cast<uint32_t*>(a_tile + 2 * kPlaneBytes + off) = w2;
        *reinterpret_cast<uint32_t*>(a_tile + 3 * kPlaneBytes + off) = w3;
      }
    }
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncthreads();

  constexpr int kTotalChunks = kTiles * kChunksPerTile;
  if (producer) {
    for (; issued < kTotalChunks; ++issued) {
      const int s = issued % kStages;
      if (!mbar_wait(empty_bar(s), ((issued / kStages) & 1) ^ 1, abort, args.err)) break;
      mbar_expect_tx(full_bar(s), kChunkBytes);
      bulk_load(b_addr + s * kChunkBytes, bsrc + size_t(issued) * kChunkBytes, kChunkBytes, full_bar(s));
    }
  } else if (warp == 5 && lane == 0) {
    bool ok = true;
    for (int j = 0; j < kTiles && ok; ++j) {
      const int b = j & 1;
      if (j >= 2 && !mbar_wait(acce_bar(b), ((j >> 1) - 1) & 1, abort, args.err)) break;
      tc_fence_after();
      const uint32_t d_tmem = tmem + uint32_t(b * 256);
      for (int c = 0; c < kChunksPerTile; ++c) {
        const int t = j * kChunksPerTile + c, s = t % kStages;
        if (!mbar_wait(full_bar(s), (t / kStages) & 1, abort, args.err)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const int kc = c >> 2, d = c & 3;
        const uint64_t a_desc = smem_desc(a_addr + d * kPlaneBytes + kc * 256, 128, 2048);
        const uint64_t b_desc = smem_desc(b_addr + s * kChunkBytes, 128, 256);
        mma_i8(d_tmem, a_desc, b_desc, c > 0 ? 1u : 0u);
        mma_commit(empty_bar(s));
      }
      if (ok) mma_commit(accf_bar(b));
    }
  } else if (warp < 4) {
    const uint32_t q = args.qinfo[2 * prime], qneg = args.qinfo[2 * prime + 1];
    const TwPair<uint32_t>* post = POST ? args.post + (size_t(prime) << kLogN) : nullptr;
    const int m = m0 + warp * 32 + lane;
    const uint32_t lane_addr = uint32_t(warp * 32) << 16;
    for (int j = 0; j < kTiles; ++j) {
      const int b = j & 1;
      // one lane waits and the verdict is broadcast, so the warp-collective
      // tcgen05.ld below always runs with all 32 lanes (or none)
      const bool ready = __shfl_sync(0xffffffffu, lane == 0 ? mbar_wait(accf_bar(b), (j >> 1) & 1, abort, args.err)
                                                           : false, 0);
      if (!ready) break;
      tc_fence_after();
#pragma unroll 1
      for (int cc = 0; cc < kTileCols / 16; ++cc) {
        uint32_t acc[4][16];
#pragma unroll
        for (int e = 0; e < 4; ++e) tmem_ld16(tmem + lane_addr + uint32_t(b * 256 + e * 64 + cc * 16), acc[e]);
        tmem_wait_ld();
        const int n0 = j * kTileCols + cc * 16;
        uint32_t res[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          uint64_t s = uint64_t(acc[0][i]) + (uint64_t(acc[1][i]) << 8) + (uint64_t(acc[2][i]) << 16) +
                       (uint64_t(acc[3][i]) << 24);
          const uint32_t mm = uint32_t(s) * qneg;
          uint32_t r = uint32_t((s + uint64_t(mm) * q) >> 32);  // S 2^-32 mod q, in [0, 2q)
          if (POST) {
            const TwPair<uint32_t> tw = post[COLUMN ? (n0 + i) * kSide + m : m * kSide + n0 + i];
            const uint32_t qh = __umulhi(r, tw.wp);
            r = r * tw.w - qh * q;  // Shoup: [0, 2q)
          }
          res[i] = r >= q ? r - q : r;
        }
        if (COLUMN) {
#pragma unroll
          for (int i = 0; i < 16; ++i) dst[(n0 + i) * kSide + m] = res[i];
        } else {
          uint4* o = reinterpret_cast<uint4*>(dst + m * kSide + n0);
#pragma unroll
          for (int i = 0; i < 4; ++i) o[i] = make_uint4(res[4 * i], res[4 * i + 1], res[4 * i + 2], res[4 * i + 3]);
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acce_bar(b));
    }
  }

  __syncthreads();
  // Drain what this CTA started before TMEM is freed and the CTA exits: all
  // MMAs (and the arrivals they signal) always, the bulk copies in flight
  // after an abort.
  if (warp == 5 && lane == 0) {
    mma_commit(drain_bar);
    mbar_wait(drain_bar, 0, nullptr, args.err);
  } else if (producer && *abort) {
    for (int t = issued - kStages < 0 ? 0 : issued - kStages; t < issued; ++t)
      mbar_wait(full_bar(t % kStages), (t / kStages) & 1, nullptr, args.err);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 5) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
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

uint32_t br8(uint32_t v) {
  uint32_t r = 0;
  for (int i = 0; i < 8; ++i, v >>= 1) r = (r << 1) | (v & 1);
  return r;
}

// Constant matrix B[k][n] of `pass` (0, 1: forward passes 1, 2; 2, 3:
// inverse passes 1, 2) as an exponent of psi modulo 2N.
uint32_t pass_exponent(int pass, uint32_t k, uint32_t n) {
  const uint32_t mask = (2u << kLogN) - 1;
  switch (pass) {
    case 0: return (256u * k * (2u * br8(n) + 1u)) & mask;              // W1[n = r][k = i1]
    case 1: return (512u * k * br8(n)) & mask;                           // W2[k = i2][n = c]
    case 2: return (0u - 512u * br8(k) * n) & mask;                      // W2'[k = c][n = i2]
    default: return (0u - 256u * n * (2u * br8(k) + 1u)) & mask;         // W1'[n = i1][k = r]
  }
}

// Byte offset of (row, k) in one B chunk (256 rows x 32 bytes, K-major).
inline size_t b_offset(uint32_t row, uint32_t kk) {
  return (row & 7) * 16 + (row >> 3) * 256 + (kk >> 4) * 128 + (kk & 15);
}

}  // namespace tcntt

// Fill the digit matrices of one pass for one prime (1 MiB at `bmat`) and,
// for passes 0 and 2, the elementwise twiddles (N pairs at `post`).
void tc_ntt_tables_host(uint64_t q, uint64_t psi, int pass, uint8_t* bmat, TwPair<uint32_t>* post) {
  using namespace tcntt;
  const uint32_t two_n = 2u << kLogN;
  std::vector<uint32_t> pw(two_n);
  pw[0] = 1;
  for (uint32_t i = 1; i < two_n; ++i) pw[i] = uint32_t(uint64_t(pw[i - 1]) * psi % q);  // q < 2^28
  uint64_t scale[4];
  for (int d = 0; d < 4; ++d) scale[d] = powmod64(2, 8 * d + 32, q);
  for (uint32_t k = 0; k < kSide; ++k) {
    for (uint32_t n = 0; n < kSide; ++n) {
      const uint64_t w = pw[pass_exponent(pass, k, n)];
      const uint32_t j = n / kTileCols, col = n % kTileCols, kc = k / 32, kk = k % 32;
      for (int d = 0; d < 4; ++d) {
        const uint32_t wd = uint32_t(w * scale[d] % q);
        uint8_t* chunk = bmat + (size_t(j) * kChunksPerTile + kc * 4 + d) * kChunkBytes;
        for (int e = 0; e < 4; ++e) chunk[b_offset(uint32_t(e) * kTileCols + col, kk)] = uint8_t(wd >> (8 * e));
      }
    }
  }
  if (post && (pass == 0 || pass == 2)) {
    const uint64_t r = powmod64(2, 30, q);
    uint64_t c = r;
    if (pass == 2) {
      const uint64_t rinv = powmod64(r, q - 2, q), ninv = powmod64((uint64_t(1) << kLogN) % q, q - 2, q);
      c = mulmod64(rinv, ninv, q);
    }
    for (uint32_t r = 0; r < kSide; ++r) {
      const uint32_t odd = 2u * br8(r) + 1u;
      for (uint32_t i2 = 0; i2 < kSide; ++i2) {
        uint32_t ex = (i2 * odd) & (two_n - 1);
        if (pass == 2) ex = (two_n - ex) & (two_n - 1);
        const uint32_t w = uint32_t(mulmod64(pw[ex], c, q));
        // forward pass 1 stores D[m = i2][n = r] column-wise (index n * 256 + m);
        // inverse pass 1 stores D[m = r][n = i2] row-wise (index m * 256 + n):
        // both are r * 256 + i2.
        post[r * kSide + i2] = TwPair<uint32_t>{w, uint32_t((uint64_t(w) << 32) / q)};
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
  std::vector<uint8_t> bm(size_t(qp) * kPassBytesPerPrime);
  std::vector<TwPair<uint32_t>> post(size_t(qp) * n);
  for (int pass = 0; pass < 4; ++pass) {
    for (int j = 0; j < qp; ++j)
      tc_ntt_tables_host(c.moduli[j], c.roots[j], pass, bm.data() + size_t(j) * kPassBytesPerPrime,
                         (pass == 0 || pass == 2) ? post.data() + size_t(j) * n : nullptr);
    t->bmat[pass] = static_cast<uint8_t*>(dev_alloc(bm.size()));
    if (!t->bmat[pass] || cudaMemcpy(t->bmat[pass], bm.data(), bm.size(), cudaMemcpyHostToDevice) != cudaSuccess)
      return give_up("tensor-core NTT digit matrices");
    if (pass == 0 || pass == 2) {
      auto*& dst = t->post[pass / 2];
      dst = static_cast<TwPair<uint32_t>*>(dev_alloc(post.size() * sizeof(post[0])));
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
template <bool COLUMN, bool POST>
int launch_pass(const Context& c, const uint32_t* in, uint32_t* out, int pass, int64_t polys, int rows,
                int row_start, cudaStream_t st) {
  using namespace tcntt;
  auto kern = k_tc_ntt_pass<COLUMN, POST>;
  if (int rc = ensure_dynamic_smem(reinterpret_cast<const void*>(kern), kSmemBytes)) return rc;
  PassArgs a{in, out, c.tc->bmat[pass], POST ? c.tc->post[pass / 2] : nullptr, c.tc->qinfo, polys / rows, rows,
             row_start, c.tc->err};
  kern<<<dim3(unsigned(polys * 2)), kThreads, kSmemBytes, st>>>(a);
  return cuda_status(cudaGetLastError(), "k_tc_ntt_pass");
}
}  // namespace

// Both passes of a direction; the second runs in place on `out` (each CTA
// reads its whole 128-row (or 128-column) slab into shared memory before it
// writes the same slab, and the two CTAs of a polynomial own disjoint slabs),
// so in == out is allowed and no scratch is needed.
int tc_ntt(Context& c, const void* in, void* out, int64_t polys, int rows, int row_start, bool inverse,
           cudaStream_t st) {
  if (int rc = tc_ntt_prepare(c)) return rc;
  if (polys == 0) return 0;
  if (polys * 2 > 0x7FFFFFFFll) return fail(-4, "too many polynomials for one launch");
  const auto* x = static_cast<const uint32_t*>(in);
  auto* y = static_cast<uint32_t*>(out);
  if (!inverse) {
    if (int rc = launch_pass<true, true>(c, x, y, 0, polys, rows, row_start, st)) return rc;
    return launch_pass<false, false>(c, y, y, 1, polys, rows, row_start, st);
  }
  if (int rc = launch_pass<false, true>(c, x, y, 2, polys, rows, row_start, st)) return rc;
  return launch_pass<true, false>(c, y, y, 3, polys, rows, row_start, st);
}

int tc_ntt_status(Context& c, int* flag) {
  std::lock_guard<std::mutex> lock(c.tc_mutex);
  *flag = 0;
  if (!c.tc) return 0;
  if (cudaError_t e = cudaMemcpy(flag, c.tc->err, sizeof(int), cudaMemcpyDeviceToHost)) return cuda_status(e, "flag");
  return cuda_status(cudaMemset(c.tc->err, 0, sizeof(int)), "flag reset");
}

}  // namespace fhb
