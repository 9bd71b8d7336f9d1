// Key switches of ciphertexts at mixed levels, driven by a device table of
// item descriptors: every stage is one launch over all items, whatever their
// levels, instead of one launch sequence per level.
//
// An item is one ciphertext (batch 1) with its own operation:
//   kind 0  HMult + relinearise + rescale of a (lhs) and b (rhs), both
//           [2, L, N] coefficient/standard, with the relinearisation key;
//   kind 1  rotation of a [2, L, N] coefficient/standard by its own Galois
//           element with its own rotation key.
// The stages mirror the fused batch path (forward NTT of the operands, the
// tensor product, the inverse NTT of d2, ModUp digits, the key-switch core
// with c0, c1 folded in for relinearisation, ModDown with the rescale or
// with sigma_g(c0)), and use the same building blocks, so every result is
// integer-equal to the per-level batch calls.  Work lists of (item, row)
// units map the cluster kernels' clusters to items; the element-wise kernels
// take the item from the grid's z dimension.
#pragma once
#include "fhb_kernels.cuh"

namespace fhb {

struct KsItem {
  int32_t kind;         // 0: HMult + relinearise + rescale, 1: rotation
  int32_t level;
  uint32_t galois;      // rotation: Galois element of the step; 1 for HMult
  uint32_t check;       // item_check() of the other fields, written by the planner
  const void* a;        // [2, L, N] coefficient/standard (lhs, or the rotated ciphertext)
  const void* b;        // HMult rhs [2, L, N] coefficient/standard; null for a rotation
  const void* key;      // [D, 2, QP0, N] NTT/Montgomery key
  void* out;            // HMult [2, L - 1, N]; rotation [2, L, N]; coefficient/standard
  void* ab;             // scratch: HMult [2 operands][2][L][N] NTT/Montgomery
  void* coef;           // scratch: HMult ct3 [3, L, N] NTT/Montgomery
  void* digits;         // scratch: [L, N] ModUp digits
  void* t0;             // scratch: [L + P, N] (d2 in the coefficient domain, then accumulator 0)
  void* t1;             // scratch: [L + P, N] accumulator 1
};

struct ItemUnit {
  int32_t item;
  int32_t row;          // forward NTT: operand * 2 L + component * L + row
};

// Check word of a descriptor: FNV-1a over every field but the check itself.
// The planner validates the fields on the host and stores the word; every
// kernel recomputes it before it uses the item, so a descriptor changed in
// device memory after planning is skipped (and reported) instead of being
// trusted for addressing.
__host__ __device__ __forceinline__ uint32_t fnv_mix(uint32_t h, uint64_t w) {
  h = (h ^ uint32_t(w)) * 16777619u;
  return (h ^ uint32_t(w >> 32)) * 16777619u;
}

__host__ __device__ __forceinline__ uint32_t item_check(const KsItem& it) {
  uint32_t h = 2166136261u;
  h = fnv_mix(h, (uint64_t(uint32_t(it.kind)) << 32) | uint32_t(it.level));
  h = fnv_mix(h, it.galois);
  const void* const ptrs[9] = {it.a, it.b, it.key, it.out, it.ab, it.coef, it.digits, it.t0, it.t1};
#pragma unroll
  for (int i = 0; i < 9; ++i) h = fnv_mix(h, uint64_t(reinterpret_cast<uintptr_t>(ptrs[i])));
  return h;
}

// Status codes of a run (the first one raised is kept).
enum ItemsStatus : int {
  kItemsOk = 0,
  kItemsBadIndex = 1,    // a work list names an item outside the plan
  kItemsBadCheck = 2,    // a descriptor no longer matches its check word
  kItemsBadRow = 3,      // a work-list row outside the item's rows
  kItemsBadKind = 4,     // the HMult list names a rotation
};

struct ItemsView {
  const KsItem* items;
  int32_t count;
  int* status;
};

__device__ __forceinline__ void items_raise(int* status, int code) {
  if (*reinterpret_cast<volatile int*>(status) == 0) atomicCAS(status, 0, code);
}

// Fetches item `idx` into `it`; false (status raised) when the index or the
// descriptor is not the planned one.
__device__ __forceinline__ bool items_fetch(const ItemsView& v, int idx, KsItem& it) {
  if (idx < 0 || idx >= v.count) {
    items_raise(v.status, kItemsBadIndex);
    return false;
  }
  it = v.items[idx];
  if (it.check != item_check(it)) {
    items_raise(v.status, kItemsBadCheck);
    return false;
  }
  return true;
}

// Tensor product of the HMult items (k_mul_ntt per item): grid (N / (256 V),
// rows, HMult items), rows past an item's level return.
template <typename T, int V>
__global__ void k_items_mul(ItemsView iv, const int32_t* __restrict__ hmult, int num_q, int log_n,
                            ChainTables<T> tabs) {
  KsItem it;
  if (!items_fetch(iv, hmult[blockIdx.z], it)) return;
  if (it.kind != 0) {
    items_raise(iv.status, kItemsBadKind);
    return;
  }
  const int limbs = num_q - it.level;
  const int row = blockIdx.y;
  const int64_t n = int64_t(1) << log_n;
  const int64_t k = (int64_t(blockIdx.x) * kEwThreads + threadIdx.x) * V;
  if (row >= limbs || k >= n) return;
  const PrimeInfo<T>& pp = tabs.prime[it.level + row];
  const T q = pp.q, ni = pp.neg_inv, tq = pp.twice_q;
  const T* ab = static_cast<const T*>(it.ab);
  const int64_t comp = int64_t(limbs) * n, i = int64_t(row) * n + k;
  const EwVec<T, V> x0 = ew_load<T, V>(ab + i), x1 = ew_load<T, V>(ab + comp + i);
  const EwVec<T, V> y0 = ew_load<T, V>(ab + 2 * comp + i), y1 = ew_load<T, V>(ab + 3 * comp + i);
  EwVec<T, V> d0, d1, d2;
#pragma unroll
  for (int e = 0; e < V; ++e) {
    d0.v[e] = Word<T>::mont(x0.v[e], y0.v[e], q, ni);
    d1.v[e] = csub(Word<T>::mont(x0.v[e], y1.v[e], q, ni) + Word<T>::mont(x1.v[e], y0.v[e], q, ni), tq);
    d2.v[e] = Word<T>::mont(x1.v[e], y1.v[e], q, ni);
  }
  T* out = static_cast<T*>(it.coef);
  ew_store<T, V>(out + i, d0);
  ew_store<T, V>(out + comp + i, d1);
  ew_store<T, V>(out + 2 * comp + i, d2);
}

// ModUp digits of every item (k_modup_digits per item): the source is d2 in
// the coefficient domain (t0) for HMult, c1 through sigma_g for a rotation.
// Grid (N / (256 V), digits, items), digits past an item's level return.
template <typename T, int V>
__global__ void k_items_modup(ItemsView iv, const LevelTables<T>* __restrict__ levels, int num_q, int log_n,
                              ChainTables<T> tabs) {
  KsItem it;
  if (!items_fetch(iv, int(blockIdx.z), it)) return;
  const LevelTables<T> lt = levels[it.level];
  if (int(blockIdx.y) >= lt.num_digits) return;
  const int64_t n = int64_t(1) << log_n;
  const int64_t k0 = (int64_t(blockIdx.x) * kEwThreads + threadIdx.x) * V;
  if (k0 >= n) return;
  using W = Word<T>;
  const int limbs = num_q - it.level;
  const DigitDesc d = lt.digits[blockIdx.y];
  const TwPair<T>* g = lt.garner + blockIdx.y * kMaxDigitWidth * kMaxDigitWidth;
  const uint32_t gi = (it.kind == 0 || it.galois == 1) ? 0u : galois_inverse_dev(it.galois, log_n);
  const T* src = it.kind == 0 ? static_cast<const T*>(it.t0) : static_cast<const T*>(it.a) + int64_t(limbs) * n;
  T* dst = static_cast<T*>(it.digits);
  EwVec<T, V> dig[kMaxDigitWidth];
  for (int r = 0; r < d.alpha; ++r) {
    const int row = d.prime0 - it.level + r;
    const T q = tabs.prime[d.prime0 + r].q;
    EwVec<T, V> x;
    if (gi == 0) {
      x = ew_load<T, V>(src + row * n + k0);
#pragma unroll
      for (int e = 0; e < V; ++e) x.v[e] = csub(x.v[e], q);
    } else {
#pragma unroll
      for (int e = 0; e < V; ++e) {
        bool neg = false;
        const int srck = galois_source(int(k0) + e, log_n, gi, neg);
        T y = csub(src[row * n + srck], q);
        x.v[e] = (neg && y) ? q - y : y;
      }
    }
    if (r > 0) {
      const TwPair<T> inv = g[r * kMaxDigitWidth + r];
#pragma unroll
      for (int e = 0; e < V; ++e) {
        T acc = 0;
        for (int i = 0; i < r; ++i) {
          const TwPair<T> c = g[r * kMaxDigitWidth + i];
          acc = csub(acc + csub(W::shoup(dig[i].v[e], c.w, c.wp, q), q), q);
        }
        x.v[e] = csub(W::shoup(csub(x.v[e] + q - acc, q), inv.w, inv.wp, q), q);
      }
    }
    dig[r] = x;
    ew_store<T, V>(dst + row * n + k0, x);
  }
}

// ModDown of every item (k_moddown per item): HMult items rescale by the
// leading prime (c0, c1 are already in the accumulators); rotations add
// sigma_g(c0).  Grid (N / 256, items), one coefficient per thread.
template <typename T>
__global__ void k_items_moddown(ItemsView iv, const LevelTables<T>* __restrict__ levels, int num_q, int num_p,
                                int log_n, ChainTables<T> tabs) {
  using W = Word<T>;
  KsItem it;
  if (!items_fetch(iv, int(blockIdx.y), it)) return;
  const int64_t n = int64_t(1) << log_n;
  const int k = int(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int level = it.level;
  const int q_limbs = num_q - level, qp0 = num_q + num_p;
  const int rescale = it.kind == 0 ? 1 : 0;
  const int out_limbs = q_limbs - rescale;
  const uint32_t gi = (it.kind == 0 || it.galois == 1) ? 0u : galois_inverse_dev(it.galois, log_n);
  bool neg = false;
  const int ak = gi ? galois_source(k, log_n, gi, neg) : k;
  const LevelTables<T> lt = levels[level];
  for (int c = 0; c < 2; ++c) {
    const T* t = static_cast<const T*>(c == 0 ? it.t0 : it.t1);
    const T* ad = (it.kind == 1 && c == 0) ? static_cast<const T*>(it.a) : nullptr;
    T e[kMaxDigitWidth];
    for (int r = 0; r < num_p; ++r) {
      const PrimeInfo<T> p = tabs.prime[num_q + r];
      T x = t[(q_limbs + r) * n + k];
      T acc = 0;
      for (int i = 0; i < r; ++i) {
        const TwPair<T> g = tabs.p_garner[r * kMaxDigitWidth + i];
        acc = csub(acc + csub(W::shoup(e[i], g.w, g.wp, p.q), p.q), p.q);
      }
      if (r > 0) {
        const TwPair<T> inv = tabs.p_garner[r * kMaxDigitWidth + r];
        x = csub(W::shoup(csub(x + p.q - acc, p.q), inv.w, inv.wp, p.q), p.q);
      }
      e[r] = x;
    }
    T* o = static_cast<T*>(it.out) + int64_t(c) * out_limbs * n;
    T v0 = 0;
    for (int i = 0; i < q_limbs; ++i) {
      const int pid = level + i;
      const PrimeInfo<T> p = tabs.prime[pid];
      T sub = 0;
      for (int r = 0; r < num_p; ++r) {
        const TwPair<T> m = tabs.p_mix[r * qp0 + pid];
        sub = csub(sub + csub(W::shoup(e[r], m.w, m.wp, p.q), p.q), p.q);
      }
      const TwPair<T> pinv = tabs.p_inv[pid];
      T v = csub(t[i * n + k] + p.q - sub, p.q);
      v = csub(W::shoup(v, pinv.w, pinv.wp, p.q), p.q);
      if (ad) {
        T x = csub(ad[i * n + ak], p.q);
        if (neg && x) x = p.q - x;
        v = csub(v + x, p.q);
      }
      if (!rescale) {
        o[i * n + k] = v;
      } else if (i == 0) {
        v0 = v;
      } else {
        const T x0 = reduce_any(v0, p);
        const TwPair<T> inv = lt.rescale_inv[pid];
        T r = csub(W::shoup(csub(v + p.q - x0, p.q), inv.w, inv.wp, p.q), p.q);
        r += (v0 > (tabs.prime[level].q >> 1)) ? 1 : 0;
        o[(i - 1) * n + k] = csub(r, p.q);
      }
    }
  }
}

// Forward NTT of the HMult operands (k_ntt_forward per row): one cluster per
// unit (item, operand 2 L + component L + row), coefficient/standard ->
// NTT/Montgomery (x R), lazy [0, 2q), into the item's `ab`.  SPLIT (int64
// chains with FP64 tables): the rows whose primes are below 2^42 (prime id
// < f64_end) run the transform in FP64 arithmetic (as k_ntt_forward's SPLIT
// form does); their lazy words may differ from the integer transform's by q,
// which the later stages (all modular, canonical at the end) do not see.
template <typename T, int LOGN, bool SPLIT = false>
__global__ void __launch_bounds__(NttGeom<T, LOGN>::kThreads)
k_items_ntt_forward(ItemsView iv, const ItemUnit* __restrict__ units, int num_q, ChainTables<T> tabs,
                    ChainTables<double> tabs64f, int f64_end) {
  using G = NttGeom<T, LOGN>;
  static_assert(!SPLIT || (sizeof(T) == 8 && NttGeom<double, LOGN>::kC == G::kC &&
                           NttGeom<double, LOGN>::kThreads == G::kThreads),
                "the FP64 rows share the integer transform's geometry");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int rank = cluster_rank<T, LOGN>();
  // every CTA of the cluster reads the same unit, so an early return is cluster-uniform
  const ItemUnit u = units[blockIdx.x / G::kC];
  KsItem it;
  if (!items_fetch(iv, u.item, it)) return;
  const int limbs = num_q - it.level;
  if (it.kind != 0) {
    items_raise(iv.status, kItemsBadKind);
    return;
  }
  if (u.row < 0 || u.row >= 4 * limbs) {
    items_raise(iv.status, kItemsBadRow);
    return;
  }
  const int op = u.row / (2 * limbs), rem = u.row - op * 2 * limbs;  // rem = component L + row
  const int pid = it.level + rem % limbs;
  const T* in = static_cast<const T*>(op == 0 ? it.a : it.b) + int64_t(rem) * G::kN;
  T* out = static_cast<T*>(it.ab) + int64_t(u.row) * G::kN + int64_t(rank) * G::kM + threadIdx.x * G::kE;
  if constexpr (SPLIT) {
    if (pid < f64_end) {
      const PrimeInfo<double> p = tabs64f.prime[pid];
      U64MontSource<true> src{reinterpret_cast<const uint64_t*>(in), p.rmod, p.rmod_s, p.q};
      double v[G::kE];
      Ntt<double, LOGN, TwGlobalQ<LOGN>>::forward_from(src, reinterpret_cast<double*>(smem_raw),
                                                       TwGlobalQ<LOGN>{tabs64f.twv_fwd + int64_t(pid) * G::kN, p.one_s},
                                                       p.q, p.one_s, rank, v);
#pragma unroll
      for (int e = 0; e < G::kE; ++e) v[e] = Word<double>::to_lazy(v[e], p.q, p.one_s);
      store_words(reinterpret_cast<uint64_t*>(out), v);
      return;
    }
  }
  const PrimeInfo<T> p = tabs.prime[pid];
  RowSource<T, true> src{in, p.rmod, p.rmod_s, p.q};
  T v[G::kE];
  Ntt<T, LOGN>::forward_from(src, reinterpret_cast<T*>(smem_raw), TwGlobal<T, LOGN>(tabs.tw_fwd + int64_t(pid) * G::kN),
                             p.q, p.twice_q, rank, v);
#pragma unroll
  for (int e = 0; e < G::kE; ++e) v[e] = csub(v[e], p.twice_q);
  store16(out, v);
}

// Inverse NTT of d2 of the HMult items (k_ntt_inverse per row): one cluster
// per unit (item, row), NTT/Montgomery -> coefficient/standard canonical,
// into the item's t0.  SPLIT: rows of primes below 2^42 in FP64 arithmetic
// (as k_ntt_inverse's SPLIT form), the same canonical words.
template <typename T, int LOGN, bool SPLIT = false>
__global__ void __launch_bounds__(NttGeom<T, LOGN>::kThreads)
k_items_ntt_inverse(ItemsView iv, const ItemUnit* __restrict__ units, int num_q, ChainTables<T> tabs,
                    ChainTables<double> tabs64f, int f64_end) {
  using G = NttGeom<T, LOGN>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int rank = cluster_rank<T, LOGN>();
  const ItemUnit u = units[blockIdx.x / G::kC];
  KsItem it;
  if (!items_fetch(iv, u.item, it)) return;
  const int limbs = num_q - it.level;
  if (it.kind != 0) {
    items_raise(iv.status, kItemsBadKind);
    return;
  }
  if (u.row < 0 || u.row >= limbs) {
    items_raise(iv.status, kItemsBadRow);
    return;
  }
  const int pid = it.level + u.row;
  const T* in = static_cast<const T*>(it.coef) + int64_t(2 * limbs + u.row) * G::kN + int64_t(rank) * G::kM +
                threadIdx.x * G::kE;
  T* out = static_cast<T*>(it.t0) + int64_t(u.row) * G::kN;
  T w[G::kE];
  load16(in, w);
  if constexpr (SPLIT) {
    if (pid < f64_end) {
      const PrimeInfo<double> p = tabs64f.prime[pid];
      double v[G::kE];
#pragma unroll
      for (int e = 0; e < G::kE; ++e) v[e] = __ull2double_rn(w[e]);
      F64OutEpilogue epi{reinterpret_cast<uint64_t*>(out), p.q, p.ninv_rinv, p.ninv_rinv_s, kInvStandard};
      Ntt<double, LOGN, TwGlobalQ<LOGN>>::inverse(reinterpret_cast<double*>(smem_raw),
                                                  TwGlobalQ<LOGN>{tabs64f.twv_inv + int64_t(pid) * G::kN, p.one_s},
                                                  p.q, p.one_s, rank, v, epi);
      return;
    }
  }
  const PrimeInfo<T> p = tabs.prime[pid];
  InvEpilogue<T> epi = make_inv_epilogue<T>(out, p, kInvStandard, true);
  Ntt<T, LOGN>::inverse(reinterpret_cast<T*>(smem_raw), TwGlobal<T, LOGN>(tabs.tw_inv + int64_t(pid) * G::kN), p.q,
                        p.twice_q, rank, w, epi);
}

// Key-switch core of every item (k_keyswitch_core per (ciphertext, row)):
// one cluster per unit (item, destination row of Q_l P).  For HMult items
// the NTT-domain ct3 is folded in (c0, c1 as P c_k, own-digit rows from c2).
// Returns false (status raised) for a unit outside its item's rows.
__device__ __forceinline__ bool items_core_unit(const ItemsView& iv, const ItemUnit& u, int num_q, int num_p,
                                                KsItem& it) {
  if (!items_fetch(iv, u.item, it)) return false;
  if (u.row < 0 || u.row >= num_q - it.level + num_p) {
    items_raise(iv.status, kItemsBadRow);
    return false;
  }
  return true;
}

template <typename T, int LOGN>
__global__ void __launch_bounds__(NttGeom<T, LOGN>::kThreads)
k_items_core(ItemsView iv, const ItemUnit* __restrict__ units, const LevelTables<T>* __restrict__ levels, int num_q,
             int num_p, ChainTables<T> tabs) {
  using G = NttGeom<T, LOGN>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const ItemUnit u = units[blockIdx.x / G::kC];  // the same unit on every CTA of the cluster
  KsItem it;
  if (!items_core_unit(iv, u, num_q, num_p, it)) return;
  const int q_limbs = num_q - it.level;
  ks_core_unit<T, LOGN, false>(static_cast<const T*>(it.digits), static_cast<const T*>(it.key),
                               static_cast<T*>(it.t0), static_cast<T*>(it.t1), 1, q_limbs, q_limbs + num_p, it.level,
                               num_q + num_p, it.kind == 0 ? static_cast<const T*>(it.coef) : nullptr,
                               int64_t(q_limbs) * G::kN, tabs, levels[it.level], 0, u.row, smem_raw,
                               cluster_rank<T, LOGN>());
}

// The same for an int64 chain with FP64 tables: the units of rows whose
// primes are below 2^42 run the FP64 body (k_keyswitch_core_split), the
// others the integer body, in one launch.  ext64f [level][digit][r][2][QP]
// of ext_digits digits per level.
template <int LOGN>
__global__ void __launch_bounds__(NttGeom<double, LOGN>::kThreads)
k_items_core_split(ItemsView iv, const ItemUnit* __restrict__ units, const LevelTables<uint64_t>* __restrict__ levels,
                   int num_q, int num_p, ChainTables<uint64_t> tabs, ChainTables<double> tabs64f,
                   const TwPair<double>* __restrict__ ext64f, int ext_digits, int f64_end) {
  using G = NttGeom<double, LOGN>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const ItemUnit u = units[blockIdx.x / G::kC];
  KsItem it;
  if (!items_core_unit(iv, u, num_q, num_p, it)) return;
  const int q_limbs = num_q - it.level, qp_limbs = q_limbs + num_p, qp0 = num_q + num_p;
  const uint64_t* ct3 = it.kind == 0 ? static_cast<const uint64_t*>(it.coef) : nullptr;
  const int rank = cluster_rank<double, LOGN>();
  const LevelTables<uint64_t> lt = levels[it.level];
  if (it.level + u.row < f64_end)
    ks_core_unit_f64<LOGN, false>(static_cast<const uint64_t*>(it.digits), static_cast<const uint64_t*>(it.key),
                                  static_cast<uint64_t*>(it.t0), static_cast<uint64_t*>(it.t1), 1, q_limbs, qp_limbs,
                                  it.level, qp0, ct3, int64_t(q_limbs) * G::kN, tabs64f, lt, ext64f, ext_digits,
                                  f64_end, 0, u.row, smem_raw, rank);
  else
    ks_core_unit<uint64_t, LOGN, false>(static_cast<const uint64_t*>(it.digits),
                                        static_cast<const uint64_t*>(it.key), static_cast<uint64_t*>(it.t0),
                                        static_cast<uint64_t*>(it.t1), 1, q_limbs, qp_limbs, it.level, qp0, ct3,
                                        int64_t(q_limbs) * G::kN, tabs, lt, 0, u.row, smem_raw, rank);
}

}  // namespace fhb
