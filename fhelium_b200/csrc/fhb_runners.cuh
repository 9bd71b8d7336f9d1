// Cluster launchers for the NTT-based kernels.  Each is explicitly
// instantiated per LOGN in its own translation unit (fhb_inst_logn.cu), so
// the kernel templates compile in parallel.
#pragma once
#include <algorithm>
#include "fhb_items.cuh"
#include "fhb_kernels.cuh"

namespace fhb {

// Rows [row_start, row_start + rows) of a transform whose leading k rows
// have primes below 2^42 and may run in FP64 arithmetic (0 when the
// context has no FP64 tables or the form is switched off).
inline int f64_rows(const Context& c, int row_start, int rows) {
  if (!c.f64_core || !c.f64_tables_ok) return 0;
  return std::max(0, std::min(rows, c.f64_prime_end - row_start));
}

template <typename T, int LOGN, int EPT = 0, typename... KArgs, typename... Args>
int launch_cluster(void (*kernel)(KArgs...), int64_t polys, size_t smem, cudaStream_t stream, Args... args) {
  using G = NttGeom<T, LOGN, EPT>;
  if (polys <= 0) return 0;
  if (polys * G::kC > 0x7fffffffLL) return fail(-6, "too many polynomials for one launch");
  const int rc = ensure_dynamic_smem(reinterpret_cast<const void*>(kernel), int(smem));
  if (rc != 0) return rc;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned(polys * G::kC));
  cfg.blockDim = dim3(G::kThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = G::kC;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = G::kC > 1 ? 1 : 0;
  return cuda_status(cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...), "cluster launch");
}

template <typename T, int LOGN>
constexpr size_t ntt_smem() {
  return size_t(NttGeom<T, LOGN>::kSmemElems) * sizeof(T);
}

// ---- per (T, LOGN) launchers --------------------------------------------
// The standalone transforms exist with 8 and 16 residues per thread (radix-8
// passes over 1024 threads or radix-16 passes over 512 for N = 2^16); the
// context's tuning values pick one per direction (0 = the ring's default).
template <typename T, int LOGN, int EPT>
int run_forward_e(const Context& c, const void* in, void* out, int64_t polys, int rows, int row_start, bool mont,
                  cudaStream_t st) {
  // the leading rows of primes below 2^42 in FP64 arithmetic (int64 chains), same launch
  const int k = sizeof(T) == 8 ? f64_rows(c, row_start, rows) : 0;
  auto launch = [&](auto kern) {
    return launch_cluster<T, LOGN, EPT>(kern, polys, ntt_smem<T, LOGN>(), st, (const T*)in, (T*)out, rows, row_start,
                                        tables<T>(c), c.t64f, k);
  };
  if constexpr (sizeof(T) == 8) {
    if (k > 0)
      return mont ? launch(k_ntt_forward<T, LOGN, false, EPT, true>) : launch(k_ntt_forward<T, LOGN, true, EPT, true>);
  }
  return mont ? launch(k_ntt_forward<T, LOGN, false, EPT>) : launch(k_ntt_forward<T, LOGN, true, EPT>);
}

template <typename T, int LOGN>
int run_forward(const Context& c, const void* in, void* out, int64_t polys, int rows, int row_start,
                bool mont, cudaStream_t st) {
  if (c.ntt_ept_fwd == 16) return run_forward_e<T, LOGN, 16>(c, in, out, polys, rows, row_start, mont, st);
  return run_forward_e<T, LOGN, 0>(c, in, out, polys, rows, row_start, mont, st);
}

template <typename T, int LOGN, int EPT>
int run_inverse_e(const Context& c, const void* in, void* out, int64_t polys, int rows, int row_start, int kind,
                  cudaStream_t st) {
  const int k = sizeof(T) == 8 ? f64_rows(c, row_start, rows) : 0;
  auto launch = [&](auto kern) {
    return launch_cluster<T, LOGN, EPT>(kern, polys, ntt_smem<T, LOGN>(), st, (const T*)in, (T*)out, rows, row_start,
                                        kind, tables<T>(c), c.t64f, k);
  };
  if constexpr (sizeof(T) == 8) {
    if (k > 0) return launch(k_ntt_inverse<T, LOGN, EPT, true>);
  }
  return launch(k_ntt_inverse<T, LOGN, EPT>);
}

template <typename T, int LOGN>
int run_inverse(const Context& c, const void* in, void* out, int64_t polys, int rows, int row_start, int kind,
                cudaStream_t st) {
  if (c.ntt_ept_inv == 16) return run_inverse_e<T, LOGN, 16>(c, in, out, polys, rows, row_start, kind, st);
  return run_inverse_e<T, LOGN, 0>(c, in, out, polys, rows, row_start, kind, st);
}

template <typename T, int LOGN>
int run_mul_coef(const Context& c, const void* a, const void* b, void* out, int64_t batch, int level,
                 cudaStream_t st) {
  const int limbs = c.num_q - level;
  const int64_t polys = 3 * batch * limbs;
  if (c.ntt_ept_inv == 16)
    return launch_cluster<T, LOGN, 16>(k_mul_to_coefficient<T, LOGN, 16>, polys, ntt_smem<T, LOGN>(), st,
                                       (const T*)a, (const T*)b, (T*)out, batch, limbs, level, tables<T>(c));
  return launch_cluster<T, LOGN>(k_mul_to_coefficient<T, LOGN>, polys, ntt_smem<T, LOGN>(), st, (const T*)a,
                                 (const T*)b, (T*)out, batch, limbs, level, tables<T>(c));
}

template <typename T, int LOGN>
int run_ks_core(const Context& c, const void* digits, const void* key, void* acc0, void* acc1, int64_t batch,
                int level, cudaStream_t st, const uint64_t* item_keys, const void* ct3, bool pre,
                int64_t ct3_pitch) {
  const int ql = c.num_q - level, qpl = ql + c.num_p;
  if (ct3_pitch <= 0) ct3_pitch = batch * ql * int64_t(c.n());  // component pitch of ct3 [3, batch, L, N]
  const auto* ik = reinterpret_cast<const unsigned long long*>(item_keys);
  auto launch_int = [&](auto kern) {
    return launch_cluster<T, LOGN>(kern, batch * qpl, KsAcc<T, LOGN>::smem_bytes(), st, (const T*)digits,
                                   (const T*)key, (T*)acc0, (T*)acc1, batch, ql, qpl, level, c.qp(), c.ks_order, ik,
                                   (const T*)ct3, ct3_pitch, tables<T>(c), level_tables<T>(c, level));
  };
  if constexpr (sizeof(T) == 8) {
    if constexpr (KsAcc<double, LOGN>::kSmem) {
      static_assert(KsAcc<double, LOGN>::smem_bytes() == KsAcc<T, LOGN>::smem_bytes(), "one smem size for both");
      // the leading Q rows whose primes are below 2^42 in FP64 arithmetic,
      // the rest (wider Q primes, the P rows) on the integer body, one launch
      const int f64_rows = c.f64_core && c.f64_tables_ok ? std::max(0, std::min(ql, c.f64_prime_end - level)) : 0;
      if (f64_rows > 0) {
        auto launch_split = [&](auto kern) {
          return launch_cluster<double, LOGN>(kern, batch * qpl, KsAcc<double, LOGN>::smem_bytes(), st,
                                              (const uint64_t*)digits, (const uint64_t*)key, (uint64_t*)acc0,
                                              (uint64_t*)acc1, batch, ql, qpl, level, c.qp(), c.ks_order, ik,
                                              (const uint64_t*)ct3, ct3_pitch, tables<uint64_t>(c),
                                              level_tables<uint64_t>(c, level), c.t64f, f64_rows, c.ext64f,
                                              c.ext64f_digits, c.f64_prime_end);
        };
        return pre ? launch_split(k_keyswitch_core_split<LOGN, true>)
                   : launch_split(k_keyswitch_core_split<LOGN, false>);
      }
    }
    if (pre) return launch_int(k_keyswitch_core<T, LOGN, true>);  // extensions of the tensor-core form
  } else {
    if (pre) return fail(-7, "the tensor-core basis conversion needs an int64 context");
  }
  return launch_int(k_keyswitch_core<T, LOGN>);
}

template <typename T, int LOGN>
int run_ks_sum(const Context& c, const void* digits, const uint64_t* key_ptrs, void* acc0, void* acc1, int giants,
               int64_t batch, int level, cudaStream_t st, bool pre) {
  const int ql = c.num_q - level, qpl = ql + c.num_p;
  if (pre) {
    if constexpr (sizeof(T) == 8) {
      return launch_cluster<T, LOGN>(k_keyswitch_sum<T, LOGN, true>, batch * qpl, KsAcc<T, LOGN>::smem_bytes(), st,
                                     (const T*)digits, reinterpret_cast<const unsigned long long*>(key_ptrs),
                                     (T*)acc0, (T*)acc1, giants, batch, ql, qpl, level, c.qp(), c.ks_order,
                                     tables<T>(c), level_tables<T>(c, level));
    } else {
      return fail(-7, "the tensor-core basis conversion needs an int64 context");
    }
  }
  return launch_cluster<T, LOGN>(k_keyswitch_sum<T, LOGN>, batch * qpl, KsAcc<T, LOGN>::smem_bytes(), st,
                                 (const T*)digits, reinterpret_cast<const unsigned long long*>(key_ptrs), (T*)acc0,
                                 (T*)acc1, giants, batch, ql, qpl, level, c.qp(), c.ks_order, tables<T>(c),
                                 level_tables<T>(c, level));
}

// Rows [0, k) of Q_l (primes below 2^42) of a key-switch kernel at `level`
// that run in FP64 arithmetic (int64 chains with FP64 tables, N <= 2^16).
template <typename T, int LOGN>
int ks_f64_rows(const Context& c, int level) {
  if constexpr (sizeof(T) == 8 && KsAcc<double, LOGN>::kSmem) {
    static_assert(KsAcc<double, LOGN>::smem_bytes() == KsAcc<T, LOGN>::smem_bytes(), "one smem size for both");
    return c.f64_core && c.f64_tables_ok ? std::max(0, std::min(c.num_q - level, c.f64_prime_end - level)) : 0;
  }
  return 0;
}

template <typename T, int LOGN>
int run_prepare(const Context& c, const void* digits, void* prepared, int64_t batch, int level,
                cudaStream_t st) {
  const int ql = c.num_q - level, qpl = ql + c.num_p;
  const int k = ks_f64_rows<T, LOGN>(c, level);
  auto launch = [&](auto kern) {
    return launch_cluster<T, LOGN>(kern, batch * qpl, KsAcc<T, LOGN>::smem_bytes(), st, (const T*)digits,
                                   (T*)prepared, batch, ql, qpl, level, c.qp(), c.ks_order, tables<T>(c),
                                   level_tables<T>(c, level), c.t64f, k, c.ext64f, c.ext64f_digits, c.f64_prime_end);
  };
  if constexpr (sizeof(T) == 8) {
    if (k > 0) return launch(k_prepare_rotation<T, LOGN, true>);
  }
  return launch(k_prepare_rotation<T, LOGN>);
}

template <typename T, int LOGN>
int run_apply_prepared(const Context& c, const void* prepared, const void* key, void* acc0, void* acc1,
                       int64_t batch, int level, uint32_t galois, cudaStream_t st) {
  const int ql = c.num_q - level, qpl = ql + c.num_p;
  const int k = ks_f64_rows<T, LOGN>(c, level);
  auto launch = [&](auto kern) {
    return launch_cluster<T, LOGN>(kern, batch * qpl, KsAcc<T, LOGN>::smem_bytes(), st, (const T*)prepared,
                                   (const T*)key, (T*)acc0, (T*)acc1, batch, qpl, level, c.qp(),
                                   galois == 1 ? 0u : galois, c.ks_order, tables<T>(c), level_tables<T>(c, level),
                                   c.t64f, k);
  };
  if constexpr (ApplyRegs<T, LOGN>::kOk) {
    if constexpr (sizeof(T) == 8) {
      if (k > 0) return launch(k_apply_prepared_rotation<T, LOGN, true>);
    }
    return launch(k_apply_prepared_rotation<T, LOGN>);
  } else {
    if constexpr (sizeof(T) == 8) {
      if (k > 0) return launch(k_apply_prepared_rotation_staged<T, LOGN, true>);
    }
    return launch(k_apply_prepared_rotation_staged<T, LOGN>);
  }
}

// ---- mixed-level item stages (fhb_items.cuh): one cluster per unit ----------
template <typename T, int LOGN>
int run_items(const Context& c, int stage, const void* items, int item_count, int* status, const void* units,
              int64_t count, cudaStream_t st, int64_t f64_units) {
  const ItemsView iv{static_cast<const KsItem*>(items), item_count, status};
  const auto* un = static_cast<const ItemUnit*>(units);
  // int64 chains with FP64 tables: the rows of primes below 2^42 in FP64 arithmetic
  const bool split = sizeof(T) == 8 && c.f64_core && c.f64_tables_ok && c.f64_prime_end > 0;
  if (stage < 2) {
    auto launch = [&](auto kern) {
      return launch_cluster<T, LOGN>(kern, count, ntt_smem<T, LOGN>(), st, iv, un, c.num_q, tables<T>(c), c.t64f,
                                     c.f64_prime_end);
    };
    if constexpr (sizeof(T) == 8) {
      if (split)
        return stage == 0 ? launch(k_items_ntt_forward<T, LOGN, true>) : launch(k_items_ntt_inverse<T, LOGN, true>);
    }
    return stage == 0 ? launch(k_items_ntt_forward<T, LOGN>) : launch(k_items_ntt_inverse<T, LOGN>);
  }
  // stage 2, the key-switch core; on an int64 chain with FP64 tables the
  // units of rows whose primes are below 2^42 run in FP64 arithmetic
  if constexpr (sizeof(T) == 8) {
    if constexpr (KsAcc<double, LOGN>::kSmem) {
      static_assert(KsAcc<double, LOGN>::smem_bytes() == KsAcc<T, LOGN>::smem_bytes(), "one smem size for both");
      if (split && f64_units > 0)
        return launch_cluster<double, LOGN>(k_items_core_split<LOGN>, count, KsAcc<double, LOGN>::smem_bytes(), st,
                                            iv, un, level_tables_dev<uint64_t>(c), c.num_q, c.num_p,
                                            tables<uint64_t>(c), c.t64f, c.ext64f, c.ext64f_digits,
                                            c.f64_prime_end);
    }
  }
  return launch_cluster<T, LOGN>(k_items_core<T, LOGN>, count, KsAcc<T, LOGN>::smem_bytes(), st, iv, un,
                                 level_tables_dev<T>(c), c.num_q, c.num_p, tables<T>(c));
}

// Explicit instantiation of every runner for one (T, LOGN).
#define FHB_INSTANTIATE_RUNNERS(T, LOGN)                                                                       \
  template int run_forward<T, LOGN>(const Context&, const void*, void*, int64_t, int, int, bool, cudaStream_t);   \
  template int run_inverse<T, LOGN>(const Context&, const void*, void*, int64_t, int, int, int, cudaStream_t);    \
  template int run_mul_coef<T, LOGN>(const Context&, const void*, const void*, void*, int64_t, int, cudaStream_t); \
  template int run_ks_core<T, LOGN>(const Context&, const void*, const void*, void*, void*, int64_t, int,        \
                                    cudaStream_t, const uint64_t*, const void*, bool, int64_t);                 \
  template int run_ks_sum<T, LOGN>(const Context&, const void*, const uint64_t*, void*, void*, int, int64_t, int, \
                                   cudaStream_t, bool);                                                         \
  template int run_prepare<T, LOGN>(const Context&, const void*, void*, int64_t, int, cudaStream_t);            \
  template int run_items<T, LOGN>(const Context&, int, const void*, int, int*, const void*, int64_t, cudaStream_t, \
                                  int64_t);                                                                     \
  template int run_apply_prepared<T, LOGN>(const Context&, const void*, const void*, void*, void*, int64_t, int, \
                                           uint32_t, cudaStream_t);

}  // namespace fhb
