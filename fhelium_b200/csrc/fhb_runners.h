// Declarations of the per-(word, LOGN) cluster launchers; definitions in
// fhb_runners.cuh, instantiated in fhb_inst_logn.cu (one object per LOGN).
#pragma once
#include <cuda_runtime.h>

#include "fhb_context.h"

namespace fhb {
template <typename T, int LOGN>
int run_forward(const Context& c, const void* in, void* out, int64_t polys, int rows, int row_start, bool mont,
                cudaStream_t st);
template <typename T, int LOGN>
int run_inverse(const Context& c, const void* in, void* out, int64_t polys, int rows, int row_start, int kind,
                cudaStream_t st);
template <typename T, int LOGN>
int run_mul_coef(const Context& c, const void* a, const void* b, void* out, int64_t batch, int level,
                 cudaStream_t st);
template <typename T, int LOGN>
int run_ks_core(const Context& c, const void* digits, const void* key, void* acc0, void* acc1, int64_t batch,
                int level, cudaStream_t st, const uint64_t* item_keys, const void* ct3, bool pre,
                int64_t ct3_pitch = 0);
template <typename T, int LOGN>
int run_ks_sum(const Context& c, const void* digits, const uint64_t* key_ptrs, void* acc0, void* acc1, int giants,
               int64_t batch, int level, cudaStream_t st, bool pre);
// Mixed-level item stages: 0 = forward NTT of the HMult operands, 1 =
// inverse NTT of d2, 2 = key-switch core; `count` units of `units`, of
// which the leading `f64_units` (stage 2) may run in FP64 arithmetic.
template <typename T, int LOGN>
int run_items(const Context& c, int stage, const void* items, int item_count, int* status, const void* units,
              int64_t count, cudaStream_t st, int64_t f64_units = 0);
template <typename T, int LOGN>
int run_prepare(const Context& c, const void* digits, void* prepared, int64_t batch, int level, cudaStream_t st);
template <typename T, int LOGN>
int run_apply_prepared(const Context& c, const void* prepared, const void* key, void* acc0, void* acc1,
                       int64_t batch, int level, uint32_t galois, cudaStream_t st);
}  // namespace fhb
