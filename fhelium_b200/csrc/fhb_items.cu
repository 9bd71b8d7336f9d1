// Mixed-level key switches as one launch per stage (C ABI: fhb_ckks_items_*).
//
// A plan is built once on the host from the caller's item descriptors and
// uploaded into a caller-provided device buffer: the device descriptors (with
// each item's scratch regions resolved), the list of HMult items, and the
// (item, row) work lists of the three cluster stages.  A run then issues six
// launches over all items, whatever their levels - forward NTT of the HMult
// operands, tensor product, inverse NTT of d2, ModUp digits, key-switch core,
// ModDown - and makes no host calls, so it can be captured in a CUDA graph
// and replayed.  The reference runs such a batch as one engine call sequence
// per ciphertext (fhelium/engine/ckks_engine.py:1530-1675, 2183-2300).
#include <algorithm>
#include <cstddef>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/fhb200.h"
#include "fhb_runners.h"
#include "fhb_items.cuh"

struct fhb_context {
  fhb::Context* impl;
};

namespace fhb {
namespace {

constexpr int64_t kRegionAlign = 256;
// the device descriptors open the plan; tests address a descriptor's level by this layout
static_assert(sizeof(KsItem) == 88 && offsetof(KsItem, level) == 4, "device descriptor layout");

int64_t align_up(int64_t x) { return (x + kRegionAlign - 1) / kRegionAlign * kRegionAlign; }

struct PlanLayout {
  int64_t items_off, hmult_off, fwd_off, inv_off, core_off, status_off, plan_bytes;
};

PlanLayout layout_of(const fhb_items_plan_info& info) {
  PlanLayout l;
  l.items_off = 0;
  l.hmult_off = align_up(int64_t(info.items) * int64_t(sizeof(KsItem)));
  l.fwd_off = l.hmult_off + align_up(int64_t(info.hmult_items) * 4);
  l.inv_off = l.fwd_off + align_up(int64_t(info.forward_units) * int64_t(sizeof(ItemUnit)));
  l.core_off = l.inv_off + align_up(int64_t(info.inverse_units) * int64_t(sizeof(ItemUnit)));
  l.status_off = l.core_off + align_up(int64_t(info.core_units) * int64_t(sizeof(ItemUnit)));
  l.plan_bytes = l.status_off + kRegionAlign;
  return l;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

class ItemsDeviceGuard {  // makes the context's device current for the call
 public:
  explicit ItemsDeviceGuard(int device) {
    cudaGetDevice(&prev_);
    if (prev_ != device) cudaSetDevice(device);
    dev_ = device;
  }
  ~ItemsDeviceGuard() {
    if (prev_ != dev_) cudaSetDevice(prev_);
  }

 private:
  int prev_ = 0, dev_ = 0;
};

// Scratch words of one item: HMult ab (4 L) + ct3 (3 L); every item digits
// (L) and the two accumulators (2 (L + P)).
int64_t item_scratch_bytes(const Context& c, const fhb_ks_item& it) {
  const int64_t l = c.num_q - it.level, lp = l + c.num_p, row = int64_t(c.n()) * (c.bits / 8);
  int64_t b = align_up(l * row) + 2 * align_up(lp * row);
  if (it.kind == FHB_ITEM_HMULT_RELIN_RESCALE) b += align_up(4 * l * row) + align_up(3 * l * row);
  return b;
}

// Leading rows of an item's Q_l whose primes are below 2^42: the key-switch
// core runs them in FP64 arithmetic (int64 chains with FP64 tables, unless
// the FP64 core is switched off).
int f64_item_rows(const Context& c, int level) {
  if (c.bits != 64 || !c.f64_tables_ok) return 0;
  return std::max(0, std::min(c.num_q - level, c.f64_prime_end - level));
}

int check_item(const Context& c, const fhb_ks_item& it, int i) {
  const std::string at = "item " + std::to_string(i) + ": ";
  if (it.kind != FHB_ITEM_HMULT_RELIN_RESCALE && it.kind != FHB_ITEM_ROTATE) return fail(-2, at + "unknown kind");
  if (it.level < 0 || it.level >= c.num_q) return fail(-4, at + "level out of range [0, num_q)");
  if (it.kind == FHB_ITEM_HMULT_RELIN_RESCALE && it.level + 1 >= c.num_q)
    return fail(-4, at + "cannot rescale at the last level");
  if (!it.a || !it.key || !it.out || (it.kind == FHB_ITEM_HMULT_RELIN_RESCALE && !it.b))
    return fail(-2, at + "NULL operand, key or output");
  if (!aligned16(it.a) || !aligned16(it.key) || !aligned16(it.out) || (it.b && !aligned16(it.b)))
    return fail(-2, at + "operands, key and output must be 16-byte aligned");
  if (it.kind == FHB_ITEM_ROTATE && (!(it.galois & 1) || it.galois >= (2u << c.log_n)))
    return fail(-5, at + "galois element must be odd and < 2N");
  return 0;
}

int run_stage(const Context& c, int stage, const ItemsView& iv, const void* units, int64_t count, cudaStream_t st,
              int64_t f64_units = 0) {
  if (count == 0) return 0;
#define FHB_ITEMS_CASE(L)                                                                                       \
  case L:                                                                                                       \
    return c.bits == 64                                                                                         \
               ? run_items<uint64_t, L>(c, stage, iv.items, iv.count, iv.status, units, count, st, f64_units) \
               : run_items<uint32_t, L>(c, stage, iv.items, iv.count, iv.status, units, count, st);
  switch (c.log_n) {
    FHB_ITEMS_CASE(12)
    FHB_ITEMS_CASE(13)
    FHB_ITEMS_CASE(14)
    FHB_ITEMS_CASE(15)
    FHB_ITEMS_CASE(16)
    FHB_ITEMS_CASE(17)
    default:
      return fail(-7, "log_n outside the supported 12..17");
  }
#undef FHB_ITEMS_CASE
}

template <typename T>
int run_elementwise(const Context& c, const char* plan, const PlanLayout& l, const fhb_items_plan_info& info,
                    cudaStream_t st) {
  constexpr int V = 16 / sizeof(T);
  const ItemsView iv{reinterpret_cast<const KsItem*>(plan + l.items_off), info.items,
                     reinterpret_cast<int*>(const_cast<char*>(plan) + l.status_off)};
  const int64_t n = c.n();
  const unsigned xb = unsigned((n / V + kEwThreads - 1) / kEwThreads);
  if (info.hmult_items > 0) {
    int rc = run_stage(c, 0, iv, plan + l.fwd_off, info.forward_units, st);
    if (rc) return rc;
    k_items_mul<T, V><<<dim3(xb, unsigned(info.max_limbs), unsigned(info.hmult_items)), kEwThreads, 0, st>>>(
        iv, reinterpret_cast<const int32_t*>(plan + l.hmult_off), c.num_q, c.log_n, tables<T>(c));
    if (int e = cuda_status(cudaGetLastError(), "k_items_mul")) return e;
    rc = run_stage(c, 1, iv, plan + l.inv_off, info.inverse_units, st);
    if (rc) return rc;
  }
  k_items_modup<T, V><<<dim3(xb, unsigned(info.max_digits), unsigned(info.items)), kEwThreads, 0, st>>>(
      iv, level_tables_dev<T>(c), c.num_q, c.log_n, tables<T>(c));
  if (int e = cuda_status(cudaGetLastError(), "k_items_modup")) return e;
  if (int rc = run_stage(c, 2, iv, plan + l.core_off, info.core_units, st, info.core_f64_units)) return rc;
  k_items_moddown<T><<<dim3(unsigned((n + 255) / 256), unsigned(info.items)), 256, 0, st>>>(
      iv, level_tables_dev<T>(c), c.num_q, c.num_p, c.log_n, tables<T>(c));
  return cuda_status(cudaGetLastError(), "k_items_moddown");
}

}  // namespace
}  // namespace fhb

using fhb::fail;

extern "C" {

int fhb_ckks_items_plan_info(const fhb_context* ctx, const fhb_ks_item* items, int count,
                             fhb_items_plan_info* info) {
  if (!ctx || !ctx->impl) return fail(-1, "context is NULL");
  if (!items || !info) return fail(-2, "NULL argument");
  if (count < 1 || count > 65535) return fail(-2, "need 1 <= count <= 65535 items");
  const fhb::Context& c = *ctx->impl;
  fhb_items_plan_info r{};
  r.items = count;
  int64_t scratch = 0;
  for (int i = 0; i < count; ++i) {
    if (int rc = fhb::check_item(c, items[i], i)) return rc;
    const int l = c.num_q - items[i].level;
    r.max_limbs = std::max(r.max_limbs, l);
    r.max_digits = std::max(r.max_digits, int(c.level_digits[items[i].level].size()));
    r.core_units += l + c.num_p;
    r.core_f64_units += fhb::f64_item_rows(c, items[i].level);
    if (items[i].kind == FHB_ITEM_HMULT_RELIN_RESCALE) {
      ++r.hmult_items;
      r.forward_units += 4 * l;
      r.inverse_units += l;
    }
    scratch += fhb::item_scratch_bytes(c, items[i]);
  }
  r.scratch_bytes = scratch;
  r.plan_bytes = fhb::layout_of(r).plan_bytes;
  *info = r;
  return 0;
}

int fhb_ckks_items_plan(const fhb_context* ctx, const fhb_ks_item* items, int count, void* plan, void* scratch,
                        const fhb_items_plan_info* info) {
  if (!ctx || !ctx->impl) return fail(-1, "context is NULL");
  const fhb::Context& c = *ctx->impl;
  fhb_items_plan_info check{};
  if (int rc = fhb_ckks_items_plan_info(ctx, items, count, &check)) return rc;
  if (!info || std::memcmp(&check, info, sizeof(check)) != 0)
    return fail(-2, "plan info does not describe these items (call fhb_ckks_items_plan_info)");
  if (!plan || !scratch || !fhb::aligned16(plan) || !fhb::aligned16(scratch))
    return fail(-2, "plan and scratch must be 16-byte aligned device buffers");
  const fhb::PlanLayout l = fhb::layout_of(*info);
  std::vector<char> host(size_t(l.plan_bytes), 0);
  auto* dev_items = reinterpret_cast<fhb::KsItem*>(host.data() + l.items_off);
  auto* hmult = reinterpret_cast<int32_t*>(host.data() + l.hmult_off);
  auto* fwd = reinterpret_cast<fhb::ItemUnit*>(host.data() + l.fwd_off);
  auto* inv = reinterpret_cast<fhb::ItemUnit*>(host.data() + l.inv_off);
  auto* core = reinterpret_cast<fhb::ItemUnit*>(host.data() + l.core_off);
  const int64_t row = int64_t(c.n()) * (c.bits / 8);
  char* sp = static_cast<char*>(scratch);
  int nh = 0, nf = 0, ni = 0;
  for (int i = 0; i < count; ++i) {
    const fhb_ks_item& src = items[i];
    const int64_t ll = c.num_q - src.level, lp = ll + c.num_p;
    fhb::KsItem d{src.kind, src.level, src.kind == FHB_ITEM_ROTATE ? src.galois : 1u, 0,
                  src.a, src.b, src.key, src.out, nullptr, nullptr, nullptr, nullptr, nullptr};
    d.digits = sp;
    sp += fhb::align_up(ll * row);
    d.t0 = sp;
    sp += fhb::align_up(lp * row);
    d.t1 = sp;
    sp += fhb::align_up(lp * row);
    if (src.kind == FHB_ITEM_HMULT_RELIN_RESCALE) {
      d.ab = sp;
      sp += fhb::align_up(4 * ll * row);
      d.coef = sp;
      sp += fhb::align_up(3 * ll * row);
      hmult[nh++] = i;
      for (int r = 0; r < 4 * ll; ++r) fwd[nf++] = fhb::ItemUnit{i, r};
      for (int r = 0; r < ll; ++r) inv[ni++] = fhb::ItemUnit{i, r};
    }
    d.check = fhb::item_check(d);
    dev_items[i] = d;
  }
  // Core work list: items of one (level, key) back to back; within such a
  // group, the context's key-switch work order picks one destination row
  // across the group's items (orders 1 and 2: concurrently resident
  // clusters share key rows in L2) or the rows of one item back to back
  // (order 0: an item's digit rows stay in L2).
  std::vector<int> order(count);
  for (int i = 0; i < count; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
    if (items[x].level != items[y].level) return items[x].level < items[y].level;
    return items[x].key < items[y].key;
  });
  int nc = 0;
  for (size_t g0 = 0; g0 < order.size();) {
    size_t g1 = g0;
    while (g1 < order.size() && items[order[g1]].level == items[order[g0]].level &&
           items[order[g1]].key == items[order[g0]].key)
      ++g1;
    const int lp = c.num_q - items[order[g0]].level + c.num_p;
    if (c.ks_order == 0) {
      for (size_t k = g0; k < g1; ++k)
        for (int r = 0; r < lp; ++r) core[nc++] = fhb::ItemUnit{order[k], r};
    } else {
      for (int r = 0; r < lp; ++r)
        for (size_t k = g0; k < g1; ++k) core[nc++] = fhb::ItemUnit{order[k], r};
    }
    g0 = g1;
  }
  fhb::ItemsDeviceGuard guard(c.device);
  return fhb::cuda_status(cudaMemcpy(plan, host.data(), host.size(), cudaMemcpyHostToDevice), "plan upload");
}

int fhb_ckks_items_status(const fhb_context* ctx, void* plan, const fhb_items_plan_info* info, int* status) {
  if (!ctx || !ctx->impl) return fail(-1, "context is NULL");
  if (!plan || !info || !status || info->items < 1) return fail(-2, "NULL plan, plan info or status");
  const fhb::Context& c = *ctx->impl;
  fhb::ItemsDeviceGuard guard(c.device);
  int* word = reinterpret_cast<int*>(static_cast<char*>(plan) + fhb::layout_of(*info).status_off);
  int value = 0;
  if (int e = fhb::cuda_status(cudaMemcpy(&value, word, sizeof(int), cudaMemcpyDeviceToHost), "status read"))
    return e;
  *status = value;
  if (value != 0)
    return fhb::cuda_status(cudaMemset(word, 0, sizeof(int)), "status reset");
  return 0;
}

int fhb_ckks_items_run(const fhb_context* ctx, const void* plan, const fhb_items_plan_info* info,
                       fhb_stream stream) {
  if (!ctx || !ctx->impl) return fail(-1, "context is NULL");
  if (!plan || !info || info->items < 1) return fail(-2, "NULL plan or empty plan info");
  const fhb::Context& c = *ctx->impl;
  fhb::ItemsDeviceGuard guard(c.device);
  const fhb::PlanLayout l = fhb::layout_of(*info);
  const char* p = static_cast<const char*>(plan);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  return c.bits == 64 ? fhb::run_elementwise<uint64_t>(c, p, l, *info, st)
                      : fhb::run_elementwise<uint32_t>(c, p, l, *info, st);
}

}  // extern "C"
