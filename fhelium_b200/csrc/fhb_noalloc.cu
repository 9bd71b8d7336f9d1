// Relinearisation that allocates nothing: its scratch is a fixed array in
// device memory that belongs to this library, instead of a buffer the caller
// provides.
//
// Who needs it: callers that can hand the library their input and output
// buffers but cannot obtain any other device memory.  Typical cases are a
// plugin running inside a host framework that owns every device byte through
// its own pool (a direct cudaMalloc would bypass the pool's accounting and may
// synchronise the whole device), and a serving loop whose latency budget
// forbids allocation on the request path.
//
// Cost and rules:
//  * The array below is FHB_NOALLOC_SCRATCH_BYTES (32 MiB).  Every GPU on which
//    this part of the library is loaded holds it until the process exits.
//  * Host code cannot use the array's name as an address: on the host it only
//    stands in for the symbol.  The device address is looked up once per
//    device with cudaGetSymbolAddress, with that device current, on the first
//    call made on that device; make that first call before any stream capture.
//  * All calls share the one array and it keeps the previous call's contents.
//    Nothing in the relinearisation needs the scratch to start at zero (every
//    scratch word is written before it is read), so it is never cleared.
//    Calls whose work can overlap on the GPU (different streams, or different
//    host threads) race on the array; serialise them.
#include <mutex>
#include <string>

#include "../../include/fhb200.h"
#include "fhb_context.h"

#define FHB_NOALLOC_SCRATCH_BYTES (int64_t{32} << 20)

static __device__ __align__(256) unsigned char g_noalloc_scratch[FHB_NOALLOC_SCRATCH_BYTES];

struct fhb_context {
  fhb::Context* impl;
};

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
void* g_scratch_address[kMaxDevices] = {};

// Device address of g_noalloc_scratch on `device` (looked up once, with the
// device current).  Returns 0 on success.
int scratch_address(int device, void** out) {
  if (device < 0 || device >= kMaxDevices) return fhb::fail(-2, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch_address[device]) {
    int prev = 0;
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) return fhb::cuda_status(e, "cudaGetDevice");
    if (prev != device && (e = cudaSetDevice(device)) != cudaSuccess) return fhb::cuda_status(e, "cudaSetDevice");
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (prev != device) cudaSetDevice(prev);
    if (e != cudaSuccess) return fhb::cuda_status(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    g_scratch_address[device] = p;
  }
  *out = g_scratch_address[device];
  return 0;
}

}  // namespace

extern "C" {

int64_t fhb_ckks_relinearize_noalloc_max_scratch_bytes(void) { return FHB_NOALLOC_SCRATCH_BYTES; }

int fhb_ckks_relinearize_noalloc(const fhb_context* ctx, const void* ct3, const void* key, void* out, int64_t batch,
                                 int level, int rescale, fhb_stream stream) {
  if (!ctx || !ctx->impl) return fhb::fail(-1, "context is NULL");
  const int64_t need = fhb_ckks_keyswitch_scratch_bytes(ctx, batch, level);
  if (need < 0) return fhb::fail(-4, "invalid batch or level");
  if (need > FHB_NOALLOC_SCRATCH_BYTES)
    return fhb::fail(-9, "fhb_ckks_relinearize_noalloc: this batch needs " + std::to_string(need) +
                             " scratch bytes, more than the library's fixed " +
                             std::to_string(FHB_NOALLOC_SCRATCH_BYTES) +
                             "; use fhb_ckks_relinearize with a caller buffer or a smaller batch");
  void* scratch = nullptr;
  const int rc = scratch_address(ctx->impl->device, &scratch);
  if (rc != 0) return rc;
  return fhb_ckks_relinearize(ctx, ct3, key, out, scratch, FHB_NOALLOC_SCRATCH_BYTES, batch, level, rescale, stream);
}

}  // extern "C"
