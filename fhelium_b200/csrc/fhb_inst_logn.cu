// Instantiates the cluster launchers for one ring degree (compiled once per
// FHB_LOGN in 12..17 by the build script).
#include "fhb_runners.cuh"

#ifndef FHB_LOGN
#error "compile with -DFHB_LOGN=<12..17>"
#endif

namespace fhb {
FHB_INSTANTIATE_RUNNERS(uint64_t, FHB_LOGN)
FHB_INSTANTIATE_RUNNERS(uint32_t, FHB_LOGN)
}  // namespace fhb
