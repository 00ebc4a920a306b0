/*
 * internal.h -- declarations shared by the library's C and CUDA sources.
 */
#ifndef CUOPO_INTERNAL_H
#define CUOPO_INTERNAL_H

#include "cuopo.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Records msg as this thread's last error and returns st. */
cuopo_status cuopo_fail(cuopo_status st, const char *msg);

/* Philox4x32-10 (Salmon et al., SC'11) + Box-Muller: value number i of the
 * stream (seed, stream_id), as the pair (re, im).  Shared by the host and
 * device noise generators. */
void cuopo_noise_pair_host(uint64_t seed, uint64_t stream_id, uint64_t i, double sigma,
                           float *re, float *im);

#ifdef __cplusplus
}

#include <nvtx3/nvToolsExt.h>

namespace cuopo {
/* A named NVTX range over the enclosing scope: the library's host calls show
 * up by name on a profiler's timeline; without a tool attached the push and
 * pop return at once. */
struct Range {
    explicit Range(const char *name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
    Range(const Range &) = delete;
    Range &operator=(const Range &) = delete;
};
}  // namespace cuopo
#endif

#endif
