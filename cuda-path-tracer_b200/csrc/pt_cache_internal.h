// pt_cache_internal.h — the radiance-cache network as the cached renderer drives it: launches
// only, no host synchronisation, batch sizes that may live on the device (so that a frame can
// be captured once as a CUDA graph and replayed).
#pragma once

#include <cuda_runtime.h>
#include "pt_host.h"

namespace ptb {
// rgb[3k..3k+2] = prediction for queries[k], k < min(count, *count_dev) (count_dev may be null).
void cache_forward(pt_cache *c, const pt_cache_query *queries, size_t count, const int32_t *count_dev, float *rgb, cudaStream_t st);
// One Adam step on the first min(count, *count_dev) samples; an empty batch changes nothing.
void cache_train(pt_cache *c, const pt_cache_query *queries, const float *targets, size_t count, const int32_t *count_dev,
                 cudaStream_t st);
void cache_bounds(const pt_cache *c, float lo[3], float hi[3]);
float cache_loss(pt_cache *c, cudaStream_t st);   // mean loss of the last step (synchronises)
void cache_status(pt_cache *c);                   // throws if a tensor-core wait expired
} // namespace ptb
