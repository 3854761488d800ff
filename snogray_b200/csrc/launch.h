// launch.h -- host-side launch helpers for the kernels in trace.cu and
// wavefront.cu.

#ifndef SNOG_LAUNCH_H
#define SNOG_LAUNCH_H

#include <cuda_runtime.h>

#include "snog_common.h"

namespace snog {

// Number of SMs of the current device (cached per device).
int num_sms();

// Blocks of THREADS threads that fill every SM exactly once (persistent
// kernels), from the occupancy calculator; cached per kernel.
int blocks_per_sm_cached(const void *kernel, int threads, int (*query)(const void *, int));

template <class K>
uint32_t resident_grid(K kernel, int threads) {
  int per_sm = blocks_per_sm_cached(reinterpret_cast<const void *>(kernel), threads,
                                    [](const void *k, int t) {
                                      int v = 0;
                                      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                                              &v, reinterpret_cast<K>(const_cast<void *>(k)), t, 0) !=
                                          cudaSuccess)
                                        v = 1;
                                      return v < 1 ? 1 : v;
                                    });
  return uint32_t(per_sm) * uint32_t(num_sms());
}

// Fill lrec (3 float4 per slot) from the surface lists and primitive records.
cudaError_t build_list_records(const uint32_t *plist, uint32_t n, const float4 *prims, float4 *lrec,
                               cudaStream_t st);

// Whether the closest-hit kernels should deal list entries in pairs for
// scene S: traces 8192 random rays through its bounding box and answers yes
// when they test more than 2.5 primitives per node visit (long lists along
// rays, as in random-triangle soups: 4.8; the terrain: 1.2).
uint32_t probe_pair_lists(const DevScene &s);

// Stack class (entries) for an octree of the given depth, 0 if too deep.
int stack_class_for_depth(uint32_t depth);

cudaError_t launch_trace_batch(const DevScene &s, const float *rays, uint32_t n, uint32_t n_closest,
                               int32_t *prim, float *t, float *nrm, unsigned long long *counters,
                               uint32_t *err, uint32_t *fetch, cudaStream_t st, int *launches);

}  // namespace snog

#endif
