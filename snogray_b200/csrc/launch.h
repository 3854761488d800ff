// launch.h -- host-side launch helpers for the kernels in trace.cu and
// wavefront.cu.

#ifndef SNOG_LAUNCH_H
#define SNOG_LAUNCH_H

#include <cuda_runtime.h>

#include "snog_common.h"

namespace snog {

// Number of SMs of the current device (cached per device).
int num_sms();

// Stack class (entries) for an octree of the given depth, 0 if too deep.
int stack_class_for_depth(uint32_t depth);

cudaError_t launch_trace_batch(const DevScene &s, const float *rays, uint32_t n, uint32_t n_closest,
                               int32_t *prim, float *t, float *nrm, unsigned long long *counters,
                               uint32_t *err, cudaStream_t st, int *launches);

}  // namespace snog

#endif
