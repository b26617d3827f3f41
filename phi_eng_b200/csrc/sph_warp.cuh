// Warp-level aggregation of bucket-count atomics, shared by the 2D and 3D
// kernel chains.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace phieng {

// Runs of equal keys over the active lanes in lane order (any active set):
// a lane starts a run unless the nearest active lane below it holds the
// same key. For the calling lane: *first = its run's first lane, *len = the
// run's active lanes, *rank = active lanes of the run below this one.
__device__ __forceinline__ void key_run(uint32_t act, uint32_t k, uint32_t lane, uint32_t* first, uint32_t* len,
                                        uint32_t* rank) {
  const uint32_t below = act & ((1u << lane) - 1u);
  const int src = below ? 31 - __clz(below) : (int)lane;
  const uint32_t prev = __shfl_sync(act, k, src);
  const bool head = !below || prev != k;
  const uint32_t heads = __ballot_sync(act, head);
  const uint32_t f = 31u - (uint32_t)__clz(heads & (0xFFFFFFFFu >> (31u - lane)));
  const uint32_t above = heads & ~(0xFFFFFFFFu >> (31u - lane));
  const uint32_t upper = above ? ((1u << (__ffs(above) - 1)) - 1u) : 0xFFFFFFFFu;  // lanes below the next run
  const uint32_t run = act & upper & ~((1u << f) - 1u);
  *first = f;
  *len = (uint32_t)__popc(run);
  *rank = (uint32_t)__popc(run & ((1u << lane) - 1u));
}

// Add a warp's keys to count[] with one atomic per run of equal keys (keys
// arrive in sorted-slot or id order, so a bucket's particles mostly sit in
// consecutive lanes; a key split over several runs takes several atomics).
__device__ __forceinline__ void count_key(uint32_t* __restrict__ count, uint32_t k) {
  const uint32_t act = __activemask();
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t first, len, rank;
  key_run(act, k, lane, &first, &len, &rank);
  if (first == lane) atomicAdd(&count[k], len);
}

}  // namespace phieng
