// Device side of the x-slab decomposition of one scene over ranks: each
// rank world steps its owned particles plus a halo of its neighbours'
// particles; these kernels fill the buffers the host sends to the
// neighbours (point-to-point, fixed size, the count travels in the buffer)
// and take the received ones in, so no count is read on the host.
//
// Every replaced slot moves its particle's bucket count from the old key to
// the new one, so the key array and the counts stay what the next sort needs
// (the force pass wrote both for the previous positions). Slot order inside
// a rank world does not matter for the results: the sort orders each bucket
// by the particles' global ids (FluidBufs::order).
#include <cuda_runtime.h>

#include <cmath>

#include "sph_device.cuh"
#include "sph_kernels.h"

namespace phieng {
namespace {

inline uint32_t cdiv(uint32_t a, uint32_t b) { return (a + b - 1) / b; }

// floor(x / h) as a saturating i32 with NaN -> 0: the column of the bucket
// key's cell (bucket_key) and of slab membership.
__device__ __forceinline__ int64_t cell_column(float x, float h) { return (int64_t)__float2int_rd(__fdiv_rn(x, h)); }

struct SlabView {
  uint32_t* hdr;  // [count, overflow, 0, 0]
  float4* rows;
  uint32_t* tags;
};

__device__ __forceinline__ SlabView slab_view(const unsigned char* p, uint32_t cap) {
  unsigned char* q = const_cast<unsigned char*>(p);
  SlabView v;
  v.hdr = reinterpret_cast<uint32_t*>(q);
  v.rows = reinterpret_cast<float4*>(q + 16);
  v.tags = reinterpret_cast<uint32_t*>(q + 16 + 16 * (size_t)cap);
  return v;
}

__device__ __forceinline__ void slab_append(unsigned char* buf, uint32_t cap, float4 s, uint32_t tag) {
  SlabView v = slab_view(buf, cap);
  const uint32_t j = atomicAdd(&v.hdr[0], 1u);
  if (j < cap) {
    v.rows[j] = s;
    v.tags[j] = tag;
  } else {
    v.hdr[1] = 1u;
  }
}

// Slot i now holds (s, tag); its bucket count follows the key.
__device__ __forceinline__ void slab_set_slot(const FluidBufs& d, const GridPlan& g, uint32_t i, float4 s,
                                              uint32_t tag) {
  const uint32_t old = d.key[i], k = bucket_key(s.x, s.y, g);
  if (old != k) {
    atomicSub(&d.count[old], 1u);
    atomicAdd(&d.count[k], 1u);
    d.key[i] = k;
  }
  d.state[i] = s;
  d.order[i] = tag;
}

__device__ __forceinline__ float4 empty_slot() { return make_float4(__int_as_float(0x7FC00000), __int_as_float(0x7FC00000), 0.0f, 0.0f); }

// Received rows of one side: min(count, cap); an overflowing sender or an
// impossible count marks the error word.
__device__ __forceinline__ uint32_t slab_received(const SlabPlan& sp, uint32_t side, SlabView v, bool report) {
  const uint32_t has = side ? sp.has_right : sp.has_left;
  if (!has) return 0u;
  const uint32_t c = v.hdr[0];
  if (report && (v.hdr[1] != 0u || c > sp.halo_cap)) atomicExch(&sp.words[1], 1u);
  return c < sp.halo_cap ? c : sp.halo_cap;
}

__global__ void k_slab_init(const uint32_t* __restrict__ order, SlabPlan sp) {
  // one block: a fixed-order compaction of the free owned slots
  __shared__ uint32_t base;
  __shared__ uint32_t wsum[32];
  if (threadIdx.x == 0) base = 0;
  __syncthreads();
  for (uint32_t i0 = 0; i0 < sp.own_cap; i0 += blockDim.x) {
    const uint32_t i = i0 + threadIdx.x;
    const bool f = i < sp.own_cap && order[i] == kSlabFree;
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    const uint32_t bal = __ballot_sync(0xFFFFFFFFu, f);
    if (lane == 0) wsum[w] = __popc(bal);
    __syncthreads();
    uint32_t off = base;
    for (uint32_t k = 0; k < w; k++) off += wsum[k];
    if (f) sp.free_stack[off + __popc(bal & ((1u << lane) - 1u))] = i;
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t t = 0;
      for (uint32_t k = 0; k < blockDim.x / 32; k++) t += wsum[k];
      base += t;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    sp.words[0] = base;
    sp.words[1] = 0u;
    sp.words[2] = 0u;
  }
}

__global__ void k_slab_pack_halo(FluidBufs d, SlabPlan sp) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= sp.own_cap) return;
  const uint32_t tag = d.order[i];
  if (tag == kSlabFree) return;
  const float4 s = d.state[i];
  const int64_t cx = cell_column(s.x, sp.h);
  if (sp.has_left && cx < (int64_t)sp.lo + kSlabHaloColumns) slab_append(sp.send[0], sp.halo_cap, s, tag);
  if (sp.has_right && cx >= (int64_t)sp.hi - kSlabHaloColumns) slab_append(sp.send[1], sp.halo_cap, s, tag);
}

__global__ void k_slab_unpack_halo(FluidBufs d, SlabPlan sp, GridPlan g) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= 2 * sp.halo_cap) return;
  const uint32_t side = j >= sp.halo_cap ? 1u : 0u, r = j - side * sp.halo_cap;
  const SlabView v = slab_view(sp.recv[side], sp.halo_cap);
  const uint32_t cnt = slab_received(sp, side, v, r == 0);
  const uint32_t i = sp.own_cap + j;
  if (r < cnt)
    slab_set_slot(d, g, i, v.rows[r], v.tags[r]);
  else if (d.order[i] != kSlabFree || finitef(d.state[i].x))
    slab_set_slot(d, g, i, empty_slot(), kSlabFree);
}

__global__ void k_slab_pack_migrants(FluidBufs d, SlabPlan sp, GridPlan g) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= sp.own_cap) return;
  const uint32_t tag = d.order[i];
  if (tag == kSlabFree) return;
  const float4 s = d.state[i];
  const int64_t cx = cell_column(s.x, sp.h);
  int side = -1;
  if (sp.has_left && cx < (int64_t)sp.lo)
    side = 0;
  else if (sp.has_right && cx >= (int64_t)sp.hi)
    side = 1;
  if (side < 0) return;
  slab_append(sp.send[side], sp.halo_cap, s, tag);
  slab_set_slot(d, g, i, empty_slot(), kSlabFree);
  const uint32_t top = atomicAdd(&sp.words[0], 1u);  // below own_cap: each slot is on the stack at most once
  if (top < sp.own_cap)
    sp.free_stack[top] = i;
  else
    atomicExch(&sp.words[1], 1u);
}

__global__ void k_slab_unpack_migrants(FluidBufs d, SlabPlan sp, GridPlan g) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= 2 * sp.halo_cap) return;
  const uint32_t side = j >= sp.halo_cap ? 1u : 0u, r = j - side * sp.halo_cap;
  const SlabView v = slab_view(sp.recv[side], sp.halo_cap);
  const uint32_t cnt = slab_received(sp, side, v, r == 0);
  if (r >= cnt) return;
  const uint32_t size = min(sp.words[0], sp.own_cap);  // not changed by this kernel
  const uint32_t p = atomicAdd(&sp.words[2], 1u);
  if (p >= size) {  // the owned region is full: the particle is lost, the run reports it
    atomicExch(&sp.words[1], 1u);
    return;
  }
  slab_set_slot(d, g, sp.free_stack[size - 1u - p], v.rows[r], v.tags[r]);
}

// Pop the slots k_slab_unpack_migrants took.
__global__ void k_slab_settle(SlabPlan sp) {
  const uint32_t size = min(sp.words[0], sp.own_cap), p = sp.words[2];
  sp.words[0] = p < size ? size - p : 0u;
  sp.words[2] = 0u;
}

}  // namespace

void enqueue_slab_init(const FluidBufs& b, const SlabPlan& sp, cudaStream_t st) {
  k_slab_init<<<1, 1024, 0, st>>>(b.order, sp);
}

void enqueue_slab_pack(const FluidBufs& b, const SlabPlan& sp, const GridPlan& g, uint32_t phase, cudaStream_t st) {
  for (int k = 0; k < 2; k++)
    if (sp.send[k]) cudaMemsetAsync(sp.send[k], 0, 16, st);
  if (sp.own_cap == 0) return;
  if (phase == 0)
    k_slab_pack_halo<<<cdiv(sp.own_cap, 256), 256, 0, st>>>(b, sp);
  else
    k_slab_pack_migrants<<<cdiv(sp.own_cap, 256), 256, 0, st>>>(b, sp, g);
}

void enqueue_slab_unpack(const FluidBufs& b, const SlabPlan& sp, const GridPlan& g, uint32_t phase, cudaStream_t st) {
  if (sp.halo_cap == 0) return;
  if (phase == 0) {
    k_slab_unpack_halo<<<cdiv(2 * sp.halo_cap, 256), 256, 0, st>>>(b, sp, g);
  } else {
    k_slab_unpack_migrants<<<cdiv(2 * sp.halo_cap, 256), 256, 0, st>>>(b, sp, g);
    k_slab_settle<<<1, 1, 0, st>>>(sp);
  }
}

}  // namespace phieng
