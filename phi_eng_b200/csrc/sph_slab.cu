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

#include <algorithm>
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

// Index of this lane's entry among the warp's `want` lanes in an array whose
// length counter is *ctr: one atomic per warp (every lane of the warp calls
// it). Returns the index (undefined where want is false).
__device__ __forceinline__ uint32_t warp_reserve(uint32_t* ctr, bool want) {
  const uint32_t m = __ballot_sync(0xFFFFFFFFu, want);
  if (m == 0u) return 0u;
  const uint32_t lane = threadIdx.x & 31u, leader = __ffs(m) - 1u;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(ctr, __popc(m));
  base = __shfl_sync(0xFFFFFFFFu, base, leader);
  return base + __popc(m & ((1u << lane) - 1u));
}

// Append (s, tag) to send[side] for the lanes with want (every lane of the
// warp calls it); rows past the capacity are dropped and show up as an
// overflowing count.
__device__ __forceinline__ void slab_append(const SlabPlan& sp, int side, bool want, float4 s, uint32_t tag) {
  SlabView v = slab_view(sp.send[side], sp.halo_cap);
  const uint32_t j = warp_reserve(&sp.words[4 + side], want);
  if (want && j < sp.halo_cap) {
    v.rows[j] = s;
    v.tags[j] = tag;
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
    for (int k = 1; k < 8; k++) sp.words[k] = 0u;
  }
}

// Blocks of whole warps, no early return: the appends are warp-collective.
// One pack per substep, after the rank's step: owned particles whose column
// left [lo, hi) go to that side as migrants (tag | kSlabMigrant; their slots
// are freed), the others within kSlabHaloColumns of a shared edge go as halo.
// phase 0 (before the first step) packs the halo only. The appends count
// into words[4 + side]; the last block to finish writes the headers. Blocks
// of whole warps and no early return: the appends are warp-collective.
__global__ void k_slab_pack(FluidBufs d, SlabPlan sp, GridPlan g, uint32_t phase) {
  // grid-stride over the owned slots (the loop bound is uniform per block)
  for (uint32_t base = blockIdx.x * blockDim.x; base < sp.own_cap; base += gridDim.x * blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    const uint32_t tag = i < sp.own_cap ? d.order[i] : kSlabFree;
    const bool live = tag != kSlabFree;
    const float4 s = live ? d.state[i] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const int64_t cx = cell_column(s.x, sp.h);
    const bool gl = phase && live && sp.has_left && cx < (int64_t)sp.lo;
    const bool gr = phase && live && !gl && sp.has_right && cx >= (int64_t)sp.hi;
    const bool stay = live && !gl && !gr;
    const bool hl = stay && sp.has_left && cx < (int64_t)sp.lo + kSlabHaloColumns;
    const bool hr = stay && sp.has_right && cx >= (int64_t)sp.hi - kSlabHaloColumns;
    if (sp.has_left) slab_append(sp, 0, gl || hl, s, gl ? (tag | kSlabMigrant) : tag);
    if (sp.has_right) slab_append(sp, 1, gr || hr, s, gr ? (tag | kSlabMigrant) : tag);
    const bool go = gl || gr;
    const uint32_t top = warp_reserve(&sp.words[0], go);  // below own_cap: each slot is on the stack at most once
    if (go) {
      slab_set_slot(d, g, i, empty_slot(), kSlabFree);
      if (top < sp.own_cap)
        sp.free_stack[top] = i;
      else
        atomicExch(&sp.words[1], 1u);
    }
  }
  __shared__ bool last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(&sp.words[2], 1u) + 1u == gridDim.x;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    for (int k = 0; k < 2; k++)
      if (sp.send[k]) {
        const uint32_t c = atomicAdd(&sp.words[4 + k], 0u);
        uint32_t* h = reinterpret_cast<uint32_t*>(sp.send[k]);
        h[0] = c;
        h[1] = c > sp.halo_cap ? 1u : 0u;
      }
    sp.words[2] = 0u;
  }
}

// One unpack per substep, after the exchange. Each side's halo region has
// 2 * halo_cap slots: slot q < halo_cap takes received row q if it is halo
// (a received migrant instead takes a free owned slot), slot halo_cap + q
// takes the row q this rank sent to that side if it was a migrant (it now
// lies within the neighbour's edge band, so it belongs to this rank's halo;
// the neighbour could not send it back in the same exchange). Every other
// halo slot is emptied. Slabs are at least 2 * kSlabHaloColumns wide, so a
// migrant from the far side never lands in the band sent to the near one.
__global__ void k_slab_unpack(FluidBufs d, SlabPlan sp, GridPlan g, uint32_t phase) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t cap = sp.halo_cap;
  if (j == 0) {  // the pack counters start from zero again (the pack has finished)
    sp.words[4] = 0u;
    sp.words[5] = 0u;
  }
  if (j >= 4 * cap) return;
  const uint32_t side = j >= 2 * cap ? 1u : 0u, q = j - side * 2 * cap;
  const uint32_t slot = sp.own_cap + j;
  const uint32_t has = side ? sp.has_right : sp.has_left;
  float4 row = empty_slot();
  uint32_t tag = kSlabFree;
  bool halo = false;
  if (has && q < cap) {
    const SlabView v = slab_view(sp.recv[side], cap);
    const uint32_t cnt = slab_received(sp, side, v, q == 0);
    if (q < cnt) {
      const uint32_t t = v.tags[q];
      const float4 r = v.rows[q];
      if (!(t & kSlabMigrant)) {
        row = r;
        tag = t;
        halo = true;
      } else if (phase == 0) {
        atomicExch(&sp.words[1], 1u);  // no particle migrates before the first step
      } else {
        // pop a free owned slot (no push runs concurrently); an empty stack is reported
        const uint32_t p = atomicSub(&sp.words[0], 1u);
        if (p == 0u || p > sp.own_cap) {
          atomicAdd(&sp.words[0], 1u);
          atomicExch(&sp.words[1], 1u);
        } else {
          slab_set_slot(d, g, sp.free_stack[p - 1u], r, t & ~kSlabMigrant);
        }
      }
    }
  } else if (has && phase == 1) {
    const uint32_t r = q - cap;
    const SlabView v = slab_view(sp.send[side], cap);
    const uint32_t cnt = min(v.hdr[0], cap);
    if (r < cnt && (v.tags[r] & kSlabMigrant)) {
      row = v.rows[r];
      tag = v.tags[r] & ~kSlabMigrant;
      halo = true;
    }
  }
  if (halo)
    slab_set_slot(d, g, slot, row, tag);
  else if (d.order[slot] != kSlabFree || finitef(d.state[slot].x))
    slab_set_slot(d, g, slot, empty_slot(), kSlabFree);
}

}  // namespace

void enqueue_slab_init(const FluidBufs& b, const SlabPlan& sp, cudaStream_t st) {
  k_slab_init<<<1, 1024, 0, st>>>(b.order, sp);
}

void enqueue_slab_pack(const FluidBufs& b, const SlabPlan& sp, const GridPlan& g, uint32_t phase, cudaStream_t st) {
  // at most sp.pack_blocks blocks: each block takes one ticket of the last-block hand-off
  const uint32_t blocks = std::min<uint32_t>(cdiv(sp.own_cap > 0 ? sp.own_cap : 1u, 256), sp.pack_blocks);
  k_slab_pack<<<blocks, 256, 0, st>>>(b, sp, g, phase);
}

void enqueue_slab_unpack(const FluidBufs& b, const SlabPlan& sp, const GridPlan& g, uint32_t phase, cudaStream_t st) {
  if (sp.halo_cap == 0) return;
  k_slab_unpack<<<cdiv(4 * sp.halo_cap, 256), 256, 0, st>>>(b, sp, g, phase);
}

}  // namespace phieng
