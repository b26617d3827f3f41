// SPH fluid step kernels for sm_100a (B200).
//
// Chain per substep (the reference's substep, crates/dynamics/src/fluid.rs:898-1136):
//   K1 keys     bucket key + bucket count per particle (rebuild_grid, :330-363)
//   K2 sort     counting sort by bucket, in-bucket rank by id = the cell lists
//               with ascending ids; the scanned counts are the K3 bucket
//               ranges, and the last kernel is the K4 gather into sorted order
//   K5 density  poly6 sum + clamp + EOS                (compute_density_pressure, :592-611)
//   K6 force    spiky pressure force (+AV, cohesion) + XSPH + cap + advect
//               + wall push-out, Jacobi reads           (:942-1094)
// K6 also writes the next substep's keys, so K1 only runs after the host
// changes the state or the bucket grid.
//
// Every neighbour walk visits, for oy = -1..1 (outer) and ox = -1..1 (inner),
// the particles of cell (cx+ox, cy+oy) in ascending id, i.e. the visit order
// of neighbors() (fluid.rs:368-386), and accumulates per thread in that order
// with no atomics, so sums are bit-identical to the reference's and runs are
// bit-reproducible.
#include <cuda_runtime.h>

#include "sph_kernels.h"
#include "sph_noise.cuh"
#include "sph_tc_net.cuh"
#include "sph_warp.cuh"

namespace phieng {

namespace {

// ---------------------------------------------------------------- K2 bucket sort
// Counting sort over the whole bucket key (a one-digit radix sort with radix
// = number of buckets), then an in-bucket rank by id, so the final order is
// exactly (key, id):
//   count   K1 / K6 add each particle to count[key] (K1 warp-aggregated,
//           K6 one atomic per particle)
//   scan    count -> start (exclusive; start doubles as the bucket range
//           table: bucket b holds slots [start[b], start[b+1])), and count
//           becomes the placement cursor
//   place   each particle takes a slot in its bucket from the cursor
//           (arrival order inside a bucket is arbitrary)
//   fixup   each particle's final slot = start[b] + (number of ids in its
//           bucket smaller than its own); gathers the state into that slot
// Buckets hold a handful of particles (a cell is h wide, the support radius),
// so the in-bucket rank is a short loop.
constexpr uint32_t kScanTile = kBucketScanTile;  // counts per scan block: 256 threads x 16

// Block-wide inclusive scan of one value per thread (256 threads).
__device__ __forceinline__ uint32_t block_incl_scan_256(uint32_t v, uint32_t* warp_tot) {
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  if (lane == 31) warp_tot[w] = x;
  __syncthreads();
  uint32_t add = 0;
  for (uint32_t k = 0; k < w; k++) add += warp_tot[k];
  return x + add;
}

// K1: key and bucket count of every particle (id order).
template <bool BATCH>
__global__ void __launch_bounds__(256) k_keys(const float4* __restrict__ state, uint32_t n, GridPlan g0,
                                              BatchTab bt, uint32_t* __restrict__ keys,
                                              uint32_t* __restrict__ count) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const GridPlan& g = BATCH ? bt.ptab[bt.pscene[i]].grid : g0;
  const float4 s = state[i];
  const uint32_t k = bucket_key(s.x, s.y, g);
  keys[i] = k;
  count_key(count, k);
}

// Sum each scan tile; the last block to finish turns the tile sums into
// exclusive tile offsets in place (no block waits on another).
__global__ void __launch_bounds__(256) k_scan_reduce(const uint32_t* __restrict__ count,
                                                     uint32_t* __restrict__ tilesum, uint32_t ntiles,
                                                     uint32_t* __restrict__ done) {
  __shared__ uint32_t warp_tot[8];
  __shared__ bool last;
  const uint32_t tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const uint4* c4 = reinterpret_cast<const uint4*>(count + (size_t)blockIdx.x * kScanTile);
  uint32_t sum = 0;
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const uint4 v = c4[r * 256 + tid];
    sum += v.x + v.y + v.z + v.w;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xFFFFFFFFu, sum, o);
  if (lane == 0) warp_tot[w] = sum;
  __syncthreads();
  if (tid == 0) {
    uint32_t t = 0;
    for (int k = 0; k < 8; k++) t += warp_tot[k];
    tilesum[blockIdx.x] = t;
    __threadfence();
    last = atomicAdd(done, 1u) + 1u == gridDim.x;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  uint32_t carry = 0;
  for (uint32_t base = 0; base < ntiles; base += 256) {
    const uint32_t i = base + tid;
    const uint32_t v = i < ntiles ? *((volatile uint32_t*)&tilesum[i]) : 0u;
    __syncthreads();  // warp_tot reuse
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
      if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) warp_tot[w] = x;
    __syncthreads();
    uint32_t add = carry;
    for (uint32_t k = 0; k < w; k++) add += warp_tot[k];
    if (i < ntiles) tilesum[i] = add + x - v;
    uint32_t chunk = 0;
    for (int k = 0; k < 8; k++) chunk += warp_tot[k];
    carry += chunk;
  }
  if (tid == 0) *done = 0;
}

// start[i] = exclusive prefix of count[i]; count[i] is overwritten with the
// same value (the placement cursor). Whole scan tiles are written with
// 16-byte stores (the arrays are padded to whole tiles); m = number of keys
// incl. the sentinel bucket, start[m] = particle count.
__global__ void __launch_bounds__(256) k_scan_down(uint32_t* __restrict__ count,
                                                   const uint32_t* __restrict__ tileoff, uint32_t m,
                                                   uint32_t* __restrict__ start) {
  __shared__ uint32_t warp_tot[8];
  const uint32_t tid = threadIdx.x;
  const uint32_t base = blockIdx.x * kScanTile + tid * 16;
  uint4* c4 = reinterpret_cast<uint4*>(count + base);
  uint32_t v[16];
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const uint4 q = c4[r];
    v[4 * r] = q.x;
    v[4 * r + 1] = q.y;
    v[4 * r + 2] = q.z;
    v[4 * r + 3] = q.w;
  }
  uint32_t sum = 0;
#pragma unroll
  for (int q = 0; q < 16; q++) sum += v[q];
  const uint32_t incl = block_incl_scan_256(sum, warp_tot);
  uint32_t run = tileoff[blockIdx.x] + incl - sum;
#pragma unroll
  for (int q = 0; q < 16; q++) {
    const uint32_t x = v[q];
    v[q] = run;
    run += x;
  }
  uint4* s4 = reinterpret_cast<uint4*>(start + base);
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const uint4 q = make_uint4(v[4 * r], v[4 * r + 1], v[4 * r + 2], v[4 * r + 3]);
    c4[r] = q;
    s4[r] = q;  // the padded tail past m gets the particle count: never read
  }
}

// Single-pass variant of k_scan_reduce + k_scan_down (decoupled look-back,
// Merrill & Garland, "Single-pass Parallel Prefix Scan with Decoupled
// Look-back", 2016), one block per supertile of kBucketScanSuper scan tiles:
// supertiles are taken in ticket order; each publishes its sum
// (flag 1) at once, then walks back over its predecessors' published values
// until it meets an inclusive prefix (flag 2), and publishes its own
// inclusive prefix. A block only waits for tiles that took an earlier ticket,
// so are already running; each wait is still bounded (kScanSpinLimit reads,
// then *err = 1 and the scan goes on with a wrong prefix). The last block to
// finish clears the tile states and counters for the next scan. ctr[0] =
// ticket, ctr[1] = finished blocks; both zero between scans. The tile whose
// ticket equals silent publishes nothing (a test of the bounded waits; the
// step passes 0xFFFFFFFF).
constexpr uint32_t kScanSpinLimit = 1u << 20;
constexpr unsigned long long kTileAgg = 1ull << 32, kTileIncl = 2ull << 32;

// Each look-back block of 256 * kLookbackSub threads scans kLookbackSub
// consecutive scan tiles (a "supertile"), 16 counts per thread: every count
// is loaded at once, as with one tile per 256-thread block, but the
// look-back chain (a block walks its predecessors 32 at a time) is
// kLookbackSub times shorter. The count arrays keep their padding to whole
// scan tiles: a thread whose tile lies past the last does nothing.
constexpr uint32_t kLookbackSub = kBucketScanSuper;
constexpr uint32_t kLookbackThreads = 256 * kLookbackSub;

// Block-wide inclusive scan of one value per thread (kLookbackThreads).
__device__ __forceinline__ uint32_t block_incl_scan_big(uint32_t v, uint32_t* warp_tot) {
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  if (lane == 31) warp_tot[w] = x;
  __syncthreads();
  uint32_t add = 0;
  for (uint32_t k = 0; k < w; k++) add += warp_tot[k];
  return x + add;
}

__global__ void __launch_bounds__(kLookbackThreads) k_scan_lookback(uint32_t* __restrict__ count, uint32_t nsub,
                                                                    uint32_t* __restrict__ start,
                                                                    unsigned long long* __restrict__ tstate,
                                                                    uint32_t* __restrict__ ctr,
                                                                    uint32_t* __restrict__ err, uint32_t silent) {
  constexpr uint32_t kWarps = kLookbackThreads / 32;
  __shared__ uint32_t warp_tot[kWarps];
  __shared__ uint32_t s_tile, s_prefix;
  __shared__ bool s_last;
  if (threadIdx.x == 0) s_tile = atomicAdd(&ctr[0], 1u);
  __syncthreads();
  const uint32_t t = s_tile;
  const bool mine = t * kLookbackSub + threadIdx.x / 256 < nsub;  // this thread's scan tile exists
  const size_t base = (size_t)t * kLookbackThreads * 16 + threadIdx.x * 16;
  uint32_t v[16];
  uint32_t sum = 0;
  if (mine) {
    const uint4* c4 = reinterpret_cast<const uint4*>(count + base);
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const uint4 q = c4[r];
      v[4 * r] = q.x;
      v[4 * r + 1] = q.y;
      v[4 * r + 2] = q.z;
      v[4 * r + 3] = q.w;
    }
#pragma unroll
    for (int q = 0; q < 16; q++) sum += v[q];
  }
  const uint32_t incl = block_incl_scan_big(sum, warp_tot);
  if (threadIdx.x < 32) {
    // warp 0: publish this supertile's sum, then look back 32 predecessors
    // at a time (lane k reads supertile t-1-k; before 0 counts as an
    // inclusive 0)
    const uint32_t lane = threadIdx.x;
    uint32_t total = 0;
    for (uint32_t k = 0; k < kWarps; k++) total += warp_tot[k];
    uint32_t excl = 0;
    if (t == 0) {
      if (lane == 0 && t != silent) atomicExch(&tstate[0], kTileIncl | total);
    } else {
      if (lane == 0 && t != silent) atomicExch(&tstate[t], kTileAgg | total);
      __syncwarp();
      volatile unsigned long long* vs = tstate;
      int64_t top = (int64_t)t - 1;
      uint32_t spins = 0;
      for (;;) {
        const int64_t idx = top - (int64_t)lane;
        unsigned long long sv;
        for (;;) {
          sv = idx >= 0 ? (unsigned long long)vs[idx] : (unsigned long long)kTileIncl;
          if (__all_sync(0xFFFFFFFFu, (sv >> 32) != 0ull)) break;
          if (++spins > kScanSpinLimit) {  // bounded: give up with a wrong prefix
            if (lane == 0) atomicExch(err, 1u);
            sv = (unsigned long long)kTileIncl;
            break;
          }
        }
        const uint32_t flag = (uint32_t)(sv >> 32);
        const uint32_t incl_lanes = __ballot_sync(0xFFFFFFFFu, flag == 2u);
        // lanes up to the nearest inclusive prefix (all 32 if none)
        const uint32_t upto = incl_lanes ? (uint32_t)(__ffs((int)incl_lanes) - 1) : 31u;
        uint32_t val = lane <= upto ? (uint32_t)sv : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) val += __shfl_xor_sync(0xFFFFFFFFu, val, o);
        excl += val;
        if (incl_lanes) break;
        top -= 32;
      }
      if (lane == 0 && t != silent) atomicExch(&tstate[t], kTileIncl | (excl + total));
    }
    if (lane == 0) s_prefix = excl;
  }
  __syncthreads();
  if (mine) {
    uint32_t run = s_prefix + incl - sum;
#pragma unroll
    for (int q = 0; q < 16; q++) {
      const uint32_t x = v[q];
      v[q] = run;
      run += x;
    }
    uint4* c4 = reinterpret_cast<uint4*>(count + base);
    uint4* s4 = reinterpret_cast<uint4*>(start + base);
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const uint4 q = make_uint4(v[4 * r], v[4 * r + 1], v[4 * r + 2], v[4 * r + 3]);
      c4[r] = q;
      s4[r] = q;  // the padded tail past the last key gets the particle count: never read
    }
  }
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(&ctr[1], 1u) + 1u == gridDim.x;
  }
  __syncthreads();
  if (s_last) {
    for (uint32_t i = threadIdx.x; i < gridDim.x; i += blockDim.x) tstate[i] = 0ull;
    if (threadIdx.x == 0) {
      ctr[0] = 0u;
      ctr[1] = 0u;
    }
  }
}

struct GatherArgs {
  const float4* state;
  const float* mass;
  const uint8_t* phase;
  float2* spos;
  float2* svel;
  float* smass;
  uint8_t* sphase;
  const uint32_t* pscene;  // batch: scene of each particle (id order), else null
  uint32_t* sscene;
};

// The particle's sorted entries at final slot f (sid only when given: the
// placement pass reads the previous sort's sid while it runs).
__device__ __forceinline__ void gather_slot(uint32_t f, uint32_t k, uint32_t id, const GatherArgs& ga,
                                            uint32_t* __restrict__ skey, uint32_t* __restrict__ sid) {
  skey[f] = k;
  if (sid) sid[f] = id;
  const float4 st = ga.state[id];
  ga.spos[f] = make_float2(st.x, st.y);
  ga.svel[f] = make_float2(st.z, st.w);
  if (ga.smass) ga.smass[f] = ga.mass[id];
  if (ga.sphase) ga.sphase[f] = ga.phase[id];
  if (ga.sscene) ga.sscene[f] = ga.pscene[id];
}

// tid entry of a slot whose particle k_place_final already put in its final
// place (ids are below 2^31)
constexpr uint32_t kPlacedFinal = 0x80000000u;

// Placement for the 2D sort, with the common case finished in place: when a
// run of equal keys in consecutive lanes is the whole bucket (its length
// equals the bucket's count) and its ids ascend lane by lane, the run's
// slots are already the final (key, id) order, so its particles are
// gathered into sorted order here and their tid entries flagged; k_fixup
// ranks only the other buckets and writes the flagged slots' sid (read here
// as the previous order). Particles keep their cell from one substep
// to the next almost always, and a bucket's particles arrive as one run in
// the previous sort's order, so most buckets finish here.
template <bool BY_SLOT>
__global__ void __launch_bounds__(256) k_place_final(const uint32_t* __restrict__ key,
                                                     const uint32_t* __restrict__ sid_prev, uint32_t n,
                                                     uint32_t* __restrict__ cursor, const uint32_t* __restrict__ start,
                                                     uint32_t* __restrict__ tkey, uint32_t* __restrict__ tid_out,
                                                     uint32_t* __restrict__ skey, const uint32_t* __restrict__ order,
                                                     GatherArgs ga) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const uint32_t id = BY_SLOT ? sid_prev[s] : s;
  const uint32_t k = key[id];
  const uint32_t act = __activemask();  // a prefix of the warp's lanes
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t first, len, rank;
  key_run(act, k, lane, &first, &len, &rank);
  uint32_t base = 0;
  if (first == lane) base = atomicAdd(&cursor[k], len);
  base = __shfl_sync(act, base, first);
  const uint32_t slot = base + rank;
  const uint32_t tag = order ? __ldg(&order[id]) : id;
  const uint32_t ptag = __shfl_sync(act, tag, lane ? lane - 1u : 0u);
  const bool asc = lane == first || ptag < tag;
  const uint32_t bad = __ballot_sync(act, !asc);
  const uint32_t run = (len >= 32u ? 0xFFFFFFFFu : ((1u << len) - 1u)) << first;
  if (len == __ldg(&start[k + 1]) - __ldg(&start[k]) && (bad & run) == 0u) {
    gather_slot(slot, k, id, ga, skey, nullptr);
    tid_out[slot] = id | kPlacedFinal;
  } else {
    tkey[slot] = k;
    tid_out[slot] = id;
  }
}

// Slot in the bucket from the cursor. BY_SLOT walks the previous sort's
// order (keys nearly sorted: a warp holds few runs of equal keys, so few
// atomics); otherwise particles are taken in id order.
template <bool BY_SLOT>
__global__ void __launch_bounds__(256) k_place(const uint32_t* __restrict__ key,
                                               const uint32_t* __restrict__ sid_prev, uint32_t n,
                                               uint32_t* __restrict__ cursor, uint32_t* __restrict__ tkey,
                                               uint32_t* __restrict__ tid_out) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const uint32_t id = BY_SLOT ? sid_prev[s] : s;
  const uint32_t k = key[id];
  // one atomic per run of equal keys in consecutive lanes; a run's lanes take
  // consecutive slots (any order inside a bucket is fine: k_fixup ranks by id)
  const uint32_t act = __activemask();
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t first, len, rank;
  key_run(act, k, lane, &first, &len, &rank);
  uint32_t base = 0;
  if (first == lane) base = atomicAdd(&cursor[k], len);
  base = __shfl_sync(act, base, first);
  const uint32_t slot = base + rank;
  tkey[slot] = k;
  tid_out[slot] = id;
}

// Final slot = bucket start + rank of the id (or its order tag) among the
// bucket's; the particle's state is gathered into that slot. With order
// tags, the sentinel bucket of non-finite particles keeps its placement
// slots: no walk visits it, and its size (a rank world's unused slots) would
// make ranking quadratic.
__device__ __forceinline__ void fixup_slot(uint32_t s, uint32_t id, const uint32_t* __restrict__ tkey,
                                           const uint32_t* __restrict__ tid_in, const uint32_t* __restrict__ start,
                                           uint32_t* __restrict__ skey, uint32_t* __restrict__ sid,
                                           const uint32_t* __restrict__ order, uint32_t sentinel,
                                           const GatherArgs& ga) {
  if (id & kPlacedFinal) {  // k_place_final finished this bucket but its sid
    sid[s] = id & ~kPlacedFinal;
    return;
  }
  const uint32_t k = tkey[s];
  const uint32_t lo = start[k], hi = start[k + 1];
  uint32_t rank = 0;
  if (order) {
    if (k == sentinel) {
      gather_slot(s, k, id, ga, skey, sid);
      return;
    }
    const uint32_t tag = __ldg(&order[id]);
    for (uint32_t j = lo; j < hi; j++) rank += __ldg(&order[__ldg(&tid_in[j])]) < tag ? 1u : 0u;
  } else {
    for (uint32_t j = lo; j < hi; j++) rank += __ldg(&tid_in[j]) < id ? 1u : 0u;
  }
  gather_slot(lo + rank, k, id, ga, skey, sid);
}

// SLOTS = 4: four slots per thread; where all four were finished by
// k_place_final (the common case) one 16-byte load and store, the others one
// by one. SLOTS = 1: one slot per thread. The same threads clear the bucket
// counts for the next sort (the placement, which used them as cursors, has
// finished): count_len is a multiple of the scan tile, so whole uint4 stores.
template <int SLOTS>
__global__ void __launch_bounds__(256) k_fixup(const uint32_t* __restrict__ tkey,
                                               const uint32_t* __restrict__ tid_in,
                                               const uint32_t* __restrict__ start, uint32_t n,
                                               uint32_t* __restrict__ skey, uint32_t* __restrict__ sid,
                                               const uint32_t* __restrict__ order, uint32_t sentinel,
                                               uint32_t* __restrict__ count, uint32_t count_len, GatherArgs ga) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (4u * t < count_len) reinterpret_cast<uint4*>(count)[t] = make_uint4(0u, 0u, 0u, 0u);
  if constexpr (SLOTS == 1) {
    if (t < n) fixup_slot(t, tid_in[t], tkey, tid_in, start, skey, sid, order, sentinel, ga);
    return;
  }
  const uint32_t s0 = 4u * t;
  if (s0 >= n) return;
  if (s0 + 3u < n) {
    const uint4 v = *reinterpret_cast<const uint4*>(tid_in + s0);
    if ((v.x & v.y & v.z & v.w) & kPlacedFinal) {
      *reinterpret_cast<uint4*>(sid + s0) =
          make_uint4(v.x & ~kPlacedFinal, v.y & ~kPlacedFinal, v.z & ~kPlacedFinal, v.w & ~kPlacedFinal);
      return;
    }
    const uint32_t ids[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int q = 0; q < 4; q++) fixup_slot(s0 + q, ids[q], tkey, tid_in, start, skey, sid, order, sentinel, ga);
    return;
  }
  for (uint32_t s = s0; s < n; s++) fixup_slot(s, tid_in[s], tkey, tid_in, start, skey, sid, order, sentinel, ga);
}

// ---------------------------------------------------------------- neighbour walk
// Visit every candidate slot j of the particle in bucket `key`, in the
// reference's order (cell rows oy = -1..1, then cells ox = -1..1, then
// ascending id). Bucket b holds slots [start[b], start[b + 1]); away from
// the wrap seam the three buckets of a row are consecutive keys, hence one
// contiguous slot range.
template <class F>
__device__ __forceinline__ void for_each_candidate(uint32_t key, const uint32_t* __restrict__ start,
                                                   const GridPlan& g, F&& f) {
  const uint32_t local = key - g.base;
  const uint32_t bx = local & g.maskw, by = local >> g.log2w;
#pragma unroll 1
  for (int oy = -1; oy <= 1; oy++) {
    const uint32_t row = g.base + (((by + (uint32_t)oy) & g.maskh) << g.log2w);
    if (bx >= 1u && bx < g.maskw) {
      const uint32_t b0 = row + bx - 1;
      const uint32_t e = __ldg(&start[b0 + 3]);
      for (uint32_t j = __ldg(&start[b0]); j < e; j++) f((int)j);
    } else {
#pragma unroll 1
      for (int ox = -1; ox <= 1; ox++) {
        const uint32_t b = row + ((bx + (uint32_t)ox) & g.maskw);
        const uint32_t e = __ldg(&start[b + 1]);
        for (uint32_t j = __ldg(&start[b]); j < e; j++) f((int)j);
      }
    }
  }
}

// ---------------------------------------------------------------- K5 density
// Per-row neighbour masks: for the candidate row oy (0..2 for oy = -1..1) of
// a particle away from the wrap seam, bit t of nmask[oy * n + s] is set iff
// slot (row start + t) is a neighbour (d2 < h*h, the particle itself
// included). A zero mask for the particle's own row (which always holds the
// particle itself) means "no masks": the row was longer than 32 slots (rows
// hold ~12 candidates at rest density) or the particle sits on the seam, and
// K6 walks the candidates itself.
constexpr uint32_t kMaskBits = 32;

// Candidate j's density contribution m_j * poly6(d2) when d2 < h*h, else +0
// (adding +0 to a non-negative sum is exact, so skipping and adding agree).
__device__ __forceinline__ float density_term(float d2, float m, const StepParams& P) {
  return d2 < P.hg2 ? __fmul_rn(m, poly6(d2, P)) : 0.0f;
}

// m_j * poly6(d2) for a candidate known to be a neighbour (poly6_nb).
template <bool WIDE>
__device__ __forceinline__ float neighbour_density_term(float d2, float m, const StepParams& P) {
  return __fmul_rn(m, poly6_nb<WIDE>(d2, P));
}

template <bool MASS, bool PHASE, bool BATCH, bool WIDE>
__global__ void __launch_bounds__(256) k_density(const float2* __restrict__ spos, const uint32_t* __restrict__ skey,
                                                 const float* __restrict__ smass,
                                                 const uint8_t* __restrict__ sphase, uint32_t n,
                                                 const uint32_t* __restrict__ start, StepParams P0, BatchTab bt,
                                                 float2* __restrict__ sdq, float* __restrict__ spres,
                                                 uint32_t* __restrict__ nmask, float2* __restrict__ svp) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const StepParams& P = scene_params<BATCH>(P0, bt.ptab, BATCH ? bt.sscene[s] : 0u);
  const uint32_t k = skey[s];
  const float2 pi = spos[s];
  float rho = 0.0f;
  uint32_t mrow[3] = {0, 0, 0};
  const GridPlan& g = P.grid;
  if (k != g.sentinel) {
    const uint32_t local = k - g.base;
    const uint32_t bx = local & g.maskw, by = local >> g.log2w;
    const bool seam = !(bx >= 1u && bx < g.maskw);
    bool masks_ok = !seam;
#pragma unroll
    for (int oy = 0; oy < 3; oy++) {
      const uint32_t row = g.base + (((by + (uint32_t)oy - 1u) & g.maskh) << g.log2w);
      if (!seam) {
        const uint32_t rs = __ldg(&start[row + bx - 1]);
        const uint32_t re = __ldg(&start[row + bx + 2]);
        uint32_t m = 0, bit = 1u;  // bit shifts out after 32 slots (then masks_ok is false)
        for (uint32_t j = rs; j < re; j++) {
          const float2 a = __ldg(&spos[j]);
          const float dx = __fsub_rn(a.x, pi.x), dy = __fsub_rn(a.y, pi.y);
          const float d2 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
          const bool nb = d2 < P.hg2;
          const float w = neighbour_density_term<WIDE>(d2, MASS ? __ldg(&smass[j]) : P.mass, P);
          rho = nb ? __fadd_rn(rho, w) : rho;
          m |= nb ? bit : 0u;
          bit <<= 1;
        }
        mrow[oy] = m;
        if (re - rs > kMaskBits) masks_ok = false;
      } else {
#pragma unroll 1
        for (int ox = -1; ox <= 1; ox++) {
          const uint32_t bb = row + ((bx + (uint32_t)ox) & g.maskw);
          const uint32_t e = __ldg(&start[bb + 1]);
          for (uint32_t j = __ldg(&start[bb]); j < e; j++) {
            const float2 a = __ldg(&spos[j]);
            const float dx = __fsub_rn(a.x, pi.x), dy = __fsub_rn(a.y, pi.y);
            const float d2 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
            rho = __fadd_rn(rho, density_term(d2, MASS ? __ldg(&smass[j]) : P.mass, P));
          }
        }
      }
    }
    if (!masks_ok) mrow[1] = 0;  // K6 walks the candidates itself
  }
  nmask[s] = mrow[0];
  nmask[n + s] = mrow[1];
  nmask[2 * (size_t)n + s] = mrow[2];
  // f32::clamp(0, 3 * max(rest_density, EPS)) (fluid.rs:605)
  float dens = rho;
  if (dens < 0.0f) dens = 0.0f;
  if (dens > P.rho_cap) dens = P.rho_cap;
  const uint32_t ph = PHASE ? min((uint32_t)sphase[s], 3u) : P.uniform_phase;
  const float p = eos(dens, P.rest[ph], P);
  const float rc = fmaxf(dens, kEps);
  const float q = __fdiv_rn(p, __fmul_rn(rc, rc));
  sdq[s] = make_float2(dens, q);
  spres[s] = p;
  // closure passes: the per-neighbour factors of the feature sums, once per
  // particle instead of once per pair (same expressions as feat_pair's)
  if (svp) svp[s] = make_float2(__fdiv_rn(MASS ? smass[s] : P.mass, rc), __fmul_rn(__fmul_rn(q, rc), rc));
}

// ---------------------------------------------------------------- K6 force + integrate
// One neighbour pair of the force loop (fluid.rs:947-990) and of the XSPH
// sum (fluid.rs:1022-1033), accumulated in the reference's order. FEAT also
// accumulates the closure network's neighbour aggregates (feat_pair). PLAIN:
// the launch's flags are known to be XSPH on, artificial viscosity and
// cohesion off, h*h <= hk*hk (plain_flags), so those tests are compiled out.
template <bool MASS, bool FEAT, bool PLAIN = false>
__device__ __forceinline__ void pair_terms(uint32_t j, float2 pi, float2 vi, float rho_i, float q_i, float m_i,
                                           const float2* __restrict__ spos, const float2* __restrict__ svel,
                                           const float2* __restrict__ sdq, const float* __restrict__ smass,
                                           const float2* __restrict__ svp, const StepParams& P, float& fx,
                                           float& fy, float& sx, float& sy, FeatAcc& fa) {
  const float2 pj = __ldg(&spos[j]);
  const float2 dqj = __ldg(&sdq[j]);
  const float2 vj = __ldg(&svel[j]);
  const float m_j = MASS ? __ldg(&smass[j]) : P.mass;
  const float rho_j = fmaxf(dqj.x, kEps);
  // delta = p_i - p_j; |delta|^2 equals the neighbour test's d2 bit for bit
  const float dx = __fsub_rn(pi.x, pj.x);
  const float dy = __fsub_rn(pi.y, pj.y);
  const float d2 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
  const float dist = __fsqrt_rn(d2);
  // spiky gradient (fluid.rs:278-285)
  float gxx = 0.0f, gyy = 0.0f;
  if (!(dist >= P.hk || dist < kEps)) {
    const float hr = __fsub_rn(P.hk, dist);
    const float sc = __fmul_rn(__fmul_rn(P.c_spiky, hr), hr);
    gxx = __fmul_rn(__fdiv_rn(dx, dist), sc);
    gyy = __fmul_rn(__fdiv_rn(dy, dist), sc);
  }
  if constexpr (FEAT) {
    // PLAIN: d2 < hg2 <= hk2, so poly6's range test passes (and the XSPH
    // term's poly6_nb is the same value)
    const float2 vp = __ldg(&svp[j]);
    feat_pair<!PLAIN>(fa, gxx, gyy, PLAIN ? poly6_nb<false>(d2, P) : poly6(d2, P), vp.x, vp.y, m_j, q_i, dqj.y,
                      __fsub_rn(vj.x, vi.x), __fsub_rn(vj.y, vi.y));
  }
  float term = __fadd_rn(q_i, dqj.y);
  if (!PLAIN && (P.flags & F_AV) && dist > kEps) {
    // Monaghan term (fluid.rs:302-317, called at :963-975)
    const float rho_bar = __fmul_rn(0.5f, __fadd_rn(rho_i, rho_j));
    const float vrx = __fsub_rn(vi.x, vj.x), vry = __fsub_rn(vi.y, vj.y);
    const float vd = __fadd_rn(__fmul_rn(vrx, dx), __fmul_rn(vry, dy));
    if (!(vd >= 0.0f)) {
      const float r_sq = __fmul_rn(dist, dist);
      const float mu =
          __fdiv_rn(__fmul_rn(P.hk, vd), __fadd_rn(r_sq, __fmul_rn(__fmul_rn(0.01f, P.hk), P.hk)));
      const float ap = __fdiv_rn(__fmul_rn(__fmul_rn(-P.av_alpha, P.c_s), mu), fmaxf(rho_bar, kEps));
      term = __fadd_rn(term, ap);
    }
  }
  const float mt = __fmul_rn(m_j, term);
  fx = __fsub_rn(fx, __fmul_rn(gxx, mt));
  fy = __fsub_rn(fy, __fmul_rn(gyy, mt));
  if (!PLAIN && (P.flags & F_COHESION) && dist > kEps) {
    // cohesion (fluid.rs:320-326, applied at :979-985)
    const float c = dist >= P.hk ? 0.0f : __fsub_rn(1.0f, __fdiv_rn(dist, P.hk));
    if (c > 0.0f) {
      const float sc = __fmul_rn(__fmul_rn(__fmul_rn(P.surface_tension, m_i), m_j), c);
      fx = __fsub_rn(fx, __fmul_rn(__fdiv_rn(dx, dist), sc));
      fy = __fsub_rn(fy, __fmul_rn(__fdiv_rn(dy, dist), sc));
    }
  }
  if (PLAIN || (P.flags & F_VISC)) {
    // XSPH (fluid.rs:1022-1033) against pre-integrate neighbours
    const float rho_bar = __fmul_rn(0.5f, __fadd_rn(rho_i, rho_j));
    const float w = PLAIN ? poly6_nb<false>(d2, P) : poly6(d2, P);
    const float mr = __fdiv_rn(m_j, rho_bar);
    sx = __fadd_rn(sx, __fmul_rn(__fmul_rn(__fsub_rn(vj.x, vi.x), mr), w));
    sy = __fadd_rn(sy, __fmul_rn(__fmul_rn(__fsub_rn(vj.y, vi.y), mr), w));
  }
}

// Neighbour sums of sorted slot s: pressure force (fx, fy) and XSPH (sx, sy),
// plus the closure aggregates when FEAT. The neighbour set comes from K5's
// row masks (bits in ascending slot order = the reference's visit order);
// particles without masks walk the candidates.
template <bool MASS, bool FEAT, bool PLAIN = false>
__device__ __forceinline__ void neighbour_sums(uint32_t s, uint32_t k, uint32_t n, float2 pi, float2 vi, float rho_i,
                                               float q_i, float m_i, const float2* __restrict__ spos,
                                               const float2* __restrict__ svel, const float2* __restrict__ sdq,
                                               const float* __restrict__ smass, const float2* __restrict__ svp,
                                               const uint32_t* __restrict__ start,
                                               const uint32_t* __restrict__ nmask, const StepParams& P, float& fx,
                                               float& fy, float& sx, float& sy, FeatAcc& fa) {
  const GridPlan& g = P.grid;
  if (k == g.sentinel) return;
  const uint32_t local = k - g.base;
  const uint32_t bx = local & g.maskw, by = local >> g.log2w;
  const uint32_t own = nmask[n + s];
  if (own != 0u) {
    // one loop over the three rows' set bits (ascending slots, row by row)
    const uint32_t rs0 = __ldg(&start[g.base + (((by - 1u) & g.maskh) << g.log2w) + bx - 1]);
    const uint32_t rs1 = __ldg(&start[g.base + ((by & g.maskh) << g.log2w) + bx - 1]);
    const uint32_t rs2 = __ldg(&start[g.base + (((by + 1u) & g.maskh) << g.log2w) + bx - 1]);
    const uint32_t m0 = nmask[s], m2 = nmask[2 * (size_t)n + s];
    // the particle's own bit (its slot in its own row, < 32 when the masks
    // are valid) is cleared: j != i (fluid.rs:947-950)
    const uint32_t own_nb = own & ~(1u << (s - rs1));
    uint32_t cur = m0;
    uint32_t row = 0, base = rs0;
    for (;;) {
      while (cur == 0u && row < 2) {
        row++;
        cur = row == 1 ? own_nb : m2;
        base = row == 1 ? rs1 : rs2;
      }
      if (cur == 0u) break;
      const uint32_t j = base + (uint32_t)(__ffs((int)cur) - 1);
      cur &= cur - 1u;
      pair_terms<MASS, FEAT, PLAIN>(j, pi, vi, rho_i, q_i, m_i, spos, svel, sdq, smass, svp, P, fx, fy, sx, sy, fa);
    }
  } else {
    for_each_candidate(k, start, g, [&](int jj) {
      const uint32_t j = (uint32_t)jj;
      const float2 pj = __ldg(&spos[j]);
      const float ex = __fsub_rn(pj.x, pi.x);
      const float ey = __fsub_rn(pj.y, pi.y);
      const float d2 = __fadd_rn(__fmul_rn(ex, ex), __fmul_rn(ey, ey));
      if (d2 < P.hg2 && j != s)
        pair_terms<MASS, FEAT, PLAIN>(j, pi, vi, rho_i, q_i, m_i, spos, svel, sdq, smass, svp, P, fx, fy, sx, sy, fa);
    });
  }
}

// integrate (fluid.rs:1003-1050) from acceleration (ax, ay) and the XSPH sum,
// then the wall pass; writes the new state, the next key and its bucket count.
// Ambient turbulence (F_TURB) joins the acceleration first, at the particle's
// pre-step position and the step's world clock. EXTRA = false compiles it and
// the polygon wall test out (the PLAIN variants, whose flags exclude both).
template <bool EXTRA = true>
__device__ __forceinline__ void integrate_write(uint32_t id, float2 pi, float2 vi, float ax, float ay, float sx,
                                                float sy, const StepParams& P, const DevBody* __restrict__ bodies,
                                                float4* __restrict__ state_out, uint32_t* __restrict__ key_out,
                                                uint32_t* __restrict__ count_out,
                                                uint32_t* __restrict__ defer = nullptr,
                                                uint32_t* __restrict__ dcount = nullptr) {
  if (EXTRA && (P.flags & F_TURB)) {
    const float2 tb = turbulence_accel(pi.x, pi.y, *P.clock, P.turb_freq, P.turb_tscale, P.turb_seed, P.turb_oct,
                                       P.flags & F_TURB_CURL, P.turb_amp);
    ax = __fadd_rn(ax, tb.x);
    ay = __fadd_rn(ay, tb.y);
  }
  float vx = __fadd_rn(vi.x, __fmul_rn(ax, P.dt));
  float vy = __fadd_rn(vi.y, __fmul_rn(ay, P.dt));
  if (P.flags & F_VISC) {
    vx = __fadd_rn(vx, __fmul_rn(sx, P.visc));
    vy = __fadd_rn(vy, __fmul_rn(sy, P.visc));
  }
  const float speed = __fsqrt_rn(__fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy)));
  if (speed > P.vmax) {
    const float sc = __fdiv_rn(P.vmax, speed);
    vx = __fmul_rn(vx, sc);
    vy = __fmul_rn(vy, sc);
  }
  if (!finitef(vx) || !finitef(vy)) {
    vx = 0.0f;
    vy = 0.0f;
  }
  float x = __fadd_rn(pi.x, __fmul_rn(vx, P.dt));
  float y = __fadd_rn(pi.y, __fmul_rn(vy, P.dt));
  if (!finitef(x) || !finitef(y)) {
    x = pi.x;
    y = pi.y;
  }
  const uint32_t r = walls<EXTRA>(x, y, vx, vy, bodies, P);
  state_out[id] = make_float4(x, y, vx, vy);
  if (P.flags & F_DYNAMIC) {
    // contacts with bodies that react run in particle order (enqueue_dynamic_walls)
    dcount[id] = r != kNoDefer ? 1u : 0u;
    if (r != kNoDefer) {
      defer[id] = r;
      return;
    }
  }
  const uint32_t nk = bucket_key(x, y, P.grid);
  key_out[id] = nk;
  // bucket counts of the next substep's sort: one atomic per particle (the
  // warp-aggregated count_key measured 1.8 us slower per 2^20-particle
  // launch here, where its match and election outweigh the atomics saved)
  atomicAdd(&count_out[nk], 1u);
}

// ---------------------------------------------------------------- boundary ghosts
// Ghost pressure on a fluid particle (fluid.rs:977-988): after its fluid
// pairs, every ghost within h of it, visited as boundary_near does (cells
// (floor(x / h) + ox, floor(y / h) + oy) for oy, ox = -1..1, h the config's
// smoothing length; each cell's ghosts in generation order), adds
// -grad W(p_i - g) * (m_g * (q_i + q_g)). Out of line: only worlds with
// ghosts pay for it.
static __device__ __noinline__ float2 ghost_force(float px, float py, float q_i, float fx, float fy,
                                                  const float2* __restrict__ gpos, const float* __restrict__ gq,
                                                  const GhostCell* __restrict__ tab, uint32_t mask, float gmass,
                                                  float hg, float hg2, float hk, float c_spiky) {
  const int32_t cx = __float2int_rd(__fdiv_rn(px, hg)), cy = __float2int_rd(__fdiv_rn(py, hg));
  for (int oy = -1; oy <= 1; oy++) {
    for (int ox = -1; ox <= 1; ox++) {
      const int32_t qx = (int32_t)((uint32_t)cx + (uint32_t)ox), qy = (int32_t)((uint32_t)cy + (uint32_t)oy);
      uint32_t slot = ghost_cell_hash(qx, qy, mask);
      GhostCell c = tab[slot];
      for (uint32_t probe = 0; probe <= mask && c.count != 0 && (c.cx != qx || c.cy != qy); probe++) {
        slot = (slot + 1) & mask;
        c = tab[slot];
      }
      if (c.count == 0 || c.cx != qx || c.cy != qy) continue;
      for (uint32_t k = c.start; k < c.start + c.count; k++) {
        const float2 g = gpos[k];
        const float ex = __fsub_rn(g.x, px), ey = __fsub_rn(g.y, py);
        if (!(__fadd_rn(__fmul_rn(ex, ex), __fmul_rn(ey, ey)) < hg2)) continue;
        const float dx = __fsub_rn(px, g.x), dy = __fsub_rn(py, g.y);
        const float dist = __fsqrt_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)));
        float gx = 0.0f, gy = 0.0f;  // spiky_grad, zero outside (EPS, h) (fluid.rs:278-285)
        if (!(dist >= hk || dist < kEps)) {
          const float hr = __fsub_rn(hk, dist);
          const float sc = __fmul_rn(__fmul_rn(c_spiky, hr), hr);
          gx = __fmul_rn(__fdiv_rn(dx, dist), sc);
          gy = __fmul_rn(__fdiv_rn(dy, dist), sc);
        }
        const float mt = __fmul_rn(gmass, __fadd_rn(q_i, gq[k]));
        fx = __fsub_rn(fx, __fmul_rn(gx, mt));
        fy = __fsub_rn(fy, __fmul_rn(gy, mt));
      }
    }
  }
  return make_float2(fx, fy);
}

// Ghost density and pressure from the fluid (compute_boundary_density_pressure,
// fluid.rs:804-818): the fluid candidates around the ghost in the reference's
// cell order, m_j * poly6 for those within h; density clamped to
// [0, 3 max(rest, EPS)], the pressure from the unclamped sum with the
// config's rest density; stored as q = p / max(density, EPS)^2.
__global__ void __launch_bounds__(256) k_ghost_density(const float2* __restrict__ spos,
                                                       const float* __restrict__ smass,
                                                       const uint32_t* __restrict__ start, StepParams P) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= P.nghost) return;
  const float2 b = P.gpos[g];
  float rho = 0.0f;
  const uint32_t key = bucket_key(b.x, b.y, P.grid);
  if (key != P.grid.sentinel) {
    const bool mass = (P.flags & F_MASS) != 0;
    for_each_candidate(key, start, P.grid, [&](int j) {
      const float2 a = __ldg(&spos[j]);
      const float dx = __fsub_rn(a.x, b.x), dy = __fsub_rn(a.y, b.y);
      rho = __fadd_rn(rho, density_term(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)),
                                        mass ? __ldg(&smass[j]) : P.mass, P));
    });
  }
  float dens = rho;
  if (dens < 0.0f) dens = 0.0f;
  if (dens > P.rho_cap) dens = P.rho_cap;
  const float p = eos(rho, P.rest0, P);
  const float rc = fmaxf(dens, kEps);
  P.gq[g] = __fdiv_rn(p, __fmul_rn(rc, rc));
}

template <bool MASS, bool DEBUG, bool BATCH, bool PLAIN>
__global__ void __launch_bounds__(256) k_force_integrate(
    const float2* __restrict__ spos, const float2* __restrict__ svel, const float2* __restrict__ sdq,
    const uint32_t* __restrict__ skey, const uint32_t* __restrict__ sid, const float* __restrict__ smass,
    uint32_t n, const uint32_t* __restrict__ start, StepParams P0, BatchTab bt, const DevBody* __restrict__ bodies,
    const uint32_t* __restrict__ nmask, float4* __restrict__ state_out, uint32_t* __restrict__ key_out,
    uint32_t* __restrict__ count_out, float2* __restrict__ dbg_force, uint32_t* __restrict__ defer,
    uint32_t* __restrict__ dcount) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const StepParams& P = scene_params<BATCH>(P0, bt.ptab, BATCH ? bt.sscene[s] : 0u);
  const uint32_t k = skey[s];
  const uint32_t id = sid[s];
  const float2 pi = spos[s];
  const float2 vi = svel[s];
  const float2 dqi = sdq[s];
  const float m_i = MASS ? smass[s] : P.mass;
  const float rho_i = fmaxf(dqi.x, kEps);
  const float q_i = dqi.y;  // p_i / (rho_i * rho_i)
  float fx = 0.0f, fy = 0.0f, sx = 0.0f, sy = 0.0f;
  FeatAcc fa;
  neighbour_sums<MASS, false, PLAIN>(s, k, n, pi, vi, rho_i, q_i, m_i, spos, svel, sdq, smass, nullptr, start, nmask,
                                     P, fx, fy, sx, sy, fa);
  if (!BATCH && !PLAIN && (P.flags & F_GHOST)) {  // PLAIN launches exclude F_GHOST (plain_flags)
    const float2 f = ghost_force(pi.x, pi.y, q_i, fx, fy, P.gpos, P.gq, P.gtab, P.gtab_mask, P.gmass, P.grid.hg,
                                 P.hg2, P.hk, P.c_spiky);
    fx = f.x;
    fy = f.y;
  }
  if (DEBUG) {
    dbg_force[id] = make_float2(fx, fy);
    return;
  }
  const float ax = __fadd_rn(P.gx, __fdiv_rn(fx, rho_i));
  const float ay = __fadd_rn(P.gy, __fdiv_rn(fy, rho_i));
  integrate_write<!PLAIN>(id, pi, vi, ax, ay, sx, sy, P, bodies, state_out, key_out, count_out, defer, dcount);
}

// ---------------------------------------------------------------- closure force pass
// The coarse step of the learned closure: the K6 neighbour pass also
// accumulates the 16 closure features; each warp then runs the closure
// network on its 32 particles on the tensor cores (two 16-row tiles) and the
// integrate adds the predicted acceleration correction
//   a_corr = y * out_scale * (h / dt^2)   (h, dt of the particle's scene)
// (the network predicts the displacement correction over the coarse step in
// units of h). It also keeps the pre-step state and density by id for the
// fallback and the density-jump check.
// FEATURES mode only writes the features (id order, 16 floats per particle)
// for the coarse step P.dt and leaves the state untouched. PLAIN as for K6
// (plain_flags); both variants give the same features and state.
// io.svp: the density pass's per-particle closure factors of this sort.
constexpr int kModeFeatures = 1;
constexpr int kModeClosure = 2;
constexpr int kXRow = 24;  // BF16 elements per staged feature row (16 + pad)

// 4 blocks per SM (64 registers, a few bytes spilled): 171 -> 152 us per
// coarse step at 2^20 particles against 3 blocks (80 registers, no spills).
template <bool MASS, bool PHASE, bool BATCH, bool PLAIN, int MODE>
__global__ void __launch_bounds__(256, 4) k_force_closure(
    const float2* __restrict__ spos, const float2* __restrict__ svel, const float2* __restrict__ sdq,
    const float* __restrict__ spres, const uint32_t* __restrict__ skey, const uint32_t* __restrict__ sid,
    const float* __restrict__ smass, const uint8_t* __restrict__ sphase, uint32_t n,
    const uint32_t* __restrict__ start, StepParams P0, BatchTab bt, const DevBody* __restrict__ bodies,
    const uint32_t* __restrict__ nmask, MlpDev mlp, ClosureIO io, float4* __restrict__ state_out,
    uint32_t* __restrict__ key_out, uint32_t* __restrict__ count_out) {
  extern __shared__ __align__(16) unsigned char closure_smem[];
  MlpSmem& sm = *reinterpret_cast<MlpSmem*>(closure_smem);
  __nv_bfloat16* sx_all = reinterpret_cast<__nv_bfloat16*>(closure_smem + sizeof(MlpSmem));
  float* sy_all = reinterpret_cast<float*>(closure_smem + sizeof(MlpSmem) + sizeof(__nv_bfloat16) * 256 * kXRow);
  if constexpr (MODE == kModeClosure) {
    mlp_load_smem(sm, mlp);
    __syncthreads();
  }
  const uint32_t s0 = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = s0 < n;
  if (MODE == kModeFeatures && !active) return;
  const uint32_t s = active ? s0 : 0u;  // idle lanes of the last warp run the network on slot 0's data
  const StepParams& P = scene_params<BATCH>(P0, bt.ptab, BATCH ? bt.sscene[s] : 0u);
  const uint32_t k = skey[s];
  const uint32_t id = sid[s];
  const float2 pi = spos[s];
  const float2 vi = svel[s];
  const float2 dqi = sdq[s];
  const float m_i = MASS ? smass[s] : P.mass;
  const float rho_i = fmaxf(dqi.x, kEps);
  const float q_i = dqi.y;
  float fx = 0.0f, fy = 0.0f, sx = 0.0f, sy = 0.0f;
  FeatAcc fa;
  neighbour_sums<MASS, true, PLAIN>(s, k, n, pi, vi, rho_i, q_i, m_i, spos, svel, sdq, smass, io.svp, start, nmask,
                                    P, fx, fy, sx, sy, fa);
  if constexpr (PLAIN) {
    fa.px = fx;  // the force sum is the pressure sum alone (feat_pair<false>)
    fa.py = fy;
  }
  const uint32_t ph = PHASE ? min((uint32_t)sphase[s], 3u) : P.uniform_phase;
  float wd, wnx, wny;
  wall_feature(pi.x, pi.y, bodies, P, wd, wnx, wny);
  float f[kFeat];
  feat_finish(fa, dqi.x, rho_i, spres[s], P.rest[ph], vi.x, vi.y, wd, wnx, wny, P, f);
  if constexpr (MODE == kModeFeatures) {
    float4* o = reinterpret_cast<float4*>(io.feat + (size_t)id * kFeat);
#pragma unroll
    for (int q = 0; q < 4; q++) o[q] = make_float4(f[4 * q], f[4 * q + 1], f[4 * q + 2], f[4 * q + 3]);
    return;
  } else {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __nv_bfloat16* xs = sx_all + warp * 32 * kXRow;
    float* ys = sy_all + warp * 64;
    mlp_normalise_row(f, sm.norm, xs + lane * kXRow);
    __syncwarp();
#pragma unroll
    for (int mt = 0; mt < 2; mt++) {
      float y[4];
      mlp_tile_forward(xs + mt * 16 * kXRow, kXRow, sm, lane, y);
      if ((lane & 3) == 0) {
        const int r = mt * 16 + (lane >> 2);
        ys[2 * r] = y[0];
        ys[2 * r + 1] = y[1];
        ys[2 * (r + 8)] = y[2];
        ys[2 * (r + 8) + 1] = y[3];
      }
    }
    __syncwarp();
    if (!active) return;
    const float acc_scale = __fdiv_rn(P.hk, __fmul_rn(P.dt, P.dt));  // h / dt^2 of this particle's scene
    const float cx = __fmul_rn(__fmul_rn(ys[2 * lane], sm.norm[2 * kFeat]), acc_scale);
    const float cy = __fmul_rn(__fmul_rn(ys[2 * lane + 1], sm.norm[2 * kFeat + 1]), acc_scale);
    io.save[id] = make_float4(pi.x, pi.y, vi.x, vi.y);
    io.rho_prev[id] = dqi.x;
    const float ax = __fadd_rn(__fadd_rn(P.gx, __fdiv_rn(fx, rho_i)), cx);
    const float ay = __fadd_rn(__fadd_rn(P.gy, __fdiv_rn(fy, rho_i)), cy);
    integrate_write<!PLAIN>(id, pi, vi, ax, ay, sx, sy, P, bodies, state_out, key_out, count_out);
  }
}

// Density checks of a coarse step, over the new sorted state after its
// density pass, each as a maximum over particles (negative values count as
// 0, a NaN as +inf): out[0] = largest per-particle density increase over the
// step, (rho'_i - rho_i) / rho0; out[1] = largest compression after the step,
// rho'_i / rho0 - 1; out[2] = largest compression before it. Float bits,
// atomicMax (all values >= 0, so the bit order is the value order and the
// maxima do not depend on the order of the atomics).
template <bool PHASE, bool BATCH>
__global__ void __launch_bounds__(256) k_closure_check(const float2* __restrict__ sdq, const uint32_t* __restrict__ sid,
                                                       const uint8_t* __restrict__ sphase, uint32_t n, StepParams P0,
                                                       BatchTab bt, const float* __restrict__ rho_prev,
                                                       unsigned int* __restrict__ out) {
  __shared__ float red[3][8];
  float v[3] = {0.0f, 0.0f, 0.0f};
  // grid-stride, then warp and block maxima: one atomic per block and value
  // (per-warp atomics on three addresses serialised to ~67 us at 2^20)
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const StepParams& P = scene_params<BATCH>(P0, bt.ptab, BATCH ? bt.sscene[s] : 0u);
    const uint32_t ph = PHASE ? min((uint32_t)sphase[s], 3u) : P.uniform_phase;
    const float r0 = fmaxf(P.rest[ph], kEps);
    const float d = sdq[s].x, d0 = rho_prev[sid[s]];
    const float q[3] = {__fdiv_rn(__fsub_rn(d, d0), r0), __fsub_rn(__fdiv_rn(d, r0), 1.0f),
                        __fsub_rn(__fdiv_rn(d0, r0), 1.0f)};
#pragma unroll
    for (int c = 0; c < 3; c++)
      v[c] = fmaxf(v[c], (q[c] != q[c]) ? __int_as_float(0x7f800000) : fmaxf(q[c], 0.0f));
  }
  const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < 3; c++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[c] = fmaxf(v[c], __shfl_xor_sync(0xFFFFFFFFu, v[c], o));
    if (lane == 0) red[c][wid] = v[c];
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    float m = 0.0f;
    for (uint32_t k = 0; k < (blockDim.x >> 5); k++) m = fmaxf(m, red[threadIdx.x][k]);
    atomicMax(&out[threadIdx.x], __float_as_uint(m));
  }
}

// ---------------------------------------------------------------- helpers
__global__ void __launch_bounds__(256) k_unsort_dp(const float2* __restrict__ sdq, const float* __restrict__ spres,
                                                   const uint32_t* __restrict__ sid, uint32_t n,
                                                   float* __restrict__ dens, float* __restrict__ pres) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  uint32_t id = sid[s];
  dens[id] = sdq[s].x;
  pres[id] = spres[s];
}

__global__ void __launch_bounds__(256) k_debug_neighbors(const float2* __restrict__ spos,
                                                         const uint32_t* __restrict__ skey,
                                                         const uint32_t* __restrict__ sid, uint32_t n,
                                                         const uint32_t* __restrict__ range, StepParams P,
                                                         uint32_t* __restrict__ counts, uint32_t* __restrict__ lists,
                                                         uint32_t max_per) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const uint32_t k = skey[s];
  const uint32_t id = sid[s];
  const float2 pi = spos[s];
  uint32_t c = 0;
  if (k != P.grid.sentinel) {
    for_each_candidate(k, range, P.grid, [&](int j) {
      float2 pj = spos[j];
      float dx = __fsub_rn(pj.x, pi.x);
      float dy = __fsub_rn(pj.y, pi.y);
      float d2 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
      if (d2 < P.hg2) {
        if (c < max_per) lists[(size_t)id * max_per + c] = sid[j];
        c++;
      }
    });
  }
  counts[id] = c;
}

__global__ void __launch_bounds__(256) k_vmax(const float4* __restrict__ state, uint32_t n,
                                              unsigned int* __restrict__ out) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  float m = 0.0f;
  for (; i < n; i += gridDim.x * blockDim.x) {
    float4 s = state[i];
    float l = __fsqrt_rn(__fadd_rn(__fmul_rn(s.z, s.z), __fmul_rn(s.w, s.w)));
    if (l > m) m = l;  // NaN never wins (f32::max semantics)
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));  // m >= 0: bit order = value order
}

// max_i x_i and max_i |v_i| (the per-step readings of fluid_dam.rs:46-52) as
// float bits. Positions can be negative: map float bits to an order-preserving
// unsigned key for the max.
__device__ __forceinline__ unsigned int f2ord(float f) {
  unsigned int u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__global__ void __launch_bounds__(256) k_front_metrics(const float4* __restrict__ state, uint32_t n,
                                                       unsigned int* __restrict__ out) {
  __shared__ unsigned int smx[8], smv[8];
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned int mx = 0u;  // below every ordered float
  float m2 = 0.0f;       // max |v|^2: sqrt is monotonic, so sqrt(max) = max(sqrt)
  for (; i < n; i += gridDim.x * blockDim.x) {
    const float4 s = state[i];
    if (s.x == s.x) mx = max(mx, f2ord(s.x));
    const float l2 = __fadd_rn(__fmul_rn(s.z, s.z), __fmul_rn(s.w, s.w));
    if (l2 > m2) m2 = l2;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mx = max(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
    m2 = fmaxf(m2, __shfl_xor_sync(0xFFFFFFFFu, m2, o));
  }
  const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
  if (lane == 0) {
    smx[wid] = mx;
    smv[wid] = __float_as_uint(m2);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (uint32_t k = 1; k < (blockDim.x >> 5); k++) {
      mx = max(mx, smx[k]);
      m2 = fmaxf(m2, __uint_as_float(smv[k]));
    }
    atomicMax(&out[0], mx);
    atomicMax(&out[1], __float_as_uint(__fsqrt_rn(m2)));  // non-negative floats order as their bits
  }
}

#include "sph_fast.cuh"
#include "sph_closure_tc.cuh"

inline uint32_t cdiv(uint32_t a, uint32_t b) { return (a + b - 1) / b; }

// The launch's flags for which the force pass compiles out the optional pair
// terms: XSPH on, artificial viscosity and cohesion off, h*h <= hk*hk (a
// batch's launch parameters carry the union of its scenes' flags).
inline bool plain_flags(uint32_t f) {
  return (f & F_VISC) && !(f & (F_AV | F_COHESION | F_WIDE_NB | F_TURB | F_GHOST | F_POLY));
}

// Tolerance-mode passes apply: requested, the plain flag set, uniform mass
// and phase (for a batch: the union of its scenes' flags).
inline bool fast_flags(uint32_t f) { return (f & F_FAST) && plain_flags(f) && !(f & (F_MASS | F_PHASE)); }

}  // namespace

void enqueue_keys(const FluidBufs& b, uint32_t n, const GridPlan& g, cudaStream_t st) {
  cudaMemsetAsync(b.count, 0, sizeof(uint32_t) * b.count_len, st);
  if (n == 0) return;
  if (b.batch.ptab)
    k_keys<true><<<cdiv(n, 256), 256, 0, st>>>(b.state, n, g, b.batch, b.key, b.count);
  else
    k_keys<false><<<cdiv(n, 256), 256, 0, st>>>(b.state, n, g, b.batch, b.key, b.count);
}

// Bucket counts -> start table (count becomes the placement cursor).
void enqueue_bucket_scan(const BucketSort& bs, uint32_t m, cudaStream_t st) {
  const uint32_t nt = cdiv(m, kScanTile);
  if (bs.tstate) {
    k_scan_lookback<<<cdiv(nt, kLookbackSub), kLookbackThreads, 0, st>>>(bs.count, nt, bs.start, bs.tstate, bs.done,
                                                                          bs.err, 0xFFFFFFFFu);
  } else {
    k_scan_reduce<<<nt, 256, 0, st>>>(bs.count, bs.tilesum, nt, bs.done);
    k_scan_down<<<nt, 256, 0, st>>>(bs.count, bs.tilesum, m, bs.start);
  }
}

void enqueue_bucket_place(const BucketSort& bs, uint32_t n, uint32_t m, bool by_slot, cudaStream_t st) {
  if (n == 0) return;
  enqueue_bucket_scan(bs, m, st);
  if (by_slot)
    k_place<true><<<cdiv(n, 256), 256, 0, st>>>(bs.key, bs.sid_prev, n, bs.count, bs.tkey, bs.tid);
  else
    k_place<false><<<cdiv(n, 256), 256, 0, st>>>(bs.key, bs.sid_prev, n, bs.count, bs.tkey, bs.tid);
}

void enqueue_sort_and_ranges(const FluidBufs& b, uint32_t n, const StepParams& P, bool by_slot, cudaStream_t st) {
  if (n == 0) return;
  const uint32_t m = P.grid.sentinel + 1;  // all buckets and the non-finite sentinel
  BucketSort bs;
  bs.count = b.count;
  bs.tilesum = b.tilesum;
  bs.done = b.done;
  bs.tstate = b.tstate;
  bs.err = b.scan_err;
  bs.start = b.start;
  bs.key = b.key;
  bs.sid_prev = b.sid;
  bs.tkey = b.tkey;
  bs.tid = b.tid;
  GatherArgs ga;
  ga.state = b.state;
  ga.mass = b.mass;
  ga.phase = b.phase;
  ga.spos = b.spos;
  ga.svel = b.svel;
  ga.smass = (P.flags & F_MASS) ? b.smass : nullptr;
  ga.sphase = (P.flags & F_PHASE) ? b.sphase : nullptr;
  ga.pscene = b.batch.pscene;
  ga.sscene = b.batch.ptab ? b.batch.sscene : nullptr;
  enqueue_bucket_scan(bs, m, st);
  if (by_slot)
    k_place_final<true><<<cdiv(n, 256), 256, 0, st>>>(b.key, b.sid, n, b.count, b.start, b.tkey, b.tid, b.skey,
                                                       b.order, ga);
  else
    k_place_final<false><<<cdiv(n, 256), 256, 0, st>>>(b.key, b.sid, n, b.count, b.start, b.tkey, b.tid, b.skey,
                                                        b.order, ga);
  // the fixup also clears the counts: the next sort's accumulate from zero
  // (K6). Four slots per thread for one world (sort 31.6 against 32.1 us at
  // 2^20 particles), one for a batch, whose many small buckets leave more
  // slots to rank (sort 160 against 168 us for 512 scenes)
  const uint32_t slots = b.batch.ptab ? 1u : 4u;
  const uint32_t threads = std::max(cdiv(n, slots), cdiv(b.count_len, 4));
  if (slots == 1)
    k_fixup<1><<<cdiv(threads, 256), 256, 0, st>>>(b.tkey, b.tid, b.start, n, b.skey, b.sid, b.order, P.grid.sentinel,
                                                   b.count, b.count_len, ga);
  else
    k_fixup<4><<<cdiv(threads, 256), 256, 0, st>>>(b.tkey, b.tid, b.start, n, b.skey, b.sid, b.order, P.grid.sentinel,
                                                   b.count, b.count_len, ga);
}

// ---------------------------------------------------------------- adaptive resolution
// FluidState2::resample (fluid.rs:826-893) after the first density pass.
// Merge: each particle i in index order whose density exceeds merge_hi takes
// in the highest-index j < i that is not yet absorbed, also exceeds merge_hi
// and lies within 0.25 h (mass and momentum conserved: v_i = (v_i m_i +
// v_j m_j) / m_t, m_i = m_t when m_t > EPS). j is found among the grid
// candidates, which hold every particle within h. Split: in index order, a
// kept particle under split_lo heavier than particle_mass / 8 becomes two
// half-mass children at x +- (0.25 h, 0) while the output holds fewer than
// MAX_PARTICLES_2D - 1. One thread: every decision depends on the earlier
// ones. Writes the new state / mass / phase to out_*, the count to *n_out.
__global__ void k_resample(uint32_t n, float4* __restrict__ state, float* __restrict__ mass,
                           const uint8_t* __restrict__ phase, const float2* __restrict__ sdq,
                           const uint32_t* __restrict__ sid, const uint32_t* __restrict__ skey,
                           const uint32_t* __restrict__ slot_of, const uint32_t* __restrict__ start, StepParams P,
                           float merge_hi, float split_lo, float min_mass, uint8_t* __restrict__ absorbed,
                           float4* __restrict__ out_state, float* __restrict__ out_mass, uint8_t* __restrict__ out_phase,
                           uint32_t out_cap, uint32_t* __restrict__ n_out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const float h = P.hk;
  const float md = __fmul_rn(0.25f, h);
  const float merge_d2 = __fmul_rn(md, md);
  for (uint32_t i = 0; i < n; i++) absorbed[i] = 0;
  for (uint32_t i = 0; i < n; i++) {
    const uint32_t si = slot_of[i];
    if (absorbed[i] || sdq[si].x <= merge_hi) continue;
    const float4 pi = state[i];
    int64_t best = -1;
    const uint32_t key = skey[si];
    if (key != P.grid.sentinel)
      for_each_candidate(key, start, P.grid, [&](int js) {
        const uint32_t j = sid[js];
        if (j >= i || absorbed[j] || sdq[js].x <= merge_hi || (int64_t)j <= best) return;
        const float4 pj = state[j];
        const float dx = __fsub_rn(pi.x, pj.x), dy = __fsub_rn(pi.y, pj.y);
        if (__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)) < merge_d2) best = j;
      });
    if (best < 0) continue;
    const uint32_t j = (uint32_t)best;
    const float mi = mass[i], mj = mass[j];
    const float mt = __fadd_rn(mi, mj);
    if (mt > kEps) {
      const float4 pj = state[j];
      state[i].z = __fdiv_rn(__fadd_rn(__fmul_rn(pi.z, mi), __fmul_rn(pj.z, mj)), mt);
      state[i].w = __fdiv_rn(__fadd_rn(__fmul_rn(pi.w, mi), __fmul_rn(pj.w, mj)), mt);
      mass[i] = mt;
    }
    absorbed[j] = 1;
  }
  uint32_t out = 0;
  const float off = __fmul_rn(0.25f, h);
  for (uint32_t i = 0; i < n; i++) {
    if (absorbed[i]) continue;
    const float4 p = state[i];
    const float m = mass[i];
    const bool split = sdq[slot_of[i]].x < split_lo && m > min_mass && out + 1 < 4096u;  // MAX_PARTICLES_2D (fluid.rs:30)
    if (out + (split ? 2u : 1u) > out_cap) {  // never with buffers sized for the bound: report, write nothing past
      *n_out = out_cap + 1u;
      return;
    }
    if (split) {
      const float half = __fmul_rn(m, 0.5f);
      out_state[out] = make_float4(__fadd_rn(p.x, off), __fadd_rn(p.y, 0.0f), p.z, p.w);
      out_mass[out] = half;
      out_phase[out++] = phase[i];
      out_state[out] = make_float4(__fsub_rn(p.x, off), __fsub_rn(p.y, 0.0f), p.z, p.w);
      out_mass[out] = half;
      out_phase[out++] = phase[i];
    } else {
      out_state[out] = p;
      out_mass[out] = m;
      out_phase[out++] = phase[i];
    }
  }
  *n_out = out;
}

// slot_of[sid[s]] = s; uniform mass / phase written out per particle first.
__global__ void k_resample_prep(const uint32_t* __restrict__ sid, uint32_t n, uint32_t* __restrict__ slot_of,
                                float* __restrict__ mass, uint8_t* __restrict__ phase, int mass_uniform,
                                float mass_value, int phase_uniform, uint8_t phase_value) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  slot_of[sid[s]] = s;
  if (mass_uniform) mass[s] = mass_value;
  if (phase_uniform) phase[s] = phase_value;
}

void enqueue_resample(const FluidBufs& b, uint32_t n, const StepParams& P, const ResampleBufs& r, float merge_hi,
                      float split_lo, float min_mass, bool mass_uniform, bool phase_uniform, cudaStream_t st) {
  if (n == 0) return;
  k_resample_prep<<<cdiv(n, 256), 256, 0, st>>>(b.sid, n, r.slot_of, b.mass, b.phase, mass_uniform ? 1 : 0, P.mass,
                                                 phase_uniform ? 1 : 0, (uint8_t)P.uniform_phase);
  k_resample<<<1, 1, 0, st>>>(n, b.state, b.mass, b.phase, b.sdq, b.sid, b.skey, r.slot_of, b.start, P, merge_hi,
                              split_lo, min_mass, r.absorbed, r.state, r.mass, r.phase, r.cap, r.n_out);
}

void enqueue_ghost_density(const FluidBufs& b, const StepParams& P, cudaStream_t st) {
  if (!(P.flags & F_GHOST) || P.nghost == 0) return;
  k_ghost_density<<<cdiv(P.nghost, 256), 256, 0, st>>>(b.spos, b.smass, b.start, P);
}

void enqueue_density(const FluidBufs& b, uint32_t n, const StepParams& P, cudaStream_t st, float2* svp) {
  if (n == 0) return;
  const bool m = (P.flags & F_MASS) != 0, ph = (P.flags & F_PHASE) != 0, bat = b.batch.ptab != nullptr;
  const bool wide = (P.flags & F_WIDE_NB) != 0;  // h <= 0, which only a snapshot can carry
  const uint32_t bs = b.block_density, g = cdiv(n, bs);
  // Tolerance mode with staging asked for: the exact density pass with its
  // neighbour rows staged in shared memory (same bits).
  if (fast_flags(P.flags) && (b.stage & 1u)) {
    const size_t sm = 3 * fast_stage_cap(bs) * sizeof(float2);
    if (bat)
      k_density_fast<true, true><<<g, bs, sm, st>>>(b.spos, b.skey, n, b.start, P, b.batch, b.sdq, b.spres, b.nmask,
                                                    svp);
    else
      k_density_fast<true, false><<<g, bs, sm, st>>>(b.spos, b.skey, n, b.start, P, b.batch, b.sdq, b.spres, b.nmask,
                                                     svp);
    return;
  }
#define PHIENG_DENSITY(M, PH, BT, WD)                                                                          \
  k_density<M, PH, BT, WD><<<g, bs, 0, st>>>(b.spos, b.skey, b.smass, b.sphase, n, b.start, P, b.batch, b.sdq, \
                                             b.spres, b.nmask, svp)
#define PHIENG_DENSITY_W(M, PH, BT)       \
  do {                                    \
    if (wide)                             \
      PHIENG_DENSITY(M, PH, BT, true);    \
    else                                  \
      PHIENG_DENSITY(M, PH, BT, false);   \
  } while (0)
  if (bat) {
    if (m && ph) PHIENG_DENSITY_W(true, true, true);
    else if (m) PHIENG_DENSITY_W(true, false, true);
    else if (ph) PHIENG_DENSITY_W(false, true, true);
    else PHIENG_DENSITY_W(false, false, true);
  } else {
    if (m && ph) PHIENG_DENSITY_W(true, true, false);
    else if (m) PHIENG_DENSITY_W(true, false, false);
    else if (ph) PHIENG_DENSITY_W(false, true, false);
    else PHIENG_DENSITY_W(false, false, false);
  }
#undef PHIENG_DENSITY_W
#undef PHIENG_DENSITY
}

void enqueue_force_integrate(const FluidBufs& b, uint32_t n, const StepParams& P, float2* dbg_force,
                             cudaStream_t st) {
  if (n == 0) return;
  const bool m = (P.flags & F_MASS) != 0, bat = b.batch.ptab != nullptr, plain = plain_flags(P.flags);
  const uint32_t bs = b.block_force, g = cdiv(n, bs);
  if (fast_flags(P.flags)) {
    const size_t sm = 9 * fast_stage_cap(bs) * sizeof(float2);
#define PHIENG_FORCE_FAST_B(STG, D, BT, BAL)                                                                       \
  k_force_fast<STG, D, BT, BAL><<<g, bs, STG ? sm : 0, st>>>(b.spos, b.svel, b.sdq, b.skey, b.sid, n, b.start, P,  \
                                                             b.batch, b.bodies, b.nmask, b.state, b.key, b.count,  \
                                                             dbg_force, b.defer, b.dcount)
#define PHIENG_FORCE_FAST(STG, D, BT) PHIENG_FORCE_FAST_B(STG, D, BT, false)
    const bool stg = (b.stage & 2u) != 0;
    const bool bal = !stg && (b.stage & 4u) != 0;  // lanes balanced by neighbour count
    if (dbg_force) {  // single worlds only
      if (stg) PHIENG_FORCE_FAST(true, true, false);
      else if (bal) PHIENG_FORCE_FAST_B(false, true, false, true);
      else PHIENG_FORCE_FAST(false, true, false);
    } else if (bat) {
      if (stg) PHIENG_FORCE_FAST(true, false, true);
      else if (bal) PHIENG_FORCE_FAST_B(false, false, true, true);
      else PHIENG_FORCE_FAST(false, false, true);
    } else {
      if (stg) PHIENG_FORCE_FAST(true, false, false);
      else if (bal) PHIENG_FORCE_FAST_B(false, false, false, true);
      else PHIENG_FORCE_FAST(false, false, false);
    }
#undef PHIENG_FORCE_FAST
#undef PHIENG_FORCE_FAST_B
    return;
  }
#define PHIENG_FORCE(M, D, BT, PL)                                                                                  \
  k_force_integrate<M, D, BT, PL><<<g, bs, 0, st>>>(b.spos, b.svel, b.sdq, b.skey, b.sid, b.smass, n, b.start, P, \
                                                    b.batch, b.bodies, b.nmask, b.state, b.key, b.count, dbg_force, \
                                                    b.defer, b.dcount)
  if (dbg_force) {
    if (m) PHIENG_FORCE(true, true, false, false);
    else PHIENG_FORCE(false, true, false, false);
  } else if (bat) {
    if (m) PHIENG_FORCE(true, false, true, false);
    else PHIENG_FORCE(false, false, true, false);
  } else if (plain) {
    if (m) PHIENG_FORCE(true, false, false, true);
    else PHIENG_FORCE(false, false, false, true);
  } else {
    if (m) PHIENG_FORCE(true, false, false, false);
    else PHIENG_FORCE(false, false, false, false);
  }
#undef PHIENG_FORCE
}

size_t closure_smem_bytes() { return sizeof(MlpSmem) + sizeof(__nv_bfloat16) * 256 * kXRow + sizeof(float) * 256 * 2; }

template <int MODE>
void launch_closure(const FluidBufs& b, uint32_t n, const StepParams& P, const MlpDev& mlp, const ClosureIO& io,
                    cudaStream_t st) {
  const bool m = (P.flags & F_MASS) != 0, ph = (P.flags & F_PHASE) != 0, bat = b.batch.ptab != nullptr;
  const bool plain = plain_flags(P.flags) && !m && !ph;
  if (MODE == kModeClosure && fast_flags(P.flags) && mlp.engine == kMlpInferMmaSync) {
    // tolerance mode, network on mma.sync warp tiles
#define PHIENG_CLOSURE_F(BT)                                                                                       \
  k_closure_fast<BT><<<cdiv(n, 256), 256, closure_smem_bytes(), st>>>(b.spos, b.svel, b.sdq, b.spres, b.skey,     \
                                                                      b.sid, n, b.start, P, b.batch, b.bodies,    \
                                                                      b.nmask, mlp, io, b.state, b.key, b.count)
    if (bat) PHIENG_CLOSURE_F(true);
    else PHIENG_CLOSURE_F(false);
#undef PHIENG_CLOSURE_F
    return;
  }
  if (MODE == kModeClosure && fast_flags(P.flags) && io.err) {
    // tolerance mode: fused pass with the network on the tcgen05 tensor cores
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint32_t blocks = min(cdiv(n, 128), (uint32_t)sms * 6u);
#define PHIENG_CLOSURE_TC(BT)                                                                                       \
  k_closure_tc<BT><<<blocks, 128, kNetSmem, st>>>(b.spos, b.svel, b.sdq, b.spres, b.skey, b.sid, n, b.start, P,     \
                                                  b.batch, b.bodies, b.nmask, mlp, io, b.state, b.key, b.count, io.err)
    if (bat) PHIENG_CLOSURE_TC(true);
    else PHIENG_CLOSURE_TC(false);
#undef PHIENG_CLOSURE_TC
    return;
  }
  const uint32_t g = cdiv(n, 256);
  const size_t sm = MODE == kModeClosure ? closure_smem_bytes() : 0;
#define PHIENG_CLOSURE_V(M, PH, BT, PL)                                                                           \
  k_force_closure<M, PH, BT, PL, MODE><<<g, 256, sm, st>>>(b.spos, b.svel, b.sdq, b.spres, b.skey, b.sid,         \
                                                           b.smass, b.sphase, n, b.start, P, b.batch, b.bodies,   \
                                                           b.nmask, mlp, io, b.state, b.key, b.count)
#define PHIENG_CLOSURE(M, PH, BT) PHIENG_CLOSURE_V(M, PH, BT, false)
  if (plain) {
    if (bat) PHIENG_CLOSURE_V(false, false, true, true);
    else PHIENG_CLOSURE_V(false, false, false, true);
  } else if (bat) {
    if (m && ph) PHIENG_CLOSURE(true, true, true);
    else if (m) PHIENG_CLOSURE(true, false, true);
    else if (ph) PHIENG_CLOSURE(false, true, true);
    else PHIENG_CLOSURE(false, false, true);
  } else {
    if (m && ph) PHIENG_CLOSURE(true, true, false);
    else if (m) PHIENG_CLOSURE(true, false, false);
    else if (ph) PHIENG_CLOSURE(false, true, false);
    else PHIENG_CLOSURE(false, false, false);
  }
#undef PHIENG_CLOSURE
#undef PHIENG_CLOSURE_V
}

void enqueue_closure_features(const FluidBufs& b, uint32_t n, const StepParams& P, float* feat, const float2* svp,
                              cudaStream_t st) {
  if (n == 0) return;
  ClosureIO io;
  io.feat = feat;
  io.svp = svp;
  launch_closure<kModeFeatures>(b, n, P, MlpDev{}, io, st);
}

void enqueue_closure_force(const FluidBufs& b, uint32_t n, const StepParams& P, const MlpDev& mlp,
                           const ClosureIO& io, cudaStream_t st) {
  if (n == 0) return;
  launch_closure<kModeClosure>(b, n, P, mlp, io, st);
}

// Running maxima of the three closure checks over a block of coarse steps:
// acc = (max out[0], max out[1], max (out[1] - out[2])), the per-step value
// of each criterion (jump, compression, growth); reset to -inf.
__global__ void k_check_fold(const unsigned int* __restrict__ out, float* __restrict__ acc, int reset) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (reset) {
    acc[0] = acc[1] = acc[2] = -INFINITY;
    return;
  }
  const float v0 = __uint_as_float(out[0]), v1 = __uint_as_float(out[1]), v2 = __uint_as_float(out[2]);
  acc[0] = fmaxf(acc[0], v0);
  acc[1] = fmaxf(acc[1], v1);
  acc[2] = fmaxf(acc[2], __fsub_rn(v1, v2));
}

void enqueue_check_fold(const unsigned int* out, float* acc, bool reset, cudaStream_t st) {
  k_check_fold<<<1, 32, 0, st>>>(out, acc, reset ? 1 : 0);
}

__global__ void k_set_word(unsigned int* p, unsigned int v) { *p = v; }

void enqueue_set_word(unsigned int* p, uint32_t v, cudaStream_t st) { k_set_word<<<1, 1, 0, st>>>(p, v); }

void enqueue_closure_check(const FluidBufs& b, uint32_t n, const StepParams& P, const float* rho_prev,
                           unsigned int* out, cudaStream_t st) {
  cudaMemsetAsync(out, 0, 3 * sizeof(unsigned int), st);
  if (n == 0) return;
  const bool ph = (P.flags & F_PHASE) != 0, bat = b.batch.ptab != nullptr;
  const uint32_t g = min(cdiv(n, 256), 148u * 8u);
  if (bat) {
    if (ph) k_closure_check<true, true><<<g, 256, 0, st>>>(b.sdq, b.sid, b.sphase, n, P, b.batch, rho_prev, out);
    else k_closure_check<false, true><<<g, 256, 0, st>>>(b.sdq, b.sid, b.sphase, n, P, b.batch, rho_prev, out);
  } else {
    if (ph) k_closure_check<true, false><<<g, 256, 0, st>>>(b.sdq, b.sid, b.sphase, n, P, b.batch, rho_prev, out);
    else k_closure_check<false, false><<<g, 256, 0, st>>>(b.sdq, b.sid, b.sphase, n, P, b.batch, rho_prev, out);
  }
}

// ---------------------------------------------------------------- bodies that react
// Ordered compaction of the deferred particles: list[dstart[i]] = i for
// every i whose flag was 1 (the scan turned the flags into their exclusive
// prefix, so a flag shows as a step between dstart[i] and dstart[i + 1]).
__global__ void __launch_bounds__(256) k_compact_deferred(const uint32_t* __restrict__ dstart, uint32_t n,
                                                          uint32_t* __restrict__ list) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && dstart[i + 1] != dstart[i]) list[dstart[i]] = i;
}

// The rest of the body loop of every deferred particle, one particle after
// the other in id order (the reference's loop order: a body's velocity after
// particle i's reactions is what particle i+1's no-slip term reads); then the
// particle's next key and bucket count.
__global__ void k_dynamic_walls(const uint32_t* __restrict__ list, const uint32_t* __restrict__ total,
                                const uint32_t* __restrict__ defer, float4* __restrict__ state,
                                const float* __restrict__ mass, uint32_t* __restrict__ key,
                                uint32_t* __restrict__ count, const DevBody* __restrict__ bodies,
                                DynBody* __restrict__ dyn, StepParams P) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const uint32_t m = *total;
  for (uint32_t t = 0; t < m; t++) {
    const uint32_t id = list[t];
    const float4 q = state[id];
    float x = q.x, y = q.y, vx = q.z, vy = q.w;
    const float mi = (P.flags & F_MASS) ? mass[id] : P.mass;
    walls_ordered(x, y, vx, vy, mi, defer[id], bodies, dyn, P);
    state[id] = make_float4(x, y, vx, vy);
    const uint32_t nk = bucket_key(x, y, P.grid);
    key[id] = nk;
    atomicAdd(&count[nk], 1u);
  }
}

// Sorted (density, q) and pressure to id order and back into the order of a
// newer sort (the buoyancy pass samples the pressure on the re-sorted grid).
__global__ void __launch_bounds__(256) k_dp_to_id(const float2* __restrict__ sdq, const float* __restrict__ spres,
                                                  const uint32_t* __restrict__ sid, uint32_t n,
                                                  float2* __restrict__ dq_id, float* __restrict__ p_id) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const uint32_t id = sid[s];
  dq_id[id] = sdq[s];
  p_id[id] = spres[s];
}

__global__ void __launch_bounds__(256) k_dp_from_id(const float2* __restrict__ dq_id, const float* __restrict__ p_id,
                                                    const uint32_t* __restrict__ sid, uint32_t n,
                                                    float2* __restrict__ sdq, float* __restrict__ spres) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const uint32_t id = sid[s];
  sdq[s] = dq_id[id];
  spres[s] = p_id[id];
}

// FluidState2::sample_pressure (fluid.rs:392-410) at a point over the sorted
// grid: h = max(smoothing_length, EPS); cells oy, ox = -1..1 around
// floor(point / h); p += m_j * (p_j / max(rho_j, EPS)) * poly6(r^2) for
// r^2 < h*h in visit order; max(p, 0).
__device__ float sample_pressure(float ptx, float pty, const float2* __restrict__ spos,
                                 const float2* __restrict__ sdq, const float* __restrict__ spres,
                                 const float* __restrict__ smass, const uint32_t* __restrict__ start,
                                 const StepParams& P) {
  const GridPlan& g = P.grid;
  const int32_t cx = __float2int_rd(__fdiv_rn(ptx, P.hk));
  const int32_t cy = __float2int_rd(__fdiv_rn(pty, P.hk));
  float p = 0.0f;
  for (int oy = -1; oy <= 1; oy++) {
    const uint32_t by = ((uint32_t)cy + (uint32_t)oy - (uint32_t)g.cy0) & g.maskh;
    for (int ox = -1; ox <= 1; ox++) {
      const uint32_t bx = ((uint32_t)cx + (uint32_t)ox - (uint32_t)g.cx0) & g.maskw;
      const uint32_t bb = g.base + (by << g.log2w) + bx;
      const uint32_t e = start[bb + 1];
      for (uint32_t j = start[bb]; j < e; j++) {
        const float2 pj = spos[j];
        const float dx = __fsub_rn(pj.x, ptx), dy = __fsub_rn(pj.y, pty);
        const float r2 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
        if (r2 < P.hk2) {
          const float mj = (P.flags & F_MASS) ? smass[j] : P.mass;
          const float pr = __fdiv_rn(spres[j], fmaxf(sdq[j].x, kEps));
          p = __fadd_rn(p, __fmul_rn(__fmul_rn(mj, pr), poly6(r2, P)));
        }
      }
    }
  }
  return fmaxf(p, 0.0f);  // f32::max(0.0); a NaN sum gives 0
}

// Buoyancy + drag on one dynamic body (fluid.rs:1103-1135): for each surface
// sample in order, the sampled pressure p > 0 gives the force
// -n * (p * area) - v_rel * (drag * area * |v_rel|) (the latter when
// |v_rel| > EPS), applied at the sample point for dt (body.rs:657-673).
__global__ void k_buoyancy(const uint32_t* __restrict__ which, uint32_t nb, const DevBody* __restrict__ bodies,
                           DynBody* __restrict__ dyn, const float4* __restrict__ samples,
                           const float* __restrict__ areas, const float2* __restrict__ spos,
                           const float2* __restrict__ sdq, const float* __restrict__ spres,
                           const float* __restrict__ smass, const uint32_t* __restrict__ start, StepParams P,
                           float drag, float dt) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nb) return;
  const uint32_t k = which[t];
  const DevBody b = bodies[P.body_first + k];
  DynBody d = dyn[k];
  bool wet = false;
  for (uint32_t q = 0; q < d.sample_count; q++) {
    const float4 sp = samples[d.sample_first + q];
    const float area = areas[d.sample_first + q];
    const float p = sample_pressure(sp.x, sp.y, spos, sdq, spres, smass, start, P);
    if (p <= 0.0f) continue;
    wet = true;
    const float rx = __fsub_rn(sp.x, b.px), ry = __fsub_rn(sp.y, b.py);
    // v + (-w r.y, w r.x) - wind
    const float vrx = __fsub_rn(__fadd_rn(d.vx, __fmul_rn(-d.w, ry)), P.wind_x);
    const float vry = __fsub_rn(__fadd_rn(d.vy, __fmul_rn(d.w, rx)), P.wind_y);
    const float speed = __fsqrt_rn(__fadd_rn(__fmul_rn(vrx, vrx), __fmul_rn(vry, vry)));
    const float pa = __fmul_rn(p, area);
    float fx = __fmul_rn(-sp.z, pa), fy = __fmul_rn(-sp.w, pa);
    if (speed > kEps) {
      const float c = __fmul_rn(__fmul_rn(drag, area), speed);
      fx = __fsub_rn(fx, __fmul_rn(vrx, c));
      fy = __fsub_rn(fy, __fmul_rn(vry, c));
    }
    if (!d.is_static) {  // RigidBody2::apply_force
      d.sleeping = 0;
      d.vx = __fadd_rn(d.vx, __fmul_rn(__fmul_rn(fx, d.inv_mass), dt));
      d.vy = __fadd_rn(d.vy, __fmul_rn(__fmul_rn(fy, d.inv_mass), dt));
      const float torque = __fsub_rn(__fmul_rn(rx, fy), __fmul_rn(ry, fx));
      d.w = __fadd_rn(d.w, __fmul_rn(__fmul_rn(torque, d.inv_inertia), dt));
    }
  }
  if (wet) d.sleeping = 0;
  dyn[k] = d;
}

void enqueue_flag_compact(uint32_t* flags, uint32_t n, uint32_t* tile, uint32_t* done, uint32_t* start,
                          uint32_t* list, cudaStream_t st) {
  if (n == 0) return;
  const uint32_t nt = cdiv(n + 1, kScanTile);
  k_scan_reduce<<<nt, 256, 0, st>>>(flags, tile, nt, done);
  k_scan_down<<<nt, 256, 0, st>>>(flags, tile, n + 1, start);
  k_compact_deferred<<<cdiv(n, 256), 256, 0, st>>>(start, n, list);
}

void enqueue_dynamic_walls(const FluidBufs& b, const DynBufs& y, uint32_t n, const StepParams& P, cudaStream_t st) {
  if (n == 0) return;
  enqueue_flag_compact(y.dcount, n, y.dtile, y.done, y.dstart, y.list, st);
  k_dynamic_walls<<<1, 32, 0, st>>>(y.list, y.dstart + n, b.defer, b.state, b.mass, b.key, b.count, b.bodies, y.dyn,
                                    P);
}

void enqueue_buoyancy(const FluidBufs& b, const DynBufs& y, uint32_t n, const StepParams& P, float drag, float dt,
                      cudaStream_t st) {
  if (n == 0 || y.nbuoy == 0) return;
  // the density pass's values by id, the grid rebuilt on the new positions
  // (from a copy of the bucket counts, which the next substep's sort needs),
  // the values gathered into the new order, then the sampling
  k_dp_to_id<<<cdiv(n, 256), 256, 0, st>>>(b.sdq, b.spres, b.sid, n, y.dq_id, y.p_id);
  cudaMemcpyAsync(y.count2, b.count, sizeof(uint32_t) * b.count_len, cudaMemcpyDeviceToDevice, st);
  FluidBufs b2 = b;
  b2.count = y.count2;
  enqueue_sort_and_ranges(b2, n, P, true, st);
  k_dp_from_id<<<cdiv(n, 256), 256, 0, st>>>(y.dq_id, y.p_id, b.sid, n, b.sdq, b.spres);
  k_buoyancy<<<cdiv(y.nbuoy, 32), 32, 0, st>>>(y.buoy, y.nbuoy, b.bodies, y.dyn, y.samples, y.areas, b.spos, b.sdq,
                                               b.spres, b.smass, b.start, P, drag, dt);
}

void enqueue_scan_silent_tile(const FluidBufs& b, uint32_t m, cudaStream_t st) {
  const uint32_t nt = cdiv(m, kScanTile);
  if (!b.tstate || cdiv(nt, kLookbackSub) < 2) return;
  k_scan_lookback<<<cdiv(nt, kLookbackSub), kLookbackThreads, 0, st>>>(b.count, nt, b.start, b.tstate, b.done,
                                                                        b.scan_err, 0u);
}

void enqueue_unsort_dp(const FluidBufs& b, uint32_t n, float* dens, float* pres, cudaStream_t st) {
  if (n == 0) return;
  k_unsort_dp<<<cdiv(n, 256), 256, 0, st>>>(b.sdq, b.spres, b.sid, n, dens, pres);
}

void enqueue_debug_neighbors(const FluidBufs& b, uint32_t n, const StepParams& P, uint32_t* counts,
                             uint32_t* lists, uint32_t max_per, cudaStream_t st) {
  if (n == 0) return;
  k_debug_neighbors<<<cdiv(n, 256), 256, 0, st>>>(b.spos, b.skey, b.sid, n, b.start, P, counts, lists, max_per);
}

void enqueue_front_metrics(const FluidBufs& b, uint32_t n, cudaStream_t st) {
  cudaMemsetAsync(b.scalar + 2, 0, 2 * sizeof(unsigned int), st);
  if (n == 0) return;
  uint32_t g = min(cdiv(n, 256), 148u * 8u);
  k_front_metrics<<<g, 256, 0, st>>>(b.state, n, b.scalar + 2);
}

void enqueue_vmax(const FluidBufs& b, uint32_t n, cudaStream_t st) {
  cudaMemsetAsync(b.scalar, 0, sizeof(unsigned int), st);
  if (n == 0) return;
  uint32_t g = min(cdiv(n, 256), 148u * 8u);
  k_vmax<<<g, 256, 0, st>>>(b.state, n, b.scalar);
}

}  // namespace phieng
