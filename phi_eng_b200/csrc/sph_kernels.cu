// SPH fluid step kernels for sm_100a (B200).
//
// Chain per substep (the reference's substep, crates/dynamics/src/fluid.rs:898-1136):
//   K1 keys     bucket key per particle                (rebuild_grid, :330-363)
//   K2 sort     stable LSD radix sort of (key, id)     (cell lists with ascending ids)
//   K4 gather   fused into the last sort pass: state -> sorted order
//   K3 ranges   [start, end) per bucket
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

namespace phieng {

namespace {

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// ---------------------------------------------------------------- K1 keys
__global__ void __launch_bounds__(256) k_keys(const float4* __restrict__ state, uint32_t n, GridPlan g,
                                              uint32_t* __restrict__ keys) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 s = state[i];
  keys[i] = bucket_key(s.x, s.y, g);
}

// ---------------------------------------------------------------- K2 radix sort
// Tile histogram of one digit: hist[d * ntiles + tile]. Warp-aggregated
// shared-memory counting (keys are spatially coherent, so digits repeat).
__global__ void __launch_bounds__(kSortThreads) k_radix_hist(const uint32_t* __restrict__ keys, uint32_t n,
                                                             uint32_t shift, uint32_t mask, uint32_t ntiles,
                                                             uint32_t* __restrict__ hist) {
  __shared__ uint32_t cnt[256];
  for (uint32_t d = threadIdx.x; d < 256; d += blockDim.x) cnt[d] = 0;
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t base = blockIdx.x * kSortTile;
#pragma unroll
  for (uint32_t r = 0; r < kSortItems; r++) {
    uint32_t idx = base + r * kSortThreads + threadIdx.x;
    bool valid = idx < n;
    uint32_t d = valid ? ((keys[idx] >> shift) & mask) : 0xFFFFFFFFu;
    uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
    if (valid && (peers & lanemask_lt()) == 0) atomicAdd(&cnt[d], (uint32_t)__popc(peers));
  }
  __syncthreads();
  for (uint32_t d = threadIdx.x; d <= mask; d += blockDim.x) hist[d * ntiles + blockIdx.x] = cnt[d];
}

struct GatherArgs {
  const float4* state;
  const float* mass;
  const uint8_t* phase;
  float2* spos;
  float2* svel;
  float* smass;
  uint8_t* sphase;
};

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

// Exclusive scan of each digit's row of tile counts, hist[d * ntiles + t],
// in place (one block per digit; rows are contiguous, so loads coalesce);
// the row total goes to tot[d]. Output offsets are then
// sum_{d' < d} tot[d'] + hist[d * ntiles + t], the first term formed by the
// scatter kernel itself.
__global__ void __launch_bounds__(256) k_radix_scan_rows(uint32_t* __restrict__ hist, uint32_t ntiles,
                                                         uint32_t* __restrict__ tot) {
  __shared__ uint32_t warp_tot[8];
  __shared__ uint32_t chunk_tot;
  uint32_t* row = hist + (size_t)blockIdx.x * ntiles;
  uint32_t carry = 0;
  for (uint32_t base = 0; base < ntiles; base += 4 * 256) {
    uint32_t v[4], s = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      uint32_t idx = base + threadIdx.x * 4 + k;
      v[k] = idx < ntiles ? row[idx] : 0u;
      s += v[k];
    }
    __syncthreads();  // warp_tot / chunk_tot reuse across chunks
    uint32_t incl = block_incl_scan_256(s, warp_tot);
    uint32_t run = carry + incl - s;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      uint32_t idx = base + threadIdx.x * 4 + k;
      if (idx < ntiles) row[idx] = run;
      run += v[k];
    }
    if (threadIdx.x == 255) chunk_tot = incl;
    __syncthreads();
    carry += chunk_tot;
  }
  if (threadIdx.x == 0) tot[blockIdx.x] = carry;
}

// Stable scatter of one digit pass. Each warp ranks its 256 keys in 8 rounds
// of 32 (item order = round-major, lane-minor = index order) with
// __match_any_sync, per-warp digit counters give the warp-local rank, a
// block scan over (digit, warp) gives the tile-local position; keys are
// staged in shared memory in tile-sorted order and written out so that each
// digit's run is contiguous. FIRST: values are the indices (ids). GATHER:
// last pass, also gathers the particle state into sorted order.
template <bool FIRST, bool GATHER>
__global__ void __launch_bounds__(kSortThreads) k_radix_scatter(const uint32_t* __restrict__ kin,
                                                                const uint32_t* __restrict__ vin,
                                                                uint32_t* __restrict__ kout,
                                                                uint32_t* __restrict__ vout, uint32_t n,
                                                                uint32_t shift, uint32_t mask, uint32_t ntiles,
                                                                const uint32_t* __restrict__ hist,
                                                                const uint32_t* __restrict__ dtot, GatherArgs ga) {
  __shared__ uint32_t wcnt[8][256];
  __shared__ uint32_t dstart[256];
  __shared__ uint32_t gofs[256];
  __shared__ uint32_t warp_tot[8];
  __shared__ uint32_t warp_tot2[8];
  __shared__ uint32_t skeys[kSortTile];
  __shared__ uint32_t svals[kSortTile];
  const uint32_t tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const uint32_t nd = mask + 1;
  for (uint32_t i = tid; i < 8 * 256; i += kSortThreads) (&wcnt[0][0])[i] = 0;
  __syncthreads();
  const uint32_t tbase = blockIdx.x * kSortTile;
  const uint32_t lt = lanemask_lt();
  uint32_t key[kSortItems], val[kSortItems], rank[kSortItems];
#pragma unroll
  for (uint32_t r = 0; r < kSortItems; r++) {
    uint32_t idx = tbase + w * (32 * kSortItems) + r * 32 + lane;
    bool valid = idx < n;
    key[r] = valid ? kin[idx] : 0xFFFFFFFFu;
    val[r] = FIRST ? idx : (valid ? vin[idx] : 0u);
    uint32_t d = valid ? ((key[r] >> shift) & mask) : 0xFFFFFFFFu;
    uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
    uint32_t before = valid ? wcnt[w][d] : 0u;
    __syncwarp();
    if (valid && (peers & lt) == 0) wcnt[w][d] = before + (uint32_t)__popc(peers);
    __syncwarp();
    rank[r] = before + (uint32_t)__popc(peers & lt);
  }
  __syncthreads();
  uint32_t tot = 0;
  if (tid < nd) {
#pragma unroll
    for (int ww = 0; ww < 8; ww++) {
      uint32_t c = wcnt[ww][tid];
      wcnt[ww][tid] = tot;
      tot += c;
    }
  }
  uint32_t incl = block_incl_scan_256(tot, warp_tot);
  const uint32_t dt = tid < nd ? dtot[tid] : 0u;
  const uint32_t dincl = block_incl_scan_256(dt, warp_tot2);
  if (tid < nd) {
    dstart[tid] = incl - tot;
    gofs[tid] = (dincl - dt) + hist[tid * ntiles + blockIdx.x];
  }
  __syncthreads();
#pragma unroll
  for (uint32_t r = 0; r < kSortItems; r++) {
    uint32_t idx = tbase + w * (32 * kSortItems) + r * 32 + lane;
    if (idx < n) {
      uint32_t d = (key[r] >> shift) & mask;
      uint32_t pos = dstart[d] + wcnt[w][d] + rank[r];
      skeys[pos] = key[r];
      svals[pos] = val[r];
    }
  }
  __syncthreads();
  const uint32_t cnt = min(kSortTile, n - tbase);
  for (uint32_t p = tid; p < cnt; p += kSortThreads) {
    uint32_t k = skeys[p];
    uint32_t d = (k >> shift) & mask;
    uint32_t g = gofs[d] + (p - dstart[d]);
    uint32_t v = svals[p];
    kout[g] = k;
    vout[g] = v;
    if (GATHER) {
      float4 s = ga.state[v];
      ga.spos[g] = make_float2(s.x, s.y);
      ga.svel[g] = make_float2(s.z, s.w);
      if (ga.smass) ga.smass[g] = ga.mass[v];
      if (ga.sphase) ga.sphase[g] = ga.phase[v];
    }
  }
}

// ---------------------------------------------------------------- K3 ranges
__global__ void __launch_bounds__(256) k_cell_ranges(const uint32_t* __restrict__ skey, uint32_t n, uint32_t nb,
                                                     int2* __restrict__ range) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  uint32_t k = skey[s];
  if (k >= nb) return;
  if (s == 0 || skey[s - 1] != k) range[k].x = (int)s;
  if (s + 1 == n || skey[s + 1] != k) range[k].y = (int)(s + 1);
}

// ---------------------------------------------------------------- neighbour walk
// Visit every candidate slot j of the particle in bucket `key`, in the
// reference's order. Away from the wrap seam the three buckets of a row are
// consecutive keys, hence one contiguous slot range.
template <class F>
__device__ __forceinline__ void for_each_candidate(uint32_t key, const int2* __restrict__ range,
                                                   const GridPlan& g, F&& f) {
  const uint32_t bx = key & g.maskw, by = key >> g.log2w;
#pragma unroll 1
  for (int oy = -1; oy <= 1; oy++) {
    const uint32_t row = ((by + (uint32_t)oy) & g.maskh) << g.log2w;
    if (bx >= 1u && bx < g.maskw) {
      int2 r0 = __ldg(&range[row + bx - 1]);
      int2 r1 = __ldg(&range[row + bx]);
      int2 r2 = __ldg(&range[row + bx + 1]);
      int s = 0x7FFFFFFF, e = 0;
      if (r0.x < r0.y) { s = r0.x; e = r0.y; }
      if (r1.x < r1.y) { s = min(s, r1.x); e = r1.y; }
      if (r2.x < r2.y) { s = min(s, r2.x); e = r2.y; }
      for (int j = s; j < e; j++) f(j);
    } else {
#pragma unroll 1
      for (int ox = -1; ox <= 1; ox++) {
        int2 r = __ldg(&range[row + ((bx + (uint32_t)ox) & g.maskw)]);
        for (int j = r.x; j < r.y; j++) f(j);
      }
    }
  }
}

// ---------------------------------------------------------------- K5 density
template <bool MASS, bool PHASE>
__global__ void __launch_bounds__(256) k_density(const float2* __restrict__ spos, const uint32_t* __restrict__ skey,
                                                 const float* __restrict__ smass,
                                                 const uint8_t* __restrict__ sphase, uint32_t n,
                                                 const int2* __restrict__ range, StepParams P,
                                                 float2* __restrict__ sdq, float* __restrict__ spres) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const uint32_t k = skey[s];
  const float2 pi = spos[s];
  float rho = 0.0f;
  if (k < P.grid.nbuckets) {
    for_each_candidate(k, range, P.grid, [&](int j) {
      float2 pj = __ldg(&spos[j]);
      float dx = __fsub_rn(pj.x, pi.x);
      float dy = __fsub_rn(pj.y, pi.y);
      float d2 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
      if (d2 < P.hg2) {
        float m = MASS ? __ldg(&smass[j]) : P.mass;
        rho = __fadd_rn(rho, __fmul_rn(m, poly6(d2, P)));
      }
    });
  }
  // f32::clamp(0, 3 * max(rest_density, EPS)) (fluid.rs:605)
  float dens = rho;
  if (dens < 0.0f) dens = 0.0f;
  if (dens > P.rho_cap) dens = P.rho_cap;
  uint32_t ph = PHASE ? min((uint32_t)sphase[s], 3u) : P.uniform_phase;
  float p = eos(dens, P.rest[ph], P);
  float rc = fmaxf(dens, kEps);
  sdq[s] = make_float2(dens, __fdiv_rn(p, __fmul_rn(rc, rc)));
  spres[s] = p;
}

// ---------------------------------------------------------------- K6 force + integrate
template <bool MASS, bool DEBUG>
__global__ void __launch_bounds__(256) k_force_integrate(
    const float2* __restrict__ spos, const float2* __restrict__ svel, const float2* __restrict__ sdq,
    const uint32_t* __restrict__ skey, const uint32_t* __restrict__ sid, const float* __restrict__ smass,
    uint32_t n, const int2* __restrict__ range, StepParams P, const DevBody* __restrict__ bodies,
    float4* __restrict__ state_out, uint32_t* __restrict__ key_out, float2* __restrict__ dbg_force) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const uint32_t k = skey[s];
  const uint32_t id = sid[s];
  const float2 pi = spos[s];
  const float2 vi = svel[s];
  const float2 dqi = sdq[s];
  const float m_i = MASS ? smass[s] : P.mass;
  const float rho_i = fmaxf(dqi.x, kEps);
  const float q_i = dqi.y;  // p_i / (rho_i * rho_i)
  const bool visc = (P.flags & F_VISC) != 0;
  const bool av = (P.flags & F_AV) != 0;
  const bool coh = (P.flags & F_COHESION) != 0;
  float fx = 0.0f, fy = 0.0f, sx = 0.0f, sy = 0.0f;
  if (k < P.grid.nbuckets) {
    for_each_candidate(k, range, P.grid, [&](int j) {
      float2 pj = __ldg(&spos[j]);
      float ex = __fsub_rn(pj.x, pi.x);
      float ey = __fsub_rn(pj.y, pi.y);
      float d2 = __fadd_rn(__fmul_rn(ex, ex), __fmul_rn(ey, ey));
      if (!(d2 < P.hg2) || (uint32_t)j == s) return;
      const float2 dqj = __ldg(&sdq[j]);
      const float2 vj = __ldg(&svel[j]);
      const float m_j = MASS ? __ldg(&smass[j]) : P.mass;
      const float rho_j = fmaxf(dqj.x, kEps);
      // delta = p_i - p_j; |delta|^2 equals d2 bit for bit (negation is exact)
      const float dx = __fsub_rn(pi.x, pj.x);
      const float dy = __fsub_rn(pi.y, pj.y);
      const float dist = __fsqrt_rn(d2);
      // spiky gradient (fluid.rs:278-285)
      float gxx = 0.0f, gyy = 0.0f;
      if (!(dist >= P.hk || dist < kEps)) {
        float hr = __fsub_rn(P.hk, dist);
        float sc = __fmul_rn(__fmul_rn(P.c_spiky, hr), hr);
        gxx = __fmul_rn(__fdiv_rn(dx, dist), sc);
        gyy = __fmul_rn(__fdiv_rn(dy, dist), sc);
      }
      float term = __fadd_rn(q_i, dqj.y);
      if (av && dist > kEps) {
        // Monaghan term (fluid.rs:302-317, called at :963-975)
        float rho_bar = __fmul_rn(0.5f, __fadd_rn(rho_i, rho_j));
        float vrx = __fsub_rn(vi.x, vj.x), vry = __fsub_rn(vi.y, vj.y);
        float vd = __fadd_rn(__fmul_rn(vrx, dx), __fmul_rn(vry, dy));
        if (!(vd >= 0.0f)) {
          float r_sq = __fmul_rn(dist, dist);
          float mu = __fdiv_rn(__fmul_rn(P.hk, vd),
                               __fadd_rn(r_sq, __fmul_rn(__fmul_rn(0.01f, P.hk), P.hk)));
          float ap = __fdiv_rn(__fmul_rn(__fmul_rn(-P.av_alpha, P.c_s), mu), fmaxf(rho_bar, kEps));
          term = __fadd_rn(term, ap);
        }
      }
      const float mt = __fmul_rn(m_j, term);
      fx = __fsub_rn(fx, __fmul_rn(gxx, mt));
      fy = __fsub_rn(fy, __fmul_rn(gyy, mt));
      if (coh && dist > kEps) {
        // cohesion (fluid.rs:320-326, applied at :979-985)
        float c = dist >= P.hk ? 0.0f : __fsub_rn(1.0f, __fdiv_rn(dist, P.hk));
        if (c > 0.0f) {
          float sc = __fmul_rn(__fmul_rn(__fmul_rn(P.surface_tension, m_i), m_j), c);
          fx = __fsub_rn(fx, __fmul_rn(__fdiv_rn(dx, dist), sc));
          fy = __fsub_rn(fy, __fmul_rn(__fdiv_rn(dy, dist), sc));
        }
      }
      if (visc) {
        // XSPH (fluid.rs:1022-1033) against pre-integrate neighbours
        float rho_bar = __fmul_rn(0.5f, __fadd_rn(rho_i, rho_j));
        float w = poly6(d2, P);
        float mr = __fdiv_rn(m_j, rho_bar);
        sx = __fadd_rn(sx, __fmul_rn(__fmul_rn(__fsub_rn(vj.x, vi.x), mr), w));
        sy = __fadd_rn(sy, __fmul_rn(__fmul_rn(__fsub_rn(vj.y, vi.y), mr), w));
      }
    });
  }
  if (DEBUG) {
    dbg_force[id] = make_float2(fx, fy);
    return;
  }
  // integrate (fluid.rs:1003-1050)
  const float ax = __fadd_rn(P.gx, __fdiv_rn(fx, rho_i));
  const float ay = __fadd_rn(P.gy, __fdiv_rn(fy, rho_i));
  float vx = __fadd_rn(vi.x, __fmul_rn(ax, P.dt));
  float vy = __fadd_rn(vi.y, __fmul_rn(ay, P.dt));
  if (visc) {
    vx = __fadd_rn(vx, __fmul_rn(sx, P.visc));
    vy = __fadd_rn(vy, __fmul_rn(sy, P.visc));
  }
  const float speed = __fsqrt_rn(__fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy)));
  if (speed > P.vmax) {
    float sc = __fdiv_rn(P.vmax, speed);
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
  walls(x, y, vx, vy, bodies, P);
  state_out[id] = make_float4(x, y, vx, vy);
  key_out[id] = bucket_key(x, y, P.grid);
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
                                                         const int2* __restrict__ range, StepParams P,
                                                         uint32_t* __restrict__ counts, uint32_t* __restrict__ lists,
                                                         uint32_t max_per) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const uint32_t k = skey[s];
  const uint32_t id = sid[s];
  const float2 pi = spos[s];
  uint32_t c = 0;
  if (k < P.grid.nbuckets) {
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
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned int mx = 0u;  // below every ordered float
  float mv = 0.0f;
  for (; i < n; i += gridDim.x * blockDim.x) {
    float4 s = state[i];
    if (s.x == s.x) mx = max(mx, f2ord(s.x));
    float l = __fsqrt_rn(__fadd_rn(__fmul_rn(s.z, s.z), __fmul_rn(s.w, s.w)));
    if (l > mv) mv = l;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mx = max(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
    mv = fmaxf(mv, __shfl_xor_sync(0xFFFFFFFFu, mv, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&out[0], mx);
    atomicMax(&out[1], __float_as_uint(mv));
  }
}

inline uint32_t cdiv(uint32_t a, uint32_t b) { return (a + b - 1) / b; }

}  // namespace

SortPlan sort_plan(uint32_t nbuckets) {
  // keys are 0..nbuckets (nbuckets = sentinel), nbuckets a power of two
  uint32_t bits = 1;
  while ((1ull << bits) <= (uint64_t)nbuckets) bits++;
  SortPlan p;
  p.passes = (bits + 7) / 8;
  p.bits = (bits + p.passes - 1) / p.passes;
  return p;
}

void enqueue_keys(const FluidBufs& b, uint32_t n, const GridPlan& g, cudaStream_t st) {
  if (n == 0) return;
  k_keys<<<cdiv(n, 256), 256, 0, st>>>(b.state, n, g, b.key);
}

void enqueue_sort_and_ranges(const FluidBufs& b, uint32_t n, const StepParams& P, cudaStream_t st) {
  if (n == 0) return;
  const SortPlan sp = sort_plan(P.grid.nbuckets);
  const uint32_t ntiles = cdiv(n, kSortTile);
  const uint32_t mask = (1u << sp.bits) - 1u;
  GatherArgs ga;
  ga.state = b.state;
  ga.mass = b.mass;
  ga.phase = b.phase;
  ga.spos = b.spos;
  ga.svel = b.svel;
  ga.smass = (P.flags & F_MASS) ? b.smass : nullptr;
  ga.sphase = (P.flags & F_PHASE) ? b.sphase : nullptr;
  const uint32_t* kin = b.key;
  const uint32_t* vin = nullptr;
  for (uint32_t pass = 0; pass < sp.passes; pass++) {
    const uint32_t shift = pass * sp.bits;
    const bool first = pass == 0;
    const bool last = pass + 1 == sp.passes;
    uint32_t* kout = last ? b.skey : ((pass & 1) ? b.kb : b.ka);
    uint32_t* vout = last ? b.sid : ((pass & 1) ? b.vb : b.va);
    k_radix_hist<<<ntiles, kSortThreads, 0, st>>>(kin, n, shift, mask, ntiles, b.hist);
    k_radix_scan_rows<<<mask + 1, 256, 0, st>>>(b.hist, ntiles, b.dtot);
    if (first && last)
      k_radix_scatter<true, true><<<ntiles, kSortThreads, 0, st>>>(kin, vin, kout, vout, n, shift, mask, ntiles,
                                                                   b.hist, b.dtot, ga);
    else if (first)
      k_radix_scatter<true, false><<<ntiles, kSortThreads, 0, st>>>(kin, vin, kout, vout, n, shift, mask, ntiles,
                                                                    b.hist, b.dtot, ga);
    else if (last)
      k_radix_scatter<false, true><<<ntiles, kSortThreads, 0, st>>>(kin, vin, kout, vout, n, shift, mask, ntiles,
                                                                    b.hist, b.dtot, ga);
    else
      k_radix_scatter<false, false><<<ntiles, kSortThreads, 0, st>>>(kin, vin, kout, vout, n, shift, mask, ntiles,
                                                                     b.hist, b.dtot, ga);
    kin = kout;
    vin = vout;
  }
  cudaMemsetAsync(b.range, 0, sizeof(int2) * (size_t)P.grid.nbuckets, st);
  k_cell_ranges<<<cdiv(n, 256), 256, 0, st>>>(b.skey, n, P.grid.nbuckets, b.range);
}

void enqueue_density(const FluidBufs& b, uint32_t n, const StepParams& P, cudaStream_t st) {
  if (n == 0) return;
  const bool m = (P.flags & F_MASS) != 0, ph = (P.flags & F_PHASE) != 0;
  const uint32_t g = cdiv(n, 256);
  if (m && ph)
    k_density<true, true><<<g, 256, 0, st>>>(b.spos, b.skey, b.smass, b.sphase, n, b.range, P, b.sdq, b.spres);
  else if (m)
    k_density<true, false><<<g, 256, 0, st>>>(b.spos, b.skey, b.smass, b.sphase, n, b.range, P, b.sdq, b.spres);
  else if (ph)
    k_density<false, true><<<g, 256, 0, st>>>(b.spos, b.skey, b.smass, b.sphase, n, b.range, P, b.sdq, b.spres);
  else
    k_density<false, false><<<g, 256, 0, st>>>(b.spos, b.skey, b.smass, b.sphase, n, b.range, P, b.sdq, b.spres);
}

void enqueue_force_integrate(const FluidBufs& b, uint32_t n, const StepParams& P, float2* dbg_force,
                             cudaStream_t st) {
  if (n == 0) return;
  const bool m = (P.flags & F_MASS) != 0;
  const uint32_t g = cdiv(n, 256);
  if (dbg_force) {
    if (m)
      k_force_integrate<true, true><<<g, 256, 0, st>>>(b.spos, b.svel, b.sdq, b.skey, b.sid, b.smass, n, b.range, P,
                                                       b.bodies, b.state, b.key, dbg_force);
    else
      k_force_integrate<false, true><<<g, 256, 0, st>>>(b.spos, b.svel, b.sdq, b.skey, b.sid, b.smass, n, b.range,
                                                        P, b.bodies, b.state, b.key, dbg_force);
  } else {
    if (m)
      k_force_integrate<true, false><<<g, 256, 0, st>>>(b.spos, b.svel, b.sdq, b.skey, b.sid, b.smass, n, b.range,
                                                        P, b.bodies, b.state, b.key, nullptr);
    else
      k_force_integrate<false, false><<<g, 256, 0, st>>>(b.spos, b.svel, b.sdq, b.skey, b.sid, b.smass, n,
                                                         b.range, P, b.bodies, b.state, b.key, nullptr);
  }
}

void enqueue_unsort_dp(const FluidBufs& b, uint32_t n, float* dens, float* pres, cudaStream_t st) {
  if (n == 0) return;
  k_unsort_dp<<<cdiv(n, 256), 256, 0, st>>>(b.sdq, b.spres, b.sid, n, dens, pres);
}

void enqueue_debug_neighbors(const FluidBufs& b, uint32_t n, const StepParams& P, uint32_t* counts,
                             uint32_t* lists, uint32_t max_per, cudaStream_t st) {
  if (n == 0) return;
  k_debug_neighbors<<<cdiv(n, 256), 256, 0, st>>>(b.spos, b.skey, b.sid, n, b.range, P, counts, lists, max_per);
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
