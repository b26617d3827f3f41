// Tolerance-mode density and force passes (K5 / K6), included by
// sph_kernels.cu inside its anonymous namespace: they use its neighbour walk
// (for_each_candidate) and integrate (integrate_write).
//
// Scope: the plain flag set (uniform mass and phase, XSPH on, no artificial
// viscosity, cohesion, turbulence, ghosts or polygons, h > 0) of a single
// world or of every scene of a batch. The neighbour sets, the sort order and
// the per-particle visit order are the exact passes': the neighbour test
// d2 < h*h keeps the reference's rounding (fluid.rs:383), so the neighbour
// lists and the row masks are the same bits.
//   density  k_density_fast is the exact density pass (the same products in
//            the same order: bit-identical results) with its neighbour rows
//            staged in shared memory, a launch shape (PhiengSphTuning.stage
//            bit 0); without staging the mode runs k_density itself.
//            Reassociating the density sum does not pay: the neighbour test
//            needs the reference's d2, which leaves one multiply per
//            candidate to save (measured slower);
//   force    one approximate reciprocal square root per pair gives the
//            distance and the direction of the spiky gradient (fluid.rs:278-285),
//            m (q_i + q_j) as one fused multiply-add, the sum accumulated
//            with fused multiply-adds (fluid.rs:942-997);
//   XSPH     (v_j - v_i) t^3 / (rho_i + rho_j) summed with one approximate
//            reciprocal per pair, scaled by 2 m c_poly6 once
//            (fluid.rs:1022-1033).
// Every operation is an explicit intrinsic in a fixed order, so a run is
// bit-reproducible; the parity tests bound the difference to the reference's
// arithmetic (force 1e-4 of the RMS from identical state). The per-particle
// epilogue (integrate, walls, next key) is the exact pass's.
//
// STAGE: the block first copies the three neighbour-row windows of its
// particles (row r's window = the union of the block's slot ranges of that
// row: contiguous, since slots are sorted by bucket and a row's three buckets
// are consecutive keys) from the sorted arrays into shared memory with
// 16-byte loads, and the loops read them there. If any window is longer than
// the block's capacity (a block across a wrapped bucket row, a crowded
// aliased row), nothing is staged and the block reads global memory.
// Staging measured slower on B200 (the rows are L1 / L2 resident) and is off
// by default.
//
// The force pass walks a thread's three rows as one flattened loop (the next
// row's range starts as soon as the current one ends), so a warp's trip count
// is the largest per-lane total, not the sum of the per-row maxima.

// Staged slots per row window for a block of `threads` threads: a block of
// B consecutive particles of one bucket row spans about B / 4 cells, i.e.
// about B + 8 slots per neighbour row at rest density.
__host__ __device__ constexpr uint32_t fast_stage_cap(uint32_t threads) { return 2 * threads + 64; }

// Row windows of the block: lo[r] <= every staged slot < hi[r]; staged iff
// hi - (lo & ~1) fits the capacity. base[r] = lo[r] & ~1 (16-byte aligned
// float2 pairs).
struct RowWindows {
  uint32_t base[3];
  uint32_t len[3];  // all 0: nothing staged
  __device__ __forceinline__ bool staged() const { return len[0] != 0u; }
};

// Block-wide min / max of the per-thread row ranges (threads without masks
// contribute nothing), then the staging decision. Every thread of the block
// must call it.
__device__ __forceinline__ RowWindows block_row_windows(const uint32_t lo[3], const uint32_t hi[3], uint32_t cap) {
  __shared__ uint32_t s_lo[3], s_hi[3];
  if (threadIdx.x < 3) {
    s_lo[threadIdx.x] = 0xFFFFFFFFu;
    s_hi[threadIdx.x] = 0u;
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < 3; r++) {
    const uint32_t a = __reduce_min_sync(0xFFFFFFFFu, lo[r]);
    const uint32_t b = __reduce_max_sync(0xFFFFFFFFu, hi[r]);
    if ((threadIdx.x & 31u) == 0u) {
      atomicMin(&s_lo[r], a);
      atomicMax(&s_hi[r], b);
    }
  }
  __syncthreads();
  RowWindows w;
  bool all = true;
#pragma unroll
  for (int r = 0; r < 3; r++) {
    const uint32_t l = s_lo[r], h = s_hi[r];
    w.base[r] = l & ~1u;
    w.len[r] = h > l ? h - w.base[r] : 0u;
    all = all && h > l && w.len[r] <= cap;
  }
  if (!all) w.len[0] = w.len[1] = w.len[2] = 0u;  // stage all three rows or none
  return w;
}

// Copy slots [base, base + len) of a float2 array into dst with 16-byte loads
// (base even, so every pair is 16-byte aligned: cudaMalloc'd arrays are).
__device__ __forceinline__ void stage_rows(float2* __restrict__ dst, const float2* __restrict__ src, uint32_t base,
                                           uint32_t len) {
  const float4* s4 = reinterpret_cast<const float4*>(src + base);
  float4* d4 = reinterpret_cast<float4*>(dst);
  const uint32_t pairs = len >> 1;
  for (uint32_t i = threadIdx.x; i < pairs; i += blockDim.x) d4[i] = __ldg(&s4[i]);
  if ((len & 1u) && threadIdx.x == 0) dst[len - 1] = __ldg(&src[base + len - 1]);
}

// The three candidate rows of a particle in bucket k away from the x seam:
// row r (oy = r - 1) holds slots [lo[r], hi[r]). Particles on the seam or
// with the sentinel key get empty ranges (lo = ~0, hi = 0).
__device__ __forceinline__ bool candidate_rows(uint32_t k, const uint32_t* __restrict__ start, const GridPlan& g,
                                               uint32_t lo[3], uint32_t hi[3]) {
  lo[0] = lo[1] = lo[2] = 0xFFFFFFFFu;
  hi[0] = hi[1] = hi[2] = 0u;
  if (k == g.sentinel) return false;
  const uint32_t local = k - g.base;
  const uint32_t bx = local & g.maskw, by = local >> g.log2w;
  if (!(bx >= 1u && bx < g.maskw)) return false;
#pragma unroll
  for (int r = 0; r < 3; r++) {
    const uint32_t row = g.base + (((by + (uint32_t)r - 1u) & g.maskh) << g.log2w);
    lo[r] = __ldg(&start[row + bx - 1]);
    hi[r] = __ldg(&start[row + bx + 2]);
  }
  return true;
}

// ---------------------------------------------------------------- K5, shared-memory-staged
template <bool STAGE, bool BATCH>
__global__ void __launch_bounds__(256) k_density_fast(const float2* __restrict__ spos,
                                                      const uint32_t* __restrict__ skey, uint32_t n,
                                                      const uint32_t* __restrict__ start, StepParams P0, BatchTab bt,
                                                      float2* __restrict__ sdq, float* __restrict__ spres,
                                                      uint32_t* __restrict__ nmask, float2* __restrict__ svp) {
  extern __shared__ __align__(16) float2 fast_win[];
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = s < n;
  // a batch: the particle's scene row (its own bucket range inside the shared key space)
  const StepParams& P = scene_params<BATCH>(P0, bt.ptab, BATCH && active ? bt.sscene[s] : 0u);
  const GridPlan& g = P.grid;
  const uint32_t k = active ? skey[s] : P0.grid.sentinel;
  uint32_t lo[3], hi[3];
  const bool rows = candidate_rows(k, start, g, lo, hi);
  RowWindows win;
  const uint32_t cap = fast_stage_cap(blockDim.x);
  if constexpr (STAGE) {
    win = block_row_windows(lo, hi, cap);
    if (win.staged()) {
#pragma unroll
      for (int r = 0; r < 3; r++) stage_rows(fast_win + r * cap, spos, win.base[r], win.len[r]);
    }
    __syncthreads();
  }
  if (!active) return;
  const float2 pi = spos[s];
  float rho = 0.0f;
  uint32_t mrow[3] = {0, 0, 0};
  bool masks_ok = rows;
  if (rows) {
    auto visit = [&](const float2 a, uint32_t& m, uint32_t bit) {
      const float dx = __fsub_rn(a.x, pi.x), dy = __fsub_rn(a.y, pi.y);
      const float d2 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));  // the reference's rounding
      const bool nb = d2 < P.hg2;
      const float w = neighbour_density_term<false>(d2, P.mass, P);  // m * poly6, the exact pass's order
      rho = nb ? __fadd_rn(rho, w) : rho;
      m |= nb ? bit : 0u;
    };
    // row by row (a flattened loop over the three rows measured slower here:
    // the candidate loop is short and its row switch costs more than the
    // lanes it keeps busy); a row's mask bit shifts out after 32 slots (then
    // masks_ok is false)
#pragma unroll
    for (int r = 0; r < 3; r++) {
      uint32_t m = 0u, bit = 1u;
      if (STAGE && win.staged()) {
        const uint32_t o = r * cap - win.base[r];  // shared index of slot j: o + j (mod 2^32)
        for (uint32_t j = lo[r]; j < hi[r]; j++, bit <<= 1) visit(fast_win[o + j], m, bit);
      } else {
        for (uint32_t j = lo[r]; j < hi[r]; j++, bit <<= 1) visit(__ldg(&spos[j]), m, bit);
      }
      mrow[r] = m;
    }
#pragma unroll
    for (int r = 0; r < 3; r++)
      if (hi[r] - lo[r] > kMaskBits) masks_ok = false;
  } else if (k != g.sentinel) {
    // x seam: the reference's cell-by-cell walk
    for_each_candidate(k, start, g, [&](int j) {
      const float2 a = __ldg(&spos[j]);
      const float dx = __fsub_rn(a.x, pi.x), dy = __fsub_rn(a.y, pi.y);
      rho = __fadd_rn(rho, density_term(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), P.mass, P));
    });
  }
  if (!masks_ok) mrow[1] = 0;  // the force pass walks the candidates itself
  nmask[s] = mrow[0];
  nmask[n + s] = mrow[1];
  nmask[2 * (size_t)n + s] = mrow[2];
  float dens = rho;
  if (dens < 0.0f) dens = 0.0f;  // f32::clamp(0, 3 * max(rest_density, EPS)) (fluid.rs:605)
  if (dens > P.rho_cap) dens = P.rho_cap;
  const float p = eos(dens, P.rest[P.uniform_phase], P);
  const float rc = fmaxf(dens, kEps);
  const float q = __fdiv_rn(p, __fmul_rn(rc, rc));
  sdq[s] = make_float2(dens, q);
  spres[s] = p;
  // closure passes: the per-neighbour factors of the feature sums, m / rho and p
  if (svp) svp[s] = make_float2(__fdiv_rn(P.mass, rc), __fmul_rn(__fmul_rn(q, rc), rc));
}

// ---------------------------------------------------------------- K6 (tolerance mode)
// One neighbour pair: pressure force into (fx, fy), the XSPH sum (before its
// 2 m c_poly6 factor) into (sx, sy).
struct FastPair {
  float2 pi, vi;
  float rho_i, mq_i;
  __device__ __forceinline__ void operator()(float2 pj, float2 vj, float2 dqj, const StepParams& P, float& fx,
                                             float& fy, float& sx, float& sy) const {
    const float dx = __fsub_rn(pi.x, pj.x);
    const float dy = __fsub_rn(pi.y, pj.y);
    const float d2 = __fmaf_rn(dx, dx, __fmul_rn(dy, dy));
    const float rinv = rsqrtf(d2);  // d2 = 0 (coincident): inf, and r below is NaN -> no gradient
    const float r = __fmul_rn(d2, rinv);
    const float hr = __fsub_rn(P.hk, r);
    const bool grad = r < P.hk && r >= kEps;  // spiky_grad's support (fluid.rs:280)
    const float gs = grad ? __fmul_rn(__fmul_rn(__fmul_rn(P.c_spiky, hr), hr), rinv) : 0.0f;
    const float c = __fmul_rn(gs, __fmaf_rn(P.mass, dqj.y, mq_i));  // m (q_i + q_j)
    fx = __fmaf_rn(-dx, c, fx);
    fy = __fmaf_rn(-dy, c, fy);
    const float t = __fsub_rn(P.hk2, d2);
    const float w = __fmul_rn(__fmul_rn(__fmul_rn(t, t), t), __fdividef(1.0f, __fadd_rn(rho_i, fmaxf(dqj.x, kEps))));
    sx = __fmaf_rn(__fsub_rn(vj.x, vi.x), w, sx);
    sy = __fmaf_rn(__fsub_rn(vj.y, vi.y), w, sy);
  }
};

// The slot a thread of a BALANCE launch takes: the block's slots ordered by
// their neighbour count (the three rows' mask bits; a slot without masks,
// which walks its candidates, counts as the largest), so the lanes of a warp
// run about as many pair iterations each. Only the lane that computes a
// particle changes, not its arithmetic or its order: results are the same.
// blockDim.x <= 256; every thread of the block calls it.
__device__ __forceinline__ uint32_t balanced_slot(const uint32_t* __restrict__ nmask, uint32_t n) {
  __shared__ uint32_t hist[64];
  __shared__ uint32_t perm[256];
  const uint32_t tid = threadIdx.x, s0 = blockIdx.x * blockDim.x + tid;
  uint32_t c = 0;
  if (s0 < n) {
    const uint32_t own = nmask[n + s0];
    c = own ? min(__popc(nmask[s0]) + __popc(own) + __popc(nmask[2 * (size_t)n + s0]), 63u) : 63u;
  }
  if (tid < 64) hist[tid] = 0u;
  __syncthreads();
  const uint32_t r = atomicAdd(&hist[c], 1u);  // rank inside the count's bin (any order will do)
  __syncthreads();
  if (tid < 32) {  // exclusive scan of the 64 bins, two per lane
    const uint32_t a = hist[2 * tid], b = hist[2 * tid + 1];
    uint32_t x = a + b;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
      if (tid >= (uint32_t)o) x += y;
    }
    const uint32_t ex = x - a - b;
    hist[2 * tid] = ex;
    hist[2 * tid + 1] = ex + a;
  }
  __syncthreads();
  perm[hist[c] + r] = s0;
  __syncthreads();
  return perm[tid];
}

// BALANCE: the block's slots reassigned to its lanes by neighbour count
// (balanced_slot); not combined with STAGE.
template <bool STAGE, bool DEBUG, bool BATCH, bool BALANCE = false>
__global__ void __launch_bounds__(256) k_force_fast(
    const float2* __restrict__ spos, const float2* __restrict__ svel, const float2* __restrict__ sdq,
    const uint32_t* __restrict__ skey, const uint32_t* __restrict__ sid, uint32_t n,
    const uint32_t* __restrict__ start, StepParams P0, BatchTab bt, const DevBody* __restrict__ bodies,
    const uint32_t* __restrict__ nmask, float4* __restrict__ state_out, uint32_t* __restrict__ key_out,
    uint32_t* __restrict__ count_out, float2* __restrict__ dbg_force, uint32_t* __restrict__ defer,
    uint32_t* __restrict__ dcount) {
  static_assert(!(STAGE && BALANCE), "staging windows assume the block's own slot order");
  extern __shared__ __align__(16) float2 fast_win[];
  const uint32_t s = BALANCE ? balanced_slot(nmask, n) : blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = s < n;
  const StepParams& P = scene_params<BATCH>(P0, bt.ptab, BATCH && active ? bt.sscene[s] : 0u);
  const GridPlan& g = P.grid;
  const uint32_t k = active ? skey[s] : P0.grid.sentinel;
  const uint32_t own = active ? nmask[n + s] : 0u;
  uint32_t lo[3], hi[3];
  const bool rows = candidate_rows(k, start, g, lo, hi) && own != 0u;
  if (!rows) {
    lo[0] = lo[1] = lo[2] = 0xFFFFFFFFu;
    hi[0] = hi[1] = hi[2] = 0u;
  }
  RowWindows win;
  const uint32_t cap = fast_stage_cap(blockDim.x);
  float2* wp = fast_win;            // [3][cap] positions
  float2* wv = fast_win + 3 * cap;  // [3][cap] velocities
  float2* wq = fast_win + 6 * cap;  // [3][cap] (density, q)
  if constexpr (STAGE) {
    win = block_row_windows(lo, hi, cap);
    if (win.staged()) {
#pragma unroll
      for (int r = 0; r < 3; r++) {
        stage_rows(wp + r * cap, spos, win.base[r], win.len[r]);
        stage_rows(wv + r * cap, svel, win.base[r], win.len[r]);
        stage_rows(wq + r * cap, sdq, win.base[r], win.len[r]);
      }
    }
    __syncthreads();
  }
  if (!active) return;
  const uint32_t id = sid[s];
  const float2 dqi = sdq[s];
  FastPair pair;
  pair.pi = spos[s];
  pair.vi = svel[s];
  pair.rho_i = fmaxf(dqi.x, kEps);
  pair.mq_i = __fmul_rn(P.mass, dqi.y);
  float fx = 0.0f, fy = 0.0f, sx = 0.0f, sy = 0.0f;
  if (rows) {
    // the three rows' neighbour bits in ascending slot order, the particle's
    // own bit cleared (j != i, fluid.rs:947-950)
    const uint32_t m1 = own & ~(1u << (s - lo[1])), m2 = nmask[2 * (size_t)n + s];
    // the three rows' set bits as one loop (ascending slots, row by row)
    auto walk = [&](auto pair_at, uint32_t o0, uint32_t o1, uint32_t o2) {
      uint32_t cur = nmask[s], row = 0, o = o0;
      for (;;) {
        while (cur == 0u && row < 2u) {
          row++;
          cur = row == 1u ? m1 : m2;
          o = row == 1u ? o1 : o2;
        }
        if (cur == 0u) break;
        const uint32_t j = o + (uint32_t)(__ffs((int)cur) - 1);
        cur &= cur - 1u;
        pair_at(j);
      }
    };
    if (STAGE && win.staged())
      walk([&](uint32_t j) { pair(wp[j], wv[j], wq[j], P, fx, fy, sx, sy); }, lo[0] - win.base[0],
           cap + lo[1] - win.base[1], 2u * cap + lo[2] - win.base[2]);
    else
      walk([&](uint32_t j) { pair(__ldg(&spos[j]), __ldg(&svel[j]), __ldg(&sdq[j]), P, fx, fy, sx, sy); }, lo[0],
           lo[1], lo[2]);
  } else if (k != g.sentinel) {
    // no masks (x seam, or a row longer than 32 slots): walk the candidates
    for_each_candidate(k, start, g, [&](int jj) {
      const uint32_t j = (uint32_t)jj;
      const float2 pj = __ldg(&spos[j]);
      const float ex = __fsub_rn(pj.x, pair.pi.x), ey = __fsub_rn(pj.y, pair.pi.y);
      if (__fadd_rn(__fmul_rn(ex, ex), __fmul_rn(ey, ey)) < P.hg2 && j != s)
        pair(pj, __ldg(&svel[j]), __ldg(&sdq[j]), P, fx, fy, sx, sy);
    });
  }
  if (DEBUG) {
    dbg_force[id] = make_float2(fx, fy);
    return;
  }
  const float xs = __fmul_rn(__fmul_rn(2.0f, P.mass), P.c_poly6);  // XSPH: m_j / rho_bar * W = 2 m c t^3 / (rho_i + rho_j)
  const float ax = __fadd_rn(P.gx, __fdiv_rn(fx, pair.rho_i));
  const float ay = __fadd_rn(P.gy, __fdiv_rn(fy, pair.rho_i));
  integrate_write<false>(id, pair.pi, pair.vi, ax, ay, __fmul_rn(sx, xs), __fmul_rn(sy, xs), P, bodies, state_out,
                         key_out, count_out, defer, dcount);
}
