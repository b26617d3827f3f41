// The coarse step of the learned closure in the tolerance mode, included by
// sph_kernels.cu after sph_fast.cuh, in two forms. k_closure_tc: one
// persistent kernel in which a CTA of 128 threads takes tiles of 128 sorted
// particles and, per tile,
//   1. walks each particle's neighbours with the tolerance-mode pair
//      arithmetic (sph_fast.cuh), accumulating the pressure force, the XSPH
//      sum and the 16 closure features (the exact pass's feature definitions,
//      sph_device.cuh feat_pair / feat_finish, with the kernel-weighted moments
//      summed without the constant poly6 factor, which their ratios cancel);
//   2. runs the network on the tile's 128 feature rows on the tcgen05 tensor
//      cores (sph_tc_net.cuh);
//   3. integrates with the predicted acceleration correction, as the exact
//      closure pass does (k_force_closure), writing the next keys and bucket
//      counts and the pre-step state / density for the fallback.
// Plain flag set only (fast_flags). A tensor-core wait that runs out sets
// *err and ends the CTA's work; the host reads the flag where it synchronises.

// One neighbour pair: FastPair's force and XSPH terms plus the feature sums.
struct FastFeatPair {
  float2 pi, vi;
  float rho_i, mq_i;
  __device__ __forceinline__ void operator()(float2 pj, float2 vj, float2 dqj, float2 vp, const StepParams& P,
                                             float& fx, float& fy, float& sx, float& sy, FeatAcc& a) const {
    const float dx = __fsub_rn(pi.x, pj.x);
    const float dy = __fsub_rn(pi.y, pj.y);
    const float d2 = __fmaf_rn(dx, dx, __fmul_rn(dy, dy));
    const float rinv = rsqrtf(d2);
    const float r = __fmul_rn(d2, rinv);
    const float hr = __fsub_rn(P.hk, r);
    const bool grad = r < P.hk && r >= kEps;
    const float gs = grad ? __fmul_rn(__fmul_rn(__fmul_rn(P.c_spiky, hr), hr), rinv) : 0.0f;  // grad = delta * gs
    const float c = __fmul_rn(gs, __fmaf_rn(P.mass, dqj.y, mq_i));
    fx = __fmaf_rn(-dx, c, fx);
    fy = __fmaf_rn(-dy, c, fy);
    const float t = __fsub_rn(P.hk2, d2);
    const float t3 = __fmul_rn(__fmul_rn(t, t), t);
    const float dvx = __fsub_rn(vj.x, vi.x), dvy = __fsub_rn(vj.y, vi.y);
    const float w = __fmul_rn(t3, __fdividef(1.0f, __fadd_rn(rho_i, fmaxf(dqj.x, kEps))));
    sx = __fmaf_rn(dvx, w, sx);
    sy = __fmaf_rn(dvy, w, sy);
    // features: V_j = vp.x = m / rho_j, p_j = vp.y
    const float gv = __fmul_rn(gs, vp.x);
    a.div = __fmaf_rn(gv, __fmaf_rn(dvx, dx, __fmul_rn(dvy, dy)), a.div);
    a.curl = __fmaf_rn(gv, __fmaf_rn(dvx, dy, -__fmul_rn(dvy, dx)), a.curl);
    const float ww = __fmul_rn(vp.x, t3);
    const float wx = __fmul_rn(ww, dvx), wy = __fmul_rn(ww, dvy);
    a.wsum = __fadd_rn(a.wsum, ww);
    a.m1x = __fadd_rn(a.m1x, wx);
    a.m1y = __fadd_rn(a.m1y, wy);
    a.m2xx = __fmaf_rn(wx, dvx, a.m2xx);
    a.m2yy = __fmaf_rn(wy, dvy, a.m2yy);
    a.pw = __fmaf_rn(ww, vp.y, a.pw);
    a.cnt++;
  }
};

// At most 6 CTAs share an SM (shared memory), so 80 registers cost nothing.
template <bool BATCH>
__global__ void __launch_bounds__(128, 6) k_closure_tc(
    const float2* __restrict__ spos, const float2* __restrict__ svel, const float2* __restrict__ sdq,
    const float* __restrict__ spres, const uint32_t* __restrict__ skey, const uint32_t* __restrict__ sid, uint32_t n,
    const uint32_t* __restrict__ start, StepParams P0, BatchTab bt, const DevBody* __restrict__ bodies,
    const uint32_t* __restrict__ nmask, MlpDev mlp, ClosureIO io, float4* __restrict__ state_out,
    uint32_t* __restrict__ key_out, uint32_t* __restrict__ count_out, uint32_t* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char net_smem[];
  TcNet net = tc_net_init(net_smem, mlp);
  bool ok = true;
  for (uint32_t base = blockIdx.x * 128u; base < n; base += gridDim.x * 128u) {
    const uint32_t s = base + threadIdx.x;
    const bool active = s < n;
    const StepParams& P = scene_params<BATCH>(P0, bt.ptab, BATCH && active ? bt.sscene[s] : 0u);
    float f[kFeat];
    float fx = 0.0f, fy = 0.0f, sx = 0.0f, sy = 0.0f;
    uint32_t id = 0;
    FastFeatPair pair;
    if (active) {
      const GridPlan& g = P.grid;
      const uint32_t k = skey[s];
      id = sid[s];
      const float2 dqi = sdq[s];
      pair.pi = spos[s];
      pair.vi = svel[s];
      pair.rho_i = fmaxf(dqi.x, kEps);
      pair.mq_i = __fmul_rn(P.mass, dqi.y);
      FeatAcc fa;
      const uint32_t own = nmask[n + s];
      uint32_t lo[3], hi[3];
      if (candidate_rows(k, start, g, lo, hi) && own != 0u) {
        uint32_t m[3] = {nmask[s], own & ~(1u << (s - lo[1])), nmask[2 * (size_t)n + s]};
#pragma unroll
        for (int r = 0; r < 3; r++) {
          uint32_t cur = m[r];
          while (cur) {
            const uint32_t j = lo[r] + (uint32_t)(__ffs((int)cur) - 1);
            cur &= cur - 1u;
            pair(__ldg(&spos[j]), __ldg(&svel[j]), __ldg(&sdq[j]), __ldg(&io.svp[j]), P, fx, fy, sx, sy, fa);
          }
        }
      } else if (k != g.sentinel) {
        for_each_candidate(k, start, g, [&](int jj) {
          const uint32_t j = (uint32_t)jj;
          const float2 pj = __ldg(&spos[j]);
          const float ex = __fsub_rn(pj.x, pair.pi.x), ey = __fsub_rn(pj.y, pair.pi.y);
          if (__fadd_rn(__fmul_rn(ex, ex), __fmul_rn(ey, ey)) < P.hg2 && j != s)
            pair(pj, __ldg(&svel[j]), __ldg(&sdq[j]), __ldg(&io.svp[j]), P, fx, fy, sx, sy, fa);
        });
      }
      fa.px = fx;  // the pressure feature is the force sum (plain flag set)
      fa.py = fy;
      float wd, wnx, wny;
      wall_feature(pair.pi.x, pair.pi.y, bodies, P, wd, wnx, wny);
      feat_finish(fa, dqi.x, pair.rho_i, spres[s], P.rest[P.uniform_phase], pair.vi.x, pair.vi.y, wd, wnx, wny, P, f);
      io.save[id] = make_float4(pair.pi.x, pair.pi.y, pair.vi.x, pair.vi.y);
      io.rho_prev[id] = dqi.x;
    } else {
#pragma unroll
      for (int q = 0; q < kFeat; q++) f[q] = net.norm()[q];  // normalises to zero; the row is discarded
    }
    float y[2];
    ok = tc_net_forward(net, f, y);
    if (!ok) break;
    if (active) {
      const float acc_scale = __fdiv_rn(P.hk, __fmul_rn(P.dt, P.dt));  // h / dt^2: y is a displacement in units of h
      const float xs = __fmul_rn(__fmul_rn(2.0f, P.mass), P.c_poly6);
      const float ax = __fadd_rn(__fadd_rn(P.gx, __fdiv_rn(fx, pair.rho_i)), __fmul_rn(y[0], acc_scale));
      const float ay = __fadd_rn(__fadd_rn(P.gy, __fdiv_rn(fy, pair.rho_i)), __fmul_rn(y[1], acc_scale));
      integrate_write<false>(id, pair.pi, pair.vi, ax, ay, __fmul_rn(sx, xs), __fmul_rn(sy, xs), P, bodies, state_out,
                             key_out, count_out);
    }
  }
  tc_net_finish(net, ok, err);
}

// The tolerance-mode coarse pass with the network on warp-level mma.sync
// tiles: the fast pair arithmetic and feature sums of k_closure_tc
// (FastFeatPair), then per warp the network on its 32 particles as in
// k_force_closure, then the corrected integrate. Plain flag set only
// (fast_flags). One 256-thread block per 256 sorted particles.
template <bool BATCH>
__global__ void __launch_bounds__(256, 4) k_closure_fast(
    const float2* __restrict__ spos, const float2* __restrict__ svel, const float2* __restrict__ sdq,
    const float* __restrict__ spres, const uint32_t* __restrict__ skey, const uint32_t* __restrict__ sid, uint32_t n,
    const uint32_t* __restrict__ start, StepParams P0, BatchTab bt, const DevBody* __restrict__ bodies,
    const uint32_t* __restrict__ nmask, MlpDev mlp, ClosureIO io, float4* __restrict__ state_out,
    uint32_t* __restrict__ key_out, uint32_t* __restrict__ count_out) {
  extern __shared__ __align__(16) unsigned char closure_smem[];
  MlpSmem& sm = *reinterpret_cast<MlpSmem*>(closure_smem);
  __nv_bfloat16* sx_all = reinterpret_cast<__nv_bfloat16*>(closure_smem + sizeof(MlpSmem));
  float* sy_all = reinterpret_cast<float*>(closure_smem + sizeof(MlpSmem) + sizeof(__nv_bfloat16) * 256 * kXRow);
  mlp_load_smem(sm, mlp);
  __syncthreads();
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = s < n;
  const StepParams& P = scene_params<BATCH>(P0, bt.ptab, BATCH && active ? bt.sscene[s] : 0u);
  float f[kFeat];
  float fx = 0.0f, fy = 0.0f, sx = 0.0f, sy = 0.0f;
  uint32_t id = 0;
  FastFeatPair pair;
  if (active) {
    const GridPlan& g = P.grid;
    const uint32_t k = skey[s];
    id = sid[s];
    const float2 dqi = sdq[s];
    pair.pi = spos[s];
    pair.vi = svel[s];
    pair.rho_i = fmaxf(dqi.x, kEps);
    pair.mq_i = __fmul_rn(P.mass, dqi.y);
    FeatAcc fa;
    const uint32_t own = nmask[n + s];
    uint32_t lo[3], hi[3];
    if (candidate_rows(k, start, g, lo, hi) && own != 0u) {
      uint32_t m[3] = {nmask[s], own & ~(1u << (s - lo[1])), nmask[2 * (size_t)n + s]};
#pragma unroll
      for (int r = 0; r < 3; r++) {
        uint32_t cur = m[r];
        while (cur) {
          const uint32_t j = lo[r] + (uint32_t)(__ffs((int)cur) - 1);
          cur &= cur - 1u;
          pair(__ldg(&spos[j]), __ldg(&svel[j]), __ldg(&sdq[j]), __ldg(&io.svp[j]), P, fx, fy, sx, sy, fa);
        }
      }
    } else if (k != g.sentinel) {
      for_each_candidate(k, start, g, [&](int jj) {
        const uint32_t j = (uint32_t)jj;
        const float2 pj = __ldg(&spos[j]);
        const float ex = __fsub_rn(pj.x, pair.pi.x), ey = __fsub_rn(pj.y, pair.pi.y);
        if (__fadd_rn(__fmul_rn(ex, ex), __fmul_rn(ey, ey)) < P.hg2 && j != s)
          pair(pj, __ldg(&svel[j]), __ldg(&sdq[j]), __ldg(&io.svp[j]), P, fx, fy, sx, sy, fa);
      });
    }
    fa.px = fx;  // the pressure feature is the force sum (plain flag set)
    fa.py = fy;
    float wd, wnx, wny;
    wall_feature(pair.pi.x, pair.pi.y, bodies, P, wd, wnx, wny);
    feat_finish(fa, dqi.x, pair.rho_i, spres[s], P.rest[P.uniform_phase], pair.vi.x, pair.vi.y, wd, wnx, wny, P, f);
    io.save[id] = make_float4(pair.pi.x, pair.pi.y, pair.vi.x, pair.vi.y);
    io.rho_prev[id] = dqi.x;
  } else {
#pragma unroll
    for (int q = 0; q < kFeat; q++) f[q] = sm.norm[q];  // normalises to zero; the row is discarded
  }
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
  const float acc_scale = __fdiv_rn(P.hk, __fmul_rn(P.dt, P.dt));  // h / dt^2: y is a displacement in units of h
  const float xsc = __fmul_rn(__fmul_rn(2.0f, P.mass), P.c_poly6);
  const float cx = __fmul_rn(__fmul_rn(ys[2 * lane], sm.norm[2 * kFeat]), acc_scale);
  const float cy = __fmul_rn(__fmul_rn(ys[2 * lane + 1], sm.norm[2 * kFeat + 1]), acc_scale);
  const float ax = __fadd_rn(__fadd_rn(P.gx, __fdiv_rn(fx, pair.rho_i)), cx);
  const float ay = __fadd_rn(__fadd_rn(P.gy, __fdiv_rn(fy, pair.rho_i)), cy);
  integrate_write<false>(id, pair.pi, pair.vi, ax, ay, __fmul_rn(sx, xsc), __fmul_rn(sy, xsc), P, bodies, state_out,
                         key_out, count_out);
}
