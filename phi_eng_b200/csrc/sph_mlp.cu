// Closure network: parameters on the device, the standalone forward pass,
// and training (forward + backward + Adam) with hand-written kernels.
//
// Training step for a minibatch of B samples drawn from (features, target)
// pairs, loss L = 1/(2B) sum_b |y_b - t_b / out_scale|^2:
//   k_mlp_train_tc    (default) each CTA takes B / gridDim samples in rounds
//                     of 128 on the 5th-generation tensor cores: forward,
//                     dH1 and the hidden layers' weight and bias gradients as
//                     tcgen05.mma chains with TMEM accumulators (the layout
//                     is described above the kernel).
//   k_mlp_train_tile  the same on warp-level mma.sync tiles:
//                     every warp runs forward and backward for 32 samples on
//                     the tensor cores (activations stay in registers or
//                     shared memory), then the CTA forms its partial weight
//                     gradients dW2 = dZ2^T H1 and dW1 = dZ1^T X with the
//                     sample dimension as K (tensor cores), dW3 and the bias
//                     gradients in FP32; one partial vector per CTA.
//   k_mlp_adam        per parameter: sum of the CTA partials in CTA order,
//                     Adam, new FP32 master and its BF16 fragment images.
//   k_mlp_advance     step counter + 1.
// No float atomics anywhere: a run is bit-reproducible.
//
// Minibatch sample k of step t is pair
//   idx = (mix64(seed ^ (t << 32) ^ k) >> 32) * npairs >> 32
// with mix64 the SplitMix64 finaliser (Steele, Lea, Flood 2014).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "phieng_sph.h"
#include "sph_mlp.cuh"
#include "sph_mlp_host.h"
#include "sph_tc_net.cuh"

static_assert(phieng::kMlpInferTcgen05 == PHIENG_MLP_TCGEN05 && phieng::kMlpInferMmaSync == PHIENG_MLP_MMA_SYNC,
              "engine codes");

namespace phieng {
namespace {

constexpr int kTrainThreads = 128;
constexpr int kTileRows = 128;  // samples per CTA round
constexpr int kXR = 24;         // staged feature row stride (BF16)
constexpr int kLdT = kTileRows + 8;
constexpr int kPartStride = 5384;  // kParams gradient entries, then the loss
constexpr float kBeta1 = 0.9f, kBeta2 = 0.999f, kAdamEps = 1e-8f;

__host__ __device__ inline uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__host__ __device__ inline uint32_t sample_index(uint64_t seed, uint32_t iter, uint32_t k, uint32_t npairs) {
  const uint64_t h = mix64(seed ^ ((uint64_t)iter << 32) ^ (uint64_t)k);
  return (uint32_t)(((h >> 32) * (uint64_t)npairs) >> 32);
}

struct TrainSmem {
  uint2 f1[kF1];
  uint2 f2[kF2];
  uint2 f3[kF3];
  uint2 f2t[kF2T];
  float bias[kBias];
  float w3[kOut * kHidden];
  float norm[kNorm];
  float tgt[kTileRows][2];
  float dy[kTileRows][2];
  float db[4][2 * kHidden];            // per-warp bias-gradient sums (b1 | b2)
  alignas(16) float z1[4][2][8][32][4];  // per warp: halved layer-1 pre-activations (z1 / 2), C-fragment order
  __nv_bfloat16 xs[kTileRows][kXR];    // x_hat, row major
  __nv_bfloat16 xt[kFeat][kLdT];       // x_hat^T
  __nv_bfloat16 h1t[kHidden][kLdT];    // H1^T
  __half h2t[kHidden][kLdT];           // H2^T (FP16, as the forward)
  __nv_bfloat16 dz2t[kHidden][kLdT];   // dZ2^T
  __nv_bfloat16 dz1t[kHidden][kLdT];   // dZ1^T
};

// Weight p of the flat parameter vector into the fragment images (F1, F2T
// BF16; F2, F3 FP16), the FP32 bias array and the FP16-rounded W3 copy (the
// forward's W3, for the backward pass).
__device__ __forceinline__ void write_weight(int p, float w, __nv_bfloat16* img, float* bias, float* w3) {
  __half* himg = reinterpret_cast<__half*>(img);
  if (p < kOffB1) {
    const int n = p / kFeat, k = p % kFeat;
    img[frag_pos(k, n, 8)] = __float2bfloat16_rn(__fmul_rn(0.5f, w));  // = bf16(w) / 2 exactly
  } else if (p < kOffW2) {
    bias[p - kOffB1] = __fmul_rn(0.5f, w);
  } else if (p < kOffB2) {
    const int q = p - kOffW2, o = q / kHidden, i = q % kHidden;
    himg[4 * kF1 + frag_pos(i, o, 8)] = __float2half_rn(__fmul_rn(0.5f, w));
    img[4 * (kF1 + kF2 + kF3) + frag_pos(o, i, 8)] = __float2bfloat16_rn(w);
  } else if (p < kOffW3) {
    bias[kHidden + (p - kOffB2)] = __fmul_rn(0.5f, w);
  } else if (p < kOffB3) {
    const int q = p - kOffW3, o = q / kHidden, n = q % kHidden;
    const __half h = __float2half_rn(w);
    himg[4 * (kF1 + kF2) + frag_pos(n, o, 1)] = h;
    w3[q] = __half2float(h);
  } else {
    bias[2 * kHidden + (p - kOffB3)] = w;
  }
}

__global__ void k_mlp_sync(const float* __restrict__ w, uint2* frag, float* bias, float* w3) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < kParams) write_weight(p, w[p], reinterpret_cast<__nv_bfloat16*>(frag), bias, w3);
}

__global__ void __launch_bounds__(128) k_mlp_forward(const float* __restrict__ x, uint32_t n, MlpDev mlp,
                                                     float* __restrict__ y) {
  __shared__ MlpSmem sm;
  __shared__ __align__(16) __nv_bfloat16 xs[128 * kXR];
  __shared__ float ys[128 * 2];
  mlp_load_smem(sm, mlp);
  __syncthreads();
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (uint32_t base = blockIdx.x * 128u; base < n; base += gridDim.x * 128u) {
    const uint32_t i = base + tid;
    float f[kFeat];
    if (i < n) {
      const float4* xi = reinterpret_cast<const float4*>(x + (size_t)i * kFeat);
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const float4 v = xi[q];
        f[4 * q] = v.x;
        f[4 * q + 1] = v.y;
        f[4 * q + 2] = v.z;
        f[4 * q + 3] = v.w;
      }
    } else {
#pragma unroll
      for (int q = 0; q < kFeat; q++) f[q] = sm.norm[q];  // normalises to zero
    }
    mlp_normalise_row(f, sm.norm, xs + tid * kXR);
    __syncwarp();
#pragma unroll
    for (int mt = 0; mt < 2; mt++) {
      float v[4];
      mlp_tile_forward(xs + (warp * 32 + mt * 16) * kXR, kXR, sm, lane, v);
      if ((lane & 3) == 0) {
        const int r = warp * 32 + mt * 16 + (lane >> 2);
        ys[2 * r] = v[0];
        ys[2 * r + 1] = v[1];
        ys[2 * (r + 8)] = v[2];
        ys[2 * (r + 8) + 1] = v[3];
      }
    }
    __syncwarp();
    if (i < n) {
      y[2 * (size_t)i] = __fmul_rn(ys[2 * tid], sm.norm[2 * kFeat]);
      y[2 * (size_t)i + 1] = __fmul_rn(ys[2 * tid + 1], sm.norm[2 * kFeat + 1]);
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------- tcgen05 forward
// The same network on the 5th-generation tensor cores (sph_tc_net.cuh): one
// CTA of 128 threads per tile of 128 rows, persistent over the tiles.
// Row i's 16 features, or the normalisation's mean (a zero input) past n.
__device__ __forceinline__ void load_features(const float* __restrict__ x, uint32_t i, uint32_t n, const float* mu,
                                              float (&f)[kFeat]) {
  if (i < n) {
    const float4* xi = reinterpret_cast<const float4*>(x + (size_t)i * kFeat);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const float4 v = xi[q];
      f[4 * q] = v.x;
      f[4 * q + 1] = v.y;
      f[4 * q + 2] = v.z;
      f[4 * q + 3] = v.w;
    }
  } else {
#pragma unroll
    for (int q = 0; q < kFeat; q++) f[q] = mu[q];
  }
}

__global__ void __launch_bounds__(128) k_mlp_forward_tc(const float* __restrict__ x, uint32_t n, MlpDev mlp,
                                                         float* __restrict__ y, uint32_t* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char tsm[];
  TcNet net = tc_net_init(tsm, mlp);
  bool ok = true;
  const uint32_t stride = gridDim.x * 128u;
  float f[kFeat];
  load_features(x, blockIdx.x * 128u + threadIdx.x, n, net.norm(), f);
  for (uint32_t base = blockIdx.x * 128u; base < n; base += stride) {
    const uint32_t i = base + threadIdx.x;
    // the next tile's features are loaded before this tile's network runs,
    // so their memory latency overlaps the tensor-core round trips
    float fn[kFeat];
    load_features(x, i + stride, n, net.norm(), fn);
    float o[2];
    ok = tc_net_forward(net, f, o);
    if (!ok) break;
    if (i < n) {
      y[2 * (size_t)i] = o[0];
      y[2 * (size_t)i + 1] = o[1];
    }
#pragma unroll
    for (int q = 0; q < kFeat; q++) f[q] = fn[q];
  }
  tc_net_finish(net, ok, err);
}

__device__ __forceinline__ void store_bf16(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }

// A packed 16-bit pair of columns (c0, c0 + 1) of row r into a transposed
// [column][row] array.
template <class T, int LD>
__device__ __forceinline__ void store_pair_t(T (*m)[LD], int c0, int r, uint32_t v) {
  static_assert(sizeof(T) == 2, "16-bit elements");
  *reinterpret_cast<uint16_t*>(&m[c0][r]) = (uint16_t)(v & 0xFFFFu);
  *reinterpret_cast<uint16_t*>(&m[c0 + 1][r]) = (uint16_t)(v >> 16);
}

// An FP16 pair as a BF16 pair (round to nearest even).
__device__ __forceinline__ uint32_t f16x2_to_bf16x2(uint32_t v) {
  const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&v));
  return pack_bf16(f.x, f.y);
}

// silu'(z) from the halved pre-activation u = z / 2 (z = 2u exactly).
__device__ __forceinline__ float dsilu_half(float u) { return dsilu_hw(__fmul_rn(2.0f, u)); }

// Sum over the 8 row groups of a warp (lanes with equal lane % 4), fixed order.
__device__ __forceinline__ float group_sum(float v) {
  v = __fadd_rn(v, __shfl_xor_sync(0xFFFFFFFFu, v, 4));
  v = __fadd_rn(v, __shfl_xor_sync(0xFFFFFFFFu, v, 8));
  v = __fadd_rn(v, __shfl_xor_sync(0xFFFFFFFFu, v, 16));
  return v;
}

__global__ void __launch_bounds__(kTrainThreads, 1)
    k_mlp_train_tile(const float* __restrict__ x, const float* __restrict__ tg, uint32_t npairs, uint32_t k0,
                     uint32_t total, uint32_t rounds, uint64_t seed, const uint32_t* __restrict__ iter_ptr, MlpDev mlp,
                     float* __restrict__ part) {
  extern __shared__ __align__(16) unsigned char train_smem[];
  TrainSmem& S = *reinterpret_cast<TrainSmem*>(train_smem);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
  for (int i = tid; i < kFragAll; i += kTrainThreads) {
    const uint2 v = mlp.frag[i];
    if (i < kF1)
      S.f1[i] = v;
    else if (i < kF1 + kF2)
      S.f2[i - kF1] = v;
    else if (i < kF1 + kF2 + kF3)
      S.f3[i - kF1 - kF2] = v;
    else
      S.f2t[i - kF1 - kF2 - kF3] = v;
  }
  for (int i = tid; i < kBias; i += kTrainThreads) S.bias[i] = mlp.bias[i];
  for (int i = tid; i < kOut * kHidden; i += kTrainThreads) S.w3[i] = mlp.w3[i];
  for (int i = tid; i < kNorm; i += kTrainThreads) S.norm[i] = mlp.norm[i];
  for (int i = tid; i < 4 * 2 * kHidden; i += kTrainThreads) (&S.db[0][0])[i] = 0.0f;
  const uint32_t iter = *iter_ptr;
  const float inv_b = __fdiv_rn(1.0f, (float)total);
  __syncthreads();
  const float inv_os0 = __fdiv_rn(1.0f, S.norm[2 * kFeat]), inv_os1 = __fdiv_rn(1.0f, S.norm[2 * kFeat + 1]);

  float acc_w2[8][4], acc_w1[2][4];
#pragma unroll
  for (int a = 0; a < 8; a++)
#pragma unroll
    for (int c = 0; c < 4; c++) acc_w2[a][c] = 0.0f;
#pragma unroll
  for (int a = 0; a < 2; a++)
#pragma unroll
    for (int c = 0; c < 4; c++) acc_w1[a][c] = 0.0f;
  float acc_w3 = 0.0f, acc_b3 = 0.0f, loss = 0.0f;

  for (uint32_t r = 0; r < rounds; r++) {
    // ---- gather 128 samples: row = warp * 32 + lane
    {
      const int row = tid;
      const uint32_t k = k0 + (blockIdx.x * rounds + r) * kTileRows + (uint32_t)row;
      const uint32_t idx = sample_index(seed, iter, k, npairs);
      const float4* xi = reinterpret_cast<const float4*>(x + (size_t)idx * kFeat);
      float f[kFeat];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const float4 v = xi[q];
        f[4 * q] = v.x;
        f[4 * q + 1] = v.y;
        f[4 * q + 2] = v.z;
        f[4 * q + 3] = v.w;
      }
      mlp_normalise_row(f, S.norm, &S.xs[row][0]);
#pragma unroll
      for (int q = 0; q < kFeat; q++) S.xt[q][row] = S.xs[row][q];
      S.tgt[row][0] = __fmul_rn(tg[2 * (size_t)idx], inv_os0);
      S.tgt[row][1] = __fmul_rn(tg[2 * (size_t)idx + 1], inv_os1);
    }
    __syncwarp();
    // ---- forward + backward, two 16-row tiles per warp
#pragma unroll 1
    for (int mt = 0; mt < 2; mt++) {
      const int r0 = warp * 32 + mt * 16;
      const int ra = r0 + g, rb = r0 + g + 8;
      uint32_t a[4];
      a[0] = lds32(&S.xs[ra][2 * t]);
      a[1] = lds32(&S.xs[rb][2 * t]);
      a[2] = lds32(&S.xs[ra][2 * t + 8]);
      a[3] = lds32(&S.xs[rb][2 * t + 8]);
      uint32_t h[4][4];
#pragma unroll
      for (int nt = 0; nt < 8; nt++) {
        const int c0 = nt * 8 + 2 * t;
        float c[4] = {S.bias[c0], S.bias[c0 + 1], S.bias[c0], S.bias[c0 + 1]};
        const uint2 b = S.f1[nt * 32 + lane];
        mma_bf16(c, a, b.x, b.y);
        // halved pre-activations u = z1 / 2, kept for the backward pass
        *reinterpret_cast<float4*>(&S.z1[warp][mt][nt][lane][0]) = make_float4(c[0], c[1], c[2], c[3]);
        const uint32_t ha = silu_half_f16x2(c[0], c[1]), hb = silu_half_f16x2(c[2], c[3]);
        h[nt >> 1][(nt & 1) * 2 + 0] = ha;
        h[nt >> 1][(nt & 1) * 2 + 1] = hb;
        // H1^T feeds dW2 = dZ2^T H1 on BF16 tensor cores
        store_pair_t(S.h1t, c0, ra, f16x2_to_bf16x2(ha));
        store_pair_t(S.h1t, c0, rb, f16x2_to_bf16x2(hb));
      }
      float z2v[8][4];
      uint32_t h2[4][4];
#pragma unroll
      for (int nt = 0; nt < 8; nt++) {
        const int c0 = nt * 8 + 2 * t;
        float c[4] = {S.bias[kHidden + c0], S.bias[kHidden + c0 + 1], S.bias[kHidden + c0], S.bias[kHidden + c0 + 1]};
#pragma unroll
        for (int kt = 0; kt < 4; kt++) {
          const uint2 b = S.f2[(kt * 8 + nt) * 32 + lane];
          mma_f16(c, h[kt], b.x, b.y);
        }
#pragma unroll
        for (int q = 0; q < 4; q++) z2v[nt][q] = c[q];  // u = z2 / 2
        const uint32_t ha = silu_half_f16x2(c[0], c[1]), hb = silu_half_f16x2(c[2], c[3]);
        h2[nt >> 1][(nt & 1) * 2 + 0] = ha;
        h2[nt >> 1][(nt & 1) * 2 + 1] = hb;
        store_pair_t(S.h2t, c0, ra, ha);
        store_pair_t(S.h2t, c0, rb, hb);
      }
      const float b30 = t == 0 ? S.bias[2 * kHidden] : 0.0f, b31 = t == 0 ? S.bias[2 * kHidden + 1] : 0.0f;
      float c3[4] = {b30, b31, b30, b31};
#pragma unroll
      for (int kt = 0; kt < 4; kt++) {
        const uint2 b = S.f3[kt * 32 + lane];
        mma_f16(c3, h2[kt], b.x, b.y);
      }
      // loss and dY on the lanes holding output columns 0 and 1
      float dyl[4] = {0.0f, 0.0f, 0.0f, 0.0f};
      if (t == 0) {
        const float e0 = __fsub_rn(c3[0], S.tgt[ra][0]);
        const float e1 = __fsub_rn(c3[1], S.tgt[ra][1]);
        const float e2 = __fsub_rn(c3[2], S.tgt[rb][0]);
        const float e3 = __fsub_rn(c3[3], S.tgt[rb][1]);
        loss = __fadd_rn(loss, __fadd_rn(__fadd_rn(__fmul_rn(e0, e0), __fmul_rn(e1, e1)),
                                         __fadd_rn(__fmul_rn(e2, e2), __fmul_rn(e3, e3))));
        dyl[0] = __fmul_rn(e0, inv_b);
        dyl[1] = __fmul_rn(e1, inv_b);
        dyl[2] = __fmul_rn(e2, inv_b);
        dyl[3] = __fmul_rn(e3, inv_b);
        S.dy[ra][0] = dyl[0];
        S.dy[ra][1] = dyl[1];
        S.dy[rb][0] = dyl[2];
        S.dy[rb][1] = dyl[3];
      }
#pragma unroll
      for (int q = 0; q < 4; q++) dyl[q] = __shfl_sync(0xFFFFFFFFu, dyl[q], lane & ~3);
      // dZ2 = (dY W3) * silu'(Z2)
      uint32_t da[4][4];
#pragma unroll
      for (int nt = 0; nt < 8; nt++) {
        const int c0 = nt * 8 + 2 * t;
        const float w00 = S.w3[c0], w01 = S.w3[c0 + 1], w10 = S.w3[kHidden + c0], w11 = S.w3[kHidden + c0 + 1];
        const float d0 = __fmul_rn(__fadd_rn(__fmul_rn(dyl[0], w00), __fmul_rn(dyl[1], w10)), dsilu_half(z2v[nt][0]));
        const float d1 = __fmul_rn(__fadd_rn(__fmul_rn(dyl[0], w01), __fmul_rn(dyl[1], w11)), dsilu_half(z2v[nt][1]));
        const float d2 = __fmul_rn(__fadd_rn(__fmul_rn(dyl[2], w00), __fmul_rn(dyl[3], w10)), dsilu_half(z2v[nt][2]));
        const float d3 = __fmul_rn(__fadd_rn(__fmul_rn(dyl[2], w01), __fmul_rn(dyl[3], w11)), dsilu_half(z2v[nt][3]));
        da[nt >> 1][(nt & 1) * 2 + 0] = pack_bf16(d0, d1);
        da[nt >> 1][(nt & 1) * 2 + 1] = pack_bf16(d2, d3);
        store_bf16(&S.dz2t[c0][ra], d0);
        store_bf16(&S.dz2t[c0 + 1][ra], d1);
        store_bf16(&S.dz2t[c0][rb], d2);
        store_bf16(&S.dz2t[c0 + 1][rb], d3);
        const float cs0 = group_sum(__fadd_rn(d0, d2)), cs1 = group_sum(__fadd_rn(d1, d3));
        if (g == 0) {
          S.db[warp][kHidden + c0] = __fadd_rn(S.db[warp][kHidden + c0], cs0);
          S.db[warp][kHidden + c0 + 1] = __fadd_rn(S.db[warp][kHidden + c0 + 1], cs1);
        }
      }
      // dH1 = dZ2 W2, dZ1 = dH1 * silu'(Z1)
#pragma unroll
      for (int nt = 0; nt < 8; nt++) {
        float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
        for (int kt = 0; kt < 4; kt++) {
          const uint2 b = S.f2t[(kt * 8 + nt) * 32 + lane];
          mma_bf16(c, da[kt], b.x, b.y);
        }
        const float4 z = *reinterpret_cast<const float4*>(&S.z1[warp][mt][nt][lane][0]);
        const float d0 = __fmul_rn(c[0], dsilu_half(z.x)), d1 = __fmul_rn(c[1], dsilu_half(z.y));
        const float d2 = __fmul_rn(c[2], dsilu_half(z.z)), d3 = __fmul_rn(c[3], dsilu_half(z.w));
        const int c0 = nt * 8 + 2 * t;
        store_bf16(&S.dz1t[c0][ra], d0);
        store_bf16(&S.dz1t[c0 + 1][ra], d1);
        store_bf16(&S.dz1t[c0][rb], d2);
        store_bf16(&S.dz1t[c0 + 1][rb], d3);
        const float cs0 = group_sum(__fadd_rn(d0, d2)), cs1 = group_sum(__fadd_rn(d1, d3));
        if (g == 0) {
          S.db[warp][c0] = __fadd_rn(S.db[warp][c0], cs0);
          S.db[warp][c0 + 1] = __fadd_rn(S.db[warp][c0 + 1], cs1);
        }
      }
    }
    __syncthreads();
    // ---- CTA weight gradients over the 128 samples of this pass
    // warp w owns rows [16w, 16w + 16) of dW2 (layer-2 outputs) and of dW1
#pragma unroll 1
    for (int kt = 0; kt < kTileRows / 16; kt++) {
      const int kc = kt * 16 + 2 * t;
      uint32_t a[4];
      a[0] = lds32(&S.dz2t[16 * warp + g][kc]);
      a[1] = lds32(&S.dz2t[16 * warp + g + 8][kc]);
      a[2] = lds32(&S.dz2t[16 * warp + g][kc + 8]);
      a[3] = lds32(&S.dz2t[16 * warp + g + 8][kc + 8]);
#pragma unroll
      for (int nt = 0; nt < 8; nt++)
        mma_bf16(acc_w2[nt], a, lds32(&S.h1t[nt * 8 + g][kc]), lds32(&S.h1t[nt * 8 + g][kc + 8]));
      a[0] = lds32(&S.dz1t[16 * warp + g][kc]);
      a[1] = lds32(&S.dz1t[16 * warp + g + 8][kc]);
      a[2] = lds32(&S.dz1t[16 * warp + g][kc + 8]);
      a[3] = lds32(&S.dz1t[16 * warp + g + 8][kc + 8]);
#pragma unroll
      for (int nt = 0; nt < 2; nt++)
        mma_bf16(acc_w1[nt], a, lds32(&S.xt[nt * 8 + g][kc]), lds32(&S.xt[nt * 8 + g][kc + 8]));
    }
    {
      // dW3[o][n] = sum_k dY[k][o] H2[k][n] and db3 (FP32, sample order)
      const int o = tid >> 6, n = tid & 63;
      for (int kk = 0; kk < kTileRows; kk++)
        acc_w3 = __fadd_rn(acc_w3, __fmul_rn(S.dy[kk][o], __half2float(S.h2t[n][kk])));
      if (tid < kOut)
        for (int kk = 0; kk < kTileRows; kk++) acc_b3 = __fadd_rn(acc_b3, S.dy[kk][tid]);
    }
    __syncthreads();
  }

  // ---- this CTA's partial gradient
  float* P = part + (size_t)blockIdx.x * kPartStride;
#pragma unroll
  for (int nt = 0; nt < 8; nt++) {
    const int i = nt * 8 + 2 * t, oa = 16 * warp + g, ob = oa + 8;
    P[kOffW2 + oa * kHidden + i] = acc_w2[nt][0];
    P[kOffW2 + oa * kHidden + i + 1] = acc_w2[nt][1];
    P[kOffW2 + ob * kHidden + i] = acc_w2[nt][2];
    P[kOffW2 + ob * kHidden + i + 1] = acc_w2[nt][3];
  }
#pragma unroll
  for (int nt = 0; nt < 2; nt++) {
    const int k = nt * 8 + 2 * t, na = 16 * warp + g, nb = na + 8;
    P[kOffW1 + na * kFeat + k] = acc_w1[nt][0];
    P[kOffW1 + na * kFeat + k + 1] = acc_w1[nt][1];
    P[kOffW1 + nb * kFeat + k] = acc_w1[nt][2];
    P[kOffW1 + nb * kFeat + k + 1] = acc_w1[nt][3];
  }
  P[kOffW3 + tid] = acc_w3;
  if (tid < kOut) P[kOffB3 + tid] = acc_b3;
  {
    const float s = __fadd_rn(__fadd_rn(S.db[0][tid], S.db[1][tid]), __fadd_rn(S.db[2][tid], S.db[3][tid]));
    if (tid < kHidden)
      P[kOffB1 + tid] = s;
    else
      P[kOffB2 + tid - kHidden] = s;
  }
  // loss: fixed-order tree within each warp, then warps in order
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) loss = __fadd_rn(loss, __shfl_xor_sync(0xFFFFFFFFu, loss, o));
  __shared__ float wl[4];
  if (lane == 0) wl[warp] = loss;
  __syncthreads();
  if (tid == 0) P[kParams] = __fadd_rn(__fadd_rn(wl[0], wl[1]), __fadd_rn(wl[2], wl[3]));
}

// ---- the training tile on the 5th-generation tensor cores (tcgen05)
//
// Same sampling, numerics and partial-gradient layout as k_mlp_train_tile;
// thread t owns sample row t of each 128-sample round, and every GEMM is one
// M = 128 tcgen05.mma chain from K-major shared-memory operands (sph_tc.cuh)
// into f32 TMEM columns:
//   Z1  [0, 64)     x_hat (W1/2)^T                       K = 16   bf16
//   Z2  [64, 128)   H1 (W2/2)^T                          K = 64   fp16
//   Y   [224, 240)  H2 W3pad^T                           K = 64   fp16
//   dH1 [64, 128)   dZ2 W2 (over Z2, once it is read)    K = 64   bf16
//   G   [128, 224)  [dZ2^T ; dZ1^T] [H1^T ; x_hat^T ; 1 ; 0]^T   K = 128 samples, bf16,
//                   accumulated over all rounds of the CTA
// G's row m < 64 holds dW2[m][:] (columns 0..63) and db2[m] (column 80, the
// ones row); row 64 + o holds dW1[o][:] (columns 64..79) and db1[o] (column
// 80); the two off-diagonal blocks are unused. dW3 and db3 are f32 sums in
// sample order from dY and the FP16 H2 tile.
constexpr uint32_t kTrW1 = 0;                       // W1 / 2   [64][16]  bf16
constexpr uint32_t kTrW2 = kTrW1 + 64 * 16 * 2;     // W2 / 2   [64][64]  fp16
constexpr uint32_t kTrW3 = kTrW2 + 64 * 64 * 2;     // W3       [16][64]  fp16 (rows 2..15 zero)
constexpr uint32_t kTrW2T = kTrW3 + 16 * 64 * 2;    // W2^T     [64][64]  bf16 (row = layer-1 unit)
constexpr uint32_t kTrX = kTrW2T + 64 * 64 * 2;     // x_hat    [128][16] bf16
constexpr uint32_t kTrA = kTrX + 128 * 16 * 2;      // H1, H2 (fp16), then dZ2 (bf16) [128][64]
constexpr uint32_t kTrGA = kTrA + 128 * 64 * 2;     // [dZ2^T ; dZ1^T]              [128][128] bf16
constexpr uint32_t kTrGB = kTrGA + 128 * 128 * 2;   // [H1^T ; x_hat^T ; 1 ; 0]     [96][128]  bf16
constexpr uint32_t kTrBias = kTrGB + 96 * 128 * 2;  // b1/2 | b2/2 | b3 (f32)
constexpr uint32_t kTrNorm = kTrBias + 4 * 256;     // mu | isd | out_scale
constexpr uint32_t kTrW3f = kTrNorm + 4 * 64;       // W3 (FP16-rounded) as f32 [2][64]
constexpr uint32_t kTrTgt = kTrW3f + 4 * 128;       // targets / out_scale [128][2]
constexpr uint32_t kTrDy = kTrTgt + 4 * 256;        // dL/dy [128][2]
constexpr uint32_t kTrLoss = kTrDy + 4 * 256;       // per-warp loss [4]
constexpr uint32_t kTrBar = kTrLoss + 16;           // mbarrier
constexpr uint32_t kTrSlot = kTrBar + 8;            // TMEM address
constexpr uint32_t kTrSmem = kTrSlot + 8;           // ~100 KB: two CTAs per SM
constexpr uint32_t kTrCols = 256;                   // two CTAs per SM use all 512 columns
constexpr uint32_t kColZ1 = 0, kColZ2 = 64, kColG = 128, kColY = 224;
constexpr uint32_t kGradN = 96;
constexpr uint32_t kTrWaitLimit = 1u << 20;
static_assert(kTrSmem % 16 == 0 && kTrBar % 8 == 0, "shared-memory layout");

// 16-bit element (row, col) of a K-major operand with 128 columns (col = sample).
__device__ __forceinline__ void st_t16(unsigned char* m, uint32_t row, uint32_t col, uint32_t v) {
  *reinterpret_cast<uint16_t*>(m + tc::kmajor_offset(row, col, 128)) = (uint16_t)v;
}

__global__ void __launch_bounds__(kTrainThreads, 1)
    k_mlp_train_tc(const float* __restrict__ x, const float* __restrict__ tg, uint32_t npairs, uint32_t k0,
                   uint32_t total, uint32_t rounds, uint64_t seed, const uint32_t* __restrict__ iter_ptr, MlpDev mlp,
                   float* __restrict__ part, uint32_t* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char tsm[];
  const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const __nv_bfloat16* img = reinterpret_cast<const __nv_bfloat16*>(mlp.frag);
  const __half* himg = reinterpret_cast<const __half*>(mlp.frag);
  for (uint32_t i = tid; i < 64 * 16; i += kTrainThreads) {
    const uint32_t o = i >> 4, k = i & 15;
    *reinterpret_cast<__nv_bfloat16*>(tsm + kTrW1 + tc::kmajor_offset(o, k, 16)) = img[frag_pos(k, o, 8)];
  }
  for (uint32_t i = tid; i < 64 * 64; i += kTrainThreads) {
    const uint32_t o = i >> 6, k = i & 63;
    *reinterpret_cast<__half*>(tsm + kTrW2 + tc::kmajor_offset(o, k, 64)) = himg[4 * kF1 + frag_pos(k, o, 8)];
    // W2^T row o (a layer-1 unit), column k (a layer-2 unit) = W2[k][o], from F2T
    *reinterpret_cast<__nv_bfloat16*>(tsm + kTrW2T + tc::kmajor_offset(o, k, 64)) =
        img[4 * (kF1 + kF2 + kF3) + frag_pos(k, o, 8)];
  }
  for (uint32_t i = tid; i < 16 * 64; i += kTrainThreads) {
    const uint32_t o = i >> 6, k = i & 63;
    *reinterpret_cast<__half*>(tsm + kTrW3 + tc::kmajor_offset(o, k, 64)) =
        o < 2 ? himg[4 * (kF1 + kF2) + frag_pos(k, o, 1)] : __float2half_rn(0.0f);
  }
  unsigned char* X = tsm + kTrX;
  unsigned char* A = tsm + kTrA;
  unsigned char* GA = tsm + kTrGA;
  unsigned char* GB = tsm + kTrGB;
  // rows 80..95 of G's B operand: ones (the bias gradients), then zeros
  for (uint32_t i = tid; i < 16 * kTileRows; i += kTrainThreads) {
    const uint32_t row = 80 + (i >> 7);
    st_t16(GB, row, i & 127, row == 80 ? 0x3F80u : 0u);  // bf16 1.0 / 0.0
  }
  float* bias = reinterpret_cast<float*>(tsm + kTrBias);
  float* norm = reinterpret_cast<float*>(tsm + kTrNorm);
  float* w3f = reinterpret_cast<float*>(tsm + kTrW3f);
  float* tgt = reinterpret_cast<float*>(tsm + kTrTgt);
  float* dy = reinterpret_cast<float*>(tsm + kTrDy);
  float* wl = reinterpret_cast<float*>(tsm + kTrLoss);
  for (uint32_t i = tid; i < kBias; i += kTrainThreads) bias[i] = mlp.bias[i];
  for (uint32_t i = tid; i < kNorm; i += kTrainThreads) norm[i] = mlp.norm[i];
  for (uint32_t i = tid; i < kOut * kHidden; i += kTrainThreads) w3f[i] = mlp.w3[i];
  uint64_t* bar = reinterpret_cast<uint64_t*>(tsm + kTrBar);
  uint32_t* slot = reinterpret_cast<uint32_t*>(tsm + kTrSlot);
  if (tid == 0) tc::mbar_init(bar, 1);
  if (warp == 0) tc::tmem_alloc(slot, kTrCols);
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tm = *slot, lanes = (warp * 32u) << 16;
  uint32_t phase = 0;
  const uint32_t iter = *iter_ptr;
  const float inv_b = __fdiv_rn(1.0f, (float)total);
  const float inv_os0 = __fdiv_rn(1.0f, norm[2 * kFeat]), inv_os1 = __fdiv_rn(1.0f, norm[2 * kFeat + 1]);
  const uint32_t aX = tc::smem_u32(X), aA = tc::smem_u32(A), aGA = tc::smem_u32(GA), aGB = tc::smem_u32(GB);
  const uint32_t aW1 = tc::smem_u32(tsm + kTrW1), aW2 = tc::smem_u32(tsm + kTrW2), aW3 = tc::smem_u32(tsm + kTrW3),
                 aW2T = tc::smem_u32(tsm + kTrW2T);

  float acc_w3 = 0.0f, acc_b3 = 0.0f, loss = 0.0f;
  bool ok = true;
  for (uint32_t r = 0; r < rounds; r++) {
    // ---- sample row tid: x_hat into X (row) and GB rows 64..79 (column), scaled target
    {
      const uint32_t k = k0 + (blockIdx.x * rounds + r) * kTileRows + tid;
      const uint32_t idx = sample_index(seed, iter, k, npairs);
      const float4* xi = reinterpret_cast<const float4*>(x + (size_t)idx * kFeat);
      float f[kFeat];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const float4 v = xi[q];
        f[4 * q] = v.x;
        f[4 * q + 1] = v.y;
        f[4 * q + 2] = v.z;
        f[4 * q + 3] = v.w;
      }
      uint32_t xp[8];
#pragma unroll
      for (int q = 0; q < 8; q++)
        xp[q] = pack_bf16(__fmul_rn(__fsub_rn(f[2 * q], norm[2 * q]), norm[kFeat + 2 * q]),
                          __fmul_rn(__fsub_rn(f[2 * q + 1], norm[2 * q + 1]), norm[kFeat + 2 * q + 1]));
      *reinterpret_cast<uint4*>(X + tc::kmajor_offset(tid, 0, 16)) = make_uint4(xp[0], xp[1], xp[2], xp[3]);
      *reinterpret_cast<uint4*>(X + tc::kmajor_offset(tid, 8, 16)) = make_uint4(xp[4], xp[5], xp[6], xp[7]);
#pragma unroll
      for (int q = 0; q < 8; q++) {
        st_t16(GB, 64 + 2 * q, tid, xp[q] & 0xFFFFu);
        st_t16(GB, 65 + 2 * q, tid, xp[q] >> 16);
      }
      tgt[2 * tid] = __fmul_rn(tg[2 * (size_t)idx], inv_os0);
      tgt[2 * tid + 1] = __fmul_rn(tg[2 * (size_t)idx + 1], inv_os1);
    }
    // ---- layer 1
    ok = tc::mma_step(bar, phase, kTrWaitLimit, [&] {
      tc::mma_f16(tm + kColZ1, tc::smem_desc(aX, 128, 256), tc::smem_desc(aW1, 128, 256),
                  tc::idesc_f16(tc::kFmtBF16, 64), 0u);
    });
    if (!ok) break;
    // H1 = silu(z1): row tid of A (fp16) and column tid of GB rows 0..63 (bf16)
#pragma unroll
    for (int half = 0; half < 2; half++) {
      float v[2][16];
#pragma unroll
      for (int q = 0; q < 2; q++) tc::tmem_ld16(tm + lanes + kColZ1 + 32 * half + 16 * q, v[q]);
      tc::tmem_wait_ld();
#pragma unroll
      for (int q = 0; q < 2; q++) {
        const int c = 32 * half + 16 * q;
        uint32_t hp[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
          hp[j] = silu_half_f16x2(__fadd_rn(v[q][2 * j], bias[c + 2 * j]), __fadd_rn(v[q][2 * j + 1], bias[c + 2 * j + 1]));
          const uint32_t b = f16x2_to_bf16x2(hp[j]);
          st_t16(GB, c + 2 * j, tid, b & 0xFFFFu);
          st_t16(GB, c + 2 * j + 1, tid, b >> 16);
        }
        *reinterpret_cast<uint4*>(A + tc::kmajor_offset(tid, c, 64)) = make_uint4(hp[0], hp[1], hp[2], hp[3]);
        *reinterpret_cast<uint4*>(A + tc::kmajor_offset(tid, c + 8, 64)) = make_uint4(hp[4], hp[5], hp[6], hp[7]);
      }
    }
    // ---- layer 2
    ok = tc::mma_step(bar, phase, kTrWaitLimit, [&] {
#pragma unroll
      for (uint32_t kk = 0; kk < 4; kk++)
        tc::mma_f16(tm + kColZ2, tc::smem_desc(aA + 256 * kk, 128, 1024), tc::smem_desc(aW2 + 256 * kk, 128, 1024),
                    tc::idesc_f16(tc::kFmtF16, 64), kk);
    });
    if (!ok) break;
    // H2 = silu(z2): row tid of A (fp16)
#pragma unroll
    for (int half = 0; half < 2; half++) {
      float v[2][16];
#pragma unroll
      for (int q = 0; q < 2; q++) tc::tmem_ld16(tm + lanes + kColZ2 + 32 * half + 16 * q, v[q]);
      tc::tmem_wait_ld();
#pragma unroll
      for (int q = 0; q < 2; q++) {
        const int c = 32 * half + 16 * q;
        const float* b = bias + kHidden + c;
        uint32_t hp[8];
#pragma unroll
        for (int j = 0; j < 8; j++)
          hp[j] = silu_half_f16x2(__fadd_rn(v[q][2 * j], b[2 * j]), __fadd_rn(v[q][2 * j + 1], b[2 * j + 1]));
        *reinterpret_cast<uint4*>(A + tc::kmajor_offset(tid, c, 64)) = make_uint4(hp[0], hp[1], hp[2], hp[3]);
        *reinterpret_cast<uint4*>(A + tc::kmajor_offset(tid, c + 8, 64)) = make_uint4(hp[4], hp[5], hp[6], hp[7]);
      }
    }
    // ---- layer 3, loss and dY = (y - t) / B
    ok = tc::mma_step(bar, phase, kTrWaitLimit, [&] {
#pragma unroll
      for (uint32_t kk = 0; kk < 4; kk++)
        tc::mma_f16(tm + kColY, tc::smem_desc(aA + 256 * kk, 128, 1024), tc::smem_desc(aW3 + 256 * kk, 128, 1024),
                    tc::idesc_f16(tc::kFmtF16, 16), kk);
    });
    if (!ok) break;
    {
      float o[2];
      tc::tmem_ld2(tm + lanes + kColY, o);
      tc::tmem_wait_ld();
      const float e0 = __fsub_rn(__fadd_rn(o[0], bias[2 * kHidden]), tgt[2 * tid]);
      const float e1 = __fsub_rn(__fadd_rn(o[1], bias[2 * kHidden + 1]), tgt[2 * tid + 1]);
      loss = __fadd_rn(loss, __fadd_rn(__fmul_rn(e0, e0), __fmul_rn(e1, e1)));
      dy[2 * tid] = __fmul_rn(e0, inv_b);
      dy[2 * tid + 1] = __fmul_rn(e1, inv_b);
    }
    __syncthreads();
    // ---- dW3[o][n] = sum_k dY[k][o] H2[k][n] and db3 (f32, sample order; H2 from A)
    {
      const uint32_t o = tid >> 6, n = tid & 63;
      for (uint32_t kk = 0; kk < kTileRows; kk++)
        acc_w3 = __fadd_rn(acc_w3, __fmul_rn(dy[2 * kk + o],
                                             __half2float(*reinterpret_cast<const __half*>(A + tc::kmajor_offset(kk, n, 64)))));
      if (tid < kOut)
        for (uint32_t kk = 0; kk < kTileRows; kk++) acc_b3 = __fadd_rn(acc_b3, dy[2 * kk + tid]);
    }
    __syncthreads();
    // ---- dZ2 = (dY W3) silu'(z2): row tid of A (bf16) and column tid of GA rows 0..63
    {
      const float dy0 = dy[2 * tid], dy1 = dy[2 * tid + 1];
#pragma unroll
      for (int half = 0; half < 2; half++) {
        float v[2][16];
#pragma unroll
        for (int q = 0; q < 2; q++) tc::tmem_ld16(tm + lanes + kColZ2 + 32 * half + 16 * q, v[q]);
        tc::tmem_wait_ld();
#pragma unroll
        for (int q = 0; q < 2; q++) {
          const int c = 32 * half + 16 * q;
          uint32_t dp[8];
#pragma unroll
          for (int j = 0; j < 8; j++) {
            const int c0 = c + 2 * j;
            const float d0 = __fmul_rn(__fadd_rn(__fmul_rn(dy0, w3f[c0]), __fmul_rn(dy1, w3f[kHidden + c0])),
                                       dsilu_half(__fadd_rn(v[q][2 * j], bias[kHidden + c0])));
            const float d1 = __fmul_rn(__fadd_rn(__fmul_rn(dy0, w3f[c0 + 1]), __fmul_rn(dy1, w3f[kHidden + c0 + 1])),
                                       dsilu_half(__fadd_rn(v[q][2 * j + 1], bias[kHidden + c0 + 1])));
            dp[j] = pack_bf16(d0, d1);
            st_t16(GA, c0, tid, dp[j] & 0xFFFFu);
            st_t16(GA, c0 + 1, tid, dp[j] >> 16);
          }
          *reinterpret_cast<uint4*>(A + tc::kmajor_offset(tid, c, 64)) = make_uint4(dp[0], dp[1], dp[2], dp[3]);
          *reinterpret_cast<uint4*>(A + tc::kmajor_offset(tid, c + 8, 64)) = make_uint4(dp[4], dp[5], dp[6], dp[7]);
        }
      }
    }
    // ---- dH1 = dZ2 W2 (over Z2, which every thread has read)
    ok = tc::mma_step(bar, phase, kTrWaitLimit, [&] {
#pragma unroll
      for (uint32_t kk = 0; kk < 4; kk++)
        tc::mma_f16(tm + kColZ2, tc::smem_desc(aA + 256 * kk, 128, 1024), tc::smem_desc(aW2T + 256 * kk, 128, 1024),
                    tc::idesc_f16(tc::kFmtBF16, 64), kk);
    });
    if (!ok) break;
    // ---- dZ1 = dH1 silu'(z1): column tid of GA rows 64..127
#pragma unroll
    for (int half = 0; half < 2; half++) {
      float v[2][16], z[2][16];
#pragma unroll
      for (int q = 0; q < 2; q++) {
        tc::tmem_ld16(tm + lanes + kColZ2 + 32 * half + 16 * q, v[q]);
        tc::tmem_ld16(tm + lanes + kColZ1 + 32 * half + 16 * q, z[q]);
      }
      tc::tmem_wait_ld();
#pragma unroll
      for (int q = 0; q < 2; q++) {
        const int c = 32 * half + 16 * q;
#pragma unroll
        for (int j = 0; j < 8; j++) {
          const int c0 = c + 2 * j;
          const float d0 = __fmul_rn(v[q][2 * j], dsilu_half(__fadd_rn(z[q][2 * j], bias[c0])));
          const float d1 = __fmul_rn(v[q][2 * j + 1], dsilu_half(__fadd_rn(z[q][2 * j + 1], bias[c0 + 1])));
          const uint32_t p = pack_bf16(d0, d1);
          st_t16(GA, 64 + c0, tid, p & 0xFFFFu);
          st_t16(GA, 65 + c0, tid, p >> 16);
        }
      }
    }
    // ---- G (+)= GA GB^T over this pass's 128 samples; the next pass's
    // operand writes wait for it
    ok = tc::mma_step(bar, phase, kTrWaitLimit, [&] {
#pragma unroll
      for (uint32_t kk = 0; kk < kTileRows / 16; kk++)
        tc::mma_f16(tm + kColG, tc::smem_desc(aGA + 256 * kk, 128, 2048), tc::smem_desc(aGB + 256 * kk, 128, 2048),
                    tc::idesc_f16(tc::kFmtBF16, kGradN), (r | kk) != 0u ? 1u : 0u);
    });
    if (!ok) break;
  }

  // ---- this CTA's partial gradient
  float* P = part + (size_t)blockIdx.x * kPartStride;
  if (ok) {
    float g[16];
    if (warp < 2) {
#pragma unroll
      for (int q = 0; q < 4; q++) {
        tc::tmem_ld16(tm + lanes + kColG + 16 * q, g);
        tc::tmem_wait_ld();
#pragma unroll
        for (int j = 0; j < 16; j++) P[kOffW2 + tid * kHidden + 16 * q + j] = g[j];
      }
    } else {
      tc::tmem_ld16(tm + lanes + kColG + 64, g);
      tc::tmem_wait_ld();
#pragma unroll
      for (int j = 0; j < 16; j++) P[kOffW1 + (tid - 64) * kFeat + j] = g[j];
    }
    tc::tmem_ld16(tm + lanes + kColG + 80, g);
    tc::tmem_wait_ld();
    if (warp < 2)
      P[kOffB2 + tid] = g[0];
    else
      P[kOffB1 + tid - 64] = g[0];
  }
  P[kOffW3 + tid] = acc_w3;
  if (tid < kOut) P[kOffB3 + tid] = acc_b3;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) loss = __fadd_rn(loss, __shfl_xor_sync(0xFFFFFFFFu, loss, o));
  if (lane == 0) wl[warp] = loss;
  __syncthreads();
  if (tid == 0) P[kParams] = __fadd_rn(__fadd_rn(wl[0], wl[1]), __fadd_rn(wl[2], wl[3]));
  if (!ok) {
    if (tid == 0) atomicExch(err, 1u);
    tc::mbar_wait(bar, phase, kTrWaitLimit);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_free(tm, kTrCols);
  }
}

// Sum of the CTA partials (CTA order) per parameter.
__device__ __forceinline__ float sum_parts(const float* __restrict__ part, uint32_t nparts, int p) {
  float g = 0.0f;
  for (uint32_t c = 0; c < nparts; c++) g = __fadd_rn(g, part[(size_t)c * kPartStride + p]);
  return g;
}

__global__ void k_mlp_reduce(const float* __restrict__ part, uint32_t nparts, float inv_2b, float* __restrict__ grad,
                             float* __restrict__ loss) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < kParams) grad[p] = sum_parts(part, nparts, p);
  if (p == kParams) *loss = __fmul_rn(sum_parts(part, nparts, kParams), inv_2b);
}

// Adam (Kingma & Ba 2015) on step t = ctr[0] + 1:
//   m = b1 m + (1 - b1) g,  v = b2 v + (1 - b2) g^2,
//   w -= lr * (m / (1 - b1^t)) / (sqrt(v / (1 - b2^t)) + eps)
__global__ void k_mlp_adam(const float* __restrict__ part, uint32_t nparts, float* __restrict__ w, float* __restrict__ m,
                           float* __restrict__ v, const uint32_t* __restrict__ ctr, float lr, float inv_2b,
                           float* __restrict__ loss_hist, uint32_t loss_base, uint32_t loss_cap, uint2* frag,
                           float* bias, float* w3) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t t0 = ctr[0];
  if (p == kParams) {
    if (loss_hist && t0 >= loss_base && t0 - loss_base < loss_cap)
      loss_hist[t0 - loss_base] = __fmul_rn(sum_parts(part, nparts, kParams), inv_2b);
    return;
  }
  if (p > kParams) return;
  const float g = sum_parts(part, nparts, p);
  const double tt = (double)t0 + 1.0;
  const float bc1 = (float)(1.0 - pow((double)kBeta1, tt));
  const float bc2 = (float)(1.0 - pow((double)kBeta2, tt));
  const float mm = __fadd_rn(__fmul_rn(kBeta1, m[p]), __fmul_rn(__fsub_rn(1.0f, kBeta1), g));
  const float vv = __fadd_rn(__fmul_rn(kBeta2, v[p]), __fmul_rn(__fsub_rn(1.0f, kBeta2), __fmul_rn(g, g)));
  const float upd = __fdiv_rn(__fdiv_rn(mm, bc1), __fadd_rn(__fsqrt_rn(__fdiv_rn(vv, bc2)), kAdamEps));
  const float ww = __fsub_rn(w[p], __fmul_rn(lr, upd));
  m[p] = mm;
  v[p] = vv;
  w[p] = ww;
  write_weight(p, ww, reinterpret_cast<__nv_bfloat16*>(frag), bias, w3);
}

__global__ void k_mlp_advance(uint32_t* ctr) { ctr[0] += 1u; }

__global__ void k_mlp_indices(uint64_t seed, uint32_t iter, uint32_t batch, uint32_t npairs, uint32_t* out) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < batch) out[k] = sample_index(seed, iter, k, npairs);
}

// Training target per particle from the fine and the coarse state:
// mode 0 (position) (x_f - x_c) / h; mode 1 (velocity) (v_f - v_c) dt / h,
// the displacement the velocity difference makes over one coarse step;
// mode 2 the mean of the two.
__global__ void k_mlp_targets(const float4* __restrict__ fine, const float4* __restrict__ coarse, uint32_t n,
                              float inv_h, float dt, uint32_t mode, float2* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 a = fine[i], b = coarse[i];
  const float px = __fmul_rn(__fsub_rn(a.x, b.x), inv_h), py = __fmul_rn(__fsub_rn(a.y, b.y), inv_h);
  const float s = __fmul_rn(dt, inv_h);
  const float vx = __fmul_rn(__fsub_rn(a.z, b.z), s), vy = __fmul_rn(__fsub_rn(a.w, b.w), s);
  if (mode == 0)
    out[i] = make_float2(px, py);
  else if (mode == 1)
    out[i] = make_float2(vx, vy);
  else
    out[i] = make_float2(__fmul_rn(0.5f, __fadd_rn(px, vx)), __fmul_rn(0.5f, __fadd_rn(py, vy)));
}

// Uniform position noise in [-amp, amp] per coordinate, from mix64 of
// (seed, particle, coordinate): the perturbed states the training pairs are
// also taken from (noise injection, Sanchez-Gonzalez et al. 2020).
__global__ void k_mlp_perturb(float4* __restrict__ state, uint32_t n, float amp, uint64_t seed) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t hx = mix64(seed ^ (2ull * i)), hy = mix64(seed ^ (2ull * i + 1ull));
  const float ux = __fmul_rn((float)(uint32_t)(hx >> 40), 1.0f / 16777216.0f);  // [0, 1)
  const float uy = __fmul_rn((float)(uint32_t)(hy >> 40), 1.0f / 16777216.0f);
  float4 s = state[i];
  s.x = __fadd_rn(s.x, __fmul_rn(amp, __fsub_rn(__fmul_rn(2.0f, ux), 1.0f)));
  s.y = __fadd_rn(s.y, __fmul_rn(amp, __fsub_rn(__fmul_rn(2.0f, uy), 1.0f)));
  state[i] = s;
}

inline uint32_t cdiv(uint32_t a, uint32_t b) { return (a + b - 1) / b; }

}  // namespace

// CTAs and rounds per CTA for a training batch (batch % 128 == 0): rounds
// grow until the grid is at most two CTAs per SM.
void mlp_grid(uint32_t batch, uint32_t* ctas, uint32_t* rounds) {
  uint32_t tiles = batch / kTileRows, r = 1;
  while (tiles / r > 296u && (tiles % (2 * r)) == 0) r *= 2;
  *ctas = tiles / r;
  *rounds = r;
}

}  // namespace phieng

using namespace phieng;

struct PhiengMlp {
  int device = -1;
  cudaStream_t stream = nullptr;
  cudaStream_t own_stream = nullptr;
  int32_t error = PHIENG_SPH_OK;
  float* w = nullptr;
  float* m = nullptr;
  float* v = nullptr;
  uint2* frag = nullptr;
  float* bias = nullptr;
  float* w3 = nullptr;
  float* norm = nullptr;
  uint32_t* ctr = nullptr;  // [0] Adam step, [1] iteration for a gradient check
  float* part = nullptr;
  uint32_t part_cap = 0;
  float* grad = nullptr;    // kParams + 1 (loss)
  float* loss_hist = nullptr;
  uint32_t loss_cap = 0;
  float* h_pinned = nullptr;
  int32_t train_engine = PHIENG_MLP_TCGEN05;
  int32_t infer_engine = PHIENG_MLP_MMA_SYNC;  // network of the tolerance-mode coarse pass (measured faster)
};

namespace {

bool mlp_ok(PhiengMlp* m, cudaError_t r) {
  if (r == cudaSuccess) return true;
  if (m->error == PHIENG_SPH_OK) m->error = PHIENG_SPH_E_CUDA;
  return false;
}

template <class T>
bool mlp_alloc(PhiengMlp* m, T*& p, size_t count) {
  return mlp_ok(m, cudaMalloc(reinterpret_cast<void**>(&p), sizeof(T) * count));
}

bool ensure_parts(PhiengMlp* m, uint32_t nparts) {
  if (m->part_cap >= nparts) return true;
  if (m->part) cudaFree(m->part);
  m->part = nullptr;
  m->part_cap = 0;
  if (!mlp_alloc(m, m->part, (size_t)nparts * kPartStride)) return false;
  m->part_cap = nparts;
  return true;
}

bool sync_images(PhiengMlp* m) {
  k_mlp_sync<<<cdiv(kParams, 256), 256, 0, m->stream>>>(m->w, m->frag, m->bias, m->w3);
  return mlp_ok(m, cudaGetLastError());
}

// After a stream synchronisation: fail (and poison the network) if a bounded
// tensor-core wait of any tcgen05 kernel of this network ran out.
bool waits_clean(PhiengMlp* m) {
  uint32_t e = 0;
  if (!mlp_ok(m, cudaMemcpy(&e, m->ctr + 2, 4, cudaMemcpyDeviceToHost))) return false;
  if (e == 0) return true;
  if (m->error == PHIENG_SPH_OK) m->error = PHIENG_SPH_E_CUDA;
  return false;
}

bool check_pairs(const float* x, const float* t, uint32_t npairs, uint32_t batch) {
  return x && t && npairs > 0 && batch > 0 && batch % kTileRows == 0;
}

// Samples [k0, k0 + batch) of a minibatch of `total` (dL/dy scaled by 1 / total).
bool launch_tile(PhiengMlp* m, const float* x, const float* t, uint32_t npairs, uint32_t batch, uint64_t seed,
                 const uint32_t* iter_ptr, uint32_t* nparts_out, uint32_t k0 = 0, uint32_t total = 0) {
  uint32_t ctas, rounds;
  mlp_grid(batch, &ctas, &rounds);
  if (!ensure_parts(m, ctas)) return false;
  MlpDev d = phieng_mlp_dev(m);
  if (total == 0) total = batch;
  if (m->train_engine == PHIENG_MLP_TCGEN05)
    k_mlp_train_tc<<<ctas, kTrainThreads, kTrSmem, m->stream>>>(x, t, npairs, k0, total, rounds, seed, iter_ptr, d,
                                                                 m->part, m->ctr + 2);
  else
    k_mlp_train_tile<<<ctas, kTrainThreads, sizeof(TrainSmem), m->stream>>>(x, t, npairs, k0, total, rounds, seed,
                                                                            iter_ptr, d, m->part);
  *nparts_out = ctas;
  return mlp_ok(m, cudaGetLastError());
}

}  // namespace

MlpDev phieng_mlp_dev(const PhiengMlp* m) {
  MlpDev d{};
  d.frag = m->frag;
  d.bias = m->bias;
  d.w3 = m->w3;
  d.norm = m->norm;
  d.engine = m->infer_engine;
  return d;
}

extern "C" {

PhiengMlp* phieng_mlp_new(uint64_t seed) {
  PhiengMlp* m = new (std::nothrow) PhiengMlp();
  if (!m) return nullptr;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    m->error = PHIENG_SPH_E_NO_DEVICE;
    return m;
  }
  m->device = dev;
  if (!mlp_ok(m, cudaStreamCreateWithFlags(&m->own_stream, cudaStreamNonBlocking))) return m;
  m->stream = m->own_stream;
  if (!mlp_alloc(m, m->w, kParams) || !mlp_alloc(m, m->m, kParams) || !mlp_alloc(m, m->v, kParams) ||
      !mlp_alloc(m, m->frag, kFragAll) || !mlp_alloc(m, m->bias, kBias) || !mlp_alloc(m, m->w3, kOut * kHidden) ||
      !mlp_alloc(m, m->norm, kNorm) || !mlp_alloc(m, m->ctr, 4) || !mlp_alloc(m, m->grad, kParams + 1))
    return m;
  // ctr[2]: set by the tcgen05 forward when one of its waits ran out
  if (!mlp_ok(m, cudaMemsetAsync(m->ctr, 0, sizeof(uint32_t) * 4, m->stream))) return m;

  if (!mlp_ok(m, cudaMallocHost(reinterpret_cast<void**>(&m->h_pinned), sizeof(float) * (kParams + kNorm + 4))))
    return m;
  if (!mlp_ok(m, cudaFuncSetAttribute(k_mlp_train_tile, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)sizeof(TrainSmem))) ||
      !mlp_ok(m, cudaFuncSetAttribute(k_mlp_train_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrSmem)))
    return m;
  // Linear-layer initialisation U(-1/sqrt(fan_in), 1/sqrt(fan_in)) from
  // SplitMix64(seed); the output layer starts at zero (no correction).
  std::vector<float> w(kParams, 0.0f), norm(kNorm, 0.0f);
  uint64_t s = seed;
  auto uni = [&](float bound) {
    const uint64_t z = mix64(s);
    s += 0x9E3779B97F4A7C15ull;
    const double u = (double)(z >> 11) * (1.0 / 9007199254740992.0);
    return (float)((2.0 * u - 1.0) * bound);
  };
  for (int i = 0; i < kHidden * kFeat; i++) w[kOffW1 + i] = uni(0.25f);
  for (int i = 0; i < kHidden; i++) w[kOffB1 + i] = uni(0.25f);
  for (int i = 0; i < kHidden * kHidden; i++) w[kOffW2 + i] = uni(0.125f);
  for (int i = 0; i < kHidden; i++) w[kOffB2 + i] = uni(0.125f);
  for (int i = 0; i < kFeat; i++) norm[kFeat + i] = 1.0f;
  norm[2 * kFeat] = norm[2 * kFeat + 1] = 1.0f;
  phieng_mlp_set_params(m, w.data(), norm.data());
  return m;
}

void phieng_mlp_free(PhiengMlp* m) {
  if (!m) return;
  if (m->device >= 0) {
    cudaStreamSynchronize(m->stream);
    cudaFree(m->w);
    cudaFree(m->m);
    cudaFree(m->v);
    cudaFree(m->frag);
    cudaFree(m->bias);
    cudaFree(m->w3);
    cudaFree(m->norm);
    cudaFree(m->ctr);
    cudaFree(m->part);
    cudaFree(m->grad);
    cudaFree(m->loss_hist);
    if (m->h_pinned) cudaFreeHost(m->h_pinned);
    if (m->own_stream) cudaStreamDestroy(m->own_stream);
  }
  delete m;
}

int32_t phieng_mlp_status(const PhiengMlp* m) { return m ? m->error : PHIENG_SPH_E_ARG; }

int32_t phieng_mlp_set_stream(PhiengMlp* m, void* stream) {
  if (!m || m->error) return 0;
  m->stream = stream ? (cudaStream_t)stream : m->own_stream;
  return 1;
}

int32_t phieng_mlp_set_params(PhiengMlp* m, const float* params, const float* norm) {
  if (!m || m->error || !params || !norm) return 0;
  if (!mlp_ok(m, cudaMemcpyAsync(m->w, params, sizeof(float) * kParams, cudaMemcpyHostToDevice, m->stream)) ||
      !mlp_ok(m, cudaMemcpyAsync(m->norm, norm, sizeof(float) * kNorm, cudaMemcpyHostToDevice, m->stream)) ||
      !mlp_ok(m, cudaMemsetAsync(m->m, 0, sizeof(float) * kParams, m->stream)) ||
      !mlp_ok(m, cudaMemsetAsync(m->v, 0, sizeof(float) * kParams, m->stream)) ||
      !mlp_ok(m, cudaMemsetAsync(m->frag, 0, sizeof(uint2) * kFragAll, m->stream)) ||
      !mlp_ok(m, cudaMemsetAsync(m->ctr, 0, sizeof(uint32_t) * 2, m->stream)))
    return 0;
  if (!sync_images(m)) return 0;
  return mlp_ok(m, cudaStreamSynchronize(m->stream)) ? 1 : 0;
}

int32_t phieng_mlp_get_params(PhiengMlp* m, float* params, float* norm) {
  if (!m || m->error) return 0;
  if (params && !mlp_ok(m, cudaMemcpyAsync(params, m->w, sizeof(float) * kParams, cudaMemcpyDeviceToHost, m->stream)))
    return 0;
  if (norm && !mlp_ok(m, cudaMemcpyAsync(norm, m->norm, sizeof(float) * kNorm, cudaMemcpyDeviceToHost, m->stream)))
    return 0;
  return mlp_ok(m, cudaStreamSynchronize(m->stream)) ? 1 : 0;
}

uint32_t phieng_mlp_step_count(PhiengMlp* m) {
  if (!m || m->error) return 0;
  uint32_t t = 0;
  if (!mlp_ok(m, cudaMemcpyAsync(m->h_pinned, m->ctr, 4, cudaMemcpyDeviceToHost, m->stream)) ||
      !mlp_ok(m, cudaStreamSynchronize(m->stream)))
    return 0;
  std::memcpy(&t, m->h_pinned, 4);
  return t;
}

int32_t phieng_mlp_forward(PhiengMlp* m, const float* x, uint32_t n, float* y) {
  if (!m || m->error || (n && (!x || !y))) return 0;
  if (n == 0) return 1;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m->device);
  const uint32_t blocks = std::min<uint32_t>(cdiv(n, 128), (uint32_t)sms * 8u);
  k_mlp_forward<<<blocks, 128, 0, m->stream>>>(x, n, phieng_mlp_dev(m), y);
  return mlp_ok(m, cudaGetLastError()) ? 1 : 0;
}

int32_t phieng_mlp_forward_tc(PhiengMlp* m, const float* x, uint32_t n, float* y) {
  if (!m || m->error || (n && (!x || !y))) return 0;
  if (n == 0) return 1;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m->device);
  const uint32_t blocks = std::min<uint32_t>(cdiv(n, 128), (uint32_t)sms * 6u);
  k_mlp_forward_tc<<<blocks, 128, kNetSmem, m->stream>>>(x, n, phieng_mlp_dev(m), y, m->ctr + 2);
  return mlp_ok(m, cudaGetLastError()) ? 1 : 0;
}

int32_t phieng_mlp_check_waits(PhiengMlp* m) {
  if (!m || m->device < 0) return 0;
  uint32_t e = 0;
  if (!mlp_ok(m, cudaMemcpyAsync(m->h_pinned, m->ctr + 2, 4, cudaMemcpyDeviceToHost, m->stream)) ||
      !mlp_ok(m, cudaStreamSynchronize(m->stream)))
    return 0;
  std::memcpy(&e, m->h_pinned, 4);
  if (e != 0 && m->error == PHIENG_SPH_OK) m->error = PHIENG_SPH_E_CUDA;
  return e == 0 ? 1 : 0;
}

int32_t phieng_mlp_grad(PhiengMlp* m, const float* x, const float* t, uint32_t npairs, uint32_t batch, uint64_t seed,
                        uint32_t iter, float* grad_host, float* loss_host) {
  if (!m || m->error || !check_pairs(x, t, npairs, batch)) return 0;
  if (!mlp_ok(m, cudaMemcpyAsync(m->ctr + 1, &iter, 4, cudaMemcpyHostToDevice, m->stream))) return 0;
  uint32_t nparts = 0;
  if (!launch_tile(m, x, t, npairs, batch, seed, m->ctr + 1, &nparts)) return 0;
  const float inv_2b = (float)(0.5 / (double)batch);
  k_mlp_reduce<<<cdiv(kParams + 1, 256), 256, 0, m->stream>>>(m->part, nparts, inv_2b, m->grad, m->grad + kParams);
  if (!mlp_ok(m, cudaGetLastError())) return 0;
  if (!mlp_ok(m, cudaMemcpyAsync(m->h_pinned, m->grad, sizeof(float) * (kParams + 1), cudaMemcpyDeviceToHost,
                                 m->stream)) ||
      !mlp_ok(m, cudaStreamSynchronize(m->stream)) || !waits_clean(m))
    return 0;
  if (grad_host) std::memcpy(grad_host, m->h_pinned, sizeof(float) * kParams);
  if (loss_host) *loss_host = m->h_pinned[kParams];
  return 1;
}

int32_t phieng_mlp_train(PhiengMlp* m, const float* x, const float* t, uint32_t npairs, uint32_t batch, uint32_t iters,
                         float lr, uint64_t seed, float* loss_hist_host) {
  if (!m || m->error || !check_pairs(x, t, npairs, batch) || !(lr > 0.0f)) return 0;
  if (iters == 0) return 1;
  if (loss_hist_host && m->loss_cap < iters) {
    cudaFree(m->loss_hist);
    m->loss_hist = nullptr;
    m->loss_cap = 0;
    if (!mlp_alloc(m, m->loss_hist, iters)) return 0;
    m->loss_cap = iters;
  }
  {
    // the partial-gradient buffer is sized here: no allocation may happen
    // while the iteration graph is being captured
    uint32_t ctas, rounds;
    mlp_grid(batch, &ctas, &rounds);
    if (!ensure_parts(m, ctas)) return 0;
  }
  const uint32_t t0 = phieng_mlp_step_count(m);
  const float inv_2b = (float)(0.5 / (double)batch);
  // one iteration = tile, Adam, advance; replayed from a graph of up to 32
  const uint32_t per_graph = std::min<uint32_t>(iters, 32u);
  auto enqueue = [&](uint32_t k, cudaStream_t st) -> bool {
    cudaStream_t keep = m->stream;
    m->stream = st;
    bool ok = true;
    for (uint32_t i = 0; i < k && ok; i++) {
      uint32_t nparts = 0;
      ok = launch_tile(m, x, t, npairs, batch, seed, m->ctr, &nparts);
      if (ok) {
        k_mlp_adam<<<cdiv(kParams + 1, 256), 256, 0, st>>>(m->part, nparts, m->w, m->m, m->v, m->ctr, lr, inv_2b,
                                                            loss_hist_host ? m->loss_hist : nullptr, t0, iters,
                                                            m->frag, m->bias, m->w3);
        k_mlp_advance<<<1, 1, 0, st>>>(m->ctr);
        ok = mlp_ok(m, cudaGetLastError());
      }
    }
    m->stream = keep;
    return ok;
  };
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ge = nullptr;
  cudaStream_t cap;
  if (!mlp_ok(m, cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking))) return 0;
  bool ok = mlp_ok(m, cudaStreamSynchronize(m->stream)) &&
            mlp_ok(m, cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
  if (ok) {
    const bool body = enqueue(per_graph, cap);
    ok = mlp_ok(m, cudaStreamEndCapture(cap, &g)) && body && mlp_ok(m, cudaGraphInstantiate(&ge, g, 0));
  }
  uint32_t done = 0;
  while (ok && done + per_graph <= iters) {
    ok = mlp_ok(m, cudaGraphLaunch(ge, m->stream));
    done += per_graph;
  }
  if (ok && done < iters) ok = enqueue(iters - done, m->stream);
  if (ge) cudaGraphExecDestroy(ge);
  if (g) cudaGraphDestroy(g);
  cudaStreamDestroy(cap);
  if (ok && loss_hist_host)
    ok = mlp_ok(m, cudaMemcpyAsync(loss_hist_host, m->loss_hist, sizeof(float) * iters, cudaMemcpyDeviceToHost,
                                   m->stream));
  if (ok) ok = mlp_ok(m, cudaStreamSynchronize(m->stream)) && waits_clean(m);
  return ok ? 1 : 0;
}

int32_t phieng_mlp_shard_grad(PhiengMlp* m, const float* x, const float* t, uint32_t npairs, uint32_t first,
                              uint32_t batch, uint32_t total, uint64_t seed, float* grad) {
  if (!m || m->error || !grad || !check_pairs(x, t, npairs, batch) || total < batch || first > total - batch)
    return 0;
  uint32_t nparts = 0;
  if (!launch_tile(m, x, t, npairs, batch, seed, m->ctr, &nparts, first, total)) return 0;
  // raw sums: the gradient already carries 1 / total, the loss is the sum of squared errors
  k_mlp_reduce<<<cdiv(kParams + 1, 256), 256, 0, m->stream>>>(m->part, nparts, 1.0f, grad, grad + kParams);
  return mlp_ok(m, cudaGetLastError()) ? 1 : 0;
}

int32_t phieng_mlp_apply_grad(PhiengMlp* m, const float* grad, float lr) {
  if (!m || m->error || !grad || !(lr > 0.0f)) return 0;
  // a single gradient vector is a partial list of length one
  k_mlp_adam<<<cdiv(kParams + 1, 256), 256, 0, m->stream>>>(grad, 1, m->w, m->m, m->v, m->ctr, lr, 0.0f, nullptr, 0,
                                                              0, m->frag, m->bias, m->w3);
  k_mlp_advance<<<1, 1, 0, m->stream>>>(m->ctr);
  return mlp_ok(m, cudaGetLastError()) ? 1 : 0;
}

int32_t phieng_mlp_set_train_engine(PhiengMlp* m, int32_t engine) {
  if (!m || m->error || (engine != PHIENG_MLP_TCGEN05 && engine != PHIENG_MLP_MMA_SYNC)) return 0;
  m->train_engine = engine;
  return 1;
}

int32_t phieng_mlp_get_train_engine(const PhiengMlp* m) { return m ? m->train_engine : -1; }

int32_t phieng_mlp_set_closure_engine(PhiengMlp* m, int32_t engine) {
  if (!m || m->error || (engine != PHIENG_MLP_TCGEN05 && engine != PHIENG_MLP_MMA_SYNC)) return 0;
  m->infer_engine = engine;
  return 1;
}

int32_t phieng_mlp_get_closure_engine(const PhiengMlp* m) { return m ? m->infer_engine : -1; }

int32_t phieng_mlp_sample_indices(uint32_t npairs, uint32_t batch, uint64_t seed, uint32_t iter, uint32_t* idx,
                                  void* stream) {
  if (!idx || npairs == 0) return 0;
  if (batch == 0) return 1;
  k_mlp_indices<<<cdiv(batch, 256), 256, 0, (cudaStream_t)stream>>>(seed, iter, batch, npairs, idx);
  return cudaGetLastError() == cudaSuccess ? 1 : 0;
}

int32_t phieng_mlp_perturb(float* state, uint32_t n, float amp, uint64_t seed, void* stream) {
  if (n && !state) return 0;
  if (n == 0) return 1;
  k_mlp_perturb<<<cdiv(n, 256), 256, 0, (cudaStream_t)stream>>>(reinterpret_cast<float4*>(state), n, amp, seed);
  return cudaGetLastError() == cudaSuccess ? 1 : 0;
}

int32_t phieng_mlp_targets(const float* fine, const float* coarse, uint32_t n, float inv_h, float dt, uint32_t mode,
                           float* out, void* stream) {
  if ((n && (!fine || !coarse || !out)) || mode > 2) return 0;
  if (n == 0) return 1;
  k_mlp_targets<<<cdiv(n, 256), 256, 0, (cudaStream_t)stream>>>(reinterpret_cast<const float4*>(fine),
                                                                 reinterpret_cast<const float4*>(coarse), n, inv_h,
                                                                 dt, mode, reinterpret_cast<float2*>(out));
  return cudaGetLastError() == cudaSuccess ? 1 : 0;
}

}  // extern "C"
