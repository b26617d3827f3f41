// Per-particle closure network: 16 -> 64 -> 64 -> 2, SiLU, on the tensor
// cores (mma.sync m16n8k16, FP32 accumulate): layer 1 on BF16 inputs and
// weights, layers 2 and 3 on FP16 activations and weights.
//
// Layout conventions shared by the inference path (fused into the coarse
// force pass), the standalone forward kernel and the training kernels:
//   parameters (FP32 masters, gradients, Adam moments), one flat vector:
//     W1[64][16] | b1[64] | W2[64][64] | b2[64] | W3[2][64] | b3[2]
//     (W[out][in]; z = W x + b)
//   normalisation: mu[16] | isd[16] | out_scale[2]; the network sees
//     x_hat = bf16((x - mu) * isd) and the caller gets y * out_scale.
//   weight fragment images (the B operand of m16n8k16 in register order):
//   one uint2 per lane per (k-tile, n-tile), so a warp loads a whole B
//   fragment with one conflict-free 64-bit shared-memory read per lane.
//     F1  B(k, n) = W1[n][k] / 2   BF16, 1 k-tile  x 8 n-tiles
//     F2  B(k, n) = W2[n][k] / 2   FP16, 4 k-tiles x 8 n-tiles
//     F3  B(k, n) = W3[n][k]       FP16, 4 k-tiles x 1 n-tile (outputs 2..7 are zero)
//     F2T B(k, n) = W2[k][n]       BF16, 4 k-tiles x 8 n-tiles (backward dH1 = dZ2 W2)
//   The hidden layers run on halved weights and biases, so their accumulators
//   hold u = z / 2 (exact: a power-of-two scale commutes with the rounding)
//   and the activation is silu(z) = u + u tanh(u) (silu_half_f16x2). Each
//   layer's bias is the accumulator's initial value.
//
// m16n8k16 register layout (PTX ISA, "Matrix Fragments for mma.m16n8k16"),
// g = lane / 4, t = lane % 4:
//   A (16x16, row major): a0 = rows g, cols 2t..2t+1; a1 = rows g+8, same
//     cols; a2 = row g, cols 2t+8..2t+9; a3 = row g+8, cols 2t+8..2t+9
//   B (16x8): b0 = k 2t..2t+1, col g; b1 = k 2t+8..2t+9, col g
//   C (16x8, f32): c0, c1 = row g, cols 2t, 2t+1; c2, c3 = row g+8
// The C fragments of n-tiles 2j and 2j+1 are, packed to FP16 pairs, exactly
// the A fragment of k-tile j of the next layer, so hidden activations stay in
// registers between layers.
#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

namespace phieng {

constexpr int kFeat = 16;
constexpr int kHidden = 64;
constexpr int kOut = 2;
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kHidden * kFeat;    // 1024
constexpr int kOffW2 = kOffB1 + kHidden;            // 1088
constexpr int kOffB2 = kOffW2 + kHidden * kHidden;  // 5184
constexpr int kOffW3 = kOffB2 + kHidden;            // 5248
constexpr int kOffB3 = kOffW3 + kOut * kHidden;     // 5376
constexpr int kParams = kOffB3 + kOut;              // 5378
constexpr int kNorm = 2 * kFeat + kOut;             // 34

constexpr int kF1 = 8 * 32;   // uint2 per image
constexpr int kF2 = 32 * 32;
constexpr int kF3 = 4 * 32;
constexpr int kF2T = 32 * 32;
constexpr int kFragAll = kF1 + kF2 + kF3 + kF2T;
constexpr int kBias = 2 * kHidden + kOut;  // b1 | b2 | b3

// Device view of a network. frag: F1 | F2 | F3 | F2T; bias (FP32): b1/2 |
// b2/2 | b3; w3 (BF16-rounded, as FP32): W3[2][64]; norm: mu | isd |
// out_scale.
struct MlpDev {
  const uint2* frag;
  const float* bias;
  const float* w3;
  const float* norm;
  // network of the tolerance-mode coarse pass: kMlpInferTcgen05 or
  // kMlpInferMmaSync (64-bit: no padding bytes, the struct is part of a graph
  // signature)
  int64_t engine;
};

// (the values of PHIENG_MLP_TCGEN05 / PHIENG_MLP_MMA_SYNC)
constexpr int32_t kMlpInferTcgen05 = 0;
constexpr int32_t kMlpInferMmaSync = 1;

// Position (in BF16 elements) of B(k, n) inside an image with nt n-tiles.
__host__ __device__ inline uint32_t frag_pos(int k, int n, int nt_count) {
  const int kt = k >> 4, kk = k & 15, nt = n >> 3, g = n & 7;
  const int reg = kk >> 3, t = (kk & 7) >> 1, half = kk & 1;
  const int lane = g * 4 + t;
  return (uint32_t)(((((kt * nt_count + nt) * 32 + lane) * 2 + reg) * 2) + half);
}

__device__ __forceinline__ void mma_f16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  // volatile keeps the MMAs in program order: without it the compiler hoists
  // every fragment load ahead and spills
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Two floats rounded to nearest-even BF16, the first in the low half.
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// Hardware tanh (PTX tanh.approx.f32); sigmoid(z) = (1 + tanh(z/2)) / 2.
__device__ __forceinline__ float tanh_hw(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float sigmoid_hw(float z) { return __fadd_rn(__fmul_rn(0.5f, tanh_hw(__fmul_rn(0.5f, z))), 0.5f); }

// Activation of two hidden units from their halved pre-activations u = z / 2,
// as an FP16 pair (first unit in the low half):
//   silu(z) = z sigmoid(z) = z (1 + tanh(z / 2)) / 2 = u + u tanh(u)
// u converted to FP16 (saturating at +-65504, so the result stays finite),
// then PTX tanh.approx.f16x2 and one fma.rn.f16x2: three instructions and one
// special-function op per pair, where FP32 takes two special-function ops.
// FP16 keeps 1 + tanh(u) near u << 0 to about the FP32 tanh.approx error;
// BF16 there loses it to cancellation (~6 % output error).
__device__ __forceinline__ uint32_t silu_half_f16x2(float u0, float u1) {
  uint32_t u, t, h;
  asm("cvt.rn.satfinite.f16x2.f32 %0, %1, %2;" : "=r"(u) : "f"(u1), "f"(u0));
  asm("tanh.approx.f16x2 %0, %1;" : "=r"(t) : "r"(u));
  asm("fma.rn.f16x2 %0, %1, %2, %1;" : "=r"(h) : "r"(u), "r"(t));
  return h;
}
// d silu / dz = s + z s (1 - s)
__device__ __forceinline__ float dsilu_hw(float z) {
  const float s = sigmoid_hw(z);
  return __fadd_rn(s, __fmul_rn(__fmul_rn(z, s), __fsub_rn(1.0f, s)));
}

__device__ __forceinline__ uint32_t lds32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

// Copy a network's fragment images, biases and normalisation into shared
// memory (any block size).
struct MlpSmem {
  uint2 f1[kF1];
  uint2 f2[kF2];
  uint2 f3[kF3];
  float bias[kBias];
  float norm[kNorm];
};

__device__ __forceinline__ void mlp_load_smem(MlpSmem& s, const MlpDev& m) {
  for (int i = threadIdx.x; i < kF1 + kF2 + kF3; i += blockDim.x) {
    const uint2 v = m.frag[i];
    if (i < kF1)
      s.f1[i] = v;
    else if (i < kF1 + kF2)
      s.f2[i - kF1] = v;
    else
      s.f3[i - kF1 - kF2] = v;
  }
  for (int i = threadIdx.x; i < kBias; i += blockDim.x) s.bias[i] = m.bias[i];
  for (int i = threadIdx.x; i < kNorm; i += blockDim.x) s.norm[i] = m.norm[i];
}

// One warp, one 16-row tile: x_hat rows (BF16, row stride ldx elements) ->
// network output before out_scale. Lanes with t == 0 receive y[g][0..1] in
// y[0..1] and y[g+8][0..1] in y[2..3]; other lanes' y hold padding columns.
__device__ __forceinline__ void mlp_tile_forward(const __nv_bfloat16* xs, int ldx, const MlpSmem& s, int lane,
                                                 float (&y)[4]) {
  const int g = lane >> 2, t = lane & 3;
  uint32_t a[4];
  a[0] = lds32(xs + g * ldx + 2 * t);
  a[1] = lds32(xs + (g + 8) * ldx + 2 * t);
  a[2] = lds32(xs + g * ldx + 2 * t + 8);
  a[3] = lds32(xs + (g + 8) * ldx + 2 * t + 8);
  uint32_t h[4][4];
#pragma unroll
  for (int nt = 0; nt < 8; nt++) {
    const float2 bb = *reinterpret_cast<const float2*>(&s.bias[nt * 8 + 2 * t]);
    float c[4] = {bb.x, bb.y, bb.x, bb.y};
    const uint2 b = s.f1[nt * 32 + lane];
    mma_bf16(c, a, b.x, b.y);
    h[nt >> 1][(nt & 1) * 2 + 0] = silu_half_f16x2(c[0], c[1]);
    h[nt >> 1][(nt & 1) * 2 + 1] = silu_half_f16x2(c[2], c[3]);
  }
  const float b30 = t == 0 ? s.bias[2 * kHidden] : 0.0f;
  const float b31 = t == 0 ? s.bias[2 * kHidden + 1] : 0.0f;
  y[0] = b30;
  y[1] = b31;
  y[2] = b30;
  y[3] = b31;
  // layer 2 two n-tiles at a time, each pair (one k-tile of layer 3) fed to
  // the output straight away: 4 live activation registers instead of 16. The
  // pair's two accumulation chains alternate (k outer), so each MMA waits on
  // the one two issues back.
#pragma unroll
  for (int j = 0; j < 4; j++) {
    float c[2][4];
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const float2 bb = *reinterpret_cast<const float2*>(&s.bias[kHidden + (2 * j + q) * 8 + 2 * t]);
      c[q][0] = bb.x;
      c[q][1] = bb.y;
      c[q][2] = bb.x;
      c[q][3] = bb.y;
    }
#pragma unroll
    for (int kt = 0; kt < 4; kt++)
#pragma unroll
      for (int q = 0; q < 2; q++) {
        const uint2 b = s.f2[(kt * 8 + 2 * j + q) * 32 + lane];
        mma_f16(c[q], h[kt], b.x, b.y);
      }
    uint32_t h2[4];
#pragma unroll
    for (int q = 0; q < 2; q++) {
      h2[q * 2 + 0] = silu_half_f16x2(c[q][0], c[q][1]);
      h2[q * 2 + 1] = silu_half_f16x2(c[q][2], c[q][3]);
    }
    const uint2 b = s.f3[j * 32 + lane];
    mma_f16(y, h2, b.x, b.y);
  }
}

// x_hat = bf16((x - mu) * isd) for one row of 16 features, stored as BF16.
__device__ __forceinline__ void mlp_normalise_row(const float (&x)[kFeat], const float* norm, __nv_bfloat16* row) {
#pragma unroll
  for (int k = 0; k < kFeat; k += 2) {
    const float a = __fmul_rn(__fsub_rn(x[k], norm[k]), norm[kFeat + k]);
    const float b = __fmul_rn(__fsub_rn(x[k + 1], norm[k + 1]), norm[kFeat + k + 1]);
    *reinterpret_cast<uint32_t*>(row + k) = pack_bf16(a, b);
  }
}

}  // namespace phieng
