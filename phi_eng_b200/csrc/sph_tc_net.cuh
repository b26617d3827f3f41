// The closure network (16 -> 64 -> 64 -> 2, sph_mlp.cuh) on the 5th-generation
// tensor cores, for a CTA of 128 threads that owns one 128-row tile at a
// time (thread t = row t). Used by the standalone forward pass
// (phieng_mlp_forward_tc) and by the fused coarse step of the tolerance mode.
//
// Operands live in shared memory in the K-major no-swizzle layout of
// sph_tc.cuh, with the numerics of the mma.sync path: x_hat and W1 / 2 as
// BF16, hidden activations, W2 / 2 and W3 as FP16; accumulators are f32 in
// 64 TMEM columns that the three layers reuse:
//   layer 1  D[:, 0:64) = x_hat (W1/2)^T        1 MMA  (K = 16)
//   layer 2  D[:, 0:64) = H1 (W2/2)^T           4 MMAs (K = 64)
//   layer 3  D[:, 0:16) = H2 W3pad^T            4 MMAs (N = 16; rows 2..15 of W3pad zero)
// A layer's MMAs are issued only after every thread has read the previous
// layer's columns (tcgen05.wait::ld, then fence / barrier / fence). Thread t
// adds the halved bias to its row, applies silu(z) = u + u tanh(u) on
// u = z / 2 as FP16 pairs and writes row t of the next operand. One thread
// issues the MMAs; each layer's completion arrives on an mbarrier whose waits
// are bounded. 64 columns per CTA: any number of CTAs that the shared memory
// lets share an SM (at most 6 at 33 KB each) fits the SM's 512 columns.
#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "sph_mlp.cuh"
#include "sph_tc.cuh"

namespace phieng {

constexpr uint32_t kNetX = 0;                      // x_hat   [128][16] bf16
constexpr uint32_t kNetA = kNetX + 128 * 16 * 2;   // H1 / H2 [128][64] fp16
constexpr uint32_t kNetW1 = kNetA + 128 * 64 * 2;  // W1 / 2  [64][16]  bf16
constexpr uint32_t kNetW2 = kNetW1 + 64 * 16 * 2;  // W2 / 2  [64][64]  fp16
constexpr uint32_t kNetW3 = kNetW2 + 64 * 64 * 2;  // W3      [16][64]  fp16
constexpr uint32_t kNetBias = kNetW3 + 16 * 64 * 2;  // b1 / 2 | b2 / 2 | b3 (f32)
constexpr uint32_t kNetNorm = kNetBias + 4 * 256;    // mu | isd | out_scale (f32)
constexpr uint32_t kNetBar = kNetNorm + 4 * 64;      // mbarrier
constexpr uint32_t kNetSlot = kNetBar + 8;           // TMEM address
constexpr uint32_t kNetSmem = kNetSlot + 8;          // dynamic shared memory of a CTA (16-byte multiple)
constexpr uint32_t kNetCols = 64;
constexpr uint32_t kNetWaitLimit = 1u << 20;

struct TcNet {
  unsigned char* sm;
  uint32_t tmem;
  uint32_t phase;
  __device__ __forceinline__ const float* norm() const { return reinterpret_cast<const float*>(sm + kNetNorm); }
  __device__ __forceinline__ const float* bias() const { return reinterpret_cast<const float*>(sm + kNetBias); }
  __device__ __forceinline__ uint64_t* bar() const { return reinterpret_cast<uint64_t*>(sm + kNetBar); }
};

// Stage the weights (from the mma.sync fragment images) and the bias /
// normalisation, set up the mbarrier and the CTA's TMEM columns. All 128
// threads call it.
__device__ __forceinline__ TcNet tc_net_init(unsigned char* sm, const MlpDev& mlp) {
  const uint32_t tid = threadIdx.x;
  const __nv_bfloat16* img = reinterpret_cast<const __nv_bfloat16*>(mlp.frag);
  const __half* himg = reinterpret_cast<const __half*>(mlp.frag);
  for (uint32_t i = tid; i < 64 * 16; i += 128) {
    const uint32_t o = i >> 4, k = i & 15;
    *reinterpret_cast<__nv_bfloat16*>(sm + kNetW1 + tc::kmajor_offset(o, k, 16)) = img[frag_pos(k, o, 8)];
  }
  for (uint32_t i = tid; i < 64 * 64; i += 128) {
    const uint32_t o = i >> 6, k = i & 63;
    *reinterpret_cast<__half*>(sm + kNetW2 + tc::kmajor_offset(o, k, 64)) = himg[4 * kF1 + frag_pos(k, o, 8)];
  }
  for (uint32_t i = tid; i < 16 * 64; i += 128) {
    const uint32_t o = i >> 6, k = i & 63;
    *reinterpret_cast<__half*>(sm + kNetW3 + tc::kmajor_offset(o, k, 64)) =
        o < 2 ? himg[4 * (kF1 + kF2) + frag_pos(k, o, 1)] : __float2half_rn(0.0f);
  }
  float* bias = reinterpret_cast<float*>(sm + kNetBias);
  float* norm = reinterpret_cast<float*>(sm + kNetNorm);
  for (uint32_t i = tid; i < kBias; i += 128) bias[i] = mlp.bias[i];
  for (uint32_t i = tid; i < kNorm; i += 128) norm[i] = mlp.norm[i];
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kNetBar);
  uint32_t* slot = reinterpret_cast<uint32_t*>(sm + kNetSlot);
  if (tid == 0) tc::mbar_init(bar, 1);
  if ((tid >> 5) == 0) tc::tmem_alloc(slot, kNetCols);
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  TcNet net;
  net.sm = sm;
  net.tmem = *slot;
  net.phase = 0;
  return net;
}

// Operand writes -> one thread issues `issue` and commits -> every thread
// waits for the completion. Returns false (for every thread) if a wait ran
// out; the phase is then left at the incomplete one.
template <class F>
__device__ __forceinline__ bool tc_net_layer(TcNet& net, F&& issue) {
  return tc::mma_step(net.bar(), net.phase, kNetWaitLimit, issue);
}

// Hidden-layer epilogue: TMEM columns [0, 64) of this thread's row plus the
// halved bias b, through silu, as FP16 into row threadIdx.x of the A operand.
// Two halves of 32 columns, to keep the registers of a fused caller low.
__device__ __forceinline__ void tc_net_hidden(const TcNet& net, const float* b) {
  const uint32_t lanes = ((threadIdx.x >> 5) * 32u) << 16;
  unsigned char* A = net.sm + kNetA;
#pragma unroll
  for (int half = 0; half < 2; half++) {
    float v[2][16];
#pragma unroll
    for (int q = 0; q < 2; q++) tc::tmem_ld16(net.tmem + lanes + 32 * half + 16 * q, v[q]);
    tc::tmem_wait_ld();
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int c = 32 * half + 16 * q;  // first unit of this group of 16
      uint32_t h[8];
#pragma unroll
      for (int j = 0; j < 8; j++)
        h[j] = silu_half_f16x2(__fadd_rn(v[q][2 * j], b[c + 2 * j]), __fadd_rn(v[q][2 * j + 1], b[c + 2 * j + 1]));
      *reinterpret_cast<uint4*>(A + tc::kmajor_offset(threadIdx.x, c, 64)) = make_uint4(h[0], h[1], h[2], h[3]);
      *reinterpret_cast<uint4*>(A + tc::kmajor_offset(threadIdx.x, c + 8, 64)) = make_uint4(h[4], h[5], h[6], h[7]);
    }
  }
}

// The network on row threadIdx.x's 16 features f (all 128 threads call it):
// y = network output times out_scale. Returns false if a wait ran out.
__device__ __forceinline__ bool tc_net_forward(TcNet& net, const float (&f)[kFeat], float (&y)[2]) {
  const float* norm = net.norm();
  const float* bias = net.bias();
  unsigned char* X = net.sm + kNetX;
  uint32_t xp[8];
#pragma unroll
  for (int k = 0; k < kFeat; k += 2)
    xp[k / 2] = pack_bf16(__fmul_rn(__fsub_rn(f[k], norm[k]), norm[kFeat + k]),
                          __fmul_rn(__fsub_rn(f[k + 1], norm[k + 1]), norm[kFeat + k + 1]));
  *reinterpret_cast<uint4*>(X + tc::kmajor_offset(threadIdx.x, 0, 16)) = make_uint4(xp[0], xp[1], xp[2], xp[3]);
  *reinterpret_cast<uint4*>(X + tc::kmajor_offset(threadIdx.x, 8, 16)) = make_uint4(xp[4], xp[5], xp[6], xp[7]);
  const uint32_t tm = net.tmem;
  const uint64_t dX = tc::smem_desc(tc::smem_u32(X), 128, 256);
  const uint64_t dW1 = tc::smem_desc(tc::smem_u32(net.sm + kNetW1), 128, 256);
  const uint32_t aA = tc::smem_u32(net.sm + kNetA), aW2 = tc::smem_u32(net.sm + kNetW2),
                 aW3 = tc::smem_u32(net.sm + kNetW3);
  if (!tc_net_layer(net, [&] { tc::mma_f16(tm, dX, dW1, tc::idesc_f16(tc::kFmtBF16, 64), 0u); })) return false;
  tc_net_hidden(net, bias);
  if (!tc_net_layer(net, [&] {
#pragma unroll
        for (uint32_t kk = 0; kk < 4; kk++)
          tc::mma_f16(tm, tc::smem_desc(aA + 256 * kk, 128, 1024), tc::smem_desc(aW2 + 256 * kk, 128, 1024),
                      tc::idesc_f16(tc::kFmtF16, 64), kk);
      }))
    return false;
  tc_net_hidden(net, bias + kHidden);
  if (!tc_net_layer(net, [&] {
#pragma unroll
        for (uint32_t kk = 0; kk < 4; kk++)
          tc::mma_f16(tm, tc::smem_desc(aA + 256 * kk, 128, 1024), tc::smem_desc(aW3 + 256 * kk, 128, 1024),
                      tc::idesc_f16(tc::kFmtF16, 16), kk);
      }))
    return false;
  float o[2];
  tc::tmem_ld2(tm + (((threadIdx.x >> 5) * 32u) << 16), o);
  tc::tmem_wait_ld();
  y[0] = __fmul_rn(__fadd_rn(o[0], bias[2 * kHidden]), norm[2 * kFeat]);
  y[1] = __fmul_rn(__fadd_rn(o[1], bias[2 * kHidden + 1]), norm[2 * kFeat + 1]);
  return true;
}

// End of the CTA's work (all threads): a wait that ran out is reported in
// *err and the MMA in flight gets one more bounded wait; then the TMEM
// columns are released.
__device__ __forceinline__ void tc_net_finish(TcNet& net, bool ok, uint32_t* err) {
  if (!ok) {
    if (threadIdx.x == 0) atomicExch(err, 1u);
    tc::mbar_wait(net.bar(), net.phase, kNetWaitLimit);
  }
  tc::fence_before_sync();
  __syncthreads();
  if ((threadIdx.x >> 5) == 0) {
    tc::fence_after_sync();
    tc::tmem_free(net.tmem, kNetCols);
  }
}

}  // namespace phieng
