// Density and pressure of a particle set with no GPU memory allocation.
//
// Who needs this: hosts that may not call cudaMalloc / cudaFree on their
// per-frame path. A game engine that drives PhiEng from its simulation
// thread cannot afford cudaMalloc there: it may synchronise the whole device
// and take milliseconds, which stalls the frame. Some hosts also reserve
// their GPU memory up front and treat any later allocation as an error.
// Such callers can run the SPH density pass through
// phieng_sph_density_noalloc, which works entirely in a fixed scratch area
// that is part of this library's device image.
//
// The scratch is one file-scope __device__ array of kScratchBytes (about
// 6 MiB): every GPU that loads the library holds it until the process exits.
// It bounds a call to kNoAllocMaxParticles particles and a bucket grid of at
// most 2^16 buckets (cells further apart share buckets; results do not
// change). Every call uses the same array, so two calls whose GPU work
// overlaps (different streams, or different host threads) race and corrupt
// each other's results; calls must be ordered on the device.
//
// The first call on a device looks up the array's device address with
// cudaGetSymbolAddress (which can trigger module loading); make that first
// call before any stream capture. The address is cached per device for the
// life of the process, so a cudaDeviceReset (which unloads the module) needs
// a process restart before the next call. Each call blocks once on the
// bounding-box read-back that sizes the bucket grid; every particle is
// phase 0.
#include <cmath>
#include <cstdio>
#include <cstring>

#include <cuda_runtime.h>

#include "../../include/phieng_sph.h"
#include "sph_kernels.h"

using namespace phieng;

namespace {

constexpr uint32_t kNoAllocMaxParticles = 65536;
constexpr uint32_t kNoAllocMaxBucketsLog2 = 16;
constexpr uint32_t kMaxBuckets = 1u << kNoAllocMaxBucketsLog2;
constexpr uint32_t kCountLen =
    ((kMaxBuckets + 1 + kBucketScanTile - 1) / kBucketScanTile) * kBucketScanTile;  // buckets + sentinel, padded
constexpr uint32_t kScanTiles = kCountLen / kBucketScanTile;
constexpr size_t kN = kNoAllocMaxParticles;

constexpr size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

// Byte offsets of the sub-arrays inside the scratch.
constexpr size_t kOffState = 0;                                          // float4 [N]
constexpr size_t kOffKey = align256(kOffState + 16 * kN);                // u32 [N]
constexpr size_t kOffTkey = align256(kOffKey + 4 * kN);                  // u32 [N]
constexpr size_t kOffTid = align256(kOffTkey + 4 * kN);                  // u32 [N]
constexpr size_t kOffSkey = align256(kOffTid + 4 * kN);                  // u32 [N]
constexpr size_t kOffSid = align256(kOffSkey + 4 * kN);                  // u32 [N]
constexpr size_t kOffSpos = align256(kOffSid + 4 * kN);                  // float2 [N]
constexpr size_t kOffSvel = align256(kOffSpos + 8 * kN);                 // float2 [N]
constexpr size_t kOffSdq = align256(kOffSvel + 8 * kN);                  // float2 [N]
constexpr size_t kOffSpres = align256(kOffSdq + 8 * kN);                 // float [N]
constexpr size_t kOffMask = align256(kOffSpres + 4 * kN);                // u32 [3N] (room for 8 B each)
constexpr size_t kOffCount = align256(kOffMask + 24 * kN);               // u32 [kCountLen]
constexpr size_t kOffStart = align256(kOffCount + 4 * (size_t)kCountLen);  // u32 [kCountLen + 1]
constexpr size_t kOffTiles = align256(kOffStart + 4 * ((size_t)kCountLen + 1));  // u32 [kScanTiles]
constexpr size_t kOffCtl = align256(kOffTiles + 4 * (size_t)kScanTiles);  // u32 [16]: done, bbox
constexpr size_t kScratchBytes = align256(kOffCtl + 64);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Device address of g_noalloc_scratch per device (host-side cache).
constexpr int kMaxDevices = 64;
void* g_scratch_addr[kMaxDevices] = {nullptr};

// Cell bounding box of the finite particles: ctl[1..4] = min cx, min cy,
// max cx, max cy as order-preserving unsigned keys (signed i32 xor 0x80000000).
__global__ void __launch_bounds__(256) k_na_pack_bbox(const float2* __restrict__ xy, uint32_t n, float hg,
                                                      float4* __restrict__ state, uint32_t* __restrict__ ctl) {
  uint32_t lo_x = 0xFFFFFFFFu, lo_y = 0xFFFFFFFFu, hi_x = 0u, hi_y = 0u;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float2 p = xy[i];
    state[i] = make_float4(p.x, p.y, 0.0f, 0.0f);
    if (isfinite(p.x) && isfinite(p.y)) {
      const uint32_t cx = (uint32_t)__float2int_rd(__fdiv_rn(p.x, hg)) ^ 0x80000000u;
      const uint32_t cy = (uint32_t)__float2int_rd(__fdiv_rn(p.y, hg)) ^ 0x80000000u;
      lo_x = min(lo_x, cx);
      lo_y = min(lo_y, cy);
      hi_x = max(hi_x, cx);
      hi_y = max(hi_y, cy);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo_x = min(lo_x, __shfl_xor_sync(0xFFFFFFFFu, lo_x, o));
    lo_y = min(lo_y, __shfl_xor_sync(0xFFFFFFFFu, lo_y, o));
    hi_x = max(hi_x, __shfl_xor_sync(0xFFFFFFFFu, hi_x, o));
    hi_y = max(hi_y, __shfl_xor_sync(0xFFFFFFFFu, hi_y, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&ctl[1], lo_x);
    atomicMin(&ctl[2], lo_y);
    atomicMax(&ctl[3], hi_x);
    atomicMax(&ctl[4], hi_y);
  }
}

inline float rmaxf(float a, float b) {
  if (a != a) return b;
  if (b != b) return a;
  return a > b ? a : b;
}

inline uint32_t pow2_at_least(uint64_t v) {
  uint32_t l = 0;
  while ((1ull << l) < v && l < 31) l++;
  return l;
}

}  // namespace

extern "C" int32_t phieng_sph_density_noalloc(const float* xy, uint32_t n, const FluidConfig2Ffi* cfg,
                                              float* density, float* pressure, void* stream) {
  if (!cfg) return PHIENG_SPH_E_ARG;
  if (n > kNoAllocMaxParticles) {
    std::fprintf(stderr, "phieng_sph_density_noalloc: %u particles exceed the fixed scratch capacity of %u\n", n,
                 kNoAllocMaxParticles);
    return PHIENG_SPH_E_TOO_LARGE;
  }
  const FluidConfig2Ffi& c = *cfg;
  if (!(std::isfinite(c.smoothing_length) && c.smoothing_length > 0.0f) || !std::isfinite(c.stiffness) ||
      !(c.gamma >= 1.0f) || !std::isfinite(c.gamma) || !(c.rest_density > 0.0f) ||
      !(c.phase_rest_density[0] > 0.0f) || !std::isfinite(c.phase_rest_density[0]) ||
      !(c.phase_mass[0] > 0.0f) || !std::isfinite(c.phase_mass[0]))
    return PHIENG_SPH_E_ARG;
  if (n == 0) return PHIENG_SPH_OK;
  if (!xy || !density || !pressure) return PHIENG_SPH_E_ARG;
  cudaStream_t st = (cudaStream_t)stream;

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return PHIENG_SPH_E_NO_DEVICE;
  }
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    const cudaError_t r = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (r != cudaSuccess || !p) {
      cudaGetLastError();
      std::fprintf(stderr, "phieng_sph_density_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(r));
      return PHIENG_SPH_E_CUDA;
    }
    g_scratch_addr[dev] = p;
  }
  unsigned char* base = static_cast<unsigned char*>(g_scratch_addr[dev]);
  uint32_t* ctl = reinterpret_cast<uint32_t*>(base + kOffCtl);

  // The array keeps the previous call's contents: reset the scan counter and
  // the bounding box before use (bucket counts are cleared by the key pass).
  if (cudaMemsetAsync(ctl, 0, sizeof(uint32_t), st) != cudaSuccess ||                // scan counter
      cudaMemsetAsync(ctl + 1, 0xFF, 2 * sizeof(uint32_t), st) != cudaSuccess ||     // bbox minima
      cudaMemsetAsync(ctl + 3, 0, 2 * sizeof(uint32_t), st) != cudaSuccess) {        // bbox maxima
    cudaGetLastError();
    return PHIENG_SPH_E_CUDA;
  }
  const float hg = c.smoothing_length;
  FluidBufs b;
  b.cap = kNoAllocMaxParticles;
  b.state = reinterpret_cast<float4*>(base + kOffState);
  b.key = reinterpret_cast<uint32_t*>(base + kOffKey);
  b.tkey = reinterpret_cast<uint32_t*>(base + kOffTkey);
  b.tid = reinterpret_cast<uint32_t*>(base + kOffTid);
  b.skey = reinterpret_cast<uint32_t*>(base + kOffSkey);
  b.sid = reinterpret_cast<uint32_t*>(base + kOffSid);
  b.spos = reinterpret_cast<float2*>(base + kOffSpos);
  b.svel = reinterpret_cast<float2*>(base + kOffSvel);
  b.sdq = reinterpret_cast<float2*>(base + kOffSdq);
  b.spres = reinterpret_cast<float*>(base + kOffSpres);
  b.nmask = reinterpret_cast<uint32_t*>(base + kOffMask);
  b.count = reinterpret_cast<uint32_t*>(base + kOffCount);
  b.start = reinterpret_cast<uint32_t*>(base + kOffStart);
  b.tilesum = reinterpret_cast<uint32_t*>(base + kOffTiles);
  b.done = ctl;

  // bucket grid from the particles' cell bounding box (one read-back)
  const uint32_t blocks = (n + 255) / 256 < 256 ? (n + 255) / 256 : 256;
  k_na_pack_bbox<<<blocks, 256, 0, st>>>(reinterpret_cast<const float2*>(xy), n, hg, b.state, ctl);
  uint32_t bbox[5];
  if (cudaMemcpyAsync(bbox, ctl, sizeof(bbox), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess) {
    cudaGetLastError();
    return PHIENG_SPH_E_CUDA;
  }
  int64_t x0 = 0, y0 = 0, sx = 1, sy = 1;
  if (bbox[1] <= bbox[3]) {
    x0 = (int32_t)(bbox[1] ^ 0x80000000u);
    y0 = (int32_t)(bbox[2] ^ 0x80000000u);
    sx = (int64_t)(int32_t)(bbox[3] ^ 0x80000000u) - x0 + 1;
    sy = (int64_t)(int32_t)(bbox[4] ^ 0x80000000u) - y0 + 1;
  }
  uint32_t lw = pow2_at_least((uint64_t)sx + 4), lh = pow2_at_least((uint64_t)sy + 4);
  if (lw < 2) lw = 2;
  if (lh < 2) lh = 2;
  while (lw + lh > kNoAllocMaxBucketsLog2) {
    if (lw >= lh && lw > 2)
      lw--;
    else
      lh--;
  }
  StepParams P;
  std::memset(&P, 0, sizeof(P));
  P.grid.log2w = lw;
  P.grid.log2h = lh;
  P.grid.maskw = (1u << lw) - 1u;
  P.grid.maskh = (1u << lh) - 1u;
  P.grid.nbuckets = 1u << (lw + lh);
  P.grid.base = 0;
  P.grid.sentinel = P.grid.nbuckets;
  P.grid.cx0 = (int32_t)(x0 - 2);
  P.grid.cy0 = (int32_t)(y0 - 2);
  P.grid.hg = hg;
  // the density-pass parameters exactly as a world step derives them
  P.hg2 = hg * hg;
  const float h = rmaxf(hg, kEps);
  P.hk = h;
  const float h2 = h * h;
  P.hk2 = h2;
  const float pi = 3.14159265358979323846f;
  P.c_poly6 = 4.0f / (pi * h2 * h2 * h2 * h2);
  P.c_spiky = -30.0f / (pi * h * h * h * h * h);
  P.rho_cap = 3.0f * rmaxf(c.rest_density, kEps);
  P.stiffness = c.stiffness;
  P.gamma = c.gamma;
  for (int k = 0; k < 4; k++) P.rest[k] = c.phase_rest_density[k];
  P.mass = rmaxf(c.phase_mass[0], 0.0f);
  P.flags = (c.gamma != 1.0f) ? (uint32_t)F_TAIT : 0u;
  P.uniform_phase = 0;
  b.count_len = (P.grid.nbuckets + 1 + kBucketScanTile - 1) / kBucketScanTile * kBucketScanTile;

  enqueue_keys(b, n, P.grid, st);
  enqueue_sort_and_ranges(b, n, P, false, st);
  enqueue_density(b, n, P, st);
  enqueue_unsort_dp(b, n, density, pressure, st);
  if (cudaGetLastError() != cudaSuccess) return PHIENG_SPH_E_CUDA;
  return PHIENG_SPH_OK;
}
