// Ambient turbulence in the fluid integrate (fluid.rs:1001-1019): the
// engine's deterministic value noise (crates/dynamics/src/noise.rs), every
// operation a correctly rounded f32 operation in the reference's order, so
// the field is bit-identical to the CPU evaluation.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace phieng {

// Integer avalanche hash (noise.rs:27-35).
__device__ __forceinline__ uint32_t noise_hash(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

// 2D lattice point + seed -> [0, 1) (noise.rs:38-47): the top 24 hash bits
// times 2^-24, both exact.
__device__ __forceinline__ float noise_lattice(int32_t ix, int32_t iy, uint32_t seed) {
  const uint32_t h = noise_hash((uint32_t)ix * 0x1f1f1f1fu + (uint32_t)iy * 0x9e3779b9u + seed);
  return __fmul_rn(__uint2float_rn(h >> 8), 1.0f / 16777216.0f);
}

// Quintic fade t*t*t*(t*(t*6 - 15) + 10) (noise.rs:64-67).
__device__ __forceinline__ float noise_fade(float t) {
  return __fmul_rn(__fmul_rn(__fmul_rn(t, t), t), __fadd_rn(__fmul_rn(t, __fsub_rn(__fmul_rn(t, 6.0f), 15.0f)), 10.0f));
}

// a + (b - a) * t (noise.rs:69-72).
__device__ __forceinline__ float noise_lerp(float a, float b, float t) { return __fadd_rn(a, __fmul_rn(__fsub_rn(b, a), t)); }

// 2D value noise in [0, 1) (noise.rs:75-87). f32 -> i32 as Rust's `as`:
// truncation, saturating, NaN -> 0 (PTX cvt.rzi.s32.f32).
__device__ __forceinline__ float value_noise2(float x, float y, uint32_t seed) {
  const float x0 = floorf(x), y0 = floorf(y);
  const int32_t xi = __float2int_rz(x0), yi = __float2int_rz(y0);
  const float tx = noise_fade(__fsub_rn(x, x0));
  const float ty = noise_fade(__fsub_rn(y, y0));
  const int32_t xi1 = (int32_t)((uint32_t)xi + 1u), yi1 = (int32_t)((uint32_t)yi + 1u);
  const float v00 = noise_lattice(xi, yi, seed);
  const float v10 = noise_lattice(xi1, yi, seed);
  const float v01 = noise_lattice(xi, yi1, seed);
  const float v11 = noise_lattice(xi1, yi1, seed);
  return noise_lerp(noise_lerp(v00, v10, tx), noise_lerp(v01, v11, tx), ty);
}

// Static fBm in [-1, 1] over oct octaves (noise.rs:115-132).
__device__ __forceinline__ float fbm2_static(float x, float y, uint32_t seed, uint32_t oct) {
  float sum = 0.0f, amp = 1.0f, freq = 1.0f, norm = 0.0f;
  for (uint32_t o = 0; o < oct; o++) {
    const float v = value_noise2(__fmul_rn(x, freq), __fmul_rn(y, freq), seed + o);
    sum = __fadd_rn(sum, __fmul_rn(amp, __fsub_rn(__fmul_rn(v, 2.0f), 1.0f)));
    norm = __fadd_rn(norm, amp);
    amp = __fmul_rn(amp, 0.5f);
    freq = __fmul_rn(freq, 2.0f);
  }
  return norm > 0.0f ? __fdiv_rn(sum, norm) : 0.0f;
}

// Time-evolving fBm (noise.rs:154-170): a fade-weighted lerp between the
// fields of the two integer time slices around t, each slice with its own
// seed seed + slice * 0x9e3779b9 (slice = t's floor as i64, saturating, then
// truncated to 32 bits).
__device__ __forceinline__ float fbm2(float x, float y, float t, uint32_t seed, uint32_t oct) {
  const float t0 = floorf(t);
  const float ft = noise_fade(__fsub_rn(t, t0));
  const long long sl = __float2ll_rz(t0);
  const uint32_t s0 = seed + (uint32_t)sl * 0x9e3779b9u;
  const uint32_t s1 = seed + ((uint32_t)sl + 1u) * 0x9e3779b9u;
  return noise_lerp(fbm2_static(x, y, s0, oct), fbm2_static(x, y, s1, oct), ft);
}

// The turbulence acceleration of a particle at (px, py) (fluid.rs:1007-1018):
// noise sampled at position * frequency and time * time_scale, either curl
// noise (central differences of the fBm potential with step 1e-3,
// noise.rs:186-193) or two fBm fields (the second seeded seed ^ 0x55aa55aa),
// clamped to length 1 as glam 0.29's Vec2::clamp_length_max(1.0) does
// (v / sqrt(|v|^2) when |v|^2 > 1), times the amplitude. Out of line: the
// force kernels only pay a call when turbulence is on.
__device__ __noinline__ float2 turbulence_accel(float px, float py, float time, float freq, float tscale,
                                                uint32_t seed, uint32_t oct, uint32_t curl, float amp) {
  const float x = __fmul_rn(px, freq), y = __fmul_rn(py, freq);
  const float t = __fmul_rn(time, tscale);
  float nx, ny;
  if (curl) {
    const float e = 1e-3f;
    const float e2 = 2.0f * 1e-3f;  // the reference's (2.0 * E), folded in f32 (exact doubling)
    const float dpdy = __fdiv_rn(__fsub_rn(fbm2(x, __fadd_rn(y, e), t, seed, oct), fbm2(x, __fsub_rn(y, e), t, seed, oct)), e2);
    const float dpdx = __fdiv_rn(__fsub_rn(fbm2(__fadd_rn(x, e), y, t, seed, oct), fbm2(__fsub_rn(x, e), y, t, seed, oct)), e2);
    nx = dpdy;
    ny = -dpdx;
  } else {
    nx = fbm2(x, y, t, seed, oct);
    ny = fbm2(x, y, t, seed ^ 0x55aa55aau, oct);
  }
  const float ls = __fadd_rn(__fmul_rn(nx, nx), __fmul_rn(ny, ny));
  if (ls > 1.0f) {
    const float l = __fsqrt_rn(ls);
    nx = __fdiv_rn(nx, l);
    ny = __fdiv_rn(ny, l);
  }
  return make_float2(__fmul_rn(nx, amp), __fmul_rn(ny, amp));
}

}  // namespace phieng
