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
static __device__ __noinline__ float2 turbulence_accel(float px, float py, float time, float freq, float tscale,
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

// ---- 3D (fluid3.rs:1090-1108) ----

// 3D lattice point + seed -> [0, 1) (noise.rs:50-60).
__device__ __forceinline__ float noise_lattice3(int32_t ix, int32_t iy, int32_t iz, uint32_t seed) {
  const uint32_t h =
      noise_hash((uint32_t)ix * 0x1f1f1f1fu + (uint32_t)iy * 0x9e3779b9u + (uint32_t)iz * 0x85ebca6bu + seed);
  return __fmul_rn(__uint2float_rn(h >> 8), 1.0f / 16777216.0f);
}

// 3D value noise in [0, 1) (noise.rs:90-111): x, then y, then z blends.
__device__ __forceinline__ float value_noise3(float x, float y, float z, uint32_t seed) {
  const float x0 = floorf(x), y0 = floorf(y), z0 = floorf(z);
  const int32_t xi = __float2int_rz(x0), yi = __float2int_rz(y0), zi = __float2int_rz(z0);
  const float tx = noise_fade(__fsub_rn(x, x0));
  const float ty = noise_fade(__fsub_rn(y, y0));
  const float tz = noise_fade(__fsub_rn(z, z0));
  const int32_t xi1 = (int32_t)((uint32_t)xi + 1u), yi1 = (int32_t)((uint32_t)yi + 1u);
  const int32_t zi1 = (int32_t)((uint32_t)zi + 1u);
  const float a = noise_lerp(noise_lerp(noise_lattice3(xi, yi, zi, seed), noise_lattice3(xi1, yi, zi, seed), tx),
                             noise_lerp(noise_lattice3(xi, yi1, zi, seed), noise_lattice3(xi1, yi1, zi, seed), tx),
                             ty);
  const float b =
      noise_lerp(noise_lerp(noise_lattice3(xi, yi, zi1, seed), noise_lattice3(xi1, yi, zi1, seed), tx),
                 noise_lerp(noise_lattice3(xi, yi1, zi1, seed), noise_lattice3(xi1, yi1, zi1, seed), tx), ty);
  return noise_lerp(a, b, tz);
}

// Static 3D fBm in [-1, 1] (noise.rs:135-152).
__device__ __forceinline__ float fbm3_static(float x, float y, float z, uint32_t seed, uint32_t oct) {
  float sum = 0.0f, amp = 1.0f, freq = 1.0f, norm = 0.0f;
  for (uint32_t o = 0; o < oct; o++) {
    const float v = value_noise3(__fmul_rn(x, freq), __fmul_rn(y, freq), __fmul_rn(z, freq), seed + o);
    sum = __fadd_rn(sum, __fmul_rn(amp, __fsub_rn(__fmul_rn(v, 2.0f), 1.0f)));
    norm = __fadd_rn(norm, amp);
    amp = __fmul_rn(amp, 0.5f);
    freq = __fmul_rn(freq, 2.0f);
  }
  return norm > 0.0f ? __fdiv_rn(sum, norm) : 0.0f;
}

// Time-evolving 3D fBm (noise.rs:173-183), time slices as fbm2.
__device__ __forceinline__ float fbm3(float x, float y, float z, float t, uint32_t seed, uint32_t oct) {
  const float t0 = floorf(t);
  const float ft = noise_fade(__fsub_rn(t, t0));
  const long long sl = __float2ll_rz(t0);
  const uint32_t s0 = seed + (uint32_t)sl * 0x9e3779b9u;
  const uint32_t s1 = seed + ((uint32_t)sl + 1u) * 0x9e3779b9u;
  return noise_lerp(fbm3_static(x, y, z, s0, oct), fbm3_static(x, y, z, s1, oct), ft);
}

// Central difference of the fBm potential with seed ps along axis ax (0 x,
// 1 y, 2 z), step 1e-3 (noise.rs:208-216).
__device__ __forceinline__ float fbm3_diff(float x, float y, float z, float t, uint32_t ps, uint32_t oct, int ax) {
  const float e = 1e-3f;
  const float e2 = 2.0f * 1e-3f;  // the reference's (2.0 * E), folded in f32 (exact doubling)
  float hi, lo;
  if (ax == 0) {
    hi = fbm3(__fadd_rn(x, e), y, z, t, ps, oct);
    lo = fbm3(__fsub_rn(x, e), y, z, t, ps, oct);
  } else if (ax == 1) {
    hi = fbm3(x, __fadd_rn(y, e), z, t, ps, oct);
    lo = fbm3(x, __fsub_rn(y, e), z, t, ps, oct);
  } else {
    hi = fbm3(x, y, __fadd_rn(z, e), t, ps, oct);
    lo = fbm3(x, y, __fsub_rn(z, e), t, ps, oct);
  }
  return __fdiv_rn(__fsub_rn(hi, lo), e2);
}

// The 3D turbulence acceleration (fluid3.rs:1096-1108): curl_3 as the
// reference computes it (noise.rs:198-222: potentials seeded seed ^
// 0x11111111 / 0x22222222 / 0x33333333, components (d/dy psi_z - d/dz psi_y,
// d/dx psi_x - d/dz psi_z, d/dx psi_y - d/dy psi_x)), or three fBm fields
// (seeds seed, seed ^ 0x55aa55aa, seed ^ 0xaa55aa55); glam 0.29's
// Vec3::clamp_length_max(1.0) (|v|^2 = (x*x + y*y) + z*z); times the
// amplitude.
static __device__ __noinline__ float3 turbulence_accel3(float px, float py, float pz, float time, float freq, float tscale,
                                                        uint32_t seed, uint32_t oct, uint32_t curl, float amp) {
  const float x = __fmul_rn(px, freq), y = __fmul_rn(py, freq), z = __fmul_rn(pz, freq);
  const float t = __fmul_rn(time, tscale);
  float nx, ny, nz;
  if (curl) {
    const uint32_t sx = seed ^ 0x11111111u, sy = seed ^ 0x22222222u, sz = seed ^ 0x33333333u;
    nx = __fsub_rn(fbm3_diff(x, y, z, t, sz, oct, 1), fbm3_diff(x, y, z, t, sy, oct, 2));
    ny = __fsub_rn(fbm3_diff(x, y, z, t, sx, oct, 0), fbm3_diff(x, y, z, t, sz, oct, 2));
    nz = __fsub_rn(fbm3_diff(x, y, z, t, sy, oct, 0), fbm3_diff(x, y, z, t, sx, oct, 1));
  } else {
    nx = fbm3(x, y, z, t, seed, oct);
    ny = fbm3(x, y, z, t, seed ^ 0x55aa55aau, oct);
    nz = fbm3(x, y, z, t, seed ^ 0xaa55aa55u, oct);
  }
  const float ls = __fadd_rn(__fadd_rn(__fmul_rn(nx, nx), __fmul_rn(ny, ny)), __fmul_rn(nz, nz));
  if (ls > 1.0f) {
    const float l = __fsqrt_rn(ls);
    nx = __fdiv_rn(nx, l);
    ny = __fdiv_rn(ny, l);
    nz = __fdiv_rn(nz, l);
  }
  return make_float3(__fmul_rn(nx, amp), __fmul_rn(ny, amp), __fmul_rn(nz, amp));
}

}  // namespace phieng
