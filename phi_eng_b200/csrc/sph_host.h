// Host-side helpers shared by the 2D and 3D worlds (sph_world.cu, sph3d.cu):
// Rust float semantics the reference relies on, the fluid config defaults
// and validation (the 2D and 3D configs share fields, defaults and rules),
// error texts.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <new>

#include <cuda_runtime.h>

#include "../../include/phieng_sph.h"

namespace phieng {
namespace host {
constexpr uint32_t kMaxAddPerCall = 1000000;    // ffi.rs:2493
constexpr float kMaxDt = 1.0f / 15.0f;          // ffi.rs:80

// Page-locked host memory when a CUDA device can be used (the particle state
// then crosses PCIe as a direct DMA, not through the driver's bounce buffer),
// ordinary memory otherwise; a 64-byte header records which.
template <class T>
struct PinnedAlloc {
  using value_type = T;
  PinnedAlloc() = default;
  template <class U>
  PinnedAlloc(const PinnedAlloc<U>&) {}
  T* allocate(size_t n) {
    const size_t bytes = n * sizeof(T) + 64;
    void* p = nullptr;
    uint8_t kind = 1;
    if (cudaHostAlloc(&p, bytes, cudaHostAllocPortable) != cudaSuccess) {
      cudaGetLastError();
      kind = 0;
      p = std::malloc(bytes);
      if (!p) throw std::bad_alloc();
    }
    static_cast<uint8_t*>(p)[0] = kind;
    return reinterpret_cast<T*>(static_cast<uint8_t*>(p) + 64);
  }
  void deallocate(T* q, size_t) {
    uint8_t* p = reinterpret_cast<uint8_t*>(q) - 64;
    if (p[0] == 1)
      cudaFreeHost(p);
    else
      std::free(p);
  }
  template <class U>
  bool operator==(const PinnedAlloc<U>&) const {
    return true;
  }
  template <class U>
  bool operator!=(const PinnedAlloc<U>&) const {
    return false;
  }
};

inline float rmaxf(float a, float b) {  // f32::max: a NaN operand loses
  if (a != a) return b;
  if (b != b) return a;
  return a > b ? a : b;
}

inline int32_t sat_floor_i32(float v) {  // `v.floor() as i32`
  float f = std::floor(v);
  if (f != f) return 0;
  if (f >= 2147483648.0f) return INT32_MAX;
  if (f <= -2147483648.0f) return INT32_MIN;
  return (int32_t)f;
}

inline uint32_t next_pow2(uint64_t v) {
  uint32_t p = 1;
  while (p < v && p < (1u << 31)) p <<= 1;
  return p;
}

inline uint32_t log2u(uint32_t v) {
  uint32_t l = 0;
  while ((1u << l) < v) l++;
  return l;
}

inline FluidConfig2Ffi default_config() {  // FluidConfig2::default (fluid.rs:142-169)
  FluidConfig2Ffi c;
  std::memset(&c, 0, sizeof(c));
  c.particle_mass = 0.0625f;
  c.rest_density = 1.0f;
  c.smoothing_length = 0.5f;
  c.stiffness = 100.0f;
  c.gamma = 1.0f;
  c.artificial_viscosity = 0.0f;
  c.surface_tension = 0.0f;
  c.cfl = 0.0f;
  c.max_substeps = 1;
  c.adaptive_resolution = 0;
  c.split_density_ratio = 0.5f;
  c.merge_density_ratio = 1.6f;
  c.boundary_particles = 0;
  c.viscosity = 0.3f;
  c.drag = 4.0f;
  c.wall_friction = 0.0f;
  c.phase_count = 1;
  for (int k = 0; k < 4; k++) {
    c.phase_rest_density[k] = 1.0f;
    c.phase_mass[k] = 0.0625f;
  }
  c.max_velocity = 30.0f;
  c.particle_radius = 0.125f;
  c.enabled = 1;
  return c;
}

// fluid2_from_ffi validation (ffi.rs:773-855).
inline bool valid_config(const FluidConfig2Ffi& c) {
  const float fs[] = {c.particle_mass,         c.rest_density,          c.smoothing_length,
                      c.stiffness,             c.gamma,                 c.artificial_viscosity,
                      c.surface_tension,       c.cfl,                   c.split_density_ratio,
                      c.merge_density_ratio,   c.viscosity,             c.drag,
                      c.wall_friction,         c.max_velocity,          c.particle_radius,
                      c.phase_rest_density[0], c.phase_rest_density[1], c.phase_rest_density[2],
                      c.phase_rest_density[3], c.phase_mass[0],         c.phase_mass[1],
                      c.phase_mass[2],         c.phase_mass[3]};
  for (float v : fs)
    if (!std::isfinite(v)) return false;
  if (c.particle_mass <= 0.0f || c.rest_density <= 0.0f || c.smoothing_length <= 0.0f || c.stiffness < 0.0f ||
      c.gamma < 1.0f || c.artificial_viscosity < 0.0f || c.artificial_viscosity > 2.0f ||
      c.surface_tension < 0.0f || c.cfl < 0.0f || c.cfl > 1.0f || c.max_substeps < 1 ||
      c.split_density_ratio <= 0.0f || c.merge_density_ratio <= 1.0f || c.viscosity < 0.0f ||
      c.viscosity > 1.0f || c.drag < 0.0f || c.wall_friction < 0.0f || c.wall_friction > 1.0f ||
      c.phase_count < 1 || c.phase_count > 4 || c.max_velocity < 0.0f || c.particle_radius < 0.0f)
    return false;
  for (int k = 0; k < 4; k++)
    if (c.phase_rest_density[k] <= 0.0f || c.phase_mass[k] <= 0.0f) return false;
  return true;
}

inline const char* error_text(int32_t e) {
  switch (e) {
    case PHIENG_SPH_OK:
      return "ok";
    case PHIENG_SPH_E_NO_DEVICE:
      return "no usable CUDA device";
    case PHIENG_SPH_E_CUDA:
      return "a CUDA call failed";
    case PHIENG_SPH_E_UNSUPPORTED:
      return "the fluid config enables adaptive resolution or boundary particles, which this library does not "
             "implement";
    case PHIENG_SPH_E_ARG:
      return "invalid argument";
    default:
      return "unknown error";
  }
}

}  // namespace host
}  // namespace phieng
