// The fluid block of the reference's binary world snapshot
// (crates/dynamics/src/snapshot.rs): encode_fluid_config2/3 + encode_fluid2/3
// (:6337-6382, :6478-6491, :6527-6572, :6662-6677), their decoders
// (:6384-6476, :6493-6525, :6573-6660, :6679-6718) and the apply step of a
// load (apply_fluid2/3, :4471-4543, :4545-4612). Little-endian; f32 as its
// bit pattern, u32, u8. Schema v5 (SNAPSHOT_SCHEMA_AMBIENT) added the EOS /
// CFL / phase fields and the per-particle mass and phase; older versions
// decode with the defaults the reference fills in. The 2D and 3D blocks are
// the same apart from the z components.
//
// Layout written for schema >= 5 (per particle: 2D 21 bytes, 3D 29 bytes):
//   particle_mass rest_density smoothing_length stiffness            4 x f32
//   gamma artificial_viscosity surface_tension cfl                    4 x f32
//   max_substeps u32, adaptive_resolution u8, split f32, merge f32,
//   boundary_particles u8, wall_friction f32,
//   phase count u8 + rest density [4] f32 + mass [4] f32
//     (a single-phase config writes 1, [1.0; 4], [particle_mass; 4])
//   viscosity drag max_velocity particle_radius                       4 x f32
//   enabled u8 (0 / 1; anything else is malformed)
//   count u32, then per particle: x y [z] vx vy [vz] f32, mass f32, phase u8
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/phieng_sph.h"

namespace phieng {
namespace snap {

constexpr uint32_t kSchemaAmbient = 5;   // SNAPSHOT_SCHEMA_AMBIENT (snapshot.rs:112)
constexpr uint32_t kSchemaLatest = 17;   // SNAPSHOT_SCHEMA_VERSION (snapshot.rs:62)

struct Particle {
  float x, y, z, vx, vy, vz, mass;
  uint8_t phase;
};

struct Block {
  FluidConfig2Ffi cfg;  // as apply_fluid2/3 leaves the world's config
  std::vector<Particle> particles;
};

inline void put_u8(std::vector<uint8_t>& o, uint8_t v) { o.push_back(v); }
inline void put_u32(std::vector<uint8_t>& o, uint32_t v) {
  for (int k = 0; k < 4; k++) o.push_back((uint8_t)(v >> (8 * k)));
}
inline void put_f32(std::vector<uint8_t>& o, float v) {
  uint32_t b;
  std::memcpy(&b, &v, 4);
  put_u32(o, b);
}

struct Reader {
  const uint8_t* p;
  uint64_t n, off = 0;
  bool ok = true;
  Reader(const uint8_t* data, uint64_t len) : p(data), n(len) {}
  bool take(uint64_t k) {
    if (!ok || n - off < k) {
      ok = false;
      return false;
    }
    return true;
  }
  uint8_t u8() {
    if (!take(1)) return 0;
    return p[off++];
  }
  uint32_t u32() {
    if (!take(4)) return 0;
    uint32_t v = 0;
    for (int k = 0; k < 4; k++) v |= (uint32_t)p[off + k] << (8 * k);
    off += 4;
    return v;
  }
  float f32() {
    const uint32_t b = u32();
    float v;
    std::memcpy(&v, &b, 4);
    return v;
  }
};

inline void encode(std::vector<uint8_t>& o, const FluidConfig2Ffi& c, const std::vector<Particle>& ps, int dim,
                   uint32_t version) {
  put_f32(o, c.particle_mass);
  put_f32(o, c.rest_density);
  put_f32(o, c.smoothing_length);
  put_f32(o, c.stiffness);
  if (version >= kSchemaAmbient) {
    put_f32(o, c.gamma);
    put_f32(o, c.artificial_viscosity);
    put_f32(o, c.surface_tension);
    put_f32(o, c.cfl);
    put_u32(o, c.max_substeps);
    put_u8(o, c.adaptive_resolution ? 1 : 0);
    put_f32(o, c.split_density_ratio);
    put_f32(o, c.merge_density_ratio);
    put_u8(o, c.boundary_particles ? 1 : 0);
    put_f32(o, c.wall_friction);
    if (c.phase_count > 1) {  // phases_config_2/3: Some only for more than one phase
      put_u8(o, c.phase_count);
      for (int k = 0; k < 4; k++) put_f32(o, c.phase_rest_density[k]);
      for (int k = 0; k < 4; k++) put_f32(o, c.phase_mass[k]);
    } else {
      put_u8(o, 1);
      for (int k = 0; k < 4; k++) put_f32(o, 1.0f);
      for (int k = 0; k < 4; k++) put_f32(o, c.particle_mass);
    }
  }
  put_f32(o, c.viscosity);
  put_f32(o, c.drag);
  put_f32(o, c.max_velocity);
  put_f32(o, c.particle_radius);
  put_u8(o, c.enabled ? 1 : 0);
  put_u32(o, (uint32_t)ps.size());
  for (const Particle& q : ps) {
    put_f32(o, q.x);
    put_f32(o, q.y);
    if (dim == 3) put_f32(o, q.z);
    put_f32(o, q.vx);
    put_f32(o, q.vy);
    if (dim == 3) put_f32(o, q.vz);
    if (version >= kSchemaAmbient) {
      put_f32(o, q.mass);
      put_u8(o, q.phase);
    }
  }
}

// Decode one fluid block and apply the load's rules to it: finite config
// scalars and particle positions / velocities, at most max_particles
// particles, phase count clamped to 1..4 (a single phase resets the phase
// tables to [1.0; 4] / [particle_mass; 4]), particle mass = stored mass if
// positive else max(particle_mass, 0). Returns false on malformed input.
inline bool decode(Reader& r, uint32_t version, int dim, uint64_t max_particles, Block& b) {
  FluidConfig2Ffi& c = b.cfg;
  std::memset(&c, 0, sizeof(c));
  c.particle_mass = r.f32();
  c.rest_density = r.f32();
  c.smoothing_length = r.f32();
  c.stiffness = r.f32();
  uint8_t count = 1;
  float rho4[4] = {1.0f, 1.0f, 1.0f, 1.0f};
  float m4[4] = {c.particle_mass, c.particle_mass, c.particle_mass, c.particle_mass};
  if (version >= kSchemaAmbient) {
    c.gamma = r.f32();
    c.artificial_viscosity = r.f32();
    c.surface_tension = r.f32();
    c.cfl = r.f32();
    c.max_substeps = r.u32();
    c.adaptive_resolution = r.u8() != 0 ? 1 : 0;
    c.split_density_ratio = r.f32();
    c.merge_density_ratio = r.f32();
    c.boundary_particles = r.u8() != 0 ? 1 : 0;
    c.wall_friction = r.f32();
    count = r.u8();
    for (int k = 0; k < 4; k++) rho4[k] = r.f32();
    for (int k = 0; k < 4; k++) m4[k] = r.f32();
  } else {  // pre-v5 defaults (snapshot.rs:712-720, :834-841)
    c.gamma = 1.0f;
    c.max_substeps = 1;
    c.split_density_ratio = 0.5f;
    c.merge_density_ratio = 1.6f;
  }
  c.viscosity = r.f32();
  c.drag = r.f32();
  c.max_velocity = r.f32();
  c.particle_radius = r.f32();
  const uint8_t en = r.u8();
  if (!r.ok || en > 1) return false;
  c.enabled = en;
  if (count > 1) {
    c.phase_count = count > 4 ? 4 : count;
    for (int k = 0; k < 4; k++) {
      c.phase_rest_density[k] = rho4[k];
      c.phase_mass[k] = m4[k];
    }
  } else {
    c.phase_count = 1;
    for (int k = 0; k < 4; k++) {
      c.phase_rest_density[k] = 1.0f;
      c.phase_mass[k] = c.particle_mass;
    }
  }
  const uint32_t n = r.u32();
  if (!r.ok || n > max_particles) return false;
  const float fin[] = {c.particle_mass, c.rest_density, c.smoothing_length, c.stiffness, c.gamma,
                       c.artificial_viscosity, c.surface_tension, c.cfl, c.viscosity, c.drag,
                       c.max_velocity, c.particle_radius};
  for (float v : fin)
    if (!std::isfinite(v)) return false;
  const uint64_t per = (dim == 3 ? 24u : 16u) + (version >= kSchemaAmbient ? 5u : 0u);
  if ((r.n - r.off) / per < n) return false;  // truncated
  b.particles.resize(n);
  const float pm = c.particle_mass > 0.0f ? c.particle_mass : 0.0f;  // max(particle_mass, 0)
  for (uint32_t i = 0; i < n; i++) {
    Particle& q = b.particles[i];
    q.x = r.f32();
    q.y = r.f32();
    q.z = dim == 3 ? r.f32() : 0.0f;
    q.vx = r.f32();
    q.vy = r.f32();
    q.vz = dim == 3 ? r.f32() : 0.0f;
    float m = 0.0f;
    q.phase = 0;
    if (version >= kSchemaAmbient) {
      m = r.f32();
      q.phase = r.u8();
    }
    q.mass = m > 0.0f ? m : pm;
    if (!std::isfinite(q.x) || !std::isfinite(q.y) || !std::isfinite(q.z) || !std::isfinite(q.vx) ||
        !std::isfinite(q.vy) || !std::isfinite(q.vz))
      return false;
  }
  return r.ok;
}

}  // namespace snap
}  // namespace phieng
