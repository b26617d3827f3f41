// ORACLE — TEST INFRASTRUCTURE ONLY (see sph_oracle.hpp).
//
// Flat C API over oracle::Fluid<float> / oracle::Fluid<double> so the Python
// tests, the smoke check and the CPU-baseline leg of the benchmark can drive
// the CPU restatement through ctypes. Nothing in the product library links
// this file.
#include <chrono>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

#include "../include/phieng_sph.h"
#include "sph_oracle.hpp"
#include "sph_oracle3.hpp"

using oracle::Fluid;
using oracle::Fluid3;

namespace {

struct Orc {
  int fp64;
  Fluid<float> f32;
  Fluid<double> f64;
};

struct Orc3 {
  int fp64;
  Fluid3<float> f32;
  Fluid3<double> f64;
};

template <class F>
void apply_config(F& f, const FluidConfig2Ffi* c) {
  auto& d = f.cfg;
  d.particle_mass = c->particle_mass;
  d.rest_density = c->rest_density;
  d.smoothing_length = c->smoothing_length;
  d.stiffness = c->stiffness;
  d.gamma = c->gamma;
  d.artificial_viscosity = c->artificial_viscosity;
  d.surface_tension = c->surface_tension;
  d.cfl = c->cfl;
  d.max_substeps = c->max_substeps;
  d.adaptive_resolution = c->adaptive_resolution != 0;
  d.split_density_ratio = c->split_density_ratio;
  d.merge_density_ratio = c->merge_density_ratio;
  d.boundary_particles = c->boundary_particles != 0;
  d.viscosity = c->viscosity;
  d.drag = c->drag;
  d.wall_friction = c->wall_friction;
  d.phase_count = c->phase_count;
  for (int k = 0; k < 4; k++) {
    d.phase_rest_density[k] = c->phase_rest_density[k];
    d.phase_mass[k] = c->phase_mass[k];
  }
  d.max_velocity = c->max_velocity;
  d.particle_radius = c->particle_radius;
  d.enabled = c->enabled != 0;
}

template <class F>
void read_config(const F& f, FluidConfig2Ffi* c) {
  std::memset(c, 0, sizeof(*c));
  const auto& d = f.cfg;
  c->particle_mass = d.particle_mass;
  c->rest_density = d.rest_density;
  c->smoothing_length = d.smoothing_length;
  c->stiffness = d.stiffness;
  c->gamma = d.gamma;
  c->artificial_viscosity = d.artificial_viscosity;
  c->surface_tension = d.surface_tension;
  c->cfl = d.cfl;
  c->max_substeps = d.max_substeps;
  c->adaptive_resolution = d.adaptive_resolution;
  c->split_density_ratio = d.split_density_ratio;
  c->merge_density_ratio = d.merge_density_ratio;
  c->boundary_particles = d.boundary_particles;
  c->viscosity = d.viscosity;
  c->drag = d.drag;
  c->wall_friction = d.wall_friction;
  c->phase_count = d.phase_count;
  for (int k = 0; k < 4; k++) {
    c->phase_rest_density[k] = d.phase_rest_density[k];
    c->phase_mass[k] = d.phase_mass[k];
  }
  c->max_velocity = d.max_velocity;
  c->particle_radius = d.particle_radius;
  c->enabled = d.enabled;
}

#define DISPATCH(o, expr)     \
  do {                        \
    if ((o)->fp64) {          \
      auto& F = (o)->f64;     \
      expr;                   \
    } else {                  \
      auto& F = (o)->f32;     \
      expr;                   \
    }                         \
  } while (0)

}  // namespace

extern "C" {

void* orc_new(int fp64) {
  Orc* o = new Orc();
  o->fp64 = fp64 ? 1 : 0;
  return o;
}

void orc_free(void* h) { delete static_cast<Orc*>(h); }

void orc_set_config(void* h, const FluidConfig2Ffi* c) {
  Orc* o = static_cast<Orc*>(h);
  DISPATCH(o, apply_config(F, c));
}

void orc_get_config(void* h, FluidConfig2Ffi* c) {
  Orc* o = static_cast<Orc*>(h);
  DISPATCH(o, read_config(F, c));
}

void orc_set_gravity(void* h, float gx, float gy) {
  Orc* o = static_cast<Orc*>(h);
  o->f32.gx = gx;
  o->f32.gy = gy;
  o->f64.gx = (double)gx;
  o->f64.gy = (double)gy;
}

// particle masses by index
uint32_t orc_masses(void* h, float* out, uint32_t max) {
  Orc* o = static_cast<Orc*>(h);
  const auto& ps = o->f32.particles;
  for (uint32_t i = 0; out && i < std::min<size_t>(ps.size(), max); i++) out[i] = ps[i].mass;
  return (uint32_t)ps.size();
}

// the boundary ghosts of the last substep, generation order
uint32_t orc_ghosts(void* h, float* xy, uint32_t max) {
  Orc* o = static_cast<Orc*>(h);
  const auto& g = o->f32.ghosts;
  for (uint32_t i = 0; xy && i < std::min<size_t>(g.size(), max); i++) {
    xy[2 * i] = g[i].x;
    xy[2 * i + 1] = g[i].y;
  }
  return (uint32_t)g.size();
}

// world.ambient.drag.wind (read by the buoyancy drag)
void orc_set_wind(void* h, float wx, float wy) {
  Orc* o = static_cast<Orc*>(h);
  o->f32.wind_x = o->f64.wind_x = wx;
  o->f32.wind_y = o->f64.wind_y = wy;
}

// world.ambient.turbulence (TurbulenceConfig2, ambient.rs:108-126)
void orc_set_turbulence(void* h, int enabled, float amp, float freq, float tscale, uint32_t seed, uint32_t octaves,
                        int divergence_free) {
  Orc* o = static_cast<Orc*>(h);
  oracle::Turbulence t;
  t.on = enabled != 0 && amp > 0.0f;
  t.amp = amp;
  t.freq = freq;
  t.tscale = tscale;
  t.seed = seed;
  t.oct = std::min<uint32_t>(octaves, 255u);
  t.curl = divergence_free != 0;
  o->f32.turb = t;
  o->f64.turb = t;
}

// noise.rs entry points in f32, for the restatement's own tests: kind 0
// value_noise_2(x, y, seed) -> out[0]; 1 fbm_2(x, y, t, seed, octaves) ->
// out[0]; 2 curl_2(x, y, t, seed, octaves) -> out[0..1]
void orc_noise2(int kind, float x, float y, float t, uint32_t seed, uint32_t octaves, float* out) {
  if (kind == 0) {
    out[0] = oracle::nz_value2<float>(x, y, seed);
  } else if (kind == 1) {
    out[0] = oracle::nz_fbm2<float>(x, y, t, seed, std::min<uint32_t>(octaves, 255u));
  } else {
    const uint32_t oct = std::min<uint32_t>(octaves, 255u);
    const float e = 1e-3f, e2 = 2.0f * 1e-3f;  // noise.rs:189-192
    out[0] = (oracle::nz_fbm2<float>(x, y + e, t, seed, oct) - oracle::nz_fbm2<float>(x, y - e, t, seed, oct)) / e2;
    out[1] = -((oracle::nz_fbm2<float>(x + e, y, t, seed, oct) - oracle::nz_fbm2<float>(x - e, y, t, seed, oct)) / e2);
  }
}

// 1 = correctly rounded power (the GPU's), 0 = the platform libm powf
void orc_set_pow_mode(void* h, int mode) {
  Orc* o = static_cast<Orc*>(h);
  o->f32.pow_mode = mode;
  o->f64.pow_mode = mode;
}

void orc_set_cap(void* h, uint32_t cap) {
  Orc* o = static_cast<Orc*>(h);
  o->f32.cap = cap;
  o->f64.cap = cap;
}

// shape 0 = circle (a = radius), 1 = box (a, b = half extents); rotation
// columns x_axis = (xax, xay), y_axis = (yax, yay).
void orc_add_body(void* h, int shape, float px, float py, float a, float b, float xax, float xay,
                  float yax, float yay) {
  Orc* o = static_cast<Orc*>(h);
  oracle::Body bd;
  bd.shape = shape;
  bd.px = px;
  bd.py = py;
  bd.a = a;
  bd.b = b;
  bd.xax = xax;
  bd.xay = xay;
  bd.yax = yax;
  bd.yay = yay;
  o->f32.bodies.push_back(bd);
  o->f64.bodies.push_back(bd);
}

// step_fluid with the caller's bodies in place of the world's (f32 oracle):
// the bodies' velocity state is updated in place (PhiengBody2 layout).
// FluidState2::step_fluid with the caller's bodies; polygon bodies
// (PHIENG_SHAPE_POLYGON) take their local vertices from poly_xy
// [2 * first[k], 2 * (first[k] + count[k])), moved by the body's transform.
void orc_step_fluid_poly(void* h, PhiengBody2* bodies, uint32_t nb, const float* poly_xy, const uint32_t* first,
                         const uint32_t* count, float dt, int mode) {
  Orc* o = static_cast<Orc*>(h);
  std::vector<oracle::Body> keep = o->f32.bodies;
  o->f32.bodies.clear();
  for (uint32_t k = 0; k < nb; k++) {
    const PhiengBody2& q = bodies[k];
    oracle::Body b;
    b.shape = q.shape_tag == PHIENG_SHAPE_CIRCLE ? 0 : q.shape_tag == PHIENG_SHAPE_POLYGON ? 2 : 1;
    if (b.shape == 2)
      for (uint32_t i = first[k]; i < first[k] + count[k]; i++) {
        const float lx = poly_xy[2 * i], ly = poly_xy[2 * i + 1];
        b.poly.push_back((q.xax * lx + q.yax * ly) + q.px);  // rotation * v + position (math.rs:58-60)
        b.poly.push_back((q.xay * lx + q.yay * ly) + q.py);
        b.poly_local.push_back(lx);
        b.poly_local.push_back(ly);
      }
    b.px = q.px;
    b.py = q.py;
    b.xax = q.xax;
    b.xay = q.xay;
    b.yax = q.yax;
    b.yay = q.yay;
    b.a = q.a;
    b.b = q.b;
    b.is_static = q.is_static != 0;
    b.sleeping = q.is_sleeping != 0;
    b.vx = q.vx;
    b.vy = q.vy;
    b.w = q.w;
    b.inv_mass = q.inv_mass;
    b.inv_inertia = q.inv_inertia;
    o->f32.bodies.push_back(b);
  }
  o->f32.step_fluid(dt, (oracle::Mode)mode);
  for (uint32_t k = 0; k < nb; k++) {
    const oracle::Body& b = o->f32.bodies[k];
    bodies[k].vx = b.vx;
    bodies[k].vy = b.vy;
    bodies[k].w = b.w;
    bodies[k].is_sleeping = b.sleeping ? 1 : 0;
  }
  o->f32.bodies = keep;
}

void orc_step_fluid(void* h, PhiengBody2* bodies, uint32_t nb, float dt, int mode) {
  orc_step_fluid_poly(h, bodies, nb, nullptr, nullptr, nullptr, dt, mode);
}

uint32_t orc_add_particles(void* h, const float* xy, const uint8_t* phases, uint32_t n) {
  Orc* o = static_cast<Orc*>(h);
  uint32_t r = 0;
  DISPATCH(o, r = (uint32_t)F.add_particles_phase(xy, phases, n));
  return r;
}

uint32_t orc_count(void* h) {
  Orc* o = static_cast<Orc*>(h);
  uint32_t r = 0;
  DISPATCH(o, r = (uint32_t)F.particles.size());
  return r;
}

void orc_clear(void* h) {
  Orc* o = static_cast<Orc*>(h);
  o->f32.particles.clear();
  o->f64.particles.clear();
}

// position + velocity of the first n particles from quads
void orc_set_state(void* h, const float* xyvv, uint32_t n) {
  Orc* o = static_cast<Orc*>(h);
  DISPATCH(o, {
    for (uint32_t i = 0; i < n && i < F.particles.size(); i++) {
      F.particles[i].x = xyvv[4 * i];
      F.particles[i].y = xyvv[4 * i + 1];
      F.particles[i].vx = xyvv[4 * i + 2];
      F.particles[i].vy = xyvv[4 * i + 3];
    }
  });
}

void orc_set_density_pressure(void* h, const float* d, const float* p, uint32_t n) {
  Orc* o = static_cast<Orc*>(h);
  DISPATCH(o, {
    for (uint32_t i = 0; i < n && i < F.particles.size(); i++) {
      if (d) F.particles[i].density = d[i];
      if (p) F.particles[i].pressure = p[i];
    }
  });
}

uint32_t orc_get_state(void* h, float* out, uint32_t max) {
  Orc* o = static_cast<Orc*>(h);
  uint32_t n = 0;
  DISPATCH(o, {
    n = (uint32_t)std::min<size_t>(max, F.particles.size());
    for (uint32_t i = 0; i < n; i++) {
      out[4 * i] = (float)F.particles[i].x;
      out[4 * i + 1] = (float)F.particles[i].y;
      out[4 * i + 2] = (float)F.particles[i].vx;
      out[4 * i + 3] = (float)F.particles[i].vy;
    }
  });
  return n;
}

uint32_t orc_get_state64(void* h, double* out, uint32_t max) {
  Orc* o = static_cast<Orc*>(h);
  uint32_t n = 0;
  DISPATCH(o, {
    n = (uint32_t)std::min<size_t>(max, F.particles.size());
    for (uint32_t i = 0; i < n; i++) {
      out[4 * i] = (double)F.particles[i].x;
      out[4 * i + 1] = (double)F.particles[i].y;
      out[4 * i + 2] = (double)F.particles[i].vx;
      out[4 * i + 3] = (double)F.particles[i].vy;
    }
  });
  return n;
}

uint32_t orc_get_density_pressure(void* h, float* d, float* p, uint32_t max) {
  Orc* o = static_cast<Orc*>(h);
  uint32_t n = 0;
  DISPATCH(o, {
    n = (uint32_t)std::min<size_t>(max, F.particles.size());
    for (uint32_t i = 0; i < n; i++) {
      if (d) d[i] = (float)F.particles[i].density;
      if (p) p[i] = (float)F.particles[i].pressure;
    }
  });
  return n;
}

uint32_t orc_get_density_pressure64(void* h, double* d, double* p, uint32_t max) {
  Orc* o = static_cast<Orc*>(h);
  uint32_t n = 0;
  DISPATCH(o, {
    n = (uint32_t)std::min<size_t>(max, F.particles.size());
    for (uint32_t i = 0; i < n; i++) {
      if (d) d[i] = (double)F.particles[i].density;
      if (p) p[i] = (double)F.particles[i].pressure;
    }
  });
  return n;
}

// World2::step (world.rs:706-732) with step_fluid (fluid.rs:541-557).
void orc_step(void* h, float dt, int mode) {
  Orc* o = static_cast<Orc*>(h);
  DISPATCH(o, F.world_step(dt, (oracle::Mode)mode));
}

// k world steps; returns wall seconds spent (for the CPU baseline).
double orc_steps(void* h, float dt, int mode, uint32_t k) {
  Orc* o = static_cast<Orc*>(h);
  auto t0 = std::chrono::steady_clock::now();
  for (uint32_t s = 0; s < k; s++) DISPATCH(o, F.world_step(dt, (oracle::Mode)mode));
  auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double>(t1 - t0).count();
}

void orc_substep(void* h, float dt, int mode) {
  Orc* o = static_cast<Orc*>(h);
  DISPATCH(o, F.substep(dt, (oracle::Mode)mode));
}

// Pass-level hooks for "from identical state" parity checks.
void orc_pass_density(void* h) {
  Orc* o = static_cast<Orc*>(h);
  DISPATCH(o, {
    F.rebuild_grid();
    F.compute_density_pressure(oracle::rmax((decltype(F.time))F.cfg.smoothing_length,
                                            (decltype(F.time))oracle::kEps));
  });
}

void orc_pass_forces(void* h) {
  Orc* o = static_cast<Orc*>(h);
  DISPATCH(o, {
    F.rebuild_grid();
    F.compute_forces(oracle::rmax((decltype(F.time))F.cfg.smoothing_length,
                                  (decltype(F.time))oracle::kEps));
  });
}

uint32_t orc_get_forces(void* h, float* fxy, uint32_t max) {
  Orc* o = static_cast<Orc*>(h);
  uint32_t n = 0;
  DISPATCH(o, {
    n = (uint32_t)std::min<size_t>(max, F.fx.size());
    for (uint32_t i = 0; i < n; i++) {
      fxy[2 * i] = (float)F.fx[i];
      fxy[2 * i + 1] = (float)F.fy[i];
    }
  });
  return n;
}

uint32_t orc_get_forces64(void* h, double* fxy, uint32_t max) {
  Orc* o = static_cast<Orc*>(h);
  uint32_t n = 0;
  DISPATCH(o, {
    n = (uint32_t)std::min<size_t>(max, F.fx.size());
    for (uint32_t i = 0; i < n; i++) {
      fxy[2 * i] = (double)F.fx[i];
      fxy[2 * i + 1] = (double)F.fy[i];
    }
  });
  return n;
}

// Neighbour list of particle i in visit order against the current state
// (rebuilds the grid first). Returns the total count (may exceed max).
uint32_t orc_neighbors(void* h, uint32_t i, uint32_t* out, uint32_t max) {
  Orc* o = static_cast<Orc*>(h);
  uint32_t n = 0;
  DISPATCH(o, {
    if (i < F.particles.size()) {
      F.rebuild_grid();
      std::vector<uint32_t> nb;
      F.neighbors_of(F.particles[i].x, F.particles[i].y, F.particles, nb);
      n = (uint32_t)nb.size();
      for (uint32_t k = 0; k < n && k < max; k++) out[k] = nb[k];
    }
  });
  return n;
}

// All neighbour lists at once: counts[i], lists[i*max_per + k].
void orc_all_neighbors(void* h, uint32_t* counts, uint32_t* lists, uint32_t max_per) {
  Orc* o = static_cast<Orc*>(h);
  DISPATCH(o, {
    F.rebuild_grid();
    std::vector<uint32_t> nb;
    for (size_t i = 0; i < F.particles.size(); i++) {
      F.neighbors_of(F.particles[i].x, F.particles[i].y, F.particles, nb);
      counts[i] = (uint32_t)nb.size();
      for (uint32_t k = 0; k < nb.size() && k < max_per; k++) lists[i * max_per + k] = nb[k];
    }
  });
}

// Cell of every particle (cx, cy) as rebuild_grid computes it (fluid.rs:350-356).
void orc_cells(void* h, int32_t* cx, int32_t* cy) {
  Orc* o = static_cast<Orc*>(h);
  DISPATCH(o, {
    for (size_t i = 0; i < F.particles.size(); i++) F.cell_of(F.particles[i].x, F.particles[i].y, cx[i], cy[i]);
  });
}

uint32_t orc_cfl_substeps(void* h, float dt) {
  Orc* o = static_cast<Orc*>(h);
  uint32_t r = 1;
  DISPATCH(o, r = F.cfl_substeps(dt));
  return r;
}

// scalar kernels for the reference's kernel-sanity tests (f32)
// Closure features (16 per particle, insertion order) for a coarse step dt.
uint32_t orc_features(void* h, float dt, float* out, uint32_t max) {
  Orc* o = static_cast<Orc*>(h);
  uint32_t r = 0;
  DISPATCH(o, {
    std::vector<decltype(F.time)> f;
    F.compute_features((decltype(F.time))dt, f);
    r = (uint32_t)std::min<size_t>(max, f.size() / 16);
    for (size_t i = 0; i < 16 * (size_t)r; i++) out[i] = (float)f[i];
  });
  return r;
}

// Extra acceleration per particle (insertion order, [n][2]) for the next
// substep only (the closure's correction).
void orc_set_extra_accel(void* h, const float* a, uint32_t n) {
  Orc* o = static_cast<Orc*>(h);
  DISPATCH(o, {
    F.extra_ax.assign(n, 0);
    F.extra_ay.assign(n, 0);
    for (uint32_t i = 0; i < n; i++) {
      F.extra_ax[i] = a[2 * i];
      F.extra_ay[i] = a[2 * i + 1];
    }
  });
}

float orc_poly6(float r2, float h) { return Fluid<float>::poly6(r2, h); }
void orc_spiky(float rx, float ry, float r, float h, float* out2) {
  Fluid<float>::spiky_grad(rx, ry, r, h, out2[0], out2[1]);
}
float orc_pressure(float d, float rho0, float k, float g) { return Fluid<float>::pressure(d, rho0, k, g, 0); }
float orc_artificial_pressure(float dx, float dy, float vrx, float vry, float r_sq, float h, float rho_bar,
                              float c, float alpha) {
  return Fluid<float>::artificial_pressure(dx, dy, vrx, vry, r_sq, h, rho_bar, c, alpha);
}
float orc_cohesion(float dist, float h) { return Fluid<float>::cohesion(dist, h); }

// ---- 3D (oracle::Fluid3: crates/dynamics/src/fluid3.rs) ----

void* orc3_new(int fp64) {
  Orc3* o = new Orc3();
  o->fp64 = fp64 ? 1 : 0;
  return o;
}

void orc3_free(void* h) { delete static_cast<Orc3*>(h); }

void orc3_set_config(void* h, const FluidConfig2Ffi* c) {
  Orc3* o = static_cast<Orc3*>(h);
  DISPATCH(o, apply_config(F, c));
}

void orc3_set_turbulence(void* h, int enabled, float amp, float freq, float tscale, uint32_t seed, uint32_t octaves,
                         int divergence_free) {
  Orc3* o = static_cast<Orc3*>(h);
  oracle::Turbulence t;
  t.on = enabled != 0 && amp > 0.0f;
  t.amp = amp;
  t.freq = freq;
  t.tscale = tscale;
  t.seed = seed;
  t.oct = std::min<uint32_t>(octaves, 255u);
  t.curl = divergence_free != 0;
  o->f32.turb = t;
  o->f64.turb = t;
}

uint32_t orc3_masses(void* h, float* out, uint32_t max) {
  Orc3* o = static_cast<Orc3*>(h);
  const auto& ps = o->f32.particles;
  for (uint32_t i = 0; out && i < std::min<size_t>(ps.size(), max); i++) out[i] = ps[i].mass;
  return (uint32_t)ps.size();
}

uint32_t orc3_ghosts(void* h, float* xyz, uint32_t max) {
  Orc3* o = static_cast<Orc3*>(h);
  const auto& g = o->f32.ghosts;
  for (uint32_t i = 0; xyz && i < std::min<size_t>(g.size(), max); i++) {
    xyz[3 * i] = g[i].x;
    xyz[3 * i + 1] = g[i].y;
    xyz[3 * i + 2] = g[i].z;
  }
  return (uint32_t)g.size();
}

void orc3_set_gravity(void* h, float gx, float gy, float gz) {
  Orc3* o = static_cast<Orc3*>(h);
  o->f32.gx = gx;
  o->f32.gy = gy;
  o->f32.gz = gz;
  o->f64.gx = (double)gx;
  o->f64.gy = (double)gy;
  o->f64.gz = (double)gz;
}

void orc3_set_pow_mode(void* h, int mode) {
  Orc3* o = static_cast<Orc3*>(h);
  o->f32.pow_mode = mode;
  o->f64.pow_mode = mode;
}

void orc3_set_cap(void* h, uint32_t cap) {
  Orc3* o = static_cast<Orc3*>(h);
  o->f32.cap = cap;
  o->f64.cap = cap;
}

// shape 0 = sphere (a = radius), 1 = box (a, b, c half extents), 2 = capsule
// (a = radius, b = half length along y); identity rotation.
void orc3_add_body(void* h, int shape, float px, float py, float pz, float a, float b, float c) {
  Orc3* o = static_cast<Orc3*>(h);
  oracle::Body3 bd;
  bd.shape = shape;
  bd.px = px;
  bd.py = py;
  bd.pz = pz;
  bd.a = a;
  bd.b = b;
  bd.c = c;
  o->f32.bodies.push_back(bd);
  o->f64.bodies.push_back(bd);
}

uint32_t orc3_add_particles(void* h, const float* xyz, const uint8_t* phases, uint32_t n) {
  Orc3* o = static_cast<Orc3*>(h);
  uint32_t r = 0;
  DISPATCH(o, r = (uint32_t)F.add_particles_phase(xyz, phases, n));
  return r;
}

uint32_t orc3_count(void* h) {
  Orc3* o = static_cast<Orc3*>(h);
  uint32_t r = 0;
  DISPATCH(o, r = (uint32_t)F.particles.size());
  return r;
}

// position + velocity of the first n particles from sextuples
void orc3_set_state(void* h, const float* q, uint32_t n) {
  Orc3* o = static_cast<Orc3*>(h);
  DISPATCH(o, {
    for (uint32_t i = 0; i < n && i < F.particles.size(); i++) {
      F.particles[i].x = q[6 * i];
      F.particles[i].y = q[6 * i + 1];
      F.particles[i].z = q[6 * i + 2];
      F.particles[i].vx = q[6 * i + 3];
      F.particles[i].vy = q[6 * i + 4];
      F.particles[i].vz = q[6 * i + 5];
    }
  });
}

uint32_t orc3_get_state(void* h, float* out, uint32_t max) {
  Orc3* o = static_cast<Orc3*>(h);
  uint32_t n = 0;
  DISPATCH(o, {
    n = (uint32_t)std::min<size_t>(max, F.particles.size());
    for (uint32_t i = 0; i < n; i++) {
      const auto& p = F.particles[i];
      float* r = out + 6 * (size_t)i;
      r[0] = (float)p.x;
      r[1] = (float)p.y;
      r[2] = (float)p.z;
      r[3] = (float)p.vx;
      r[4] = (float)p.vy;
      r[5] = (float)p.vz;
    }
  });
  return n;
}

uint32_t orc3_get_density_pressure(void* h, float* d, float* p, uint32_t max) {
  Orc3* o = static_cast<Orc3*>(h);
  uint32_t n = 0;
  DISPATCH(o, {
    n = (uint32_t)std::min<size_t>(max, F.particles.size());
    for (uint32_t i = 0; i < n; i++) {
      if (d) d[i] = (float)F.particles[i].density;
      if (p) p[i] = (float)F.particles[i].pressure;
    }
  });
  return n;
}

// World3::step's fluid phase (world.rs:2670-2697 with fluid3.rs:591-605).
void orc3_step(void* h, float dt, int mode) {
  Orc3* o = static_cast<Orc3*>(h);
  DISPATCH(o, F.world_step(dt, (oracle::Mode)mode));
}

double orc3_steps(void* h, float dt, int mode, uint32_t k) {
  Orc3* o = static_cast<Orc3*>(h);
  auto t0 = std::chrono::steady_clock::now();
  for (uint32_t s = 0; s < k; s++) DISPATCH(o, F.world_step(dt, (oracle::Mode)mode));
  auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double>(t1 - t0).count();
}

float orc3_time(void* h) {
  Orc3* o = static_cast<Orc3*>(h);
  float t = 0.0f;
  DISPATCH(o, t = (float)F.time);
  return t;
}

// Density pass, then (forces != 0) the force pass, on the current state.
void orc3_passes(void* h, int forces) {
  Orc3* o = static_cast<Orc3*>(h);
  DISPATCH(o, {
    using R = decltype(F.time);
    const R hk = oracle::rmax((R)F.cfg.smoothing_length, (R)oracle::kEps);
    F.rebuild_grid();
    F.compute_density_pressure(hk);
    if (forces) F.compute_forces(hk);
  });
}

uint32_t orc3_get_forces(void* h, float* fxyz, uint32_t max) {
  Orc3* o = static_cast<Orc3*>(h);
  uint32_t n = 0;
  DISPATCH(o, {
    n = (uint32_t)std::min<size_t>(max, F.fx.size());
    for (uint32_t i = 0; i < n; i++) {
      fxyz[3 * i] = (float)F.fx[i];
      fxyz[3 * i + 1] = (float)F.fy[i];
      fxyz[3 * i + 2] = (float)F.fz[i];
    }
  });
  return n;
}

// Neighbour list of particle i in visit order (rebuilds the grid first).
uint32_t orc3_neighbors(void* h, uint32_t i, uint32_t* out, uint32_t max) {
  Orc3* o = static_cast<Orc3*>(h);
  uint32_t n = 0;
  DISPATCH(o, {
    if (i < F.particles.size()) {
      F.rebuild_grid();
      std::vector<uint32_t> nb;
      const auto& p = F.particles[i];
      F.neighbors_of(p.x, p.y, p.z, F.particles, nb);
      n = (uint32_t)nb.size();
      for (uint32_t k = 0; k < n && k < max; k++) out[k] = nb[k];
    }
  });
  return n;
}

uint32_t orc3_cfl_substeps(void* h, float dt) {
  Orc3* o = static_cast<Orc3*>(h);
  uint32_t r = 1;
  DISPATCH(o, r = F.cfl_substeps(dt));
  return r;
}

// Particle vs one static body (fluid3.rs:471-590); returns 1 on contact.
int orc3_collide(int shape, float a, float b, float c, float px, float py, float pz, float pr, float* out4) {
  oracle::Body3 bd;
  bd.shape = shape;
  bd.a = a;
  bd.b = b;
  bd.c = c;
  float nx = 0, ny = 0, nz = 0, depth = 0;
  const bool hit = Fluid3<float>::collide(px, py, pz, pr, bd, nx, ny, nz, depth);
  out4[0] = nx;
  out4[1] = ny;
  out4[2] = nz;
  out4[3] = depth;
  return hit ? 1 : 0;
}

// FluidState3::step_fluid with the caller's bodies (PhiengBody3 layout), in
// place of the world's statics; vx .. wz and is_sleeping are updated in
// place. Hull bodies (PHIENG_SHAPE3_HULL) take their local vertices from
// hull_xyz [3 * first[k], 3 * (first[k] + count[k])), moved by the body's
// transform (rotation * v + position, math.rs:94-96).
void orc3_step_fluid(void* h, PhiengBody3* bodies, uint32_t nb, const float* hull_xyz, const uint32_t* first,
                     const uint32_t* count, float dt, int mode) {
  Orc3* o = static_cast<Orc3*>(h);
  std::vector<oracle::Body3> keep = o->f32.bodies;
  o->f32.bodies.clear();
  for (uint32_t k = 0; k < nb; k++) {
    const PhiengBody3& q = bodies[k];
    oracle::Body3 b;
    b.shape = (int)q.shape_tag;
    b.px = q.px, b.py = q.py, b.pz = q.pz;
    b.a = q.a, b.b = q.b, b.c = q.c;
    b.rotated = true;
    b.qx = q.qx, b.qy = q.qy, b.qz = q.qz, b.qw = q.qw;
    b.is_static = q.is_static != 0;
    b.sleeping = q.is_sleeping != 0;
    b.vx = q.vx, b.vy = q.vy, b.vz = q.vz;
    b.wx = q.wx, b.wy = q.wy, b.wz = q.wz;
    b.inv_mass = q.inv_mass;
    for (int i = 0; i < 9; i++) b.inv_inertia[i] = q.inv_inertia[i];
    if (b.shape == 3)
      for (uint32_t i = first[k]; i < first[k] + count[k]; i++) {
        float x, y, z;
        oracle::qrot(q.qx, q.qy, q.qz, q.qw, hull_xyz[3 * i], hull_xyz[3 * i + 1], hull_xyz[3 * i + 2], x, y, z);
        b.hull.push_back(x + q.px);
        b.hull.push_back(y + q.py);
        b.hull.push_back(z + q.pz);
      }
    o->f32.bodies.push_back(b);
  }
  o->f32.step_fluid(dt, (oracle::Mode)mode);
  for (uint32_t k = 0; k < nb; k++) {
    const oracle::Body3& b = o->f32.bodies[k];
    bodies[k].vx = b.vx, bodies[k].vy = b.vy, bodies[k].vz = b.vz;
    bodies[k].wx = b.wx, bodies[k].wy = b.wy, bodies[k].wz = b.wz;
    bodies[k].is_sleeping = b.sleeping ? 1 : 0;
  }
  o->f32.bodies = keep;
}

void orc3_set_wind(void* h, float x, float y, float z) {
  Orc3* o = static_cast<Orc3*>(h);
  o->f32.wind_x = o->f64.wind_x = x;
  o->f32.wind_y = o->f64.wind_y = y;
  o->f32.wind_z = o->f64.wind_z = z;
}

// Rotation of a vector by a quaternion, the world inverse inertia and the
// buoyancy samples of one body, as the fluid phase computes them.
void orc3_qrot(float qx, float qy, float qz, float qw, const float* v, float* out) {
  oracle::qrot(qx, qy, qz, qw, v[0], v[1], v[2], out[0], out[1], out[2]);
}
void orc3_world_inv_inertia(float qx, float qy, float qz, float qw, const float* inv_i, float* out) {
  oracle::world_inv_inertia(qx, qy, qz, qw, inv_i, out);
}
uint32_t orc3_surface_samples(const PhiengBody3* q, float* out, uint32_t max) {
  oracle::Body3 b;
  b.shape = (int)q->shape_tag;
  b.px = q->px, b.py = q->py, b.pz = q->pz;
  b.a = q->a, b.b = q->b, b.c = q->c;
  b.qx = q->qx, b.qy = q->qy, b.qz = q->qz, b.qw = q->qw;
  std::vector<float> s;
  oracle::surface_samples3(b, s);
  for (size_t i = 0; out && i < std::min<size_t>(s.size(), 7 * (size_t)max); i++) out[i] = s[i];
  return (uint32_t)(s.size() / 7);
}

float orc3_poly6(float r2, float h) { return Fluid3<float>::poly6(r2, h); }
void orc3_spiky(float rx, float ry, float rz, float r, float h, float* out3) {
  Fluid3<float>::spiky_grad(rx, ry, rz, r, h, out3[0], out3[1], out3[2]);
}

}  // extern "C"
