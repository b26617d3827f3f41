// ORACLE — TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the reference 2D SPH fluid step (PhiEng
// `crates/dynamics/src/fluid.rs`, `FluidState2::step_fluid` -> `substep`).
// It is the numeric ground truth for the CUDA path: only the tests, the
// smoke check and the CPU-baseline leg of the benchmark may link it. The
// product library never calls into this file.
//
// Parity status: the reference's Rust step cannot be compiled in this
// environment (no cargo/rustc) and its own tests pin no numeric results of
// the SPH step, so this restatement is pinned by (a) the reference's
// behavioural tests re-run on it (tests/test_behaviour.py), (b) the one
// bit-pinned arithmetic identity of the reference (linear EOS,
// fluid.rs:1326-1329), (c) an FP64 twin that bounds its f32 error, and
// (d) a second restatement written from the reference's C# solver
// (oracle/fluid_cs.py, src/PhiEng.Dynamics/FluidSolver.cs), which this one
// matches bit for bit on the scene of the reference's own C#-vs-Rust
// equivalence test (tests/PhiEng.Tests/EquivalenceTests.cs:122-176;
// tests/test_oracle_pin.py).
//
// Arithmetic contract: every expression keeps the reference's evaluation
// order (glam 0.29 Vec2 ops are component-wise IEEE f32; Rust never
// contracts a*b+c into an FMA). Build with -ffp-contract=off and without
// -ffast-math. `powf` is the platform libm one, as Rust's `f32::powf` is.
//
// Two integrate modes:
//   REF_SEQ  the reference's in-place Gauss-Seidel sweep (fluid.rs:1003-1050:
//            particle i reads the already-advected state of every j < i);
//   JACOBI   every read comes from the pre-integrate state (what a parallel
//            GPU integrate computes; the CUDA path is bit-exact to this).
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <unordered_map>
#include <vector>

namespace oracle {

enum Mode { REF_SEQ = 0, JACOBI = 1 };

// crates/math/src/math.rs:3-4
constexpr float kEps = 1e-6f;
constexpr float kEpsSq = 1e-12f;

// FluidConfig2 (fluid.rs:54-140) with its Default (fluid.rs:142-169).
struct Config {
  float particle_mass = 0.0625f;
  float rest_density = 1.0f;
  float smoothing_length = 0.5f;
  float stiffness = 100.0f;
  float gamma = 1.0f;
  float artificial_viscosity = 0.0f;
  float surface_tension = 0.0f;
  float cfl = 0.0f;
  uint32_t max_substeps = 1;
  bool adaptive_resolution = false;
  float split_density_ratio = 0.5f;
  float merge_density_ratio = 1.6f;
  bool boundary_particles = false;
  float viscosity = 0.3f;
  float drag = 4.0f;
  float wall_friction = 0.0f;
  uint8_t phase_count = 1;
  float phase_rest_density[4] = {1.0f, 1.0f, 1.0f, 1.0f};
  float phase_mass[4] = {0.0625f, 0.0625f, 0.0625f, 0.0625f};
  float max_velocity = 30.0f;
  float particle_radius = 0.125f;
  bool enabled = true;
};

// A static rigid body as the fluid sees it (body.rs:573-607): a circle or a
// box with a Transform2 (math.rs:34-60: position + glam Mat2 columns).
struct Body {
  int shape = 1;  // 0 = circle (a = radius), 1 = box (a, b = half extents), 2 = polygon
  std::vector<float> poly;  // polygon: world-space vertices x0, y0, x1, y1, ... (transform_point of the local ones)
  std::vector<float> poly_local;  // polygon: the body-frame vertices (boundary ghosts sample these)
  float px = 0, py = 0;
  float xax = 1, xay = 0, yax = 0, yay = 1;  // rotation columns x_axis, y_axis
  float a = 0, b = 0;
  // RigidBody2 velocity state (body.rs:560-700): statics take no reaction
  bool is_static = true, sleeping = false;
  float vx = 0, vy = 0, w = 0, inv_mass = 0, inv_inertia = 0;

  // apply_impulse (body.rs:675-687)
  void apply_impulse(float jx, float jy, float qx, float qy) {
    if (is_static) return;
    sleeping = false;
    vx = vx + jx * inv_mass;
    vy = vy + jy * inv_mass;
    float rx = qx - px, ry = qy - py;
    float torque = rx * jy - ry * jx;
    w = w + torque * inv_inertia;
  }
  // apply_force (body.rs:657-673)
  void apply_force(float fx, float fy, float qx, float qy, float dt) {
    if (is_static) return;
    sleeping = false;
    vx = vx + fx * inv_mass * dt;
    vy = vy + fy * inv_mass * dt;
    float rx = qx - px, ry = qy - py;
    float torque = rx * fy - ry * fx;
    w = w + torque * inv_inertia * dt;
  }
};

template <class R>
struct Particle {
  R x, y, vx, vy;
  R density, pressure, mass;
  uint8_t phase;
};

template <class R>
struct Consts;
template <>
struct Consts<float> {
  // std::f32::consts::PI
  static float pi() { return 3.14159265358979323846f; }
};
template <>
struct Consts<double> {
  static double pi() { return 3.14159265358979323846; }
};

// `f32 as i32` / `f64 as i32`: saturating, NaN -> 0 (Rust semantics).
template <class R>
inline int32_t sat_i32(R v) {
  if (v != v) return 0;
  if (v >= (R)2147483648.0) return INT32_MAX;
  if (v <= (R)-2147483648.0) return INT32_MIN;
  return (int32_t)v;
}

template <class R>
inline bool finite(R v) {
  return std::isfinite(v);
}

// Rust f32::max / f32::min ignore a NaN operand.
template <class R>
inline R rmax(R a, R b) {
  if (a != a) return b;
  if (b != b) return a;
  return a > b ? a : b;
}
// Rust f32::clamp (NaN passes through).
template <class R>
inline R rclamp(R x, R lo, R hi) {
  if (x < lo) x = lo;
  if (x > hi) x = hi;
  return x;
}

// x^g for the Tait EOS (fluid.rs:295: `(density / rho0).powf(gamma)`).
// pow_mode 1 (default): the correctly rounded f32 power, evaluated in double
//   (binary exponentiation for an integer g in [1, 64], else double pow) and
//   rounded once; this is the GPU's arithmetic.
// pow_mode 0: the platform libm powf, which Rust's f32::powf calls; glibc's
//   powf is off by one ulp from the correctly rounded result on ~0.07% of
//   inputs in [0.5, 3) for g = 7.
inline float powf_cr(float x, float g) {
  if (g >= 1.0f && g <= 64.0f && g == std::floor(g)) {
    unsigned e = (unsigned)g;
    double b = (double)x, r = 1.0;
    while (e) {
      if (e & 1u) r = r * b;
      e >>= 1;
      if (e) b = b * b;
    }
    return (float)r;
  }
  return (float)pow((double)x, (double)g);
}

template <class R>
inline R rpow(R a, R b, int mode);
template <>
inline float rpow<float>(float a, float b, int mode) {
  return mode == 0 ? powf(a, b) : powf_cr(a, b);
}
template <>
inline double rpow<double>(double a, double b, int) {
  return pow(a, b);
}

// ---- ambient turbulence (crates/dynamics/src/noise.rs, fluid.rs:1001-1019) ----
struct Turbulence {
  bool on = false;  // enabled && amplitude > 0 (fluid.rs:1002)
  float amp = 0, freq = 1, tscale = 1;
  uint32_t seed = 0, oct = 3;  // octaves as stored (u8); clamped to 1..8 where used
  bool curl = false;
};

// integer avalanche hash (noise.rs:27-35)
inline uint32_t nz_hash(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

// Rust's `f as i32` / `f as i64`: truncate, saturate, NaN -> 0
template <class I, class R>
inline I rust_as_int(R v) {
  if (v != v) return 0;
  const R lo = (R)std::numeric_limits<I>::min(), hi = (R)std::numeric_limits<I>::max();
  if (v <= lo) return std::numeric_limits<I>::min();
  if (v >= hi) return std::numeric_limits<I>::max();
  return (I)v;
}

template <class R>
inline R nz_lattice(int32_t ix, int32_t iy, uint32_t seed) {  // noise.rs:38-47
  const uint32_t h = nz_hash((uint32_t)ix * 0x1f1f1f1fu + (uint32_t)iy * 0x9e3779b9u + seed);
  return (R)(h >> 8) * (R)(1.0f / 16777216.0f);
}

template <class R>
inline R nz_fade(R t) {  // noise.rs:64-67
  return t * t * t * (t * (t * (R)6 - (R)15) + (R)10);
}

template <class R>
inline R nz_lerp(R a, R b, R t) {
  return a + (b - a) * t;
}

template <class R>
inline R nz_value2(R x, R y, uint32_t seed) {  // noise.rs:75-87
  const R x0 = std::floor(x), y0 = std::floor(y);
  const int32_t xi = rust_as_int<int32_t>(x0), yi = rust_as_int<int32_t>(y0);
  const R tx = nz_fade(x - x0), ty = nz_fade(y - y0);
  const int32_t xi1 = (int32_t)((uint32_t)xi + 1u), yi1 = (int32_t)((uint32_t)yi + 1u);
  const R v00 = nz_lattice<R>(xi, yi, seed), v10 = nz_lattice<R>(xi1, yi, seed);
  const R v01 = nz_lattice<R>(xi, yi1, seed), v11 = nz_lattice<R>(xi1, yi1, seed);
  return nz_lerp(nz_lerp(v00, v10, tx), nz_lerp(v01, v11, tx), ty);
}

template <class R>
inline R nz_fbm2_static(R x, R y, uint32_t seed, uint32_t oct) {  // noise.rs:115-132
  R sum = 0, amp = 1, freq = 1, norm = 0;
  for (uint32_t o = 0; o < oct; o++) {
    sum += amp * (nz_value2(x * freq, y * freq, seed + o) * (R)2 - (R)1);
    norm += amp;
    amp *= (R)0.5;
    freq *= (R)2;
  }
  return norm > (R)0 ? sum / norm : (R)0;
}

template <class R>
inline R nz_fbm2(R x, R y, R t, uint32_t seed, uint32_t octaves) {  // noise.rs:160-170
  const uint32_t oct = std::min<uint32_t>(std::max<uint32_t>(octaves, 1u), 8u);
  const R t0 = std::floor(t);
  const R ft = nz_fade(t - t0);
  const int64_t sl = rust_as_int<int64_t>(t0);
  const uint32_t s0 = seed + (uint32_t)sl * 0x9e3779b9u;
  const uint32_t s1 = seed + (uint32_t)((uint64_t)sl + 1u) * 0x9e3779b9u;
  return nz_lerp(nz_fbm2_static(x, y, s0, oct), nz_fbm2_static(x, y, s1, oct), ft);
}

// acceleration added at (px, py) and clock `time` (fluid.rs:1007-1018);
// clamp_length_max(1.0) as glam 0.29 (v / sqrt(|v|^2) when |v|^2 > 1)
template <class R>
inline void turbulence_accel(const Turbulence& tb, R px, R py, R time, R& ax, R& ay) {
  const R x = px * (R)tb.freq, y = py * (R)tb.freq;
  const R t = time * (R)tb.tscale;
  R nx, ny;
  if (tb.curl) {  // noise.rs:186-193
    const R e = (R)1e-3f, e2 = (R)(2.0f * 1e-3f);
    const R dpdy = (nz_fbm2(x, y + e, t, tb.seed, tb.oct) - nz_fbm2(x, y - e, t, tb.seed, tb.oct)) / e2;
    const R dpdx = (nz_fbm2(x + e, y, t, tb.seed, tb.oct) - nz_fbm2(x - e, y, t, tb.seed, tb.oct)) / e2;
    nx = dpdy;
    ny = -dpdx;
  } else {
    nx = nz_fbm2(x, y, t, tb.seed, tb.oct);
    ny = nz_fbm2(x, y, t, tb.seed ^ 0x55aa55aau, tb.oct);
  }
  const R ls = nx * nx + ny * ny;
  if (ls > (R)1) {
    const R l = std::sqrt(ls);
    nx = nx / l;
    ny = ny / l;
  }
  ax = ax + nx * (R)tb.amp;
  ay = ay + ny * (R)tb.amp;
}

template <class R>
class Fluid {
 public:
  Config cfg;
  std::vector<Particle<R>> particles;
  std::vector<Body> bodies;
  R gx = (R)0.0f, gy = (R)-9.81f;  // World2::new gravity (world.rs:338)
  R time = 0;
  Turbulence turb;    // world.ambient.turbulence
  float wind_x = 0, wind_y = 0;  // world.ambient.drag.wind
  size_t cap = 4096;  // MAX_PARTICLES_2D (fluid.rs:30); lifted by the caller
  int pow_mode = 1;   // see powf_cr

  // last-substep scratch exposed for per-pass parity dumps
  std::vector<R> fx, fy;
  // per-particle acceleration added in the integrate (the learned closure's
  // correction; empty = none), consumed by the next substep
  std::vector<R> extra_ax, extra_ay;

  // ---- kernels (fluid.rs:265-326) ----
  // poly6: 4/(pi h^8)(h^2-r^2)^3, zero beyond h (fluid.rs:265-273)
  static R poly6(R r2, R h) {
    if (r2 >= h * h || r2 < (R)0) return (R)0;
    R h2 = h * h;
    R t = h2 - r2;
    return (R)4.0 / (Consts<R>::pi() * h2 * h2 * h2 * h2) * t * t * t;
  }
  // spiky gradient (fluid.rs:278-285)
  static void spiky_grad(R rx, R ry, R r, R h, R& gxo, R& gyo) {
    if (r >= h || r < (R)kEps) {
      gxo = 0;
      gyo = 0;
      return;
    }
    R s = (R)-30.0 / (Consts<R>::pi() * h * h * h * h * h) * (h - r) * (h - r);
    gxo = rx / r * s;
    gyo = ry / r * s;
  }
  // equation of state (fluid.rs:290-297)
  static R pressure(R density, R rest_density, R stiffness, R gamma, int pow_mode = 1) {
    if (gamma == (R)1.0) {
      return rmax(stiffness * (density - rest_density), (R)0);
    }
    R rho0 = rmax(rest_density, (R)kEps);
    return rmax(stiffness * rho0 * (rpow(density / rho0, gamma, pow_mode) - (R)1.0), (R)0);
  }
  // Monaghan artificial viscosity (fluid.rs:302-317)
  static R artificial_pressure(R dx, R dy, R vrx, R vry, R r_sq, R h, R rho_bar, R c, R alpha) {
    R vd = vrx * dx + vry * dy;
    if (vd >= (R)0) return (R)0;
    R mu = h * vd / (r_sq + (R)0.01f * h * h);
    return -alpha * c * mu / rmax(rho_bar, (R)kEps);
  }
  // cohesion (fluid.rs:320-326)
  static R cohesion(R dist, R h) { return dist >= h ? (R)0 : (R)1.0 - dist / h; }

  // ---- insert (fluid.rs:232-257) ----
  size_t add_particles_phase(const float* xy, const uint8_t* ph, size_t n_in) {
    size_t room = cap > particles.size() ? cap - particles.size() : 0;
    size_t n = std::min(room, n_in);
    for (size_t i = 0; i < n; i++) {
      uint8_t p = ph ? ph[i] : 0;
      size_t k = std::min<size_t>(p, 3);
      Particle<R> q;
      q.x = (R)xy[2 * i];
      q.y = (R)xy[2 * i + 1];
      q.vx = 0;
      q.vy = 0;
      q.density = (R)cfg.phase_rest_density[k];
      q.pressure = 0;
      q.mass = rmax((R)cfg.phase_mass[k], (R)0);
      q.phase = p;
      particles.push_back(q);
    }
    return n;
  }

  // ---- adaptive resolution: FluidState2::resample (fluid.rs:826-893) ----
  void resample(R h) {
    const float rest = std::max(cfg.rest_density, kEps);
    const R split_lo = (R)(cfg.split_density_ratio * rest);
    const R merge_hi = (R)(cfg.merge_density_ratio * rest);
    const R min_mass = (R)(std::max(cfg.particle_mass, kEps) * 0.125f);
    const size_t n = particles.size();
    std::vector<char> absorbed(n, 0);
    const R md = (R)0.25 * h;
    const R merge_d2 = md * md;
    for (size_t i = 0; i < n; i++) {
      if (absorbed[i] || particles[i].density <= merge_hi) continue;
      for (size_t j = i; j-- > 0;) {  // j = i - 1 down to 0
        if (absorbed[j] || particles[j].density <= merge_hi) continue;
        const R dx = particles[i].x - particles[j].x, dy = particles[i].y - particles[j].y;
        if (dx * dx + dy * dy < merge_d2) {
          const R mi = particles[i].mass, mj = particles[j].mass;
          const R mt = mi + mj;
          if (mt > (R)kEps) {
            particles[i].vx = (particles[i].vx * mi + particles[j].vx * mj) / mt;
            particles[i].vy = (particles[i].vy * mi + particles[j].vy * mj) / mt;
            particles[i].mass = mt;
          }
          absorbed[j] = 1;
          break;
        }
      }
    }
    std::vector<Particle<R>> out;
    out.reserve(n);
    const R off = (R)0.25 * h;
    for (size_t i = 0; i < n; i++) {
      if (absorbed[i]) continue;
      const Particle<R>& p = particles[i];
      if (p.density < split_lo && p.mass > min_mass && out.size() + 1 < 4096) {  // MAX_PARTICLES_2D
        Particle<R> a = p, b = p;
        a.mass = b.mass = p.mass * (R)0.5;
        a.x = p.x + off;
        a.y = p.y + (R)0;
        b.x = p.x - off;
        b.y = p.y - (R)0;
        out.push_back(a);
        out.push_back(b);
      } else {
        out.push_back(p);
      }
    }
    particles.swap(out);
  }

  // ---- boundary ghosts (fluid.rs:617-818) ----
  struct Ghost {
    float x, y;
    R density, pressure;
  };
  std::vector<Ghost> ghosts;
  std::unordered_map<uint64_t, std::vector<uint32_t>> ghost_grid;

  // refresh_boundaries (fluid.rs:665-741) + rebuild_boundary_grid
  // (fluid.rs:744-756) from the static bodies, in f32 as the reference. Its
  // output is a function of the bodies and the config only, so regenerating
  // every substep gives what the reference's fingerprint-triggered refresh
  // keeps.
  void refresh_ghosts() {
    ghosts.clear();
    ghost_grid.clear();
    const float hk = std::max(cfg.smoothing_length, kEps);
    const float spacing = std::max(hk * 0.5f, kEps);
    const float pi = Consts<float>::pi();
    auto cnt = [](float v) -> uint64_t {  // `as usize`, at least 1
      uint64_t n = (v > 0.0f) ? (v >= 1.8446744e19f ? UINT64_MAX : (uint64_t)v) : 0;
      return std::max<uint64_t>(n, 1);
    };
    for (const Body& b : bodies) {
      if (!b.is_static) continue;
      auto put = [&](float lx, float ly) {
        ghosts.push_back({(b.xax * lx + b.yax * ly) + b.px, (b.xay * lx + b.yay * ly) + b.py, 0, 0});
      };
      if (b.shape == 0) {
        const uint64_t n = cnt(std::ceil((2.0f * pi * b.a) / spacing));
        for (uint64_t k = 0; k < n; k++) {
          const float a = 2.0f * pi * (float)k / (float)n;
          put(std::cos(a) * b.a, std::sin(a) * b.a);
        }
      } else if (b.shape == 1) {
        const float hx = b.a, hy = b.b;
        // fluid.rs:686-691: (origin, tangent) per edge, in this order
        const float o[4][2] = {{-hx, -hy}, {-hx, hy}, {-hx, -hy}, {hx, -hy}};
        const float tg[4][2] = {{0, 1}, {0, 1}, {1, 0}, {1, 0}};
        for (int e = 0; e < 4; e++) {
          const float ext = (tg[e][0] == 1.0f) ? hx : hy;
          const uint64_t n = cnt(std::ceil((2.0f * ext) / spacing));
          for (uint64_t k = 0; k < n; k++) {
            const float t = ((float)k + 0.5f) / (float)n;
            const float sc = 2.0f * ext * t;
            put(o[e][0] + tg[e][0] * sc, o[e][1] + tg[e][1] * sc);
          }
        }
      } else {
        const size_t nv = b.poly_local.size() / 2;
        for (size_t e = 0; e < nv; e++) {
          const size_t f = (e + 1) % nv;
          const float ax = b.poly_local[2 * e], ay = b.poly_local[2 * e + 1];
          const float ex = b.poly_local[2 * f] - ax, ey = b.poly_local[2 * f + 1] - ay;
          const float len = std::sqrt(ex * ex + ey * ey);
          if (len < kEps) continue;
          const uint64_t n = cnt(std::ceil(len / spacing));
          for (uint64_t k = 0; k < n; k++) {
            const float t = ((float)k + 0.5f) / (float)n;
            put(ax + ex * t, ay + ey * t);
          }
        }
      }
    }
    for (uint32_t i = 0; i < ghosts.size(); i++) {
      const Ghost& g = ghosts[i];
      if (!std::isfinite(g.x) || !std::isfinite(g.y)) continue;
      ghost_grid[cell_key(sat_i32(std::floor(g.x / hk)), sat_i32(std::floor(g.y / hk)))].push_back(i);
    }
  }

  // compute_boundary_density_pressure (fluid.rs:804-818)
  void ghost_density(R h) {
    std::vector<uint32_t> nb;
    for (Ghost& g : ghosts) {
      neighbors_of((R)g.x, (R)g.y, particles, nb);
      R rho = 0;
      for (uint32_t j : nb) {
        const R dx = particles[j].x - (R)g.x, dy = particles[j].y - (R)g.y;
        rho += particles[j].mass * poly6(dx * dx + dy * dy, h);
      }
      g.density = rclamp(rho, (R)0, (R)3 * rmax((R)cfg.rest_density, (R)kEps));
      g.pressure = pressure(rho, (R)cfg.rest_density, (R)cfg.stiffness, (R)cfg.gamma, pow_mode);
    }
  }

  // ghost pressure on a fluid particle (fluid.rs:977-988), after its fluid
  // pairs: boundary_near's cells and filter, -grad W * (m_g (q_i + q_g))
  void ghost_pressure_force(R px, R py, R q_i, R h, R& fxi, R& fyi) const {
    const R hg = (R)cfg.smoothing_length;
    const R m = (R)std::max(cfg.particle_mass, kEps);
    int32_t cx, cy;
    cell_of(px, py, cx, cy);
    for (int oy = -1; oy <= 1; oy++) {
      for (int ox = -1; ox <= 1; ox++) {
        auto it = ghost_grid.find(cell_key((int32_t)((uint32_t)cx + (uint32_t)ox), (int32_t)((uint32_t)cy + (uint32_t)oy)));
        if (it == ghost_grid.end()) continue;
        for (uint32_t k : it->second) {
          const Ghost& g = ghosts[k];
          const R ex = (R)g.x - px, ey = (R)g.y - py;
          if (!(ex * ex + ey * ey < hg * hg)) continue;
          const R dx = px - (R)g.x, dy = py - (R)g.y;
          const R dist = std::sqrt(dx * dx + dy * dy);
          R gx, gy;
          spiky_grad(dx, dy, dist, h, gx, gy);
          const R rb = rmax(g.density, (R)kEps);
          const R s = m * (q_i + g.pressure / (rb * rb));
          fxi -= gx * s;
          fyi -= gy * s;
        }
      }
    }
  }

  // ---- grid (fluid.rs:330-386) ----
  static uint64_t cell_key(int32_t cx, int32_t cy) {
    return ((uint64_t)(uint32_t)cx << 32) | (uint64_t)(uint32_t)cy;
  }
  std::unordered_map<uint64_t, std::vector<uint32_t>> grid;

  void cell_of(R x, R y, int32_t& cx, int32_t& cy) const {
    R hg = (R)cfg.smoothing_length;  // rebuild_grid / neighbors use the raw h
    cx = sat_i32(std::floor(x / hg));
    cy = sat_i32(std::floor(y / hg));
  }

  void rebuild_grid() {
    for (auto& kv : grid) kv.second.clear();
    for (size_t i = 0; i < particles.size(); i++) {
      const auto& p = particles[i];
      if (!finite(p.x) || !finite(p.y)) continue;
      int32_t cx, cy;
      cell_of(p.x, p.y, cx, cy);
      grid[cell_key(cx, cy)].push_back((uint32_t)i);
    }
  }

  // neighbours of the point (px, py) against the positions in `ps`
  // (fluid.rs:368-386): oy outer, ox inner, in-cell ids ascending, kept
  // when |x_j - x|^2 < h*h. Cells beyond the i32 range cannot exist.
  void neighbors_of(R px, R py, const std::vector<Particle<R>>& ps, std::vector<uint32_t>& out) const {
    out.clear();
    R hg = (R)cfg.smoothing_length;
    int32_t cx, cy;
    cell_of(px, py, cx, cy);
    for (int oy = -1; oy <= 1; oy++) {
      int64_t yy = (int64_t)cy + oy;
      if (yy < INT32_MIN || yy > INT32_MAX) continue;
      for (int ox = -1; ox <= 1; ox++) {
        int64_t xx = (int64_t)cx + ox;
        if (xx < INT32_MIN || xx > INT32_MAX) continue;
        auto it = grid.find(cell_key((int32_t)xx, (int32_t)yy));
        if (it == grid.end()) continue;
        for (uint32_t j : it->second) {
          R dx = ps[j].x - px;
          R dy = ps[j].y - py;
          R d2 = dx * dx + dy * dy;
          if (d2 < hg * hg) out.push_back(j);
        }
      }
    }
  }

  // ---- density + pressure (fluid.rs:592-611) ----
  void compute_density_pressure(R h) {
    std::vector<uint32_t> nb;
    R rho_cap = (R)3.0 * rmax((R)cfg.rest_density, (R)kEps);
    for (size_t i = 0; i < particles.size(); i++) {
      neighbors_of(particles[i].x, particles[i].y, particles, nb);
      R pix = particles[i].x, piy = particles[i].y;
      R rho = 0;
      for (uint32_t j : nb) {
        R dx = particles[j].x - pix;
        R dy = particles[j].y - piy;
        R r2 = dx * dx + dy * dy;
        rho += particles[j].mass * poly6(r2, h);
      }
      particles[i].density = rclamp(rho, (R)0, rho_cap);
    }
    for (auto& p : particles) {
      R rho0 = (R)cfg.phase_rest_density[std::min<int>(p.phase, 3)];
      p.pressure = pressure(p.density, rho0, (R)cfg.stiffness, (R)cfg.gamma, pow_mode);
    }
  }

  // ---- pressure force (+AV, cohesion) (fluid.rs:942-997) ----
  void compute_forces(R h) {
    std::vector<uint32_t> nb;
    size_t n = particles.size();
    fx.assign(n, (R)0);
    fy.assign(n, (R)0);
    R c_s = std::sqrt(rmax((R)cfg.stiffness, (R)0));
    for (size_t i = 0; i < n; i++) {
      neighbors_of(particles[i].x, particles[i].y, particles, nb);
      R pix = particles[i].x, piy = particles[i].y;
      R vix = particles[i].vx, viy = particles[i].vy;
      R rho_i = rmax(particles[i].density, (R)kEps);
      R p_i = particles[i].pressure;
      R fxi = 0, fyi = 0;
      for (uint32_t j : nb) {
        if (j == i) continue;
        const auto& pj = particles[j];
        R rho_j = rmax(pj.density, (R)kEps);
        R dx = pix - pj.x;
        R dy = piy - pj.y;
        R dist = std::sqrt(dx * dx + dy * dy);
        R gxx, gyy;
        spiky_grad(dx, dy, dist, h, gxx, gyy);
        R term = p_i / (rho_i * rho_i) + pj.pressure / (rho_j * rho_j);
        if ((R)cfg.artificial_viscosity > (R)0 && dist > (R)kEps) {
          R rho_bar = (R)0.5 * (rho_i + rho_j);
          term += artificial_pressure(dx, dy, vix - pj.vx, viy - pj.vy, dist * dist, h, rho_bar, c_s,
                                      (R)cfg.artificial_viscosity);
        }
        R mt = pj.mass * term;
        fxi -= gxx * mt;
        fyi -= gyy * mt;
        if ((R)cfg.surface_tension > (R)0 && dist > (R)kEps) {
          R coh = cohesion(dist, h);
          if (coh > (R)0) {
            R s = (R)cfg.surface_tension * particles[i].mass * pj.mass * coh;
            fxi -= dx / dist * s;
            fyi -= dy / dist * s;
          }
        }
      }
      if (cfg.boundary_particles) ghost_pressure_force(pix, piy, p_i / (rho_i * rho_i), h, fxi, fyi);
      fx[i] = fxi;
      fy[i] = fyi;
    }
  }

  // ---- integrate: gravity + pressure, XSPH, cap, advect (fluid.rs:1003-1050) ----
  void integrate(R h, R dt, Mode mode) {
    std::vector<uint32_t> nb;
    size_t n = particles.size();
    std::vector<Particle<R>> snap;
    if (mode == JACOBI) snap = particles;
    const std::vector<Particle<R>>& src = (mode == JACOBI) ? snap : particles;
    R visc = (R)cfg.viscosity;
    R vmax = (R)cfg.max_velocity;
    for (size_t i = 0; i < n; i++) {
      // REF_SEQ reads the live array: j < i are already advected.
      neighbors_of(src[i].x, src[i].y, src, nb);
      R rho_i = rmax(src[i].density, (R)kEps);
      R ax = gx + fx[i] / rho_i;
      R ay = gy + fy[i] / rho_i;
      if (extra_ax.size() == n) {
        ax = ax + extra_ax[i];
        ay = ay + extra_ay[i];
      }
      if (turb.on) turbulence_accel(turb, src[i].x, src[i].y, time, ax, ay);
      R vx = src[i].vx + ax * dt;
      R vy = src[i].vy + ay * dt;
      if (visc > (R)0) {
        R pix = src[i].x, piy = src[i].y;
        R sx = 0, sy = 0;
        for (uint32_t j : nb) {
          if (j == i) continue;
          const auto& pj = src[j];
          R rho_bar = (R)0.5 * (rho_i + rmax(pj.density, (R)kEps));
          R dx = pj.x - pix;
          R dy = pj.y - piy;
          R w = poly6(dx * dx + dy * dy, h);
          R mr = pj.mass / rho_bar;
          sx += (pj.vx - src[i].vx) * mr * w;
          sy += (pj.vy - src[i].vy) * mr * w;
        }
        vx += sx * visc;
        vy += sy * visc;
      }
      R speed = std::sqrt(vx * vx + vy * vy);
      if (speed > vmax) {
        R sc = vmax / speed;
        vx *= sc;
        vy *= sc;
      }
      if (!finite(vx) || !finite(vy)) {
        vx = 0;
        vy = 0;
      }
      R nx = src[i].x + vx * dt;
      R ny = src[i].y + vy * dt;
      if (!finite(nx) || !finite(ny)) {
        nx = src[i].x;
        ny = src[i].y;
      }
      particles[i].vx = vx;
      particles[i].vy = vy;
      particles[i].x = nx;
      particles[i].y = ny;
    }
  }

  // ---- particle vs static body (fluid.rs:463-533, circle + box) ----
  // Returns false when separated; else the normal and depth.
  static bool collide(R px, R py, R pr, const Body& b, R& nx, R& ny, R& depth) {
    R qx, qy;
    return collide_pt(px, py, pr, b, nx, ny, depth, qx, qy);
  }
  // ... and the contact point on the body surface (circle: position +
  // normal * radius; box: transform_point(clamped))
  // ---- polygon bodies: fluid.rs:518-530 and crates/collision/src/sat.rs ----
  // glam Vec2::normalize_or_zero: v * (1 / |v|) if that is finite and > 0
  static void unit_or_zero(R x, R y, R& ox, R& oy) {
    const R rcp = (R)1 / std::sqrt(x * x + y * y);
    if (std::isfinite(rcp) && rcp > (R)0) {
      ox = x * rcp;
      oy = y * rcp;
    } else {
      ox = 0;
      oy = 0;
    }
  }
  // project_polygon (sat.rs:88-99); std::fmin / fmax keep the non-NaN, as f32::min / max
  static void poly_extent(const std::vector<float>& v, R ax, R ay, R& lo, R& hi) {
    lo = (R)std::numeric_limits<float>::max();
    hi = -(R)std::numeric_limits<float>::max();
    for (size_t i = 0; i + 1 < v.size(); i += 2) {
      const R d = ax * (R)v[i] + ay * (R)v[i + 1];
      lo = std::fmin(lo, d);
      hi = std::fmax(hi, d);
    }
  }
  // edge k's normalised (-e.y, e.x); false for |e|^2 < EPS_SQ
  static bool edge_unit_normal(const std::vector<float>& v, size_t k, R& nx, R& ny) {
    const size_t n = v.size() / 2, j = (k + 1) % n;
    const R ex = (R)v[2 * j] - (R)v[2 * k], ey = (R)v[2 * j + 1] - (R)v[2 * k + 1];
    if (ex * ex + ey * ey < (R)kEpsSq) return false;
    unit_or_zero(-ey, ex, nx, ny);
    return true;
  }
  // point_in_polygon (sat.rs:203-220), even-odd rule
  static bool inside_poly(R x, R y, const std::vector<float>& v) {
    const size_t n = v.size() / 2;
    bool in = false;
    for (size_t i = 0, j = n - 1; i < n; j = i++) {
      const R xi = v[2 * i], yi = v[2 * i + 1], xj = v[2 * j], yj = v[2 * j + 1];
      if ((yi > y) != (yj > y) && x < (xj - xi) * (y - yi) / (yj - yi) + xi) in = !in;
    }
    return in;
  }
  // sat_circle_polygon (sat.rs:104-200)
  static bool circle_poly_sat(R cx, R cy, R r, const std::vector<float>& v, R& ax, R& ay, R& pen) {
    const size_t n = v.size() / 2;
    if (n < 3 || r <= (R)0) return false;
    R best = (R)std::numeric_limits<float>::max(), bx = 0, by = 0;
    for (size_t k = 0; k < n; k++) {
      R ux, uy, lo, hi;
      if (!edge_unit_normal(v, k, ux, uy)) continue;
      poly_extent(v, ux, uy, lo, hi);
      const R c = ux * cx + uy * cy;
      if (hi < c - r || c + r < lo) return false;
      const R ov = std::fmin(hi, c + r) - std::fmax(lo, c - r);
      if (ov < best) {
        best = ov;
        bx = ux;
        by = uy;
      }
    }
    size_t kc = 0;  // the closest vertex (first of equals)
    R dbest = (cx - (R)v[0]) * (cx - (R)v[0]) + (cy - (R)v[1]) * (cy - (R)v[1]);
    for (size_t k = 1; k < n; k++) {
      const R dx = cx - (R)v[2 * k], dy = cy - (R)v[2 * k + 1];
      const R d = dx * dx + dy * dy;
      if (d < dbest) {
        dbest = d;
        kc = k;
      }
    }
    const R wx = cx - (R)v[2 * kc], wy = cy - (R)v[2 * kc + 1];
    if (wx * wx + wy * wy >= (R)kEpsSq) {
      R ux, uy, lo, hi;
      unit_or_zero(wx, wy, ux, uy);
      if (!(ux == (R)0 && uy == (R)0)) {
        poly_extent(v, ux, uy, lo, hi);
        const R c = ux * cx + uy * cy;
        if (hi < c - r || c + r < lo) return false;
      }
    }
    if (inside_poly(cx, cy, v)) {
      R far = -(R)std::numeric_limits<float>::max(), fx = 0, fy = 0;
      for (size_t k = 0; k < n; k++) {
        R ux, uy;
        if (!edge_unit_normal(v, k, ux, uy)) continue;
        const R d = ux * ((R)v[2 * k] - cx) + uy * ((R)v[2 * k + 1] - cy);
        if (d > far) {
          far = d;
          fx = ux;
          fy = uy;
        }
      }
      if (fx == (R)0 && fy == (R)0) return false;
      ax = -fx;
      ay = -fy;
      pen = r - far;
      return true;
    }
    if (bx == (R)0 && by == (R)0) return false;
    ax = bx;
    ay = by;
    pen = best;
    return true;
  }

  static bool collide_pt(R px, R py, R pr, const Body& b, R& nx, R& ny, R& depth, R& qx, R& qy) {
    if (b.shape == 2) {
      R ax, ay, pen;
      if (!circle_poly_sat(px, py, pr, b.poly, ax, ay, pen)) return false;
      R sx = 0, sy = 0;  // polygon_centroid: sum from zero, divided by the count
      for (size_t i = 0; i + 1 < b.poly.size(); i += 2) {
        sx = sx + (R)b.poly[i];
        sy = sy + (R)b.poly[i + 1];
      }
      const R cnt = (R)(float)(b.poly.size() / 2);
      const R cenx = sx / cnt, ceny = sy / cnt;
      if ((px - cenx) * ax + (py - ceny) * ay < (R)0) {  // orient_normal(axis, centroid, particle)
        ax = -ax;
        ay = -ay;
      }
      nx = ax;
      ny = ay;
      depth = pen;
      qx = px - ax * pr;
      qy = py - ay * pr;
      return true;
    }
    if (b.shape == 0) {
      R dx = px - (R)b.px;
      R dy = py - (R)b.py;
      R dist = std::sqrt(dx * dx + dy * dy);
      R radius = (R)b.a;
      if (dist >= radius + pr) return false;
      if (dist > (R)kEps) {
        nx = dx / dist;
        ny = dy / dist;
      } else {
        nx = 1;
        ny = 0;
      }
      depth = radius + pr - dist;
      qx = (R)b.px + nx * radius;
      qy = (R)b.py + ny * radius;
      return true;
    }
    R hx = (R)b.a, hy = (R)b.b;
    R rx = px - (R)b.px;
    R ry = py - (R)b.py;
    R xax = (R)b.xax, xay = (R)b.xay, yax = (R)b.yax, yay = (R)b.yay;
    // fluid.rs:483-489 literally: x_axis.x*rel.x + y_axis.x*rel.y (this is
    // R*rel, not R^T*rel as its comment says; identical for unrotated walls).
    R lx = xax * rx + yax * ry;
    R ly = xay * rx + yay * ry;
    R cxl = rclamp(lx, -hx, hx);
    R cyl = rclamp(ly, -hy, hy);
    R ddx = lx - cxl;
    R ddy = ly - cyl;
    if (ddx * ddx + ddy * ddy > (R)kEpsSq) {
      R dist = std::sqrt(ddx * ddx + ddy * ddy);
      if (dist >= pr) return false;
      R lnx = ddx / dist, lny = ddy / dist;
      // glam Mat2 * Vec2: x_axis * v.x + y_axis * v.y
      nx = xax * lnx + yax * lny;
      ny = xay * lnx + yay * lny;
      depth = pr - dist;
      qx = (xax * cxl + yax * cyl) + (R)b.px;
      qy = (xay * cxl + yay * cyl) + (R)b.py;
      return true;
    }
    R dxp = hx - std::fabs(lx);
    R dyp = hy - std::fabs(ly);
    // `signum().copysign(1.0)` is always +1 (NaN keeps a NaN): the eject
    // normal is always +x or +y in the box frame (fluid.rs:504-516).
    R lnx, lny;
    if (dxp < dyp) {
      lnx = (lx != lx) ? lx : (R)1;
      lny = 0;
      depth = pr + dxp;
    } else {
      lnx = 0;
      lny = (ly != ly) ? ly : (R)1;
      depth = pr + dyp;
    }
    if (lnx != lnx) lnx = std::fabs(lnx);
    if (lny != lny) lny = std::fabs(lny);
    nx = xax * lnx + yax * lny;
    ny = xay * lnx + yay * lny;
    qx = (xax * cxl + yax * cyl) + (R)b.px;
    qy = (xay * cxl + yay * cyl) + (R)b.py;
    return true;
  }

  // boundary pass (fluid.rs:1056-1094): push out, remove the approach
  // velocity, impulse n * (vn * m) on the body, then the no-slip pull toward
  // the body's tangential velocity with its reaction -dv * m. Statics take
  // no impulse (body.rs:675-687) and walls have zero velocity.
  void boundaries() {
    R pr = rmax((R)cfg.particle_radius, (R)0);
    for (auto& p : particles) {
      for (Body& b : bodies) {
        R nx, ny, depth, qx, qy;
        if (!collide_pt(p.x, p.y, pr, b, nx, ny, depth, qx, qy)) continue;
        if (depth <= (R)0) continue;
        p.x = p.x + nx * depth;
        p.y = p.y + ny * depth;
        R vn = p.vx * nx + p.vy * ny;
        if (vn < (R)0) {
          p.vx -= nx * vn;
          p.vy -= ny * vn;
          if (!b.is_static) b.sleeping = false;
          b.apply_impulse((float)(nx * (vn * p.mass)), (float)(ny * (vn * p.mass)), (float)qx, (float)qy);
          if ((R)cfg.wall_friction > (R)0) {
            R mu = rclamp((R)cfg.wall_friction, (R)0, (R)1);
            R vtx = p.vx, vty = p.vy;
            R wvx = (R)b.vx, wvy = (R)b.vy;
            R wdot = wvx * nx + wvy * ny;
            R wtx = wvx - nx * wdot;
            R wty = wvy - ny * wdot;
            R dvx = (wtx - vtx) * mu;
            R dvy = (wty - vty) * mu;
            p.vx += dvx;
            p.vy += dvy;
            b.apply_impulse((float)(-dvx * p.mass), (float)(-dvy * p.mass), (float)qx, (float)qy);
          }
        }
      }
    }
  }

  // ---- buoyancy + drag (fluid.rs:388-458, :1103-1135) ----
  // sample_pressure: p(x) = sum m_j (p_j / max(rho_j, EPS)) poly6(|x - x_j|^2)
  // over the grid cells around floor(x / h), h = max(smoothing_length, EPS)
  R sample_pressure(R ptx, R pty) const {
    R h = rmax((R)cfg.smoothing_length, (R)kEps);
    int32_t cx = sat_i32(std::floor(ptx / h)), cy = sat_i32(std::floor(pty / h));
    R p = 0;
    for (int oy = -1; oy <= 1; oy++)
      for (int ox = -1; ox <= 1; ox++) {
        int64_t xx = (int64_t)cx + ox, yy = (int64_t)cy + oy;
        if (xx < INT32_MIN || xx > INT32_MAX || yy < INT32_MIN || yy > INT32_MAX) continue;
        auto it = grid.find(cell_key((int32_t)xx, (int32_t)yy));
        if (it == grid.end()) continue;
        for (uint32_t j : it->second) {
          const auto& pj = particles[j];
          R dx = pj.x - ptx, dy = pj.y - pty;
          R r2 = dx * dx + dy * dy;
          if (r2 < h * h) p += pj.mass * (pj.pressure / rmax(pj.density, (R)kEps)) * poly6(r2, h);
        }
      }
    return rmax(p, (R)0);
  }
  // surface_samples: circles 12 perimeter points, boxes 4 per edge
  static void surface_samples(const Body& b, std::vector<float>& out) {  // (x, y, nx, ny, area) each
    if (b.shape == 2) return;  // polygons are impulse-coupled only (fluid.rs:415-418)
    const float pi = Consts<float>::pi();
    auto push = [&](float lx, float ly, float nlx, float nly, float area) {
      out.push_back((b.xax * lx + b.yax * ly) + b.px);
      out.push_back((b.xay * lx + b.yay * ly) + b.py);
      out.push_back(b.xax * nlx + b.yax * nly);
      out.push_back(b.xay * nlx + b.yay * nly);
      out.push_back(area);
    };
    if (b.shape == 0) {
      const int n = 12;
      float area = 2.0f * pi * b.a / (float)n;
      for (int k = 0; k < n; k++) {
        float a = 2.0f * pi * (float)k / (float)n;
        float c = cosf(a), sn = sinf(a);
        push(c * b.a, sn * b.a, c, sn, area);
      }
    } else {
      float hx = b.a, hy = b.b;
      float area = 4.0f * (hx + hy) / 16.0f;
      const float e[4][5] = {{0, -1, -hx, -hy, 1}, {0, 1, -hx, hy, 1}, {-1, 0, -hx, -hy, 0}, {1, 0, hx, -hy, 0}};
      for (int q = 0; q < 4; q++)
        for (int k = 0; k < 4; k++) {
          float t = ((float)k + 0.5f) / 4.0f;
          bool along_x = e[q][4] != 0;
          float extent = along_x ? hx : hy;
          float sc = 2.0f * extent * t;
          float tx = along_x ? 1.0f : 0.0f, ty = along_x ? 0.0f : 1.0f;
          push(e[q][2] + tx * sc, e[q][3] + ty * sc, e[q][0], e[q][1], area);
        }
    }
  }
  void buoyancy(R dt) {
    rebuild_grid();
    std::vector<float> smp;
    for (Body& b : bodies) {
      if (b.is_static) continue;
      smp.clear();
      surface_samples(b, smp);
      if (smp.empty()) continue;
      float drag = std::max(cfg.drag, 0.0f);
      bool wet = false;
      for (size_t q = 0; q < smp.size(); q += 5) {
        float ptx = smp[q], pty = smp[q + 1], nx = smp[q + 2], ny = smp[q + 3], area = smp[q + 4];
        float p = (float)sample_pressure((R)ptx, (R)pty);
        if (p <= 0.0f) continue;
        wet = true;
        float rx = ptx - b.px, ry = pty - b.py;
        float vrx = (b.vx + (-b.w * ry)) - wind_x;  // against ambient.drag.wind (fluid.rs:1121-1124)
        float vry = (b.vy + (b.w * rx)) - wind_y;
        float speed = std::sqrt(vrx * vrx + vry * vry);
        float fx = -nx * (p * area), fy = -ny * (p * area);
        if (speed > kEps) {
          float c = drag * area * speed;
          fx -= vrx * c;
          fy -= vry * c;
        }
        b.apply_force(fx, fy, ptx, pty, (float)dt);
      }
      if (wet) b.sleeping = false;
    }
  }
  bool any_dynamic() const {
    for (const Body& b : bodies)
      if (!b.is_static) return true;
    return false;
  }

  // ---- CFL substeps (fluid.rs:562-588) ----
  uint32_t cfl_substeps(R dt) const {
    uint32_t mx = std::max<uint32_t>(cfg.max_substeps, 1);
    if ((R)cfg.cfl <= (R)0 || mx <= 1) return 1;
    R h = rmax((R)cfg.smoothing_length, (R)kEps);
    R rho0 = rmax((R)cfg.rest_density, (R)kEps);
    R c0;
    if ((R)cfg.gamma == (R)1.0)
      c0 = std::sqrt(rmax((R)cfg.stiffness, (R)0));
    else
      c0 = std::sqrt((R)cfg.gamma * rmax((R)cfg.stiffness, (R)0) * rho0);
    R vm = 0;
    for (const auto& p : particles) vm = rmax(vm, std::sqrt(p.vx * p.vx + p.vy * p.vy));
    R speed = c0 + vm;
    if (!finite(speed) || speed <= (R)kEps) return 1;
    R dt_max = (R)cfg.cfl * h / speed;
    if (!finite(dt_max) || dt_max <= (R)0) return 1;
    R q = std::ceil(dt / dt_max);
    int64_t k;
    if (q != q)
      k = 0;
    else if (q >= (R)9.2233720368547758e18)
      k = INT64_MAX;
    else if (q <= (R)-9.2233720368547758e18)
      k = INT64_MIN;
    else
      k = (int64_t)q;
    if (k < 1) k = 1;
    if (k > (int64_t)mx) k = mx;
    return (uint32_t)k;
  }

  // ---- closure-network inputs (no reference counterpart) ----
  // The 16 inputs of the learned closure for every particle at the current
  // state, for a coarse step dt. Restates the GPU closure pass
  // (feat_pair / wall_feature / feat_finish) operation for operation: the
  // neighbour aggregates run over j != i in the reference's visit order with
  // the pressure force's pair arithmetic (fluid.rs:942-997), then the
  // nearest static body within 3h, then the scaled feature vector.
  void wall_feature(R x, R y, R h, R& fd, R& fnx, R& fny) const {
    const R lim = (R)3.0 * h;
    R best = lim, bnx = 0, bny = 0;
    for (const Body& b : bodies) {
      const R ha = (R)b.a, hb = b.shape == 0 ? (R)b.a : (R)b.b;
      // the world's padded bounding box (phieng_world_add_body)
      const R ex = (std::fabs((R)b.xax) * ha + std::fabs((R)b.yax) * hb) * (R)1.001f + (R)1e-30f;
      const R ey = (std::fabs((R)b.xay) * ha + std::fabs((R)b.yay) * hb) * (R)1.001f + (R)1e-30f;
      if (std::fabs(x - (R)b.px) > ex + lim || std::fabs(y - (R)b.py) > ey + lim) continue;
      R d, nx, ny;
      if (b.shape == 0) {
        const R dx = x - (R)b.px, dy = y - (R)b.py;
        const R dist = std::sqrt(dx * dx + dy * dy);
        d = dist - (R)b.a;
        if (dist > (R)kEps) {
          nx = dx / dist;
          ny = dy / dist;
        } else {
          nx = 1;
          ny = 0;
        }
      } else {
        const R rx = x - (R)b.px, ry = y - (R)b.py;
        const R lx = (R)b.xax * rx + (R)b.yax * ry;
        const R ly = (R)b.xay * rx + (R)b.yay * ry;
        const R qx = std::fabs(lx) - (R)b.a, qy = std::fabs(ly) - (R)b.b;
        R lnx, lny;
        if (qx > (R)0 || qy > (R)0) {
          const R ox = qx > (R)0 ? qx : (R)0, oy = qy > (R)0 ? qy : (R)0;
          d = std::sqrt(ox * ox + oy * oy);
          lnx = std::copysign(ox, lx) / d;
          lny = std::copysign(oy, ly) / d;
        } else if (qx >= qy) {
          d = qx;
          lnx = std::copysign((R)1, lx);
          lny = 0;
        } else {
          d = qy;
          lnx = 0;
          lny = std::copysign((R)1, ly);
        }
        nx = (R)b.xax * lnx + (R)b.yax * lny;
        ny = (R)b.xay * lnx + (R)b.yay * lny;
      }
      if (d < best) {
        best = d;
        bnx = nx;
        bny = ny;
      }
    }
    fd = (best > -h ? best : -h) / h;
    fnx = bnx;
    fny = bny;
  }

  void compute_features(R dt, std::vector<R>& out) {
    const R h = rmax((R)cfg.smoothing_length, (R)kEps);
    rebuild_grid();
    compute_density_pressure(h);
    const size_t n = particles.size();
    out.assign(16 * n, (R)0);
    std::vector<uint32_t> nb;
    const R ih = (R)1 / h;
    const R s1 = dt * ih, s2 = s1 * s1, s3 = dt * dt * ih;
    for (size_t i = 0; i < n; i++) {
      const auto& pi = particles[i];
      neighbors_of(pi.x, pi.y, particles, nb);
      const R rho_i = rmax(pi.density, (R)kEps);
      const R q_i = pi.pressure / (rho_i * rho_i);
      R px = 0, py = 0, div = 0, curl = 0, wsum = 0, m1x = 0, m1y = 0, m2xx = 0, m2yy = 0, pw = 0;
      uint32_t cnt = 0;
      for (uint32_t j : nb) {
        if (j == i) continue;
        const auto& pj = particles[j];
        const R rho_j = rmax(pj.density, (R)kEps);
        const R dx = pi.x - pj.x, dy = pi.y - pj.y;
        const R d2 = dx * dx + dy * dy;
        const R dist = std::sqrt(d2);
        R gxx, gyy;
        spiky_grad(dx, dy, dist, h, gxx, gyy);
        const R w = poly6(d2, h);
        const R q_j = pj.pressure / (rho_j * rho_j);
        const R mt = pj.mass * (q_i + q_j);
        px = px - gxx * mt;
        py = py - gyy * mt;
        const R vol = pj.mass / rho_j;
        const R dvx = pj.vx - pi.vx, dvy = pj.vy - pi.vy;
        div = div + vol * (dvx * gxx + dvy * gyy);
        curl = curl + vol * (dvx * gyy - dvy * gxx);
        const R ww = vol * w;
        wsum = wsum + ww;
        const R wx = ww * dvx, wy = ww * dvy;
        m1x = m1x + wx;
        m1y = m1y + wy;
        m2xx = m2xx + wx * dvx;
        m2yy = m2yy + wy * dvy;
        pw = pw + ww * (q_j * rho_j * rho_j);
        cnt++;
      }
      R wd, wnx, wny;
      wall_feature(pi.x, pi.y, h, wd, wnx, wny);
      const R r0 = rmax((R)cfg.phase_rest_density[std::min<int>(pi.phase, 3)], (R)kEps);
      const R kr = (R)cfg.stiffness * r0;
      R* f = &out[16 * i];
      f[0] = pi.density / r0 - (R)1;
      f[1] = kr > (R)0 ? pi.pressure / kr : (R)0;
      f[2] = div * dt;
      f[3] = curl * dt;
      f[4] = (R)cnt * (R)0.0625f;
      f[5] = wd;
      f[6] = wnx;
      f[7] = wny;
      const R iw = wsum > (R)0 ? (R)1 / wsum : (R)0;
      f[8] = m1x * iw * s1;
      f[9] = m1y * iw * s1;
      f[10] = m2xx * iw * s2;
      f[11] = kr > (R)0 ? (pi.pressure - pw * iw) / kr : (R)0;
      f[12] = m2yy * iw * s2;
      f[13] = px / rho_i * s3;
      f[14] = py / rho_i * s3;
      f[15] = std::sqrt(pi.vx * pi.vx + pi.vy * pi.vy) * s1;
    }
  }

  // ---- one substep (fluid.rs:898-1136) for the dam-break feature set ----
  void substep(R dt, Mode mode) {
    R h = rmax((R)cfg.smoothing_length, (R)kEps);
    rebuild_grid();
    compute_density_pressure(h);
    if (cfg.adaptive_resolution) {  // fluid.rs:915-919
      resample(h);
      rebuild_grid();
      compute_density_pressure(h);
    }
    if (cfg.boundary_particles) {  // fluid.rs:929-937
      refresh_ghosts();
      ghost_density(h);
    }
    compute_forces(h);
    integrate(h, dt, mode);
    extra_ax.clear();
    extra_ay.clear();
    boundaries();
    // the trailing rebuild_grid + buoyancy pass (fluid.rs:1102-1135) acts on
    // dynamic bodies only and leaves the particle state unchanged
    if (any_dynamic()) buoyancy(dt);
  }

  // FluidState2::step_fluid (fluid.rs:541-557): no clock
  void step_fluid(R dt, Mode mode) {
    if (!cfg.enabled || particles.empty() || dt <= (R)0) return;
    uint32_t n = cfl_substeps(dt);
    R sub = dt / (R)n;
    for (uint32_t k = 0; k < n; k++) substep(sub, mode);
  }

  // ---- step_fluid (fluid.rs:541-557) inside World2::step (world.rs:706-732) ----
  void world_step(R dt, Mode mode) {
    if (cfg.enabled && !particles.empty() && dt > (R)0) {
      uint32_t n = cfl_substeps(dt);
      R sub = dt / (R)n;
      for (uint32_t k = 0; k < n; k++) substep(sub, mode);
    }
    time += dt;
  }
};

}  // namespace oracle
