// ORACLE — TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the reference's 3D SPH fluid step
// (crates/dynamics/src/fluid3.rs), for the static-wall feature set the GPU
// 3D path implements: particles, hash grid, density + EOS, pressure force
// (+ Monaghan AV, cohesion), XSPH integrate in the reference's in-place order
// (REF_SEQ) or in Jacobi order (what the GPU computes), sphere / box / capsule
// walls with wall friction, CFL substeps. Rigid bodies added through the C
// ABI (phieng_world3_add_body, crates/engine/src/ffi.rs:3703-3760) carry the
// identity rotation, so the box and capsule local frames are the world axes:
// glam's quaternion products with the identity return the vector unchanged.
// Float arithmetic follows glam 0.29's scalar Vec3 (dot = (x*x + y*y) + z*z,
// component-wise operators); built with -ffp-contract=off.
// Pinned against a second statement of the algorithm by the reference's
// authors, the C# solver (src/PhiEng.Dynamics/FluidSolver3.cs, restated in
// oracle/fluid3_cs.py): bit-identical in REF_SEQ order on the reference's
// own 3D equivalence scene (tests/PhiEng.Tests/EquivalenceTests.cs:177-225,
// 30 steps) and on a five-box tank with CFL substeps and wall friction
// (tests/test_oracle_pin.py).
#pragma once

#include <algorithm>
#include <map>
#include <tuple>
#include <cmath>
#include <cstdint>
#include <unordered_map>
#include <vector>

#include "sph_oracle.hpp"

namespace oracle {

// ---- 3D ambient turbulence (noise.rs:50-222, fluid3.rs:1090-1108) ----
template <class R>
inline R nz_lattice3(int32_t ix, int32_t iy, int32_t iz, uint32_t seed) {  // noise.rs:50-60
  const uint32_t h = nz_hash((uint32_t)ix * 0x1f1f1f1fu + (uint32_t)iy * 0x9e3779b9u + (uint32_t)iz * 0x85ebca6bu + seed);
  return (R)(h >> 8) * (R)(1.0f / 16777216.0f);
}

template <class R>
inline R nz_value3(R x, R y, R z, uint32_t seed) {  // noise.rs:90-111
  const R x0 = std::floor(x), y0 = std::floor(y), z0 = std::floor(z);
  const int32_t xi = rust_as_int<int32_t>(x0), yi = rust_as_int<int32_t>(y0), zi = rust_as_int<int32_t>(z0);
  const R tx = nz_fade(x - x0), ty = nz_fade(y - y0), tz = nz_fade(z - z0);
  const int32_t x1 = (int32_t)((uint32_t)xi + 1u), y1 = (int32_t)((uint32_t)yi + 1u), z1 = (int32_t)((uint32_t)zi + 1u);
  const R v000 = nz_lattice3<R>(xi, yi, zi, seed), v100 = nz_lattice3<R>(x1, yi, zi, seed);
  const R v010 = nz_lattice3<R>(xi, y1, zi, seed), v110 = nz_lattice3<R>(x1, y1, zi, seed);
  const R v001 = nz_lattice3<R>(xi, yi, z1, seed), v101 = nz_lattice3<R>(x1, yi, z1, seed);
  const R v011 = nz_lattice3<R>(xi, y1, z1, seed), v111 = nz_lattice3<R>(x1, y1, z1, seed);
  const R a = nz_lerp(nz_lerp(v000, v100, tx), nz_lerp(v010, v110, tx), ty);
  const R b = nz_lerp(nz_lerp(v001, v101, tx), nz_lerp(v011, v111, tx), ty);
  return nz_lerp(a, b, tz);
}

template <class R>
inline R nz_fbm3_static(R x, R y, R z, uint32_t seed, uint32_t oct) {  // noise.rs:135-152
  R sum = 0, amp = 1, freq = 1, norm = 0;
  for (uint32_t o = 0; o < oct; o++) {
    sum += amp * (nz_value3(x * freq, y * freq, z * freq, seed + o) * (R)2 - (R)1);
    norm += amp;
    amp *= (R)0.5;
    freq *= (R)2;
  }
  return norm > (R)0 ? sum / norm : (R)0;
}

template <class R>
inline R nz_fbm3(R x, R y, R z, R t, uint32_t seed, uint32_t octaves) {  // noise.rs:173-183
  const uint32_t oct = std::min<uint32_t>(std::max<uint32_t>(octaves, 1u), 8u);
  const R t0 = std::floor(t);
  const R ft = nz_fade(t - t0);
  const int64_t sl = rust_as_int<int64_t>(t0);
  const uint32_t s0 = seed + (uint32_t)sl * 0x9e3779b9u;
  const uint32_t s1 = seed + (uint32_t)((uint64_t)sl + 1u) * 0x9e3779b9u;
  return nz_lerp(nz_fbm3_static(x, y, z, s0, oct), nz_fbm3_static(x, y, z, s1, oct), ft);
}

template <class R>
inline void turbulence_accel3(const Turbulence& tb, R px, R py, R pz, R time, R& ax, R& ay, R& az) {
  const R x = px * (R)tb.freq, y = py * (R)tb.freq, z = pz * (R)tb.freq;
  const R t = time * (R)tb.tscale;
  R nx, ny, nz;
  if (tb.curl) {  // curl_3 (noise.rs:198-222), components exactly as written there
    const R e = (R)1e-3f, e2 = (R)(2.0f * 1e-3f);
    const uint32_t oc = tb.oct;
    auto px_ = [&](R a, R b, R c) { return nz_fbm3(a, b, c, t, tb.seed ^ 0x11111111u, oc); };
    auto py_ = [&](R a, R b, R c) { return nz_fbm3(a, b, c, t, tb.seed ^ 0x22222222u, oc); };
    auto pz_ = [&](R a, R b, R c) { return nz_fbm3(a, b, c, t, tb.seed ^ 0x33333333u, oc); };
    auto ddx = [&](auto f) { return (f(x + e, y, z) - f(x - e, y, z)) / e2; };
    auto ddy = [&](auto f) { return (f(x, y + e, z) - f(x, y - e, z)) / e2; };
    auto ddz = [&](auto f) { return (f(x, y, z + e) - f(x, y, z - e)) / e2; };
    nx = ddy(pz_) - ddz(py_);
    ny = ddx(px_) - ddz(pz_);
    nz = ddx(py_) - ddy(px_);
  } else {
    nx = nz_fbm3(x, y, z, t, tb.seed, tb.oct);
    ny = nz_fbm3(x, y, z, t, tb.seed ^ 0x55aa55aau, tb.oct);
    nz = nz_fbm3(x, y, z, t, tb.seed ^ 0xaa55aa55u, tb.oct);
  }
  const R ls = nx * nx + ny * ny + nz * nz;  // glam Vec3 dot: (x*x + y*y) + z*z
  if (ls > (R)1) {
    const R l = std::sqrt(ls);
    nx = nx / l;
    ny = ny / l;
    nz = nz / l;
  }
  ax = ax + nx * (R)tb.amp;
  ay = ay + ny * (R)tb.amp;
  az = az + nz * (R)tb.amp;
}

// ---- rigid bodies of the fluid phase (RigidBody3, body.rs:902-956, 1324-1361) ----
// Rotation of v by the unit quaternion (b, w) = (qx, qy, qz, qw), the
// expansion of q v q* for |q| = 1:
//   v' = (v (w^2 - b.b) + b (2 (v.b))) + (b x v) (2 w)
// evaluated in this order. glam 0.29's Quat * Vec3 sums the same three
// terms; its association is not pinned here (no Rust toolchain on this
// image), so rotated bodies are checked against this restatement only.
template <class R>
inline R vdot3(R ax, R ay, R az, R bx, R by, R bz) {  // glam Vec3::dot: (x x' + y y') + z z'
  return ax * bx + ay * by + az * bz;
}
template <class R>
inline void qrot(R qx, R qy, R qz, R qw, R vx, R vy, R vz, R& ox, R& oy, R& oz) {
  const R s = qw * qw - vdot3(qx, qy, qz, qx, qy, qz);
  const R d = vdot3(vx, vy, vz, qx, qy, qz) * (R)2;
  const R w2 = qw * (R)2;
  const R cx = qy * vz - qz * vy, cy = qz * vx - qx * vz, cz = qx * vy - qy * vx;
  ox = (vx * s + qx * d) + cx * w2;
  oy = (vy * s + qy * d) + cy * w2;
  oz = (vz * s + qz * d) + cz * w2;
}

// Mat3::from_quat for a unit quaternion (column-major: x_axis, y_axis,
// z_axis), with x2 = x + x etc.: the standard rotation matrix.
inline void mat3_from_quat(float x, float y, float z, float w, float m[9]) {
  const float x2 = x + x, y2 = y + y, z2 = z + z;
  const float xx = x * x2, xy = x * y2, xz = x * z2, yy = y * y2, yz = y * z2, zz = z * z2;
  const float wx = w * x2, wy = w * y2, wz = w * z2;
  m[0] = 1.0f - (yy + zz), m[1] = xy + wz, m[2] = xz - wy;
  m[3] = xy - wz, m[4] = 1.0f - (xx + zz), m[5] = yz + wx;
  m[6] = xz + wy, m[7] = yz - wx, m[8] = 1.0f - (xx + yy);
}
// c = a * b, column by column: a * v = (x_axis v.x + y_axis v.y) + z_axis v.z
inline void mat3_mul(const float a[9], const float b[9], float c[9]) {
  for (int j = 0; j < 3; j++)
    for (int i = 0; i < 3; i++) c[3 * j + i] = (a[i] * b[3 * j] + a[3 + i] * b[3 * j + 1]) + a[6 + i] * b[3 * j + 2];
}
// RigidBody3::world_inv_inertia (body.rs:1328-1331): (R I^-1) R^T
inline void world_inv_inertia(float qx, float qy, float qz, float qw, const float inv_i[9], float out[9]) {
  float r[9], rt[9], t[9];
  mat3_from_quat(qx, qy, qz, qw, r);
  for (int j = 0; j < 3; j++)
    for (int i = 0; i < 3; i++) rt[3 * j + i] = r[3 * i + j];
  mat3_mul(r, inv_i, t);
  mat3_mul(t, rt, out);
}

struct Body3 {
  int shape = 1;  // 0 sphere (a = radius), 1 box (a, b, c half extents), 2 capsule (a = radius, b = half length along y), 3 hull
  float px = 0, py = 0, pz = 0;
  float a = 0, b = 0, c = 0;
  // a body of the fluid phase with the engine's bodies (step_fluid): its
  // rotation, motion and mass properties; hull vertices moved by the
  // transform (rotation * v + position, math.rs:94-96)
  bool rotated = false;
  float qx = 0, qy = 0, qz = 0, qw = 1;
  bool is_static = true, sleeping = false;
  float vx = 0, vy = 0, vz = 0, wx = 0, wy = 0, wz = 0;
  float inv_mass = 0;
  float inv_inertia[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  std::vector<float> hull;  // world-space xyz

  // RigidBody3::apply_impulse (body.rs:1349-1361)
  void apply_impulse(float jx, float jy, float jz, float ptx, float pty, float ptz) {
    if (is_static) return;
    sleeping = false;
    vx = vx + jx * inv_mass;
    vy = vy + jy * inv_mass;
    vz = vz + jz * inv_mass;
    const float rx = ptx - px, ry = pty - py, rz = ptz - pz;
    const float tx = ry * jz - rz * jy, ty = rz * jx - rx * jz, tz = rx * jy - ry * jx;
    float iw[9];
    world_inv_inertia(qx, qy, qz, qw, inv_inertia, iw);
    wx = wx + ((iw[0] * tx + iw[3] * ty) + iw[6] * tz);
    wy = wy + ((iw[1] * tx + iw[4] * ty) + iw[7] * tz);
    wz = wz + ((iw[2] * tx + iw[5] * ty) + iw[8] * tz);
  }
  // RigidBody3::apply_force (body.rs:1334-1346): impulse F dt at the point
  void apply_force(float fx, float fy, float fz, float ptx, float pty, float ptz, float dt) {
    if (is_static) return;
    sleeping = false;
    vx = vx + (fx * inv_mass) * dt;
    vy = vy + (fy * inv_mass) * dt;
    vz = vz + (fz * inv_mass) * dt;
    const float rx = ptx - px, ry = pty - py, rz = ptz - pz;
    const float tx = ry * fz - rz * fy, ty = rz * fx - rx * fz, tz = rx * fy - ry * fx;
    float iw[9];
    world_inv_inertia(qx, qy, qz, qw, inv_inertia, iw);
    wx = wx + ((iw[0] * tx + iw[3] * ty) + iw[6] * tz) * dt;
    wy = wy + ((iw[1] * tx + iw[4] * ty) + iw[7] * tz) * dt;
    wz = wz + ((iw[2] * tx + iw[5] * ty) + iw[8] * tz) * dt;
  }
};

// Surface samples (point, outward normal, area) of a dynamic body for the
// buoyancy pass (fluid3.rs:371-467): 14 sphere directions, 4 per box face
// (every face's points at its fixed coordinate -he, as written), two rings
// of 8 plus the poles for a capsule; none for hulls. Appends 7 floats each.
inline void surface_samples3(const Body3& b, std::vector<float>& out) {
  const float pi = 3.14159265358979323846f;
  auto push = [&](float lx, float ly, float lz, float nlx, float nly, float nlz, float area) {
    float x, y, z, nx, ny, nz;
    qrot(b.qx, b.qy, b.qz, b.qw, lx, ly, lz, x, y, z);  // transform_point
    qrot(b.qx, b.qy, b.qz, b.qw, nlx, nly, nlz, nx, ny, nz);
    out.insert(out.end(), {x + b.px, y + b.py, z + b.pz, nx, ny, nz, area});
  };
  if (b.shape == 0) {
    const float r = b.a;
    float dirs[14][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    const float sg[8][3] = {{1, 1, 1}, {1, 1, -1}, {1, -1, 1}, {1, -1, -1},
                            {-1, 1, 1}, {-1, 1, -1}, {-1, -1, 1}, {-1, -1, -1}};
    for (int k = 0; k < 8; k++) {  // normalize_or_zero: v * (1 / |v|)
      const float rcp = 1.0f / std::sqrt(vdot3(sg[k][0], sg[k][1], sg[k][2], sg[k][0], sg[k][1], sg[k][2]));
      for (int a = 0; a < 3; a++) dirs[6 + k][a] = sg[k][a] * rcp;
    }
    const float area = 4.0f * pi * r * r / 14.0f;
    for (auto& d : dirs) push(d[0] * r, d[1] * r, d[2] * r, d[0], d[1], d[2], area);
  } else if (b.shape == 1) {
    const float hx = b.a, hy = b.b, hz = b.c;
    const float area = 8.0f * (hx * hy + hy * hz + hz * hx) / 24.0f;
    const struct { float n[3]; float fixed; int axis; } faces[6] = {
        {{0, 1, 0}, -hy, 0}, {{0, -1, 0}, -hy, 0}, {{1, 0, 0}, -hx, 1},
        {{-1, 0, 0}, -hx, 1}, {{0, 0, 1}, -hz, 2}, {{0, 0, -1}, -hz, 2}};
    const float ts[4][2] = {{-0.75f, -0.75f}, {0.75f, -0.75f}, {-0.75f, 0.75f}, {0.75f, 0.75f}};
    for (const auto& f : faces)
      for (const auto& t : ts) {
        if (f.axis == 0) push(hx * t[0], f.fixed, hz * t[1], f.n[0], f.n[1], f.n[2], area);
        else if (f.axis == 1) push(f.fixed, hy * t[0], hz * t[1], f.n[0], f.n[1], f.n[2], area);
        else push(hx * t[0], hy * t[1], f.fixed, f.n[0], f.n[1], f.n[2], area);
      }
  } else if (b.shape == 2) {
    const float r = b.a, hl = b.b;
    const float side = 4.0f * pi * r * hl / 16.0f, cap = 2.0f * pi * r * r;
    for (float sy : {-hl * 0.5f, hl * 0.5f})
      for (int k = 0; k < 8; k++) {
        const float a = 2.0f * pi * (float)k / 8.0f;
        const float c = std::cos(a), s = std::sin(a);
        // dir * r + Y * sy
        push(c * r + 0.0f * sy, 0.0f * r + 1.0f * sy, s * r + 0.0f * sy, c, 0.0f, s, side);
      }
    for (float s : {-1.0f, 1.0f}) {
      const float len = hl + r;
      push((0.0f * s) * len, (1.0f * s) * len, (0.0f * s) * len, 0.0f * s, 1.0f * s, 0.0f * s, cap);
    }
  }
}

template <class R>
struct Particle3 {
  R x, y, z, vx, vy, vz;
  R density, pressure, mass;
  uint8_t phase;
};

template <class R>
class Fluid3 {
 public:
  Config cfg;  // FluidConfig3 has the same fields and defaults as FluidConfig2 (fluid3.rs:51-137)
  std::vector<Particle3<R>> particles;
  std::vector<Body3> bodies;
  R gx = 0, gy = (R)-9.81f, gz = 0;  // World3::new gravity
  R time = 0;
  Turbulence turb;  // world.ambient.turbulence
  float wind_x = 0, wind_y = 0, wind_z = 0;  // world.ambient.drag.wind (buoyancy drag)

  // ---- boundary ghosts (fluid3.rs:719-922), regenerated every substep (a
  // function of the static bodies and the config only) ----
  struct Ghost3 {
    float x, y, z;
    R density, pressure;
  };
  std::vector<Ghost3> ghosts;
  std::map<std::tuple<int32_t, int32_t, int32_t>, std::vector<uint32_t>> ghost_grid;

  static int32_t as_i32(float v) {
    if (v != v) return 0;
    if (v <= -2147483648.0f) return INT32_MIN;
    if (v >= 2147483648.0f) return INT32_MAX;
    return (int32_t)v;
  }
  void refresh_ghosts() {
    ghosts.clear();
    ghost_grid.clear();
    const float hk = std::max(cfg.smoothing_length, kEps);
    const float sp = std::max(hk * 0.5f, kEps), sp2 = sp * sp;
    const float pi = Consts<float>::pi();
    auto count = [](float v, float hi) -> uint64_t {  // .ceil().clamp(1, hi) as usize
      return v != v ? 0 : (uint64_t)std::min(std::max(std::ceil(v), 1.0f), hi);
    };
    for (const Body3& b : bodies) {
      // identity rotation: glam Mat3 * Vec3 = (x_axis*x + y_axis*y) + z_axis*z, then + position
      auto put = [&](float x, float y, float z) {
        ghosts.push_back({((1.0f * x + 0.0f * y) + 0.0f * z) + b.px, ((0.0f * x + 1.0f * y) + 0.0f * z) + b.py,
                          ((0.0f * x + 0.0f * y) + 1.0f * z) + b.pz, 0, 0});
      };
      if (b.shape == 0) {
        const float r = b.a;
        const uint64_t n = count((4.0f * pi * r * r) / sp2, 512.0f);
        const float golden = pi * (3.0f - std::sqrt(5.0f));
        for (uint64_t k = 0; k < n; k++) {
          const float z = 1.0f - 2.0f * ((float)k + 0.5f) / (float)n;
          const float rr = std::sqrt(1.0f - z * z);
          const float th = golden * (float)k;
          put(std::cos(th) * rr * r, z * r, std::sin(th) * rr * r);
        }
      } else if (b.shape == 1) {
        const float he[3] = {b.a, b.b, b.c};
        const struct { float fixed; int axis; } faces[6] = {{-he[1], 0}, {-he[1], 0}, {-he[0], 1},
                                                            {-he[0], 1}, {-he[2], 2}, {-he[2], 2}};
        for (const auto& f : faces) {
          const float area = f.axis == 0 ? 4.0f * he[1] * he[2] : f.axis == 1 ? 4.0f * he[0] * he[2] : 4.0f * he[0] * he[1];
          const uint64_t n = count(area / sp2, 512.0f);
          for (uint64_t k = 0; k < n; k++) {
            const float t = ((float)k + 0.5f) / (float)n;
            float l[3] = {0.0f, 0.0f, f.fixed};
            const float u = (2.0f * t - 1.0f), v = (2.0f * std::fmod(t * 7.0f, 1.0f) - 1.0f);
            if (f.axis == 0) {
              l[1] = u * he[1];
              l[2] = v * he[2];
            } else if (f.axis == 1) {
              l[0] = u * he[0];
              l[2] = v * he[2];
            } else {
              l[0] = u * he[0];
              l[1] = v * he[1];
            }
            put(l[0], l[1], l[2]);
          }
        }
      } else {
        const float r = b.a, hl = b.b;
        const uint64_t n = count((4.0f * pi * r * hl) / sp2, 256.0f);
        const float ys[2] = {-hl * 0.5f, hl * 0.5f};
        for (float sy : ys)
          for (uint64_t k = 0; k < n; k++) {
            const float a = 2.0f * pi * (float)k / (float)n;
            put(std::cos(a) * r, sy, std::sin(a) * r);
          }
        const float ss[2] = {-1.0f, 1.0f};
        for (float s : ss) put((0.0f * s) * (hl + r), (1.0f * s) * (hl + r), (0.0f * s) * (hl + r));
      }
    }
    for (uint32_t i = 0; i < ghosts.size(); i++) {
      const Ghost3& g = ghosts[i];
      if (!std::isfinite(g.x)) continue;
      ghost_grid[{as_i32(std::floor(g.x / hk)), as_i32(std::floor(g.y / hk)), as_i32(std::floor(g.z / hk))}].push_back(i);
    }
  }
  void ghost_density(R h) {
    std::vector<uint32_t> nb;
    for (Ghost3& g : ghosts) {
      neighbors_of((R)g.x, (R)g.y, (R)g.z, particles, nb);
      R rho = 0;
      for (uint32_t j : nb) {
        const R dx = particles[j].x - (R)g.x, dy = particles[j].y - (R)g.y, dz = particles[j].z - (R)g.z;
        rho += particles[j].mass * poly6(dx * dx + dy * dy + dz * dz, h);
      }
      g.density = rclamp(rho, (R)0, (R)3 * rmax((R)cfg.rest_density, (R)kEps));
      g.pressure = Fluid<R>::pressure(rho, (R)cfg.rest_density, (R)cfg.stiffness, (R)cfg.gamma, pow_mode);
    }
  }
  void ghost_force(R px, R py, R pz, R q_i, R h, R& f0, R& f1, R& f2) const {
    const R hg = (R)cfg.smoothing_length;
    const R m = (R)std::max(cfg.particle_mass, kEps);
    const int32_t cx = sat_i32(std::floor(px / hg)), cy = sat_i32(std::floor(py / hg)), cz = sat_i32(std::floor(pz / hg));
    for (int oz = -1; oz <= 1; oz++)
      for (int oy = -1; oy <= 1; oy++)
        for (int ox = -1; ox <= 1; ox++) {
          auto it = ghost_grid.find({(int32_t)((uint32_t)cx + (uint32_t)ox), (int32_t)((uint32_t)cy + (uint32_t)oy),
                                     (int32_t)((uint32_t)cz + (uint32_t)oz)});
          if (it == ghost_grid.end()) continue;
          for (uint32_t k : it->second) {
            const Ghost3& g = ghosts[k];
            const R ex = (R)g.x - px, ey = (R)g.y - py, ez = (R)g.z - pz;
            if (!(ex * ex + ey * ey + ez * ez < hg * hg)) continue;
            const R dx = px - (R)g.x, dy = py - (R)g.y, dz = pz - (R)g.z;
            const R dist = std::sqrt(dx * dx + dy * dy + dz * dz);
            R g0, g1, g2;
            spiky_grad(dx, dy, dz, dist, h, g0, g1, g2);
            const R rb = rmax(g.density, (R)kEps);
            const R s = m * (q_i + g.pressure / (rb * rb));
            f0 -= g0 * s;
            f1 -= g1 * s;
            f2 -= g2 * s;
          }
        }
  }
  size_t cap = 4096;
  int pow_mode = 1;
  std::vector<R> fx, fy, fz;

  static R dot3(R ax, R ay, R az, R bx, R by, R bz) { return ax * bx + ay * by + az * bz; }

  // poly6 (fluid3.rs:220-229): 315/(64 pi h^9) (h^2 - r^2)^3
  static R poly6(R r2, R h) {
    if (r2 >= h * h || r2 < (R)0) return (R)0;
    R h2 = h * h;
    R t = h2 - r2;
    return (R)315.0 / ((R)64.0 * Consts<R>::pi() * h2 * h2 * h2 * h2 * h) * t * t * t;
  }
  // spiky gradient (fluid3.rs:232-240): -45/(pi h^6) (h - r)^2 r_vec / r
  static void spiky_grad(R rx, R ry, R rz, R r, R h, R& gx_, R& gy_, R& gz_) {
    if (r >= h || r < (R)kEps) {
      gx_ = gy_ = gz_ = 0;
      return;
    }
    R s = (R)-45.0 / (Consts<R>::pi() * h * h * h * h * h * h) * (h - r) * (h - r);
    gx_ = rx / r * s;
    gy_ = ry / r * s;
    gz_ = rz / r * s;
  }
  static R pressure(R density, R rest_density, R stiffness, R gamma, int pow_mode = 1) {
    return Fluid<R>::pressure(density, rest_density, stiffness, gamma, pow_mode);
  }
  // Monaghan term (fluid3.rs:254-270)
  static R artificial_pressure(R dx, R dy, R dz, R vx, R vy, R vz, R r_sq, R h, R rho_bar, R c, R alpha) {
    R vd = dot3(vx, vy, vz, dx, dy, dz);
    if (vd >= (R)0) return (R)0;
    R mu = h * vd / (r_sq + (R)0.01f * h * h);
    return -alpha * c * mu / rmax(rho_bar, (R)kEps);
  }
  static R cohesion(R dist, R h) { return dist >= h ? (R)0 : (R)1.0 - dist / h; }

  size_t add_particles_phase(const float* xyz, const uint8_t* ph, size_t n_in) {
    size_t room = cap > particles.size() ? cap - particles.size() : 0;
    size_t n = std::min(room, n_in);
    for (size_t i = 0; i < n; i++) {
      uint8_t p = ph ? ph[i] : 0;
      size_t k = std::min<size_t>(p, 3);
      Particle3<R> q;
      q.x = (R)xyz[3 * i];
      q.y = (R)xyz[3 * i + 1];
      q.z = (R)xyz[3 * i + 2];
      q.vx = q.vy = q.vz = 0;
      q.density = (R)cfg.phase_rest_density[k];
      q.pressure = 0;
      q.mass = rmax((R)cfg.phase_mass[k], (R)0);
      q.phase = p;
      particles.push_back(q);
    }
    return n;
  }

  // ---- grid (fluid3.rs:282-343) ----
  struct Key {
    int32_t x, y, z;
    bool operator==(const Key& o) const { return x == o.x && y == o.y && z == o.z; }
  };
  struct KeyHash {
    size_t operator()(const Key& k) const {
      return ((size_t)(uint32_t)k.x * 73856093u) ^ ((size_t)(uint32_t)k.y * 19349663u) ^ ((size_t)(uint32_t)k.z * 83492791u);
    }
  };
  std::unordered_map<Key, std::vector<uint32_t>, KeyHash> grid;

  void cell_of(R x, R y, R z, int32_t& cx, int32_t& cy, int32_t& cz) const {
    R hg = (R)cfg.smoothing_length;
    cx = sat_i32(std::floor(x / hg));
    cy = sat_i32(std::floor(y / hg));
    cz = sat_i32(std::floor(z / hg));
  }
  void rebuild_grid() {
    for (auto& kv : grid) kv.second.clear();
    for (size_t i = 0; i < particles.size(); i++) {
      const auto& p = particles[i];
      if (!finite(p.x) || !finite(p.y) || !finite(p.z)) continue;
      Key k;
      cell_of(p.x, p.y, p.z, k.x, k.y, k.z);
      grid[k].push_back((uint32_t)i);
    }
  }
  // oz outer, oy, ox inner; ids ascending; keep d2 < h*h (includes i)
  void neighbors_of(R px, R py, R pz, const std::vector<Particle3<R>>& ps, std::vector<uint32_t>& out) const {
    out.clear();
    R hg = (R)cfg.smoothing_length;
    int32_t cx, cy, cz;
    cell_of(px, py, pz, cx, cy, cz);
    for (int oz = -1; oz <= 1; oz++)
      for (int oy = -1; oy <= 1; oy++)
        for (int ox = -1; ox <= 1; ox++) {
          int64_t xx = (int64_t)cx + ox, yy = (int64_t)cy + oy, zz = (int64_t)cz + oz;
          if (xx < INT32_MIN || xx > INT32_MAX || yy < INT32_MIN || yy > INT32_MAX || zz < INT32_MIN ||
              zz > INT32_MAX)
            continue;
          auto it = grid.find(Key{(int32_t)xx, (int32_t)yy, (int32_t)zz});
          if (it == grid.end()) continue;
          for (uint32_t j : it->second) {
            R dx = ps[j].x - px, dy = ps[j].y - py, dz = ps[j].z - pz;
            R d2 = dot3(dx, dy, dz, dx, dy, dz);
            if (d2 < hg * hg) out.push_back(j);
          }
        }
  }

  // ---- density + pressure (fluid3.rs:639-658) ----
  void compute_density_pressure(R h) {
    std::vector<uint32_t> nb;
    R rho_cap = (R)3.0 * rmax((R)cfg.rest_density, (R)kEps);
    for (size_t i = 0; i < particles.size(); i++) {
      const auto& pi = particles[i];
      neighbors_of(pi.x, pi.y, pi.z, particles, nb);
      R rho = 0;
      for (uint32_t j : nb) {
        R dx = particles[j].x - pi.x, dy = particles[j].y - pi.y, dz = particles[j].z - pi.z;
        rho += particles[j].mass * poly6(dot3(dx, dy, dz, dx, dy, dz), h);
      }
      particles[i].density = rclamp(rho, (R)0, rho_cap);
    }
    for (auto& p : particles) {
      R rho0 = (R)cfg.phase_rest_density[std::min<int>(p.phase, 3)];
      p.pressure = pressure(p.density, rho0, (R)cfg.stiffness, (R)cfg.gamma, pow_mode);
    }
  }

  // ---- pressure force (+AV, cohesion) (fluid3.rs:1040-1090) ----
  void compute_forces(R h) {
    std::vector<uint32_t> nb;
    size_t n = particles.size();
    fx.assign(n, 0);
    fy.assign(n, 0);
    fz.assign(n, 0);
    R c_s = std::sqrt(rmax((R)cfg.stiffness, (R)0));
    for (size_t i = 0; i < n; i++) {
      const auto& P = particles[i];
      neighbors_of(P.x, P.y, P.z, particles, nb);
      R rho_i = rmax(P.density, (R)kEps);
      R p_i = P.pressure;
      R fxi = 0, fyi = 0, fzi = 0;
      for (uint32_t j : nb) {
        if (j == i) continue;
        const auto& pj = particles[j];
        R rho_j = rmax(pj.density, (R)kEps);
        R dx = P.x - pj.x, dy = P.y - pj.y, dz = P.z - pj.z;
        R dist = std::sqrt(dot3(dx, dy, dz, dx, dy, dz));
        R gx_, gy_, gz_;
        spiky_grad(dx, dy, dz, dist, h, gx_, gy_, gz_);
        R term = p_i / (rho_i * rho_i) + pj.pressure / (rho_j * rho_j);
        if ((R)cfg.artificial_viscosity > (R)0 && dist > (R)kEps) {
          R rho_bar = (R)0.5 * (rho_i + rho_j);
          term += artificial_pressure(dx, dy, dz, P.vx - pj.vx, P.vy - pj.vy, P.vz - pj.vz, dist * dist, h, rho_bar,
                                      c_s, (R)cfg.artificial_viscosity);
        }
        R mt = pj.mass * term;
        fxi -= gx_ * mt;
        fyi -= gy_ * mt;
        fzi -= gz_ * mt;
        if ((R)cfg.surface_tension > (R)0 && dist > (R)kEps) {
          R coh = cohesion(dist, h);
          if (coh > (R)0) {
            R s = (R)cfg.surface_tension * P.mass * pj.mass * coh;
            fxi -= dx / dist * s;
            fyi -= dy / dist * s;
            fzi -= dz / dist * s;
          }
        }
      }
      if (cfg.boundary_particles) ghost_force(P.x, P.y, P.z, p_i / (rho_i * rho_i), h, fxi, fyi, fzi);
      fx[i] = fxi;
      fy[i] = fyi;
      fz[i] = fzi;
    }
  }

  // ---- integrate (fluid3.rs:1092-1138) ----
  void integrate(R h, R dt, Mode mode) {
    std::vector<uint32_t> nb;
    size_t n = particles.size();
    std::vector<Particle3<R>> snap;
    if (mode == JACOBI) snap = particles;
    const std::vector<Particle3<R>>& src = (mode == JACOBI) ? snap : particles;
    R visc = (R)cfg.viscosity, vmax = (R)cfg.max_velocity;
    for (size_t i = 0; i < n; i++) {
      neighbors_of(src[i].x, src[i].y, src[i].z, src, nb);
      R rho_i = rmax(src[i].density, (R)kEps);
      R ax = gx + fx[i] / rho_i, ay = gy + fy[i] / rho_i, az = gz + fz[i] / rho_i;
      if (turb.on) turbulence_accel3(turb, src[i].x, src[i].y, src[i].z, time, ax, ay, az);
      R vx = src[i].vx + ax * dt, vy = src[i].vy + ay * dt, vz = src[i].vz + az * dt;
      if (visc > (R)0) {
        R sx = 0, sy = 0, sz = 0;
        for (uint32_t j : nb) {
          if (j == i) continue;
          const auto& pj = src[j];
          R rho_bar = (R)0.5 * (rho_i + rmax(pj.density, (R)kEps));
          R dx = pj.x - src[i].x, dy = pj.y - src[i].y, dz = pj.z - src[i].z;
          R w = poly6(dot3(dx, dy, dz, dx, dy, dz), h);
          R mr = pj.mass / rho_bar;
          sx += (pj.vx - src[i].vx) * mr * w;
          sy += (pj.vy - src[i].vy) * mr * w;
          sz += (pj.vz - src[i].vz) * mr * w;
        }
        vx += sx * visc;
        vy += sy * visc;
        vz += sz * visc;
      }
      R speed = std::sqrt(dot3(vx, vy, vz, vx, vy, vz));
      if (speed > vmax) {
        R sc = vmax / speed;
        vx *= sc;
        vy *= sc;
        vz *= sc;
      }
      if (!finite(vx) || !finite(vy) || !finite(vz)) vx = vy = vz = 0;
      R nx = src[i].x + vx * dt, ny = src[i].y + vy * dt, nz = src[i].z + vz * dt;
      if (!finite(nx) || !finite(ny) || !finite(nz)) {
        nx = src[i].x;
        ny = src[i].y;
        nz = src[i].z;
      }
      particles[i].vx = vx;
      particles[i].vy = vy;
      particles[i].vz = vz;
      particles[i].x = nx;
      particles[i].y = ny;
      particles[i].z = nz;
    }
  }

  // ---- particle vs static body (fluid3.rs:471-590, identity rotation) ----
  static bool collide(R px, R py, R pz, R pr, const Body3& b, R& nx, R& ny, R& nz, R& depth) {
    R rx = px - (R)b.px, ry = py - (R)b.py, rz = pz - (R)b.pz;
    if (b.shape == 0) {
      R dist = std::sqrt(dot3(rx, ry, rz, rx, ry, rz));
      R radius = (R)b.a;
      if (dist >= radius + pr) return false;
      if (dist > (R)kEps) {
        nx = rx / dist;
        ny = ry / dist;
        nz = rz / dist;
      } else {
        nx = 1;
        ny = 0;
        nz = 0;
      }
      depth = radius + pr - dist;
      return true;
    }
    if (b.shape == 1) {
      R hx = (R)b.a, hy = (R)b.b, hz = (R)b.c;
      R cxl = rclamp(rx, -hx, hx), cyl = rclamp(ry, -hy, hy), czl = rclamp(rz, -hz, hz);
      R ddx = rx - cxl, ddy = ry - cyl, ddz = rz - czl;
      if (dot3(ddx, ddy, ddz, ddx, ddy, ddz) > (R)kEpsSq) {
        R dist = std::sqrt(dot3(ddx, ddy, ddz, ddx, ddy, ddz));
        if (dist >= pr) return false;
        nx = ddx / dist;
        ny = ddy / dist;
        nz = ddz / dist;
        depth = pr - dist;
        return true;
      }
      R dx = hx - std::fabs(rx), dy = hy - std::fabs(ry), dz = hz - std::fabs(rz);
      // signum().copysign(1.0) = +1 (a NaN stays a positive NaN)
      if (dx <= dy && dx <= dz) {
        nx = (rx != rx) ? std::fabs(rx) : (R)1;
        ny = 0;
        nz = 0;
        depth = pr + dx;
      } else if (dy <= dz) {
        nx = 0;
        ny = (ry != ry) ? std::fabs(ry) : (R)1;
        nz = 0;
        depth = pr + dy;
      } else {
        nx = 0;
        ny = 0;
        nz = (rz != rz) ? std::fabs(rz) : (R)1;
        depth = pr + dz;
      }
      return true;
    }
    // capsule along local y
    R r = (R)b.a, hl = (R)b.b;
    R sy = rclamp(ry, -hl, hl);
    R ddx = rx, ddy = ry - sy, ddz = rz;
    if (dot3(ddx, ddy, ddz, ddx, ddy, ddz) > (R)kEpsSq) {
      R dist = std::sqrt(dot3(ddx, ddy, ddz, ddx, ddy, ddz));
      if (dist >= r + pr) return false;
      nx = ddx / dist;
      ny = ddy / dist;
      nz = ddz / dist;
      depth = r + pr - dist;
      return true;
    }
    // on the axis: radial direction (x, 0, z) by glam's normalize_or_zero
    // (multiplication by the reciprocal length), else +x
    R l2 = dot3(rx, (R)0, rz, rx, (R)0, rz);
    if (l2 > (R)kEpsSq) {
      R rcp = (R)1 / std::sqrt(l2);
      if (finite(rcp) && rcp > (R)0) {
        nx = rx * rcp;
        ny = (R)0 * rcp;
        nz = rz * rcp;
      } else {
        nx = ny = nz = 0;
      }
    } else {
      nx = 1;
      ny = 0;
      nz = 0;
    }
    depth = pr + r - std::sqrt(dot3(ddx, ddy, ddz, ddx, ddy, ddz));
    return true;
  }

  // boundary pass (fluid3.rs:1140-1176): statics, no impulse
  void boundaries() {
    R pr = rmax((R)cfg.particle_radius, (R)0);
    for (auto& p : particles) {
      for (const Body3& b : bodies) {
        R nx, ny, nz, depth;
        if (!collide(p.x, p.y, p.z, pr, b, nx, ny, nz, depth)) continue;
        if (depth <= (R)0) continue;
        p.x = p.x + nx * depth;
        p.y = p.y + ny * depth;
        p.z = p.z + nz * depth;
        R vn = dot3(p.vx, p.vy, p.vz, nx, ny, nz);
        if (vn < (R)0) {
          p.vx -= nx * vn;
          p.vy -= ny * vn;
          p.vz -= nz * vn;
          if ((R)cfg.wall_friction > (R)0) {
            R mu = rclamp((R)cfg.wall_friction, (R)0, (R)1);
            R vtx = p.vx, vty = p.vy, vtz = p.vz;
            R wvx = 0, wvy = 0, wvz = 0;
            R wdot = dot3(wvx, wvy, wvz, nx, ny, nz);
            R wtx = wvx - nx * wdot, wty = wvy - ny * wdot, wtz = wvz - nz * wdot;
            R dvx = (wtx - vtx) * mu, dvy = (wty - vty) * mu, dvz = (wtz - vtz) * mu;
            p.vx += dvx;
            p.vy += dvy;
            p.vz += dvz;
          }
        }
      }
    }
  }

  // ---- the fluid phase with the engine's bodies (fluid3.rs:591-607, 1140-1213) ----
  // Particle vs a body with its transform (fluid3.rs:471-586); also the
  // contact point on the body. local = inverse(rotation) * (p - position),
  // the inverse of a unit quaternion being its conjugate.
  static bool collide_q(R px, R py, R pz, R pr, const Body3& b, R& nx, R& ny, R& nz, R& depth, R& cx, R& cy,
                        R& cz) {
    const R qx = (R)b.qx, qy = (R)b.qy, qz = (R)b.qz, qw = (R)b.qw;
    const R bx = (R)b.px, by = (R)b.py, bz = (R)b.pz;
    R rx = px - bx, ry = py - by, rz = pz - bz;
    if (b.shape == 0) {
      R dist = std::sqrt(dot3(rx, ry, rz, rx, ry, rz));
      R radius = (R)b.a;
      if (dist >= radius + pr) return false;
      if (dist > (R)kEps) {
        nx = rx / dist, ny = ry / dist, nz = rz / dist;
      } else {
        nx = 1, ny = 0, nz = 0;
      }
      depth = radius + pr - dist;
      cx = bx + nx * radius, cy = by + ny * radius, cz = bz + nz * radius;
      return true;
    }
    if (b.shape == 3) {  // nearest vertex sphere; the first of equal depths
      bool hit = false;
      R best = 0;
      for (size_t k = 0; k + 2 < b.hull.size(); k += 3) {
        const R vx = (R)b.hull[k], vy = (R)b.hull[k + 1], vz = (R)b.hull[k + 2];
        const R dx = px - vx, dy = py - vy, dz = pz - vz;
        const R dist = std::sqrt(dot3(dx, dy, dz, dx, dy, dz));
        if (!(dist < pr)) continue;
        const R d = pr - dist;
        if (hit && best >= d) continue;
        hit = true;
        best = d;
        if (dist > (R)kEps) {
          nx = dx / dist, ny = dy / dist, nz = dz / dist;
        } else {
          nx = 1, ny = 0, nz = 0;
        }
        depth = d;
        cx = vx, cy = vy, cz = vz;
      }
      return hit;
    }
    R lx, ly, lz;
    qrot(-qx, -qy, -qz, qw, rx, ry, rz, lx, ly, lz);
    if (b.shape == 1) {
      const R hx = (R)b.a, hy = (R)b.b, hz = (R)b.c;
      const R kx = rclamp(lx, -hx, hx), ky = rclamp(ly, -hy, hy), kz = rclamp(lz, -hz, hz);
      const R ddx = lx - kx, ddy = ly - ky, ddz = lz - kz;
      if (dot3(ddx, ddy, ddz, ddx, ddy, ddz) > (R)kEpsSq) {
        const R dist = std::sqrt(dot3(ddx, ddy, ddz, ddx, ddy, ddz));
        if (dist >= pr) return false;
        qrot(qx, qy, qz, qw, ddx / dist, ddy / dist, ddz / dist, nx, ny, nz);
        depth = pr - dist;
      } else {
        // least-penetration axis, sign signum().copysign(1.0) = +1 (NaN: |NaN|)
        const R dx = hx - std::fabs(lx), dy = hy - std::fabs(ly), dz = hz - std::fabs(lz);
        R ax = 0, ay = 0, az = 0, s, d;
        if (dx <= dy && dx <= dz) {
          ax = 1, s = (lx != lx) ? std::fabs(lx) : (R)1, d = dx;
        } else if (dy <= dz) {
          ay = 1, s = (ly != ly) ? std::fabs(ly) : (R)1, d = dy;
        } else {
          az = 1, s = (lz != lz) ? std::fabs(lz) : (R)1, d = dz;
        }
        qrot(qx, qy, qz, qw, ax * s, ay * s, az * s, nx, ny, nz);
        depth = pr + d;
      }
      qrot(qx, qy, qz, qw, kx, ky, kz, cx, cy, cz);
      cx = cx + bx, cy = cy + by, cz = cz + bz;
      return true;
    }
    // capsule along the local y axis
    const R r = (R)b.a, hl = (R)b.b;
    const R sy = rclamp(ly, -hl, hl);
    const R ddx = lx - (R)0, ddy = ly - sy, ddz = lz - (R)0;
    const R l2 = dot3(ddx, ddy, ddz, ddx, ddy, ddz);
    R ox, oy, oz;  // local contact point seg + dir * r
    if (l2 > (R)kEpsSq) {
      const R dist = std::sqrt(l2);
      if (dist >= r + pr) return false;
      qrot(qx, qy, qz, qw, ddx / dist, ddy / dist, ddz / dist, nx, ny, nz);
      depth = r + pr - dist;
      R ux = 0, uy = 0, uz = 0;  // diff.normalize_or_zero()
      const R rcp = (R)1 / std::sqrt(l2);
      if (finite(rcp) && rcp > (R)0) ux = ddx * rcp, uy = ddy * rcp, uz = ddz * rcp;
      ox = (R)0 + ux * r, oy = sy + uy * r, oz = (R)0 + uz * r;
    } else {
      // on the axis: the radial direction (x, 0, z), else +x
      R ux = 1, uy = 0, uz = 0;
      const R q2 = dot3(lx, (R)0, lz, lx, (R)0, lz);
      if (q2 > (R)kEpsSq) {
        const R rcp = (R)1 / std::sqrt(q2);
        if (finite(rcp) && rcp > (R)0) {
          ux = lx * rcp, uy = (R)0 * rcp, uz = lz * rcp;
        } else {
          ux = uy = uz = 0;
        }
      }
      qrot(qx, qy, qz, qw, ux, uy, uz, nx, ny, nz);
      depth = pr + r - std::sqrt(l2);
      ox = (R)0 + ux * r, oy = sy + uy * r, oz = (R)0 + uz * r;
    }
    qrot(qx, qy, qz, qw, ox, oy, oz, cx, cy, cz);
    cx = cx + bx, cy = cy + by, cz = cz + bz;
    return true;
  }

  // boundary pass with reactions (fluid3.rs:1140-1178), particle by particle
  void boundaries_q() {
    R pr = rmax((R)cfg.particle_radius, (R)0);
    for (auto& p : particles) {
      for (Body3& b : bodies) {
        R nx, ny, nz, depth, cx, cy, cz;
        if (!collide_q(p.x, p.y, p.z, pr, b, nx, ny, nz, depth, cx, cy, cz)) continue;
        if (depth <= (R)0) continue;
        p.x = p.x + nx * depth;
        p.y = p.y + ny * depth;
        p.z = p.z + nz * depth;
        R vn = dot3(p.vx, p.vy, p.vz, nx, ny, nz);
        if (vn < (R)0) {
          p.vx -= nx * vn;
          p.vy -= ny * vn;
          p.vz -= nz * vn;
          if (!b.is_static) b.sleeping = false;
          const R vm = vn * p.mass;
          b.apply_impulse((float)(nx * vm), (float)(ny * vm), (float)(nz * vm), (float)cx, (float)cy, (float)cz);
          if ((R)cfg.wall_friction > (R)0) {
            R mu = rclamp((R)cfg.wall_friction, (R)0, (R)1);
            R vtx = p.vx, vty = p.vy, vtz = p.vz;
            R wvx = (R)b.vx, wvy = (R)b.vy, wvz = (R)b.vz;
            R wdot = dot3(wvx, wvy, wvz, nx, ny, nz);
            R wtx = wvx - nx * wdot, wty = wvy - ny * wdot, wtz = wvz - nz * wdot;
            R dvx = (wtx - vtx) * mu, dvy = (wty - vty) * mu, dvz = (wtz - vtz) * mu;
            p.vx += dvx;
            p.vy += dvy;
            p.vz += dvz;
            b.apply_impulse((float)(-dvx * p.mass), (float)(-dvy * p.mass), (float)(-dvz * p.mass), (float)cx,
                            (float)cy, (float)cz);
          }
        }
      }
    }
  }

  // FluidState3::sample_pressure (fluid3.rs:345-369): sum over the 27 cells
  // around floor(point / h), h = max(smoothing_length, EPS), of
  // m_j (p_j / max(rho_j, EPS)) poly6(r^2) for r^2 < h*h; max(p, 0)
  R sample_pressure3(R ptx, R pty, R ptz) const {
    const R h = rmax((R)cfg.smoothing_length, (R)kEps);
    const int32_t cx = sat_i32(std::floor(ptx / h)), cy = sat_i32(std::floor(pty / h)), cz = sat_i32(std::floor(ptz / h));
    R p = 0;
    for (int oz = -1; oz <= 1; oz++)
      for (int oy = -1; oy <= 1; oy++)
        for (int ox = -1; ox <= 1; ox++) {
          const int64_t xx = (int64_t)cx + ox, yy = (int64_t)cy + oy, zz = (int64_t)cz + oz;
          if (xx < INT32_MIN || xx > INT32_MAX || yy < INT32_MIN || yy > INT32_MAX || zz < INT32_MIN ||
              zz > INT32_MAX)
            continue;
          auto it = grid.find(Key{(int32_t)xx, (int32_t)yy, (int32_t)zz});
          if (it == grid.end()) continue;
          for (uint32_t j : it->second) {
            const auto& pj = particles[j];
            const R dx = pj.x - ptx, dy = pj.y - pty, dz = pj.z - ptz;
            const R r2 = dot3(dx, dy, dz, dx, dy, dz);
            if (r2 < h * h) p += pj.mass * (pj.pressure / rmax(pj.density, (R)kEps)) * poly6(r2, h);
          }
        }
    return rmax(p, (R)0);
  }

  // buoyancy + drag over the dynamic bodies' surfaces (fluid3.rs:1180-1213)
  void buoyancy3(R dt) {
    rebuild_grid();
    std::vector<float> smp;
    for (Body3& b : bodies) {
      if (b.is_static) continue;
      smp.clear();
      surface_samples3(b, smp);
      if (smp.empty()) continue;
      const float drag = std::max(cfg.drag, 0.0f);
      bool wet = false;
      for (size_t q = 0; q < smp.size(); q += 7) {
        const float ptx = smp[q], pty = smp[q + 1], ptz = smp[q + 2];
        const float nx = smp[q + 3], ny = smp[q + 4], nz = smp[q + 5], area = smp[q + 6];
        const float p = (float)sample_pressure3((R)ptx, (R)pty, (R)ptz);
        if (p <= 0.0f) continue;
        wet = true;
        const float rx = ptx - b.px, ry = pty - b.py, rz = ptz - b.pz;
        // (velocity + angular_velocity x r) - wind
        const float vrx = (b.vx + (b.wy * rz - b.wz * ry)) - wind_x;
        const float vry = (b.vy + (b.wz * rx - b.wx * rz)) - wind_y;
        const float vrz = (b.vz + (b.wx * ry - b.wy * rx)) - wind_z;
        const float speed = std::sqrt(vrx * vrx + vry * vry + vrz * vrz);
        const float pa = p * area;
        float fx = -nx * pa, fy = -ny * pa, fz = -nz * pa;
        if (speed > kEps) {
          const float c = drag * area * speed;
          fx -= vrx * c;
          fy -= vry * c;
          fz -= vrz * c;
        }
        b.apply_force(fx, fy, fz, ptx, pty, ptz, (float)dt);
      }
      if (wet) b.sleeping = false;
    }
  }

  void substep_bodies(R dt, Mode mode) {
    R h = rmax((R)cfg.smoothing_length, (R)kEps);
    rebuild_grid();
    compute_density_pressure(h);
    if (cfg.boundary_particles) {
      refresh_ghosts();
      ghost_density(h);
    }
    compute_forces(h);
    integrate(h, dt, mode);
    boundaries_q();
    bool dyn = false;
    for (const Body3& b : bodies) dyn = dyn || !b.is_static;
    if (dyn) buoyancy3(dt);
  }

  // FluidState3::step_fluid (fluid3.rs:591-607) with `bodies` as the
  // engine's bodies: no clock
  void step_fluid(R dt, Mode mode) {
    if (!cfg.enabled || particles.empty() || !(dt > (R)0)) return;
    uint32_t n = cfl_substeps(dt);
    R sub = dt / (R)n;
    for (uint32_t k = 0; k < n; k++) substep_bodies(sub, mode);
  }

  // CFL substeps (fluid3.rs:610-637)
  uint32_t cfl_substeps(R dt) const {
    uint32_t mx = std::max<uint32_t>(cfg.max_substeps, 1);
    if ((R)cfg.cfl <= (R)0 || mx <= 1) return 1;
    R h = rmax((R)cfg.smoothing_length, (R)kEps);
    R rho0 = rmax((R)cfg.rest_density, (R)kEps);
    R c0 = ((R)cfg.gamma == (R)1.0) ? std::sqrt(rmax((R)cfg.stiffness, (R)0))
                                    : std::sqrt((R)cfg.gamma * rmax((R)cfg.stiffness, (R)0) * rho0);
    R vm = 0;
    for (const auto& p : particles) vm = rmax(vm, std::sqrt(dot3(p.vx, p.vy, p.vz, p.vx, p.vy, p.vz)));
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
    k = std::max<int64_t>(1, std::min<int64_t>(k, mx));
    return (uint32_t)k;
  }

  // FluidState3::resample (fluid3.rs:923-990)
  void resample(R h) {
    const float rest = std::max(cfg.rest_density, kEps);
    const R split_lo = (R)(cfg.split_density_ratio * rest), merge_hi = (R)(cfg.merge_density_ratio * rest);
    const R min_mass = (R)(std::max(cfg.particle_mass, kEps) * 0.125f);
    const size_t n = particles.size();
    std::vector<char> absorbed(n, 0);
    const R md = (R)0.25 * h, merge_d2 = md * md;
    for (size_t i = 0; i < n; i++) {
      if (absorbed[i] || particles[i].density <= merge_hi) continue;
      for (size_t j = i; j-- > 0;) {
        if (absorbed[j] || particles[j].density <= merge_hi) continue;
        const R dx = particles[i].x - particles[j].x, dy = particles[i].y - particles[j].y;
        const R dz = particles[i].z - particles[j].z;
        if (dx * dx + dy * dy + dz * dz < merge_d2) {
          const R mi = particles[i].mass, mj = particles[j].mass, mt = mi + mj;
          if (mt > (R)kEps) {
            particles[i].vx = (particles[i].vx * mi + particles[j].vx * mj) / mt;
            particles[i].vy = (particles[i].vy * mi + particles[j].vy * mj) / mt;
            particles[i].vz = (particles[i].vz * mi + particles[j].vz * mj) / mt;
            particles[i].mass = mt;
          }
          absorbed[j] = 1;
          break;
        }
      }
    }
    std::vector<Particle3<R>> out;
    const R off = (R)0.25 * h;
    for (size_t i = 0; i < n; i++) {
      if (absorbed[i]) continue;
      const Particle3<R>& p = particles[i];
      if (p.density < split_lo && p.mass > min_mass && out.size() + 1 < 4096) {  // MAX_PARTICLES_3D
        Particle3<R> a = p, b = p;
        a.mass = b.mass = p.mass * (R)0.5;
        a.x = p.x + off, a.y = p.y + (R)0, a.z = p.z + (R)0;
        b.x = p.x - off, b.y = p.y - (R)0, b.z = p.z - (R)0;
        out.push_back(a);
        out.push_back(b);
      } else {
        out.push_back(p);
      }
    }
    particles.swap(out);
  }

  void substep(R dt, Mode mode) {
    R h = rmax((R)cfg.smoothing_length, (R)kEps);
    rebuild_grid();
    compute_density_pressure(h);
    if (cfg.adaptive_resolution) {  // fluid3.rs:1008-1016
      resample(h);
      rebuild_grid();
      compute_density_pressure(h);
    }
    if (cfg.boundary_particles) {  // fluid3.rs:1018-1026
      refresh_ghosts();
      ghost_density(h);
    }
    compute_forces(h);
    integrate(h, dt, mode);
    boundaries();
  }

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
