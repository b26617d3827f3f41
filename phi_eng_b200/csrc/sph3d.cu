// 3D SPH fluid step (crates/dynamics/src/fluid3.rs) on the GPU, behind the
// engine's phieng_world3_* C ABI (crates/engine/src/ffi.rs:3199-3760).
//
// Same design as the 2D chain (sph_kernels.cu): a power-of-two bucket grid
// over cells of size h, bucket = ((cz - cz0) mod D) * H * W + ((cy - cy0) mod
// H) * W + ((cx - cx0) mod W); a counting sort by bucket with the in-bucket
// rank by id (the shared scan + placement of sph_kernels.cu, a 3D gather
// here), so each particle's candidates are 9 contiguous slot ranges (rows
// oz, oy = -1..1 of three consecutive x cells) visited in the reference's
// order (oz outer, oy, ox inner, ascending id, fluid3.rs:319-343); the
// density pass records one 32-bit neighbour mask per row and the force pass
// walks them. Arithmetic is glam 0.29's scalar Vec3 in f32 (dot =
// (x*x + y*y) + z*z, component-wise operators), IEEE division and square
// root, no FMA contraction: per-pair results are bit-identical to the
// reference's. The integrate reads pre-step neighbour state (Jacobi), as in
// 2D. Static sphere / box / capsule walls as phieng_world3_add_body creates
// them (identity rotation: glam's quaternion products with the identity
// return the vector unchanged).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/phieng_sph.h"
#include "sph_host.h"
#include "sph_kernels.h"
#include "sph_noise.cuh"
#include "sph_snapshot.h"
#include "sph_warp.cuh"

using namespace phieng;
using namespace phieng::host;

namespace phieng {
namespace {

constexpr uint32_t kMaxParticles3D = 4096;  // MAX_PARTICLES_3D (fluid3.rs:28)

// Most particles one 3D resample pass (fluid3.rs:923-990) can leave from n:
// a split only happens while the output holds fewer than MAX_PARTICLES_3D - 1
// particles, so at most MAX_PARTICLES_3D / 2 particles split.
inline uint32_t resample_bound3(uint32_t n) { return n + std::min(n, kMaxParticles3D / 2); }
constexpr uint32_t kMaskBits3 = 32;

struct GridPlan3 {
  int32_t cx0, cy0, cz0;
  uint32_t log2w, log2h, log2d;
  uint32_t maskw, maskh, maskd;
  uint32_t nbuckets;
  float hg;
  uint32_t sentinel;
};

// One cell of the 3D boundary ghosts' hash grid (count 0 = empty slot).
struct GhostCell3 {
  int32_t cx, cy, cz;
  uint32_t start, count;
};

__host__ __device__ inline uint32_t ghost_cell_hash3(int32_t cx, int32_t cy, int32_t cz, uint32_t mask) {
  uint32_t h = (uint32_t)cx * 0x9E3779B1u ^ ((uint32_t)cy * 0x85EBCA77u) ^ ((uint32_t)cz * 0xC2B2AE3Du + 0x165667B1u);
  h ^= h >> 15;
  return h & mask;
}

// A body of phieng_sph3_step_fluid as the boundary pass reads it: shape (0
// sphere, 1 box, 2 capsule, 3 hull), position, rotation (unit quaternion),
// shape sizes, the half extents of its padded world bounding box, dyn = the
// body takes reactions or moves (its contacts run in the ordered pass), and
// for a hull its world-space vertices [vfirst, vfirst + vcount).
struct DevBodyQ3 {
  int32_t shape;
  uint32_t dyn;
  float px, py, pz;
  float qx, qy, qz, qw;
  float a, b, c;
  float ex, ey, ez;
  uint32_t vfirst, vcount;
};

// The motion state of a body in the fluid phase (RigidBody3): velocity,
// angular velocity, inverse mass, the world inverse inertia R I^-1 R^T
// (column-major, fixed over the call: the transform does not change), the
// flags, and its buoyancy samples [sample_first, sample_first + sample_count).
struct DynBody3 {
  float vx, vy, vz, wx, wy, wz;
  float inv_mass;
  float iw[9];
  uint32_t is_static, sleeping, sample_first, sample_count;
};

struct StepParams3 {
  GridPlan3 grid;
  float hg2, hk, hk2;
  float c_poly6;  // 315/(64 PI h2 h2 h2 h2 h), as fluid3.rs:228 evaluates it
  float c_spiky;  // -45/(PI h h h h h h), as fluid3.rs:238
  float rho_cap;
  float stiffness, gamma;
  float rest[4];
  float mass, visc, vmax, dt;
  float gx, gy, gz;
  float pr, pr_pad, mu, av_alpha, c_s, surface_tension;
  uint32_t flags, nbodies, uniform_phase;
  // ambient turbulence (F_TURB; TurbulenceConfig3, ambient.rs:251-266)
  float turb_amp, turb_freq, turb_tscale;
  uint32_t turb_seed, turb_oct;  // octaves already clamped to 1..8
  const float* clock;            // device word holding the world clock of the current step
  // boundary ghosts (F_GHOST, fluid3.rs:719-922): cell-grouped positions,
  // their q = p / max(rho, EPS)^2 this substep, the cell table
  const float4* gpos;
  float* gq;
  const GhostCell3* gtab;
  uint32_t gtab_mask, nghost;
  float gmass, rest0;
  // the engine's bodies (F_QBODIES, phieng_sph3_step_fluid): replace the
  // world's statics; with F_DYNAMIC a particle's contact with a body that
  // reacts defers the rest of its body loop to the ordered pass (defer[id] =
  // the body it resumes from, dcount[id] = 1)
  const DevBodyQ3* qbodies;
  const float4* hullv;
  uint32_t* defer;
  uint32_t* dcount;
};

// Static body: shape 0 sphere (a = radius), 1 box (a, b, c half extents),
// 2 capsule (a = radius, b = half length along y); ex, ey, ez = half extents
// of its axis-aligned bounding box padded by 0.1%.
struct DevBody3 {
  int32_t shape;
  float px, py, pz;
  float a, b, c;
  float ex, ey, ez;
};

__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz) {
  return __fadd_rn(__fadd_rn(__fmul_rn(ax, bx), __fmul_rn(ay, by)), __fmul_rn(az, bz));
}

__device__ __forceinline__ uint32_t bucket_key3(float x, float y, float z, const GridPlan3& g) {
  if (!isfinite(x) || !isfinite(y) || !isfinite(z)) return g.sentinel;
  const int32_t cx = __float2int_rd(__fdiv_rn(x, g.hg));
  const int32_t cy = __float2int_rd(__fdiv_rn(y, g.hg));
  const int32_t cz = __float2int_rd(__fdiv_rn(z, g.hg));
  const uint32_t bx = ((uint32_t)cx - (uint32_t)g.cx0) & g.maskw;
  const uint32_t by = ((uint32_t)cy - (uint32_t)g.cy0) & g.maskh;
  const uint32_t bz = ((uint32_t)cz - (uint32_t)g.cz0) & g.maskd;
  return (bz << (g.log2w + g.log2h)) | (by << g.log2w) | bx;
}

// poly6 (fluid3.rs:220-229): (((c * t) * t) * t)
__device__ __forceinline__ float poly6_3(float r2, const StepParams3& P) {
  if (r2 >= P.hk2 || r2 < 0.0f) return 0.0f;
  const float t = __fsub_rn(P.hk2, r2);
  return __fmul_rn(__fmul_rn(__fmul_rn(P.c_poly6, t), t), t);
}

// Candidate j's density term m_j * poly6(d2) when d2 < h*h (a neighbour), else +0
__device__ __forceinline__ float contrib3(float d2, float m, const StepParams3& P) {
  return d2 < P.hg2 ? __fmul_rn(m, poly6_3(d2, P)) : 0.0f;
}

// Particle vs static body (fluid3.rs:471-590) with the identity rotation.
__device__ __forceinline__ bool collide3(float px, float py, float pz, float pr, const DevBody3& b, float& nx,
                                         float& ny, float& nz, float& depth) {
  const float rx = __fsub_rn(px, b.px), ry = __fsub_rn(py, b.py), rz = __fsub_rn(pz, b.pz);
  if (b.shape == 0) {
    const float dist = __fsqrt_rn(dot3(rx, ry, rz, rx, ry, rz));
    const float rr = __fadd_rn(b.a, pr);
    if (dist >= rr) return false;
    if (dist > kEps) {
      nx = __fdiv_rn(rx, dist);
      ny = __fdiv_rn(ry, dist);
      nz = __fdiv_rn(rz, dist);
    } else {
      nx = 1.0f;
      ny = 0.0f;
      nz = 0.0f;
    }
    depth = __fsub_rn(rr, dist);
    return true;
  }
  if (b.shape == 1) {
    float cxl = rx, cyl = ry, czl = rz;  // f32::clamp (NaN passes through)
    if (cxl < -b.a) cxl = -b.a;
    if (cxl > b.a) cxl = b.a;
    if (cyl < -b.b) cyl = -b.b;
    if (cyl > b.b) cyl = b.b;
    if (czl < -b.c) czl = -b.c;
    if (czl > b.c) czl = b.c;
    const float ddx = __fsub_rn(rx, cxl), ddy = __fsub_rn(ry, cyl), ddz = __fsub_rn(rz, czl);
    const float l2 = dot3(ddx, ddy, ddz, ddx, ddy, ddz);
    if (l2 > kEpsSq) {
      const float dist = __fsqrt_rn(l2);
      if (dist >= pr) return false;
      nx = __fdiv_rn(ddx, dist);
      ny = __fdiv_rn(ddy, dist);
      nz = __fdiv_rn(ddz, dist);
      depth = __fsub_rn(pr, dist);
      return true;
    }
    const float dx = __fsub_rn(b.a, fabsf(rx)), dy = __fsub_rn(b.b, fabsf(ry)), dz = __fsub_rn(b.c, fabsf(rz));
    // signum().copysign(1.0) = +1 (a NaN stays a positive NaN)
    if (dx <= dy && dx <= dz) {
      nx = (rx != rx) ? fabsf(rx) : 1.0f;
      ny = 0.0f;
      nz = 0.0f;
      depth = __fadd_rn(pr, dx);
    } else if (dy <= dz) {
      nx = 0.0f;
      ny = (ry != ry) ? fabsf(ry) : 1.0f;
      nz = 0.0f;
      depth = __fadd_rn(pr, dy);
    } else {
      nx = 0.0f;
      ny = 0.0f;
      nz = (rz != rz) ? fabsf(rz) : 1.0f;
      depth = __fadd_rn(pr, dz);
    }
    return true;
  }
  // capsule along y: closest point on the segment [-hl, hl]
  float sy = ry;
  if (sy < -b.b) sy = -b.b;
  if (sy > b.b) sy = b.b;
  const float ddx = rx, ddy = __fsub_rn(ry, sy), ddz = rz;
  const float l2 = dot3(ddx, ddy, ddz, ddx, ddy, ddz);
  if (l2 > kEpsSq) {
    const float dist = __fsqrt_rn(l2);
    const float rr = __fadd_rn(b.a, pr);
    if (dist >= rr) return false;
    nx = __fdiv_rn(ddx, dist);
    ny = __fdiv_rn(ddy, dist);
    nz = __fdiv_rn(ddz, dist);
    depth = __fsub_rn(rr, dist);
    return true;
  }
  // on the axis: push radially, glam normalize_or_zero of (x, 0, z)
  // (multiplication by the reciprocal length), else +x
  const float r2 = dot3(rx, 0.0f, rz, rx, 0.0f, rz);
  if (r2 > kEpsSq) {
    const float rcp = __fdiv_rn(1.0f, __fsqrt_rn(r2));
    if (isfinite(rcp) && rcp > 0.0f) {
      nx = __fmul_rn(rx, rcp);
      ny = __fmul_rn(0.0f, rcp);
      nz = __fmul_rn(rz, rcp);
    } else {
      nx = ny = nz = 0.0f;
    }
  } else {
    nx = 1.0f;
    ny = 0.0f;
    nz = 0.0f;
  }
  depth = __fsub_rn(__fadd_rn(pr, b.a), __fsqrt_rn(l2));
  return true;
}

// Boundary pass (fluid3.rs:1140-1176); statics take no impulse.
__device__ __forceinline__ void walls3(float& x, float& y, float& z, float& vx, float& vy, float& vz,
                                       const DevBody3* __restrict__ bodies, const StepParams3& P) {
  for (uint32_t k = 0; k < P.nbodies; k++) {
    const DevBody3* bp = bodies + k;
    if (fabsf(x - __ldg(&bp->px)) > __ldg(&bp->ex) + P.pr_pad || fabsf(y - __ldg(&bp->py)) > __ldg(&bp->ey) + P.pr_pad ||
        fabsf(z - __ldg(&bp->pz)) > __ldg(&bp->ez) + P.pr_pad)
      continue;
    const DevBody3 b = *bp;
    float nx, ny, nz, depth;
    if (!collide3(x, y, z, P.pr, b, nx, ny, nz, depth)) continue;
    if (depth <= 0.0f) continue;
    x = __fadd_rn(x, __fmul_rn(nx, depth));
    y = __fadd_rn(y, __fmul_rn(ny, depth));
    z = __fadd_rn(z, __fmul_rn(nz, depth));
    const float vn = dot3(vx, vy, vz, nx, ny, nz);
    if (vn < 0.0f) {
      vx = __fsub_rn(vx, __fmul_rn(nx, vn));
      vy = __fsub_rn(vy, __fmul_rn(ny, vn));
      vz = __fsub_rn(vz, __fmul_rn(nz, vn));
      if (P.flags & F_FRICTION) {
        const float vtx = vx, vty = vy, vtz = vz;
        const float wdot = dot3(0.0f, 0.0f, 0.0f, nx, ny, nz);
        const float wtx = __fsub_rn(0.0f, __fmul_rn(nx, wdot));
        const float wty = __fsub_rn(0.0f, __fmul_rn(ny, wdot));
        const float wtz = __fsub_rn(0.0f, __fmul_rn(nz, wdot));
        vx = __fadd_rn(vx, __fmul_rn(__fsub_rn(wtx, vtx), P.mu));
        vy = __fadd_rn(vy, __fmul_rn(__fsub_rn(wty, vty), P.mu));
        vz = __fadd_rn(vz, __fmul_rn(__fsub_rn(wtz, vtz), P.mu));
      }
    }
  }
}

// ---------------------------------------------------------------- the engine's bodies
// Rotation of v by the unit quaternion (b, w) = (qx, qy, qz, qw), the
// expansion of q v q*: (v (w^2 - b.b) + b (2 (v.b))) + (b x v) (2 w), in this
// order (the host restates it for hull vertices and buoyancy samples).
__device__ __forceinline__ void qrot3(float qx, float qy, float qz, float qw, float vx, float vy, float vz, float& ox,
                                      float& oy, float& oz) {
  const float s = __fsub_rn(__fmul_rn(qw, qw), dot3(qx, qy, qz, qx, qy, qz));
  const float d = __fmul_rn(dot3(vx, vy, vz, qx, qy, qz), 2.0f);
  const float w2 = __fmul_rn(qw, 2.0f);
  const float cx = __fsub_rn(__fmul_rn(qy, vz), __fmul_rn(qz, vy));
  const float cy = __fsub_rn(__fmul_rn(qz, vx), __fmul_rn(qx, vz));
  const float cz = __fsub_rn(__fmul_rn(qx, vy), __fmul_rn(qy, vx));
  ox = __fadd_rn(__fadd_rn(__fmul_rn(vx, s), __fmul_rn(qx, d)), __fmul_rn(cx, w2));
  oy = __fadd_rn(__fadd_rn(__fmul_rn(vy, s), __fmul_rn(qy, d)), __fmul_rn(cy, w2));
  oz = __fadd_rn(__fadd_rn(__fmul_rn(vz, s), __fmul_rn(qz, d)), __fmul_rn(cz, w2));
}

__device__ __forceinline__ float clampf_rs(float x, float lo, float hi) {  // f32::clamp: NaN passes through
  if (x < lo) x = lo;
  if (x > hi) x = hi;
  return x;
}

// Particle vs a body with its transform (fluid3.rs:471-586): outward normal,
// depth and the contact point on the body. The local frame is
// inverse(rotation) * (p - position), the conjugate for a unit quaternion.
__device__ __noinline__ bool collide_q3(float px, float py, float pz, float pr, const DevBodyQ3& b,
                                        const float4* __restrict__ hullv, float& nx, float& ny, float& nz,
                                        float& depth, float& cx, float& cy, float& cz) {
  const float rx = __fsub_rn(px, b.px), ry = __fsub_rn(py, b.py), rz = __fsub_rn(pz, b.pz);
  if (b.shape == 0) {
    const float dist = __fsqrt_rn(dot3(rx, ry, rz, rx, ry, rz));
    if (dist >= __fadd_rn(b.a, pr)) return false;
    if (dist > kEps) {
      nx = __fdiv_rn(rx, dist), ny = __fdiv_rn(ry, dist), nz = __fdiv_rn(rz, dist);
    } else {
      nx = 1.0f, ny = 0.0f, nz = 0.0f;
    }
    depth = __fsub_rn(__fadd_rn(b.a, pr), dist);
    cx = __fadd_rn(b.px, __fmul_rn(nx, b.a));
    cy = __fadd_rn(b.py, __fmul_rn(ny, b.a));
    cz = __fadd_rn(b.pz, __fmul_rn(nz, b.a));
    return true;
  }
  if (b.shape == 3) {  // nearest vertex sphere of radius pr; the first of equal depths
    bool hit = false;
    float best = 0.0f;
    for (uint32_t k = 0; k < b.vcount; k++) {
      const float4 v = hullv[b.vfirst + k];
      const float dx = __fsub_rn(px, v.x), dy = __fsub_rn(py, v.y), dz = __fsub_rn(pz, v.z);
      const float dist = __fsqrt_rn(dot3(dx, dy, dz, dx, dy, dz));
      if (!(dist < pr)) continue;
      const float d = __fsub_rn(pr, dist);
      if (hit && best >= d) continue;
      hit = true;
      best = d;
      if (dist > kEps) {
        nx = __fdiv_rn(dx, dist), ny = __fdiv_rn(dy, dist), nz = __fdiv_rn(dz, dist);
      } else {
        nx = 1.0f, ny = 0.0f, nz = 0.0f;
      }
      depth = d;
      cx = v.x, cy = v.y, cz = v.z;
    }
    return hit;
  }
  float lx, ly, lz;
  qrot3(-b.qx, -b.qy, -b.qz, b.qw, rx, ry, rz, lx, ly, lz);
  float ox, oy, oz;  // local contact point
  if (b.shape == 1) {
    const float kx = clampf_rs(lx, -b.a, b.a), ky = clampf_rs(ly, -b.b, b.b), kz = clampf_rs(lz, -b.c, b.c);
    const float ddx = __fsub_rn(lx, kx), ddy = __fsub_rn(ly, ky), ddz = __fsub_rn(lz, kz);
    const float l2 = dot3(ddx, ddy, ddz, ddx, ddy, ddz);
    if (l2 > kEpsSq) {
      const float dist = __fsqrt_rn(l2);
      if (dist >= pr) return false;
      qrot3(b.qx, b.qy, b.qz, b.qw, __fdiv_rn(ddx, dist), __fdiv_rn(ddy, dist), __fdiv_rn(ddz, dist), nx, ny, nz);
      depth = __fsub_rn(pr, dist);
    } else {
      // least-penetration axis, sign signum().copysign(1.0) = +1 (NaN: |NaN|)
      const float dx = __fsub_rn(b.a, fabsf(lx)), dy = __fsub_rn(b.b, fabsf(ly)), dz = __fsub_rn(b.c, fabsf(lz));
      float ax = 0.0f, ay = 0.0f, az = 0.0f, sg, d;
      if (dx <= dy && dx <= dz) {
        ax = 1.0f, sg = (lx != lx) ? fabsf(lx) : 1.0f, d = dx;
      } else if (dy <= dz) {
        ay = 1.0f, sg = (ly != ly) ? fabsf(ly) : 1.0f, d = dy;
      } else {
        az = 1.0f, sg = (lz != lz) ? fabsf(lz) : 1.0f, d = dz;
      }
      qrot3(b.qx, b.qy, b.qz, b.qw, __fmul_rn(ax, sg), __fmul_rn(ay, sg), __fmul_rn(az, sg), nx, ny, nz);
      depth = __fadd_rn(pr, d);
    }
    ox = kx, oy = ky, oz = kz;
  } else {
    // capsule along the local y axis: closest point on the segment [-hl, hl]
    const float r = b.a, sy = clampf_rs(ly, -b.b, b.b);
    const float ddx = __fsub_rn(lx, 0.0f), ddy = __fsub_rn(ly, sy), ddz = __fsub_rn(lz, 0.0f);
    const float l2 = dot3(ddx, ddy, ddz, ddx, ddy, ddz);
    float ux, uy, uz;  // diff.normalize_or_zero(), or the radial direction on the axis
    if (l2 > kEpsSq) {
      const float dist = __fsqrt_rn(l2);
      if (dist >= __fadd_rn(r, pr)) return false;
      qrot3(b.qx, b.qy, b.qz, b.qw, __fdiv_rn(ddx, dist), __fdiv_rn(ddy, dist), __fdiv_rn(ddz, dist), nx, ny, nz);
      depth = __fsub_rn(__fadd_rn(r, pr), dist);
      const float rcp = __fdiv_rn(1.0f, __fsqrt_rn(l2));
      if (isfinite(rcp) && rcp > 0.0f) {
        ux = __fmul_rn(ddx, rcp), uy = __fmul_rn(ddy, rcp), uz = __fmul_rn(ddz, rcp);
      } else {
        ux = uy = uz = 0.0f;
      }
    } else {
      ux = 1.0f, uy = 0.0f, uz = 0.0f;
      const float q2 = dot3(lx, 0.0f, lz, lx, 0.0f, lz);
      if (q2 > kEpsSq) {
        const float rcp = __fdiv_rn(1.0f, __fsqrt_rn(q2));
        if (isfinite(rcp) && rcp > 0.0f) {
          ux = __fmul_rn(lx, rcp), uy = __fmul_rn(0.0f, rcp), uz = __fmul_rn(lz, rcp);
        } else {
          ux = uy = uz = 0.0f;
        }
      }
      qrot3(b.qx, b.qy, b.qz, b.qw, ux, uy, uz, nx, ny, nz);
      depth = __fsub_rn(__fadd_rn(pr, r), __fsqrt_rn(l2));
    }
    ox = __fadd_rn(0.0f, __fmul_rn(ux, r)), oy = __fadd_rn(sy, __fmul_rn(uy, r)), oz = __fadd_rn(0.0f, __fmul_rn(uz, r));
  }
  qrot3(b.qx, b.qy, b.qz, b.qw, ox, oy, oz, cx, cy, cz);
  cx = __fadd_rn(cx, b.px), cy = __fadd_rn(cy, b.py), cz = __fadd_rn(cz, b.pz);
  return true;
}

// The parallel part of the boundary pass over the engine's bodies
// (fluid3.rs:1140-1178): plain walls (statics at rest) in body order;
// returns kNoDefer, or the index of the first body marked dyn that the
// particle touches, the state left as it was before that body.
__device__ __forceinline__ uint32_t walls3q(float& x, float& y, float& z, float& vx, float& vy, float& vz,
                                            const StepParams3& P) {
  for (uint32_t k = 0; k < P.nbodies; k++) {
    const DevBodyQ3* bp = P.qbodies + k;
    // bounding-box reject (the extents include the particle radius)
    if (fabsf(x - __ldg(&bp->px)) > __ldg(&bp->ex) || fabsf(y - __ldg(&bp->py)) > __ldg(&bp->ey) ||
        fabsf(z - __ldg(&bp->pz)) > __ldg(&bp->ez))
      continue;
    const DevBodyQ3 b = *bp;
    float nx, ny, nz, depth, cx, cy, cz;
    if (!collide_q3(x, y, z, P.pr, b, P.hullv, nx, ny, nz, depth, cx, cy, cz)) continue;
    if (depth <= 0.0f) continue;
    if (b.dyn) return k;
    x = __fadd_rn(x, __fmul_rn(nx, depth));
    y = __fadd_rn(y, __fmul_rn(ny, depth));
    z = __fadd_rn(z, __fmul_rn(nz, depth));
    const float vn = dot3(vx, vy, vz, nx, ny, nz);
    if (vn < 0.0f) {
      vx = __fsub_rn(vx, __fmul_rn(nx, vn));
      vy = __fsub_rn(vy, __fmul_rn(ny, vn));
      vz = __fsub_rn(vz, __fmul_rn(nz, vn));
      if (P.flags & F_FRICTION) {  // the wall's velocity is zero
        const float wdot = dot3(0.0f, 0.0f, 0.0f, nx, ny, nz);
        const float wtx = __fsub_rn(0.0f, __fmul_rn(nx, wdot));
        const float wty = __fsub_rn(0.0f, __fmul_rn(ny, wdot));
        const float wtz = __fsub_rn(0.0f, __fmul_rn(nz, wdot));
        vx = __fadd_rn(vx, __fmul_rn(__fsub_rn(wtx, vx), P.mu));
        vy = __fadd_rn(vy, __fmul_rn(__fsub_rn(wty, vy), P.mu));
        vz = __fadd_rn(vz, __fmul_rn(__fsub_rn(wtz, vz), P.mu));
      }
    }
  }
  return kNoDefer;
}

// (Iw * t): (x_axis t.x + y_axis t.y) + z_axis t.z
__device__ __forceinline__ void mat3_vec(const float* m, float tx, float ty, float tz, float& ox, float& oy,
                                         float& oz) {
  ox = __fadd_rn(__fadd_rn(__fmul_rn(m[0], tx), __fmul_rn(m[3], ty)), __fmul_rn(m[6], tz));
  oy = __fadd_rn(__fadd_rn(__fmul_rn(m[1], tx), __fmul_rn(m[4], ty)), __fmul_rn(m[7], tz));
  oz = __fadd_rn(__fadd_rn(__fmul_rn(m[2], tx), __fmul_rn(m[5], ty)), __fmul_rn(m[8], tz));
}

// RigidBody3::apply_impulse (body.rs:1349-1361): statics ignore it; a
// dynamic body wakes, v += J * inv_mass, w += Iw (r x J).
__device__ __forceinline__ void apply_impulse3(DynBody3& d, float bpx, float bpy, float bpz, float jx, float jy,
                                               float jz, float qx, float qy, float qz) {
  if (d.is_static) return;
  d.sleeping = 0;
  d.vx = __fadd_rn(d.vx, __fmul_rn(jx, d.inv_mass));
  d.vy = __fadd_rn(d.vy, __fmul_rn(jy, d.inv_mass));
  d.vz = __fadd_rn(d.vz, __fmul_rn(jz, d.inv_mass));
  const float rx = __fsub_rn(qx, bpx), ry = __fsub_rn(qy, bpy), rz = __fsub_rn(qz, bpz);
  const float tx = __fsub_rn(__fmul_rn(ry, jz), __fmul_rn(rz, jy));
  const float ty = __fsub_rn(__fmul_rn(rz, jx), __fmul_rn(rx, jz));
  const float tz = __fsub_rn(__fmul_rn(rx, jy), __fmul_rn(ry, jx));
  float ax, ay, az;
  mat3_vec(d.iw, tx, ty, tz, ax, ay, az);
  d.wx = __fadd_rn(d.wx, ax);
  d.wy = __fadd_rn(d.wy, ay);
  d.wz = __fadd_rn(d.wz, az);
}

// The body loop of one particle from body k0 on with the reactions
// (fluid3.rs:1140-1178): push out, remove the approach velocity, impulse
// n * (vn * m), then the no-slip pull toward the body's velocity and its
// reaction -dv * m. Run in particle order.
__device__ void walls3q_ordered(float& x, float& y, float& z, float& vx, float& vy, float& vz, float m, uint32_t k0,
                                DynBody3* __restrict__ dyn, const StepParams3& P) {
  for (uint32_t k = k0; k < P.nbodies; k++) {
    const DevBodyQ3 b = P.qbodies[k];
    if (fabsf(x - b.px) > b.ex || fabsf(y - b.py) > b.ey || fabsf(z - b.pz) > b.ez) continue;
    float nx, ny, nz, depth, cx, cy, cz;
    if (!collide_q3(x, y, z, P.pr, b, P.hullv, nx, ny, nz, depth, cx, cy, cz)) continue;
    if (depth <= 0.0f) continue;
    x = __fadd_rn(x, __fmul_rn(nx, depth));
    y = __fadd_rn(y, __fmul_rn(ny, depth));
    z = __fadd_rn(z, __fmul_rn(nz, depth));
    const float vn = dot3(vx, vy, vz, nx, ny, nz);
    if (!(vn < 0.0f)) continue;
    vx = __fsub_rn(vx, __fmul_rn(nx, vn));
    vy = __fsub_rn(vy, __fmul_rn(ny, vn));
    vz = __fsub_rn(vz, __fmul_rn(nz, vn));
    float wvx = 0.0f, wvy = 0.0f, wvz = 0.0f;
    DynBody3* d = b.dyn ? dyn + k : nullptr;
    if (d) {
      if (!d->is_static) d->sleeping = 0;
      const float vm = __fmul_rn(vn, m);
      apply_impulse3(*d, b.px, b.py, b.pz, __fmul_rn(nx, vm), __fmul_rn(ny, vm), __fmul_rn(nz, vm), cx, cy, cz);
      wvx = d->vx, wvy = d->vy, wvz = d->vz;
    }
    if (P.flags & F_FRICTION) {
      const float vtx = vx, vty = vy, vtz = vz;
      const float wdot = dot3(wvx, wvy, wvz, nx, ny, nz);
      const float wtx = __fsub_rn(wvx, __fmul_rn(nx, wdot));
      const float wty = __fsub_rn(wvy, __fmul_rn(ny, wdot));
      const float wtz = __fsub_rn(wvz, __fmul_rn(nz, wdot));
      const float dvx = __fmul_rn(__fsub_rn(wtx, vtx), P.mu);
      const float dvy = __fmul_rn(__fsub_rn(wty, vty), P.mu);
      const float dvz = __fmul_rn(__fsub_rn(wtz, vtz), P.mu);
      vx = __fadd_rn(vx, dvx);
      vy = __fadd_rn(vy, dvy);
      vz = __fadd_rn(vz, dvz);
      if (d)
        apply_impulse3(*d, b.px, b.py, b.pz, __fmul_rn(-dvx, m), __fmul_rn(-dvy, m), __fmul_rn(-dvz, m), cx, cy,
                       cz);
    }
  }
}

// ---------------------------------------------------------------- kernels
__global__ void __launch_bounds__(256) k_keys3(const float4* __restrict__ pos, uint32_t n, GridPlan3 g,
                                               uint32_t* __restrict__ keys, uint32_t* __restrict__ count) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 p = pos[i];
  const uint32_t k = bucket_key3(p.x, p.y, p.z, g);
  keys[i] = k;
  count_key(count, k);
}

// In-bucket rank by id, then the gather into sorted order.
__global__ void __launch_bounds__(256) k_fixup3(const uint32_t* __restrict__ tkey, const uint32_t* __restrict__ tid_in,
                                                const uint32_t* __restrict__ start, uint32_t n,
                                                uint32_t* __restrict__ skey, uint32_t* __restrict__ sid,
                                                const float4* __restrict__ pos, const float4* __restrict__ vel,
                                                const float* __restrict__ mass, const uint8_t* __restrict__ phase,
                                                float4* __restrict__ spos, float4* __restrict__ svel,
                                                float* __restrict__ smass, uint8_t* __restrict__ sphase) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const uint32_t k = tkey[s];
  const uint32_t id = tid_in[s];
  const uint32_t lo = start[k], hi = start[k + 1];
  uint32_t rank = 0;
  for (uint32_t j = lo; j < hi; j++) rank += __ldg(&tid_in[j]) < id ? 1u : 0u;
  const uint32_t f = lo + rank;
  skey[f] = k;
  sid[f] = id;
  spos[f] = pos[id];
  svel[f] = vel[id];
  if (smass) smass[f] = mass[id];
  if (sphase) sphase[f] = phase[id];
}

__device__ __forceinline__ uint32_t row_base3(uint32_t by, uint32_t bz, int r, const GridPlan3& g) {
  const uint32_t oz = (uint32_t)(r / 3) - 1u, oy = (uint32_t)(r % 3) - 1u;
  return (((bz + oz) & g.maskd) << (g.log2w + g.log2h)) | (((by + oy) & g.maskh) << g.log2w);
}

// Density + EOS (fluid3.rs:639-658) in sorted order; per-row neighbour masks
// (bit t of nmask[r * n + s]: slot row_start + t is a neighbour). A zero mask
// for the particle's own row (r = 4) means no masks (seam or > 32 slots).
template <bool MASS, bool PHASE, bool WIDE>
__global__ void __launch_bounds__(256) k_density3(const float4* __restrict__ spos, const uint32_t* __restrict__ skey,
                                                  const float* __restrict__ smass, const uint8_t* __restrict__ sphase,
                                                  uint32_t n, const uint32_t* __restrict__ start, StepParams3 P,
                                                  float2* __restrict__ sdq, float* __restrict__ spres,
                                                  uint32_t* __restrict__ nmask) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const uint32_t k = skey[s];
  const float4 pi = spos[s];
  float rho = 0.0f;
  const GridPlan3& g = P.grid;
  if (k != g.sentinel) {
    const uint32_t bx = k & g.maskw, by = (k >> g.log2w) & g.maskh, bz = k >> (g.log2w + g.log2h);
    if (bx >= 1u && bx < g.maskw) {
      // the three x cells of each row are consecutive buckets: one slot range
      bool masked = true;
      uint32_t m_own = 0;
      // the rows' slot ranges, loaded up front
      uint32_t rsa[9], rea[9];
#pragma unroll
      for (int r = 0; r < 9; r++) {
        const uint32_t row = row_base3(by, bz, r, g);
        rsa[r] = __ldg(&start[row + bx - 1]);
        rea[r] = __ldg(&start[row + bx + 2]);
      }
#pragma unroll
      for (int r = 0; r < 9; r++) {
        const uint32_t rs = rsa[r], re = rea[r];
        uint32_t m = 0, bit = 1u;  // bit shifts out after 32 slots (then masked is false)
        for (uint32_t j = rs; j < re; j++) {
          const float4 a = __ldg(&spos[j]);
          const float dx = __fsub_rn(a.x, pi.x), dy = __fsub_rn(a.y, pi.y), dz = __fsub_rn(a.z, pi.z);
          const float d2 = dot3(dx, dy, dz, dx, dy, dz);
          const bool nb = d2 < P.hg2;
          const float w = __fmul_rn(MASS ? __ldg(&smass[j]) : P.mass, poly6_nb<WIDE>(d2, P));
          rho = nb ? __fadd_rn(rho, w) : rho;
          m |= nb ? bit : 0u;
          bit <<= 1;
        }
        if (re - rs > kMaskBits3) masked = false;
        if (r == 4) m_own = m;
        else nmask[(size_t)r * n + s] = m;
      }
      nmask[4 * (size_t)n + s] = masked ? m_own : 0u;
    } else {
      // seam column: the x cells wrap, visit bucket by bucket
#pragma unroll 1
      for (int r = 0; r < 9; r++) {
        const uint32_t row = row_base3(by, bz, r, g);
#pragma unroll 1
        for (int ox = -1; ox <= 1; ox++) {
          const uint32_t bb = row | ((bx + (uint32_t)ox) & g.maskw);
          const uint32_t e = __ldg(&start[bb + 1]);
          for (uint32_t j = __ldg(&start[bb]); j < e; j++) {
            const float4 a = __ldg(&spos[j]);
            const float dx = __fsub_rn(a.x, pi.x), dy = __fsub_rn(a.y, pi.y), dz = __fsub_rn(a.z, pi.z);
            rho = __fadd_rn(rho, contrib3(dot3(dx, dy, dz, dx, dy, dz), MASS ? __ldg(&smass[j]) : P.mass, P));
          }
        }
      }
      nmask[4 * (size_t)n + s] = 0u;
    }
  } else {
    nmask[4 * (size_t)n + s] = 0u;
  }
  float dens = rho;
  if (dens < 0.0f) dens = 0.0f;
  if (dens > P.rho_cap) dens = P.rho_cap;
  const uint32_t ph = PHASE ? min((uint32_t)sphase[s], 3u) : P.uniform_phase;
  const float p = eos(dens, P.rest[ph], P);
  const float rc = fmaxf(dens, kEps);
  sdq[s] = make_float2(dens, __fdiv_rn(p, __fmul_rn(rc, rc)));
  spres[s] = p;
}

// One neighbour pair of the force loop (fluid3.rs:1040-1084) and of the XSPH
// sum (fluid3.rs:1111-1123), accumulated in the reference's order.
template <bool MASS, bool PLAIN>
__device__ __forceinline__ void pair3(uint32_t j, float4 pi, float4 vi, float rho_i, float q_i, float m_i,
                                      const float4* __restrict__ spos, const float4* __restrict__ svel,
                                      const float2* __restrict__ sdq, const float* __restrict__ smass,
                                      const StepParams3& P, float (&f)[3], float (&sm)[3]) {
  const float4 pj = __ldg(&spos[j]);
  const float2 dqj = __ldg(&sdq[j]);
  const float4 vj = __ldg(&svel[j]);
  const float m_j = MASS ? __ldg(&smass[j]) : P.mass;
  const float rho_j = fmaxf(dqj.x, kEps);
  const float dx = __fsub_rn(pi.x, pj.x), dy = __fsub_rn(pi.y, pj.y), dz = __fsub_rn(pi.z, pj.z);
  const float d2 = dot3(dx, dy, dz, dx, dy, dz);
  const float dist = __fsqrt_rn(d2);
  float g0 = 0.0f, g1 = 0.0f, g2 = 0.0f;
  if (!(dist >= P.hk || dist < kEps)) {
    const float hr = __fsub_rn(P.hk, dist);
    const float sc = __fmul_rn(__fmul_rn(P.c_spiky, hr), hr);
    g0 = __fmul_rn(__fdiv_rn(dx, dist), sc);
    g1 = __fmul_rn(__fdiv_rn(dy, dist), sc);
    g2 = __fmul_rn(__fdiv_rn(dz, dist), sc);
  }
  float term = __fadd_rn(q_i, dqj.y);
  if (!PLAIN && (P.flags & F_AV) && dist > kEps) {
    const float rho_bar = __fmul_rn(0.5f, __fadd_rn(rho_i, rho_j));
    const float vd = dot3(__fsub_rn(vi.x, vj.x), __fsub_rn(vi.y, vj.y), __fsub_rn(vi.z, vj.z), dx, dy, dz);
    if (!(vd >= 0.0f)) {
      const float r_sq = __fmul_rn(dist, dist);
      const float mu = __fdiv_rn(__fmul_rn(P.hk, vd), __fadd_rn(r_sq, __fmul_rn(__fmul_rn(0.01f, P.hk), P.hk)));
      term = __fadd_rn(term, __fdiv_rn(__fmul_rn(__fmul_rn(-P.av_alpha, P.c_s), mu), fmaxf(rho_bar, kEps)));
    }
  }
  const float mt = __fmul_rn(m_j, term);
  f[0] = __fsub_rn(f[0], __fmul_rn(g0, mt));
  f[1] = __fsub_rn(f[1], __fmul_rn(g1, mt));
  f[2] = __fsub_rn(f[2], __fmul_rn(g2, mt));
  if (!PLAIN && (P.flags & F_COHESION) && dist > kEps) {
    const float c = dist >= P.hk ? 0.0f : __fsub_rn(1.0f, __fdiv_rn(dist, P.hk));
    if (c > 0.0f) {
      const float sc = __fmul_rn(__fmul_rn(__fmul_rn(P.surface_tension, m_i), m_j), c);
      f[0] = __fsub_rn(f[0], __fmul_rn(__fdiv_rn(dx, dist), sc));
      f[1] = __fsub_rn(f[1], __fmul_rn(__fdiv_rn(dy, dist), sc));
      f[2] = __fsub_rn(f[2], __fmul_rn(__fdiv_rn(dz, dist), sc));
    }
  }
  if (PLAIN || (P.flags & F_VISC)) {
    const float rho_bar = __fmul_rn(0.5f, __fadd_rn(rho_i, rho_j));
    const float w = PLAIN ? poly6_nb<false>(d2, P) : poly6_3(d2, P);
    const float mr = __fdiv_rn(m_j, rho_bar);
    sm[0] = __fadd_rn(sm[0], __fmul_rn(__fmul_rn(__fsub_rn(vj.x, vi.x), mr), w));
    sm[1] = __fadd_rn(sm[1], __fmul_rn(__fmul_rn(__fsub_rn(vj.y, vi.y), mr), w));
    sm[2] = __fadd_rn(sm[2], __fmul_rn(__fmul_rn(__fsub_rn(vj.z, vi.z), mr), w));
  }
}

// The tolerance mode's pair (plain flag set, uniform mass): the same pairs
// in the same order as pair3 with reassociated arithmetic, as the 2D pass
// does: one approximate reciprocal square root for the spiky direction and
// one approximate reciprocal for the XSPH weight 1 / (rho_i + rho_j) per
// pair, fused multiply-adds. The XSPH sum leaves out its constant factor
// 2 m c_poly6 (m / rho_bar * poly6 = 2 m c_poly6 t^3 / (rho_i + rho_j)),
// which k_force3 applies once per particle. mq_i = m q_i.
__device__ __forceinline__ void pair3_fast(uint32_t j, float4 pi, float4 vi, float rho_i, float mq_i,
                                           const float4* __restrict__ spos, const float4* __restrict__ svel,
                                           const float2* __restrict__ sdq, const StepParams3& P, float (&f)[3],
                                           float (&sm)[3]) {
  const float4 pj = __ldg(&spos[j]);
  const float2 dqj = __ldg(&sdq[j]);
  const float4 vj = __ldg(&svel[j]);
  const float dx = __fsub_rn(pi.x, pj.x), dy = __fsub_rn(pi.y, pj.y), dz = __fsub_rn(pi.z, pj.z);
  const float d2 = __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmul_rn(dz, dz)));
  const float rinv = rsqrtf(d2);  // d2 = 0 (coincident): inf, and r below is NaN -> no gradient
  const float r = __fmul_rn(d2, rinv);
  const float hr = __fsub_rn(P.hk, r);
  const bool grad = r < P.hk && r >= kEps;  // spiky_grad's support
  const float gs = grad ? __fmul_rn(__fmul_rn(__fmul_rn(P.c_spiky, hr), hr), rinv) : 0.0f;
  const float c = __fmul_rn(gs, __fmaf_rn(P.mass, dqj.y, mq_i));  // m (q_i + q_j)
  f[0] = __fmaf_rn(-dx, c, f[0]);
  f[1] = __fmaf_rn(-dy, c, f[1]);
  f[2] = __fmaf_rn(-dz, c, f[2]);
  const float t = __fsub_rn(P.hk2, d2);
  const float w = __fmul_rn(__fmul_rn(__fmul_rn(t, t), t), __fdividef(1.0f, __fadd_rn(rho_i, fmaxf(dqj.x, kEps))));
  sm[0] = __fmaf_rn(__fsub_rn(vj.x, vi.x), w, sm[0]);
  sm[1] = __fmaf_rn(__fsub_rn(vj.y, vi.y), w, sm[1]);
  sm[2] = __fmaf_rn(__fsub_rn(vj.z, vi.z), w, sm[2]);
}

// Ghost pressure on a fluid particle (fluid3.rs:1073-1083), after its fluid
// pairs: boundary_near's cells (oz, oy, ox = -1..1 around floor(p / h), h
// the config's smoothing length) and filter, -grad W * (m_g (q_i + q_g)).
static __device__ __noinline__ float3 ghost_force3(float4 pi, float q_i, float f0, float f1, float f2,
                                                   const StepParams3 P) {
  const float hg = P.grid.hg;
  const int32_t cx = __float2int_rd(__fdiv_rn(pi.x, hg)), cy = __float2int_rd(__fdiv_rn(pi.y, hg));
  const int32_t cz = __float2int_rd(__fdiv_rn(pi.z, hg));
  for (int oz = -1; oz <= 1; oz++)
    for (int oy = -1; oy <= 1; oy++)
      for (int ox = -1; ox <= 1; ox++) {
        const int32_t qx = (int32_t)((uint32_t)cx + (uint32_t)ox), qy = (int32_t)((uint32_t)cy + (uint32_t)oy);
        const int32_t qz = (int32_t)((uint32_t)cz + (uint32_t)oz);
        uint32_t slot = ghost_cell_hash3(qx, qy, qz, P.gtab_mask);
        GhostCell3 c = P.gtab[slot];
        for (uint32_t probe = 0; probe <= P.gtab_mask && c.count != 0 && (c.cx != qx || c.cy != qy || c.cz != qz);
             probe++) {
          slot = (slot + 1) & P.gtab_mask;
          c = P.gtab[slot];
        }
        if (c.count == 0 || c.cx != qx || c.cy != qy || c.cz != qz) continue;
        for (uint32_t k = c.start; k < c.start + c.count; k++) {
          const float4 g = P.gpos[k];
          const float ex = __fsub_rn(g.x, pi.x), ey = __fsub_rn(g.y, pi.y), ez = __fsub_rn(g.z, pi.z);
          if (!(dot3(ex, ey, ez, ex, ey, ez) < P.hg2)) continue;
          const float dx = __fsub_rn(pi.x, g.x), dy = __fsub_rn(pi.y, g.y), dz = __fsub_rn(pi.z, g.z);
          const float dist = __fsqrt_rn(dot3(dx, dy, dz, dx, dy, dz));
          float g0 = 0.0f, g1 = 0.0f, g2 = 0.0f;
          if (!(dist >= P.hk || dist < kEps)) {
            const float hr = __fsub_rn(P.hk, dist);
            const float sc = __fmul_rn(__fmul_rn(P.c_spiky, hr), hr);
            g0 = __fmul_rn(__fdiv_rn(dx, dist), sc);
            g1 = __fmul_rn(__fdiv_rn(dy, dist), sc);
            g2 = __fmul_rn(__fdiv_rn(dz, dist), sc);
          }
          const float mt = __fmul_rn(P.gmass, __fadd_rn(q_i, P.gq[k]));
          f0 = __fsub_rn(f0, __fmul_rn(g0, mt));
          f1 = __fsub_rn(f1, __fmul_rn(g1, mt));
          f2 = __fsub_rn(f2, __fmul_rn(g2, mt));
        }
      }
  return make_float3(f0, f1, f2);
}

// Ghost density and pressure from the fluid (fluid3.rs:906-921): the 27
// cells around the ghost bucket by bucket in the reference's order, m_j *
// poly6 for candidates within h; density clamped, pressure from the
// unclamped sum with the config's rest density; stored as q.
template <bool MASS>
__global__ void __launch_bounds__(256) k_ghost_density3(const float4* __restrict__ spos,
                                                        const float* __restrict__ smass,
                                                        const uint32_t* __restrict__ start, StepParams3 P) {
  const uint32_t gi = blockIdx.x * blockDim.x + threadIdx.x;
  if (gi >= P.nghost) return;
  const float4 b = P.gpos[gi];
  const GridPlan3& g = P.grid;
  float rho = 0.0f;
  const uint32_t k = bucket_key3(b.x, b.y, b.z, g);
  if (k != g.sentinel) {
    const uint32_t bx = k & g.maskw, by = (k >> g.log2w) & g.maskh, bz = k >> (g.log2w + g.log2h);
#pragma unroll 1
    for (int r = 0; r < 9; r++) {
      const uint32_t row = row_base3(by, bz, r, g);
#pragma unroll 1
      for (int ox = -1; ox <= 1; ox++) {
        const uint32_t bb = row | ((bx + (uint32_t)ox) & g.maskw);
        const uint32_t e = __ldg(&start[bb + 1]);
        for (uint32_t j = __ldg(&start[bb]); j < e; j++) {
          const float4 a = __ldg(&spos[j]);
          const float dx = __fsub_rn(a.x, b.x), dy = __fsub_rn(a.y, b.y), dz = __fsub_rn(a.z, b.z);
          rho = __fadd_rn(rho, contrib3(dot3(dx, dy, dz, dx, dy, dz), MASS ? __ldg(&smass[j]) : P.mass, P));
        }
      }
    }
  }
  float dens = rho;
  if (dens < 0.0f) dens = 0.0f;
  if (dens > P.rho_cap) dens = P.rho_cap;
  const float p = eos(rho, P.rest0, P);
  const float rc = fmaxf(dens, kEps);
  P.gq[gi] = __fdiv_rn(p, __fmul_rn(rc, rc));
}

// FluidState3::resample (fluid3.rs:923-990), one thread as the 2D pass:
// merges (index order, highest-index dense neighbour j < i within 0.25 h
// among the 27-cell grid candidates, mass and momentum conserved), then
// splits into half-mass children at x +- (0.25 h, 0, 0) while the output
// holds fewer than MAX_PARTICLES_3D - 1.
__global__ void k_resample3(uint32_t n, float4* __restrict__ pos, float4* __restrict__ vel, float* __restrict__ mass,
                            const uint8_t* __restrict__ phase, const float2* __restrict__ sdq,
                            const uint32_t* __restrict__ sid, const uint32_t* __restrict__ skey,
                            const uint32_t* __restrict__ slot_of, const uint32_t* __restrict__ start, StepParams3 P,
                            float merge_hi, float split_lo, float min_mass, uint8_t* __restrict__ absorbed,
                            float4* __restrict__ out_pos, float4* __restrict__ out_vel, float* __restrict__ out_mass,
                            uint8_t* __restrict__ out_phase, uint32_t out_cap, uint32_t* __restrict__ n_out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const GridPlan3& g = P.grid;
  const float md = __fmul_rn(0.25f, P.hk), merge_d2 = __fmul_rn(md, md);
  for (uint32_t i = 0; i < n; i++) absorbed[i] = 0;
  for (uint32_t i = 0; i < n; i++) {
    const uint32_t si = slot_of[i];
    if (absorbed[i] || sdq[si].x <= merge_hi) continue;
    const float4 pi = pos[i];
    int64_t best = -1;
    const uint32_t k = skey[si];
    if (k != g.sentinel) {
      const uint32_t bx = k & g.maskw, by = (k >> g.log2w) & g.maskh, bz = k >> (g.log2w + g.log2h);
      for (int r = 0; r < 9; r++) {
        const uint32_t row = row_base3(by, bz, r, g);
        for (int ox = -1; ox <= 1; ox++) {
          const uint32_t bb = row | ((bx + (uint32_t)ox) & g.maskw);
          for (uint32_t js = start[bb]; js < start[bb + 1]; js++) {
            const uint32_t j = sid[js];
            if (j >= i || absorbed[j] || sdq[js].x <= merge_hi || (int64_t)j <= best) continue;
            const float4 pj = pos[j];
            const float dx = __fsub_rn(pi.x, pj.x), dy = __fsub_rn(pi.y, pj.y), dz = __fsub_rn(pi.z, pj.z);
            if (dot3(dx, dy, dz, dx, dy, dz) < merge_d2) best = j;
          }
        }
      }
    }
    if (best < 0) continue;
    const uint32_t j = (uint32_t)best;
    const float mi = mass[i], mj = mass[j];
    const float mt = __fadd_rn(mi, mj);
    if (mt > kEps) {
      const float4 vi = vel[i], vj = vel[j];
      vel[i] = make_float4(__fdiv_rn(__fadd_rn(__fmul_rn(vi.x, mi), __fmul_rn(vj.x, mj)), mt),
                           __fdiv_rn(__fadd_rn(__fmul_rn(vi.y, mi), __fmul_rn(vj.y, mj)), mt),
                           __fdiv_rn(__fadd_rn(__fmul_rn(vi.z, mi), __fmul_rn(vj.z, mj)), mt), vi.w);
      mass[i] = mt;
    }
    absorbed[j] = 1;
  }
  uint32_t out = 0;
  const float off = __fmul_rn(0.25f, P.hk);
  for (uint32_t i = 0; i < n; i++) {
    if (absorbed[i]) continue;
    const float4 p = pos[i], v = vel[i];
    const float m = mass[i];
    const bool split = sdq[slot_of[i]].x < split_lo && m > min_mass && out + 1 < 4096u;  // MAX_PARTICLES_3D (fluid3.rs:28)
    if (out + (split ? 2u : 1u) > out_cap) {  // never with buffers sized for the bound: report, write nothing past
      *n_out = out_cap + 1u;
      return;
    }
    if (split) {
      const float half = __fmul_rn(m, 0.5f);
      out_pos[out] = make_float4(__fadd_rn(p.x, off), __fadd_rn(p.y, 0.0f), __fadd_rn(p.z, 0.0f), p.w);
      out_vel[out] = v;
      out_mass[out] = half;
      out_phase[out++] = phase[i];
      out_pos[out] = make_float4(__fsub_rn(p.x, off), __fsub_rn(p.y, 0.0f), __fsub_rn(p.z, 0.0f), p.w);
      out_vel[out] = v;
      out_mass[out] = half;
      out_phase[out++] = phase[i];
    } else {
      out_pos[out] = p;
      out_vel[out] = v;
      out_mass[out] = m;
      out_phase[out++] = phase[i];
    }
  }
  *n_out = out;
}

__global__ void k_resample_prep3(const uint32_t* __restrict__ sid, uint32_t n, uint32_t* __restrict__ slot_of,
                                 float* __restrict__ mass, uint8_t* __restrict__ phase, int mass_uniform,
                                 float mass_value, int phase_uniform, uint8_t phase_value) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  slot_of[sid[s]] = s;
  if (mass_uniform) mass[s] = mass_value;
  if (phase_uniform) phase[s] = phase_value;
}

// Force + XSPH + integrate + walls (fluid3.rs:1040-1176); writes the new
// state (id order), the next key and its bucket count. DEBUG: forces only.
// FAST (tolerance mode; PLAIN, uniform mass): pair3_fast's arithmetic.
template <bool MASS, bool DEBUG, bool PLAIN, bool FAST = false>
__global__ void __launch_bounds__(256) k_force3(const float4* __restrict__ spos, const float4* __restrict__ svel,
                                                const float2* __restrict__ sdq, const uint32_t* __restrict__ skey,
                                                const uint32_t* __restrict__ sid, const float* __restrict__ smass,
                                                uint32_t n, const uint32_t* __restrict__ start, StepParams3 P,
                                                const DevBody3* __restrict__ bodies,
                                                const uint32_t* __restrict__ nmask, float4* __restrict__ pos_out,
                                                float4* __restrict__ vel_out, uint32_t* __restrict__ key_out,
                                                uint32_t* __restrict__ count_out, float4* __restrict__ dbg) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const uint32_t k = skey[s];
  const uint32_t id = sid[s];
  const float4 pi = spos[s];
  const float4 vi = svel[s];
  const float2 dqi = sdq[s];
  const float m_i = MASS ? smass[s] : P.mass;
  const float rho_i = fmaxf(dqi.x, kEps);
  const float q_i = dqi.y;
  const float mq_i = __fmul_rn(P.mass, q_i);
  float f[3] = {0.0f, 0.0f, 0.0f}, sm[3] = {0.0f, 0.0f, 0.0f};
  const GridPlan3& g = P.grid;
  if (k != g.sentinel) {
    const uint32_t bx = k & g.maskw, by = (k >> g.log2w) & g.maskh, bz = k >> (g.log2w + g.log2h);
    if (nmask[4 * (size_t)n + s] != 0u) {
      // the nine rows' masks and first slots, loaded up front (independent
      // loads; none inside the divergent row advance below)
      uint32_t mk[9], bs[9];
#pragma unroll
      for (int r = 0; r < 9; r++) {
        mk[r] = nmask[(size_t)r * n + s];
        bs[r] = __ldg(&start[row_base3(by, bz, r, g) + bx - 1]);
      }
      mk[4] &= ~(1u << (s - bs[4]));  // the particle's own bit: j != i
      // one loop over the set bits of all rows (ascending slots, row by row),
      // so a warp runs as many pair iterations as its busiest lane has
      // neighbours
      uint32_t cur = mk[0], base = bs[0];
      int r = 0;
      for (;;) {
        while (cur == 0u && r < 8) {
          r++;
#pragma unroll
          for (int t = 1; t < 9; t++)
            if (t == r) {
              cur = mk[t];
              base = bs[t];
            }
        }
        if (cur == 0u) break;
        const uint32_t j = base + (uint32_t)(__ffs((int)cur) - 1);
        cur &= cur - 1u;
        if constexpr (FAST)
          pair3_fast(j, pi, vi, rho_i, mq_i, spos, svel, sdq, P, f, sm);
        else
          pair3<MASS, PLAIN>(j, pi, vi, rho_i, q_i, m_i, spos, svel, sdq, smass, P, f, sm);
      }
    } else {
#pragma unroll 1
      for (int r = 0; r < 9; r++) {
        const uint32_t row = row_base3(by, bz, r, g);
#pragma unroll 1
        for (int ox = -1; ox <= 1; ox++) {
          const uint32_t bb = row | ((bx + (uint32_t)ox) & g.maskw);
          const uint32_t e = __ldg(&start[bb + 1]);
          for (uint32_t j = __ldg(&start[bb]); j < e; j++) {
            const float4 a = __ldg(&spos[j]);
            const float ex = __fsub_rn(a.x, pi.x), ey = __fsub_rn(a.y, pi.y), ez = __fsub_rn(a.z, pi.z);
            if (dot3(ex, ey, ez, ex, ey, ez) < P.hg2 && j != s) {
              if constexpr (FAST)
                pair3_fast(j, pi, vi, rho_i, mq_i, spos, svel, sdq, P, f, sm);
              else
                pair3<MASS, PLAIN>(j, pi, vi, rho_i, q_i, m_i, spos, svel, sdq, smass, P, f, sm);
            }
          }
        }
      }
    }
  }
  if constexpr (FAST) {
    const float xs = __fmul_rn(__fmul_rn(2.0f, P.mass), P.c_poly6);  // pair3_fast's XSPH factor
    sm[0] = __fmul_rn(sm[0], xs);
    sm[1] = __fmul_rn(sm[1], xs);
    sm[2] = __fmul_rn(sm[2], xs);
  }
  if (!PLAIN && (P.flags & F_GHOST)) {  // PLAIN launches exclude F_GHOST
    const float3 gf = ghost_force3(pi, q_i, f[0], f[1], f[2], P);
    f[0] = gf.x;
    f[1] = gf.y;
    f[2] = gf.z;
  }
  if (DEBUG) {
    dbg[id] = make_float4(f[0], f[1], f[2], 0.0f);
    return;
  }
  float ax = __fadd_rn(P.gx, __fdiv_rn(f[0], rho_i));
  float ay = __fadd_rn(P.gy, __fdiv_rn(f[1], rho_i));
  float az = __fadd_rn(P.gz, __fdiv_rn(f[2], rho_i));
  if (!PLAIN && (P.flags & F_TURB)) {  // fluid3.rs:1096-1108, at the pre-step position and the step's clock
    const float3 tb = turbulence_accel3(pi.x, pi.y, pi.z, *P.clock, P.turb_freq, P.turb_tscale, P.turb_seed,
                                        P.turb_oct, P.flags & F_TURB_CURL, P.turb_amp);
    ax = __fadd_rn(ax, tb.x);
    ay = __fadd_rn(ay, tb.y);
    az = __fadd_rn(az, tb.z);
  }
  float vx = __fadd_rn(vi.x, __fmul_rn(ax, P.dt));
  float vy = __fadd_rn(vi.y, __fmul_rn(ay, P.dt));
  float vz = __fadd_rn(vi.z, __fmul_rn(az, P.dt));
  if (P.flags & F_VISC) {
    vx = __fadd_rn(vx, __fmul_rn(sm[0], P.visc));
    vy = __fadd_rn(vy, __fmul_rn(sm[1], P.visc));
    vz = __fadd_rn(vz, __fmul_rn(sm[2], P.visc));
  }
  const float speed = __fsqrt_rn(dot3(vx, vy, vz, vx, vy, vz));
  if (speed > P.vmax) {
    const float sc = __fdiv_rn(P.vmax, speed);
    vx = __fmul_rn(vx, sc);
    vy = __fmul_rn(vy, sc);
    vz = __fmul_rn(vz, sc);
  }
  if (!isfinite(vx) || !isfinite(vy) || !isfinite(vz)) vx = vy = vz = 0.0f;
  float x = __fadd_rn(pi.x, __fmul_rn(vx, P.dt));
  float y = __fadd_rn(pi.y, __fmul_rn(vy, P.dt));
  float z = __fadd_rn(pi.z, __fmul_rn(vz, P.dt));
  if (!isfinite(x) || !isfinite(y) || !isfinite(z)) {
    x = pi.x;
    y = pi.y;
    z = pi.z;
  }
  if (P.flags & F_QBODIES) {
    // the engine's bodies (phieng_sph3_step_fluid)
    const uint32_t r = walls3q(x, y, z, vx, vy, vz, P);
    pos_out[id] = make_float4(x, y, z, 0.0f);
    vel_out[id] = make_float4(vx, vy, vz, 0.0f);
    if (P.flags & F_DYNAMIC) {
      // contacts with bodies that react run in particle order (k_dynamic_walls3)
      P.dcount[id] = r != kNoDefer ? 1u : 0u;
      if (r != kNoDefer) {
        P.defer[id] = r;
        return;
      }
    }
  } else {
    walls3(x, y, z, vx, vy, vz, bodies, P);
    pos_out[id] = make_float4(x, y, z, 0.0f);
    vel_out[id] = make_float4(vx, vy, vz, 0.0f);
  }
  const uint32_t nk = bucket_key3(x, y, z, g);
  key_out[id] = nk;
  atomicAdd(&count_out[nk], 1u);  // one atomic per particle, as the 2D force pass
}

__global__ void __launch_bounds__(256) k_vmax3(const float4* __restrict__ vel, uint32_t n, unsigned int* out) {
  float m = 0.0f;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float4 v = vel[i];
    const float l = __fsqrt_rn(dot3(v.x, v.y, v.z, v.x, v.y, v.z));
    if (l > m) m = l;  // NaN never wins (f32::max semantics)
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

__global__ void __launch_bounds__(256) k_unsort3(const float2* __restrict__ sdq, const float* __restrict__ spres,
                                                 const uint32_t* __restrict__ sid, uint32_t n, float* dens,
                                                 float* pres) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  dens[sid[s]] = sdq[s].x;
  pres[sid[s]] = spres[s];
}

// The rest of the body loop of every deferred particle, one after the other
// in id order (a body's velocity after particle i's reactions is what
// particle i+1's no-slip term reads); then its next key and bucket count.
__global__ void k_dynamic_walls3(const uint32_t* __restrict__ list, const uint32_t* __restrict__ total,
                                 float4* __restrict__ pos, float4* __restrict__ vel, const float* __restrict__ mass,
                                 uint32_t* __restrict__ key, uint32_t* __restrict__ count, DynBody3* __restrict__ dyn,
                                 StepParams3 P) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const uint32_t m = *total;
  for (uint32_t t = 0; t < m; t++) {
    const uint32_t id = list[t];
    const float4 p = pos[id], v = vel[id];
    float x = p.x, y = p.y, z = p.z, vx = v.x, vy = v.y, vz = v.z;
    const float mi = (P.flags & F_MASS) ? mass[id] : P.mass;
    walls3q_ordered(x, y, z, vx, vy, vz, mi, P.defer[id], dyn, P);
    pos[id] = make_float4(x, y, z, 0.0f);
    vel[id] = make_float4(vx, vy, vz, 0.0f);
    const uint32_t nk = bucket_key3(x, y, z, P.grid);
    key[id] = nk;
    count_key(count, nk);
  }
}

// Sorted (density, q) and pressure to id order, and back into the order of
// a newer sort (the buoyancy pass samples the pressure on the re-sorted grid).
__global__ void __launch_bounds__(256) k_dp_to_id3(const float2* __restrict__ sdq, const float* __restrict__ spres,
                                                   const uint32_t* __restrict__ sid, uint32_t n,
                                                   float2* __restrict__ dq_id, float* __restrict__ p_id) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const uint32_t id = sid[s];
  dq_id[id] = sdq[s];
  p_id[id] = spres[s];
}

__global__ void __launch_bounds__(256) k_dp_from_id3(const float2* __restrict__ dq_id,
                                                     const float* __restrict__ p_id,
                                                     const uint32_t* __restrict__ sid, uint32_t n,
                                                     float2* __restrict__ sdq, float* __restrict__ spres) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const uint32_t id = sid[s];
  sdq[s] = dq_id[id];
  spres[s] = p_id[id];
}

// FluidState3::sample_pressure (fluid3.rs:345-369) over the sorted grid:
// cells oz, oy, ox = -1..1 around floor(point / h), h = max(smoothing_length,
// EPS), each bucket's particles in id order (others aliased into the bucket
// lie at least 3 h away); p += m_j (p_j / max(rho_j, EPS)) poly6(r^2) for
// r^2 < h*h; max(p, 0).
__device__ float sample_pressure3(float ptx, float pty, float ptz, const float4* __restrict__ spos,
                                  const float2* __restrict__ sdq, const float* __restrict__ spres,
                                  const float* __restrict__ smass, const uint32_t* __restrict__ start,
                                  const StepParams3& P) {
  const GridPlan3& g = P.grid;
  const int32_t cx = __float2int_rd(__fdiv_rn(ptx, P.hk));
  const int32_t cy = __float2int_rd(__fdiv_rn(pty, P.hk));
  const int32_t cz = __float2int_rd(__fdiv_rn(ptz, P.hk));
  float p = 0.0f;
  for (int oz = -1; oz <= 1; oz++) {
    const uint32_t bz = ((uint32_t)cz + (uint32_t)oz - (uint32_t)g.cz0) & g.maskd;
    for (int oy = -1; oy <= 1; oy++) {
      const uint32_t by = ((uint32_t)cy + (uint32_t)oy - (uint32_t)g.cy0) & g.maskh;
      for (int ox = -1; ox <= 1; ox++) {
        const uint32_t bx = ((uint32_t)cx + (uint32_t)ox - (uint32_t)g.cx0) & g.maskw;
        const uint32_t bb = (bz << (g.log2w + g.log2h)) | (by << g.log2w) | bx;
        const uint32_t e = start[bb + 1];
        for (uint32_t j = start[bb]; j < e; j++) {
          const float4 pj = spos[j];
          const float dx = __fsub_rn(pj.x, ptx), dy = __fsub_rn(pj.y, pty), dz = __fsub_rn(pj.z, ptz);
          const float r2 = dot3(dx, dy, dz, dx, dy, dz);
          if (r2 < P.hk2) {
            const float mj = (P.flags & F_MASS) ? smass[j] : P.mass;
            const float pr = __fdiv_rn(spres[j], fmaxf(sdq[j].x, kEps));
            p = __fadd_rn(p, __fmul_rn(__fmul_rn(mj, pr), poly6_3(r2, P)));
          }
        }
      }
    }
  }
  return fmaxf(p, 0.0f);  // f32::max(0.0): a NaN sum gives 0
}

// Buoyancy + drag on one dynamic body (fluid3.rs:1180-1213): for each
// surface sample in order (point and area in samples[2 q], outward normal in
// samples[2 q + 1]), a sampled pressure p > 0 gives the force
// -n (p A) - v_rel (drag A |v_rel|) (the latter when |v_rel| > EPS), v_rel =
// (v + w x r) - wind, applied at the point for dt (RigidBody3::apply_force,
// body.rs:1334-1346).
__global__ void k_buoyancy3(const uint32_t* __restrict__ which, uint32_t nb, DynBody3* __restrict__ dyn,
                            const float4* __restrict__ samples, const float4* __restrict__ spos,
                            const float2* __restrict__ sdq, const float* __restrict__ spres,
                            const float* __restrict__ smass, const uint32_t* __restrict__ start, StepParams3 P,
                            float drag, float dt, float wind_x, float wind_y, float wind_z) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nb) return;
  const uint32_t k = which[t];
  const DevBodyQ3 b = P.qbodies[k];
  DynBody3 d = dyn[k];
  bool wet = false;
  for (uint32_t q = 0; q < d.sample_count; q++) {
    const float4 sp = samples[2 * (size_t)(d.sample_first + q)];
    const float4 sn = samples[2 * (size_t)(d.sample_first + q) + 1];
    const float p = sample_pressure3(sp.x, sp.y, sp.z, spos, sdq, spres, smass, start, P);
    if (p <= 0.0f) continue;
    wet = true;
    const float rx = __fsub_rn(sp.x, b.px), ry = __fsub_rn(sp.y, b.py), rz = __fsub_rn(sp.z, b.pz);
    const float vrx = __fsub_rn(__fadd_rn(d.vx, __fsub_rn(__fmul_rn(d.wy, rz), __fmul_rn(d.wz, ry))), wind_x);
    const float vry = __fsub_rn(__fadd_rn(d.vy, __fsub_rn(__fmul_rn(d.wz, rx), __fmul_rn(d.wx, rz))), wind_y);
    const float vrz = __fsub_rn(__fadd_rn(d.vz, __fsub_rn(__fmul_rn(d.wx, ry), __fmul_rn(d.wy, rx))), wind_z);
    const float speed = __fsqrt_rn(dot3(vrx, vry, vrz, vrx, vry, vrz));
    const float pa = __fmul_rn(p, sp.w);
    float fx = __fmul_rn(-sn.x, pa), fy = __fmul_rn(-sn.y, pa), fz = __fmul_rn(-sn.z, pa);
    if (speed > kEps) {
      const float c = __fmul_rn(__fmul_rn(drag, sp.w), speed);
      fx = __fsub_rn(fx, __fmul_rn(vrx, c));
      fy = __fsub_rn(fy, __fmul_rn(vry, c));
      fz = __fsub_rn(fz, __fmul_rn(vrz, c));
    }
    if (!d.is_static) {  // RigidBody3::apply_force
      d.sleeping = 0;
      d.vx = __fadd_rn(d.vx, __fmul_rn(__fmul_rn(fx, d.inv_mass), dt));
      d.vy = __fadd_rn(d.vy, __fmul_rn(__fmul_rn(fy, d.inv_mass), dt));
      d.vz = __fadd_rn(d.vz, __fmul_rn(__fmul_rn(fz, d.inv_mass), dt));
      const float tx = __fsub_rn(__fmul_rn(ry, fz), __fmul_rn(rz, fy));
      const float ty = __fsub_rn(__fmul_rn(rz, fx), __fmul_rn(rx, fz));
      const float tz = __fsub_rn(__fmul_rn(rx, fy), __fmul_rn(ry, fx));
      float ax, ay, az;
      mat3_vec(d.iw, tx, ty, tz, ax, ay, az);
      d.wx = __fadd_rn(d.wx, __fmul_rn(ax, dt));
      d.wy = __fadd_rn(d.wy, __fmul_rn(ay, dt));
      d.wz = __fadd_rn(d.wz, __fmul_rn(az, dt));
    }
  }
  if (wet) d.sleeping = 0;
  dyn[k] = d;
}

inline uint32_t cdiv(uint32_t a, uint32_t b) { return (a + b - 1) / b; }

}  // namespace
}  // namespace phieng

// ---------------------------------------------------------------- the 3D world
// AmbientConfig3::default (ambient.rs): everything off, air density 1,
// turbulence frequency 1, time scale 1, 3 octaves.
AmbientConfig3Ffi default_ambient3() {
  AmbientConfig3Ffi a;
  std::memset(&a, 0, sizeof(a));
  a.air_density = 1.0f;
  a.turbulence_frequency = 1.0f;
  a.turbulence_time_scale = 1.0f;
  a.turbulence_octaves = 3;
  return a;
}

constexpr uint32_t kClockWord3 = 16;  // scalar word holding the step's world clock (turbulence)

struct World3 {
  FluidConfig3Ffi cfg = default_config();
  // arithmetic of the plain force pass (phieng_sph3_set_precision)
  uint32_t precision = PHIENG_SPH_EXACT;
  AmbientConfig3Ffi ambient = default_ambient3();
  float gx = 0.0f, gy = -9.81f, gz = 0.0f;  // World3::new gravity
  float time = 0.0f;
  std::vector<DevBody3> bodies;
  // boundary ghosts (boundary_particles): regenerated when their inputs change
  std::string ghost_sig;
  std::vector<float4> h_gpos;
  uint64_t ghost_regens = 0;
  uint32_t nghost = 0, ghost_cap = 0, gtab_cap = 0, gtab_mask = 0;
  float4* d_gpos = nullptr;
  float* d_gq = nullptr;
  GhostCell3* d_gtab = nullptr;
  // adaptive resolution scratch (capacity = dcap when allocated)
  uint32_t* rs_slot = nullptr;
  uint8_t* rs_absorbed = nullptr;
  float4 *rs_pos = nullptr, *rs_vel = nullptr;
  float* rs_mass = nullptr;
  uint8_t* rs_phase = nullptr;
  uint32_t rs_cap = 0;
  bool bodies_dirty = true;
  uint32_t cap = kMaxParticles3D;
  uint32_t n = 0;
  std::vector<float4> h_pos, h_vel;
  std::vector<float> h_mass, h_dens, h_pres;  // density / pressure as of dp_dev == false
  std::vector<uint8_t> h_phase;
  bool mass_uniform = true, phase_uniform = true;
  float mass_value = 0.0f;
  uint32_t phase_value = 0;
  bool host_valid = true, dev_valid = false, aux_valid = false, keys_valid = false;
  bool dp_dev = false;  // the sorted density / pressure on the device are newer than h_dens / h_pres
  bool plan_valid = false;
  uint32_t sid_perm_n = 0;
  GridPlan3 plan{};
  int device = -1;
  cudaStream_t own_stream = nullptr, stream = nullptr;
  bool user_stream = false;
  int32_t error = PHIENG_SPH_OK;
  uint64_t substeps = 0;
  // device arrays
  uint32_t dcap = 0;
  float4 *pos = nullptr, *vel = nullptr, *spos = nullptr, *svel = nullptr;
  float *mass = nullptr, *smass = nullptr, *spres = nullptr, *tmp = nullptr;
  uint8_t *phase = nullptr, *sphase = nullptr;
  uint32_t *key = nullptr, *tkey = nullptr, *tid = nullptr, *skey = nullptr, *sid = nullptr, *nmask = nullptr;
  float2* sdq = nullptr;
  uint32_t *count = nullptr, *start = nullptr, *tilesum = nullptr, *scalar = nullptr;
  unsigned long long* tstate = nullptr;  // single-pass scan tile states
  uint32_t count_len = 0, range_cap = 0;
  DevBody3* dbodies = nullptr;
  uint32_t bodies_cap = 0;
  unsigned int* h_pinned = nullptr;
  cudaGraphExec_t gexec = nullptr;
  std::string gsig;
  bool profiling = false;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  // the fluid phase with the engine's bodies (phieng_sph3_step_fluid)
  DevBodyQ3* d_qbodies = nullptr;
  DynBody3* d_dyn = nullptr;
  uint32_t* d_buoy = nullptr;
  uint32_t qbody_cap = 0;
  float4* d_samples = nullptr;  // two per sample: (point, area), (normal, 0)
  uint32_t sample_cap = 0;
  float4* d_hullv = nullptr;
  uint32_t hull_cap = 0;
  uint32_t *d_defer = nullptr, *d_dcount = nullptr, *d_dstart = nullptr, *d_dtile = nullptr, *d_list = nullptr;
  float2* d_dq_id = nullptr;
  float* d_p_id = nullptr;
  uint32_t dyn_pcap = 0;
  uint32_t* d_count2 = nullptr;
  uint32_t count2_cap = 0;
};

namespace {

bool ok3(World3* w, cudaError_t r) {
  if (r == cudaSuccess) return true;
  cudaGetLastError();
  if (w->error == PHIENG_SPH_OK) w->error = PHIENG_SPH_E_CUDA;
  return false;
}

template <class T>
void dfree3(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

template <class T>
bool dalloc3(World3* w, T*& p, size_t count) {
  return ok3(w, cudaMalloc(&p, sizeof(T) * std::max<size_t>(count, 1)));
}

void release_graph3(World3* w) {
  if (w->gexec) cudaGraphExecDestroy(w->gexec);
  w->gexec = nullptr;
  w->gsig.clear();
}

void free_particles3(World3* w) {
  dfree3(w->pos), dfree3(w->vel), dfree3(w->spos), dfree3(w->svel), dfree3(w->mass), dfree3(w->smass);
  dfree3(w->spres), dfree3(w->tmp), dfree3(w->phase), dfree3(w->sphase), dfree3(w->key), dfree3(w->tkey);
  dfree3(w->tid), dfree3(w->skey), dfree3(w->sid), dfree3(w->nmask), dfree3(w->sdq);
  w->dcap = 0;
}

bool ensure_device3(World3* w) {
  if (w->device >= 0) return true;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    w->error = PHIENG_SPH_E_NO_DEVICE;
    return false;
  }
  int dev = 0;
  if (!ok3(w, cudaGetDevice(&dev))) return false;
  if (!ok3(w, cudaStreamCreateWithFlags(&w->own_stream, cudaStreamNonBlocking))) return false;
  if (!w->user_stream) w->stream = w->own_stream;
  if (!ok3(w, cudaMalloc(&w->scalar, 128)) || !ok3(w, cudaMemset(w->scalar, 0, 128))) return false;
  if (!ok3(w, cudaMallocHost(&w->h_pinned, 64))) return false;
  w->device = dev;
  return true;
}

bool ensure_capacity3(World3* w, uint32_t need) {
  if (need <= w->dcap && w->pos) return true;
  cudaStreamSynchronize(w->stream);
  free_particles3(w);
  release_graph3(w);
  const uint32_t c = std::max<uint32_t>(need, 1024);
  const bool ok = dalloc3(w, w->pos, c) && dalloc3(w, w->vel, c) && dalloc3(w, w->spos, c) && dalloc3(w, w->svel, c) &&
                  dalloc3(w, w->mass, c) && dalloc3(w, w->smass, c) && dalloc3(w, w->spres, c) &&
                  dalloc3(w, w->tmp, 2 * (size_t)c) && dalloc3(w, w->phase, c) && dalloc3(w, w->sphase, c) &&
                  dalloc3(w, w->key, c) && dalloc3(w, w->tkey, c) && dalloc3(w, w->tid, c) && dalloc3(w, w->skey, c) &&
                  dalloc3(w, w->sid, c) && dalloc3(w, w->nmask, 9 * (size_t)c) && dalloc3(w, w->sdq, c);
  if (!ok) {
    free_particles3(w);
    return false;
  }
  w->dcap = c;
  w->dev_valid = w->aux_valid = w->keys_valid = false;
  w->sid_perm_n = 0;
  return true;
}

bool ensure_host3(World3* w) {
  if (w->host_valid) return true;
  if (!ok3(w, cudaMemcpyAsync(w->h_pos.data(), w->pos, sizeof(float4) * w->n, cudaMemcpyDeviceToHost, w->stream)) ||
      !ok3(w, cudaMemcpyAsync(w->h_vel.data(), w->vel, sizeof(float4) * w->n, cudaMemcpyDeviceToHost, w->stream)) ||
      !ok3(w, cudaStreamSynchronize(w->stream)))
    return false;
  w->host_valid = true;
  return true;
}

// Bring the density / pressure of the last density pass (sorted order on the
// device) back to insertion order on the host.
bool ensure_host_dp3(World3* w) {
  if (!w->dp_dev) return true;
  k_unsort3<<<cdiv(w->n, 256), 256, 0, w->stream>>>(w->sdq, w->spres, w->sid, w->n, w->tmp, w->tmp + w->dcap);
  if (!ok3(w, cudaGetLastError()) ||
      !ok3(w, cudaMemcpyAsync(w->h_dens.data(), w->tmp, sizeof(float) * w->n, cudaMemcpyDeviceToHost, w->stream)) ||
      !ok3(w, cudaMemcpyAsync(w->h_pres.data(), w->tmp + w->dcap, sizeof(float) * w->n, cudaMemcpyDeviceToHost,
                              w->stream)) ||
      !ok3(w, cudaStreamSynchronize(w->stream)))
    return false;
  w->dp_dev = false;
  return true;
}

void plan_grid3(World3* w) {
  const float hg = w->cfg.smoothing_length;
  int64_t lo[3] = {INT64_MAX, INT64_MAX, INT64_MAX}, hi[3] = {INT64_MIN, INT64_MIN, INT64_MIN};
  for (uint32_t i = 0; i < w->n; i++) {
    const float4 p = w->h_pos[i];
    if (!std::isfinite(p.x) || !std::isfinite(p.y) || !std::isfinite(p.z)) continue;
    const int32_t c[3] = {sat_floor_i32(p.x / hg), sat_floor_i32(p.y / hg), sat_floor_i32(p.z / hg)};
    for (int a = 0; a < 3; a++) {
      lo[a] = std::min<int64_t>(lo[a], c[a]);
      hi[a] = std::max<int64_t>(hi[a], c[a]);
    }
  }
  if (lo[0] > hi[0]) lo[0] = lo[1] = lo[2] = hi[0] = hi[1] = hi[2] = 0;
  uint32_t lg[3];  // log2 of the buckets along x, y, z (each >= 2)
  int64_t mg[3];
  for (int a = 0; a < 3; a++) {
    const int64_t ext = hi[a] - lo[a] + 1;
    mg[a] = std::max<int64_t>(2, ext / 8);
    lg[a] = std::max<uint32_t>(2, log2u(next_pow2((uint64_t)(ext + 2 * mg[a]))));
  }
  // bucket budget: ~2 per particle (each bucket costs ~20 B of scan traffic),
  // 2^12 .. 2^24; halve the longest axis until the grid fits
  const uint32_t lb = std::min<uint32_t>(24, std::max<uint32_t>(12, log2u(next_pow2(2ull * w->n))));
  while (lg[0] + lg[1] + lg[2] > lb) {
    int a = 0;
    for (int b = 1; b < 3; b++)
      if (lg[b] > lg[a]) a = b;
    if (lg[a] <= 2) break;
    lg[a]--;
  }
  GridPlan3 g;
  g.log2w = lg[0];
  g.log2h = lg[1];
  g.log2d = lg[2];
  g.maskw = (1u << lg[0]) - 1;
  g.maskh = (1u << lg[1]) - 1;
  g.maskd = (1u << lg[2]) - 1;
  g.nbuckets = 1u << (lg[0] + lg[1] + lg[2]);
  g.sentinel = g.nbuckets;
  g.cx0 = (int32_t)std::max<int64_t>(INT32_MIN, lo[0] - mg[0]);
  g.cy0 = (int32_t)std::max<int64_t>(INT32_MIN, lo[1] - mg[1]);
  g.cz0 = (int32_t)std::max<int64_t>(INT32_MIN, lo[2] - mg[2]);
  g.hg = hg;
  w->plan = g;
  w->plan_valid = true;
  w->keys_valid = false;
}

bool ensure_range3(World3* w) {
  const uint32_t m = w->plan.sentinel + 1;
  const uint32_t tiles = (m + kBucketScanTile - 1) / kBucketScanTile;
  if (w->count && w->range_cap >= w->plan.nbuckets) {
    w->count_len = tiles * kBucketScanTile;
    return true;
  }
  cudaStreamSynchronize(w->stream);
  dfree3(w->count), dfree3(w->start), dfree3(w->tilesum), dfree3(w->tstate);
  release_graph3(w);
  const uint32_t len = tiles * kBucketScanTile;
  if (!dalloc3(w, w->count, len) || !dalloc3(w, w->start, (size_t)len + 1) || !dalloc3(w, w->tilesum, tiles) ||
      !dalloc3(w, w->tstate, tiles))
    return false;
  if (!ok3(w, cudaMemsetAsync(w->count, 0, sizeof(uint32_t) * len, w->stream)) ||
      !ok3(w, cudaMemsetAsync(w->tstate, 0, sizeof(unsigned long long) * tiles, w->stream)))
    return false;
  w->range_cap = w->plan.nbuckets;
  w->count_len = len;
  w->keys_valid = false;
  return true;
}

bool ensure_bodies3(World3* w) {
  if (!w->bodies_dirty) return true;
  const uint32_t nb = (uint32_t)w->bodies.size();
  if (nb > w->bodies_cap || !w->dbodies) {
    cudaStreamSynchronize(w->stream);
    dfree3(w->dbodies);
    release_graph3(w);
    const uint32_t c = std::max<uint32_t>(16, nb);
    if (!dalloc3(w, w->dbodies, c)) return false;
    w->bodies_cap = c;
  }
  if (nb && !ok3(w, cudaMemcpyAsync(w->dbodies, w->bodies.data(), sizeof(DevBody3) * nb, cudaMemcpyHostToDevice,
                                    w->stream)))
    return false;
  w->bodies_dirty = false;
  return true;
}

void enqueue_keys3(World3* w, cudaStream_t st) {
  cudaMemsetAsync(w->count, 0, sizeof(uint32_t) * w->count_len, st);
  if (w->n) k_keys3<<<cdiv(w->n, 256), 256, 0, st>>>(w->pos, w->n, w->plan, w->key, w->count);
}

bool prepare3(World3* w) {
  if (w->error != PHIENG_SPH_OK) return false;
  if (!ensure_device3(w)) return false;
  if (!w->dev_valid) {
    // adaptive resolution: room for what a resample pass can output
    if (!ensure_capacity3(w, w->cfg.adaptive_resolution ? std::max(resample_bound3(w->n), kMaxParticles3D) : w->n))
      return false;
    if (!w->plan_valid) plan_grid3(w);
    if (w->n && (!ok3(w, cudaMemcpyAsync(w->pos, w->h_pos.data(), sizeof(float4) * w->n, cudaMemcpyHostToDevice,
                                         w->stream)) ||
                 !ok3(w, cudaMemcpyAsync(w->vel, w->h_vel.data(), sizeof(float4) * w->n, cudaMemcpyHostToDevice,
                                         w->stream))))
      return false;
    w->dev_valid = true;
    w->keys_valid = false;
  }
  if (!w->aux_valid && (!w->mass_uniform || !w->phase_uniform) && w->n) {
    if (!ok3(w, cudaMemcpyAsync(w->mass, w->h_mass.data(), sizeof(float) * w->n, cudaMemcpyHostToDevice, w->stream)) ||
        !ok3(w, cudaMemcpyAsync(w->phase, w->h_phase.data(), w->n, cudaMemcpyHostToDevice, w->stream)))
      return false;
    w->aux_valid = true;
  }
  if (!w->plan_valid) {
    if (!ensure_host3(w)) return false;
    plan_grid3(w);
  }
  if (!ensure_range3(w) || !ensure_bodies3(w)) return false;
  if (!w->keys_valid) {
    enqueue_keys3(w, w->stream);
    w->keys_valid = true;
  }
  return ok3(w, cudaGetLastError());
}

// ---- boundary ghosts (fluid3.rs:719-922) ----
int32_t as_i32_3(float v) {  // Rust `as i32`: truncate, saturate, NaN -> 0
  if (v != v) return 0;
  if (v <= -2147483648.0f) return INT32_MIN;
  if (v >= 2147483648.0f) return INT32_MAX;
  return (int32_t)v;
}
uint64_t ghost_count3(float v, float hi) {  // `.ceil().clamp(1.0, hi) as usize` (NaN -> 0)
  if (v != v) return 0;
  return (uint64_t)std::min(std::max(std::ceil(v), 1.0f), hi);
}

// refresh_boundaries (fluid3.rs:719-855) for the world's static spheres,
// boxes and capsules (identity rotation: transform_point = (x_axis * v.x +
// y_axis * v.y + z_axis * v.z) + position, evaluated as glam's Mat3 * Vec3),
// at spacing max(h * 0.5, EPS).
void generate_ghosts3(const std::vector<DevBody3>& bodies, float hk, std::vector<float4>& out) {
  const float spacing = std::max(hk * 0.5f, kEps);
  const float sp2 = spacing * spacing;  // powi(2)
  const float pi = 3.14159265358979323846f;
  out.clear();
  for (const DevBody3& b : bodies) {
    auto put = [&](float x, float y, float z) {
      const float wx = ((1.0f * x + 0.0f * y) + 0.0f * z) + b.px;
      const float wy = ((0.0f * x + 1.0f * y) + 0.0f * z) + b.py;
      const float wz = ((0.0f * x + 0.0f * y) + 1.0f * z) + b.pz;
      out.push_back(make_float4(wx, wy, wz, 0.0f));
    };
    if (b.shape == 0) {  // sphere: golden-angle spiral
      const float r = b.a;
      const uint64_t n = ghost_count3((4.0f * pi * r * r) / sp2, 512.0f);
      const float golden = pi * (3.0f - std::sqrt(5.0f));
      for (uint64_t k = 0; k < n; k++) {
        const float z = 1.0f - 2.0f * ((float)k + 0.5f) / (float)n;
        const float rr = std::sqrt(1.0f - z * z);
        const float th = golden * (float)k;
        put(std::cos(th) * rr * r, z * r, std::sin(th) * rr * r);
      }
    } else if (b.shape == 1) {  // box: six faces, (7 t) mod 1 across each
      const float hx = b.a, hy = b.b, hz = b.c;
      const float fixed[6] = {-hy, -hy, -hx, -hx, -hz, -hz};
      const int axis[6] = {0, 0, 1, 1, 2, 2};
      for (int f = 0; f < 6; f++) {
        const int ax = axis[f];
        const float area = ax == 0 ? 4.0f * hy * hz : ax == 1 ? 4.0f * hx * hz : 4.0f * hx * hy;
        const uint64_t n = ghost_count3(area / sp2, 512.0f);
        for (uint64_t k = 0; k < n; k++) {
          const float t = ((float)k + 0.5f) / (float)n;
          const float u = 2.0f * t - 1.0f, v = 2.0f * std::fmod(t * 7.0f, 1.0f) - 1.0f;
          float lx = 0.0f, ly = 0.0f, lz = fixed[f];
          if (ax == 0) {
            ly = u * hy;
            lz = v * hz;
          } else if (ax == 1) {
            lx = u * hx;
            lz = v * hz;
          } else {
            lx = u * hx;
            ly = v * hy;
          }
          put(lx, ly, lz);
        }
      }
    } else {  // capsule along y: two rings at +-hl / 2, then the two poles
      const float r = b.a, hl = b.b;
      const uint64_t n = ghost_count3((4.0f * pi * r * hl) / sp2, 256.0f);
      for (float sy : {-hl * 0.5f, hl * 0.5f})
        for (uint64_t k = 0; k < n; k++) {
          const float a = 2.0f * pi * (float)k / (float)n;
          put(std::cos(a) * r, sy, std::sin(a) * r);
        }
      for (float sg : {-1.0f, 1.0f}) {
        const float len = hl + r;
        put((0.0f * sg) * len, (1.0f * sg) * len, (0.0f * sg) * len);  // Vec3::Y * s * (hl + r)
      }
    }
  }
}

// Ghosts of the static bodies `bodies` (the world's own, or the statics of a
// fluid-phase call), regenerated when they or the kernel config change.
bool refresh_ghosts3(World3* w, const std::vector<DevBody3>& bodies) {
  const FluidConfig3Ffi& c = w->cfg;
  std::string sig;
  auto add = [&](const void* p, size_t n) { sig.append((const char*)p, n); };
  add(&c.smoothing_length, 4);
  add(&c.particle_mass, 4);
  add(&c.rest_density, 4);
  for (const DevBody3& b : bodies) add(&b, sizeof(DevBody3));
  if (sig == w->ghost_sig && w->d_gtab) return true;
  const float hk = std::max(c.smoothing_length, kEps);
  std::vector<float4> raw;
  generate_ghosts3(bodies, hk, raw);
  std::vector<std::pair<std::pair<int64_t, int32_t>, uint32_t>> order;  // ((x, y), z) cell key, index
  std::vector<int32_t> cell(3 * raw.size());
  for (uint32_t i = 0; i < raw.size(); i++) {
    if (!std::isfinite(raw[i].x)) continue;  // rebuild_boundary_grid checks x only (fluid3.rs:842-844)
    const int32_t cx = as_i32_3(std::floor(raw[i].x / hk)), cy = as_i32_3(std::floor(raw[i].y / hk));
    const int32_t cz = as_i32_3(std::floor(raw[i].z / hk));
    cell[3 * i] = cx, cell[3 * i + 1] = cy, cell[3 * i + 2] = cz;
    order.push_back({{((int64_t)cx << 32) | (uint32_t)cy, cz}, i});
  }
  std::stable_sort(order.begin(), order.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
  std::vector<float4> gpos(order.size());
  std::vector<GhostCell3> cells;
  for (size_t k = 0; k < order.size(); k++) {
    const uint32_t i = order[k].second;
    gpos[k] = raw[i];
    if (cells.empty() || cells.back().cx != cell[3 * i] || cells.back().cy != cell[3 * i + 1] ||
        cells.back().cz != cell[3 * i + 2])
      cells.push_back({cell[3 * i], cell[3 * i + 1], cell[3 * i + 2], (uint32_t)k, 0});
    cells.back().count++;
  }
  uint32_t tsize = 16;
  while (tsize < 2 * cells.size()) tsize <<= 1;
  std::vector<GhostCell3> tab(tsize, GhostCell3{0, 0, 0, 0, 0});
  for (const GhostCell3& gc : cells) {
    uint32_t slot = ghost_cell_hash3(gc.cx, gc.cy, gc.cz, tsize - 1);
    while (tab[slot].count != 0) slot = (slot + 1) & (tsize - 1);
    tab[slot] = gc;
  }
  const uint32_t ng = (uint32_t)gpos.size();
  if (ng > w->ghost_cap || !w->d_gpos) {
    cudaStreamSynchronize(w->stream);
    dfree3(w->d_gpos), dfree3(w->d_gq);
    const uint32_t cp = std::max<uint32_t>(ng, 64);
    if (!dalloc3(w, w->d_gpos, cp) || !dalloc3(w, w->d_gq, cp)) return false;
    w->ghost_cap = cp;
  }
  if (tsize > w->gtab_cap) {
    cudaStreamSynchronize(w->stream);
    dfree3(w->d_gtab);
    if (!dalloc3(w, w->d_gtab, tsize)) return false;
    w->gtab_cap = tsize;
  }
  if ((ng && !ok3(w, cudaMemcpyAsync(w->d_gpos, gpos.data(), sizeof(float4) * ng, cudaMemcpyHostToDevice, w->stream))) ||
      !ok3(w, cudaMemcpyAsync(w->d_gtab, tab.data(), sizeof(GhostCell3) * tsize, cudaMemcpyHostToDevice, w->stream)) ||
      !ok3(w, cudaStreamSynchronize(w->stream)))
    return false;
  w->nghost = ng;
  w->gtab_mask = tsize - 1;
  w->ghost_sig = sig;
  w->h_gpos = std::move(gpos);
  w->ghost_regens++;
  return true;
}

StepParams3 make_params3(const World3* w, float dt) {
  StepParams3 P;
  std::memset(&P, 0, sizeof(P));
  const FluidConfig3Ffi& c = w->cfg;
  P.grid = w->plan;
  const float hg = c.smoothing_length;
  P.hg2 = hg * hg;
  const float h = rmaxf(hg, kEps);
  P.hk = h;
  const float h2 = h * h;
  P.hk2 = h2;
  const float pi = 3.14159265358979323846f;
  P.c_poly6 = 315.0f / (64.0f * pi * h2 * h2 * h2 * h2 * h);
  P.c_spiky = -45.0f / (pi * h * h * h * h * h * h);
  P.rho_cap = 3.0f * rmaxf(c.rest_density, kEps);
  P.stiffness = c.stiffness;
  P.gamma = c.gamma;
  for (int k = 0; k < 4; k++) P.rest[k] = c.phase_rest_density[k];
  P.mass = w->mass_value;
  P.visc = c.viscosity;
  P.vmax = c.max_velocity;
  P.dt = dt;
  P.gx = w->gx;
  P.gy = w->gy;
  P.gz = w->gz;
  P.pr = rmaxf(c.particle_radius, 0.0f);
  P.pr_pad = P.pr * 1.001f + 1e-30f;
  float mu = c.wall_friction;
  if (mu < 0.0f) mu = 0.0f;
  if (mu > 1.0f) mu = 1.0f;
  P.mu = mu;
  P.av_alpha = c.artificial_viscosity;
  P.c_s = std::sqrt(rmaxf(c.stiffness, 0.0f));
  P.surface_tension = c.surface_tension;
  uint32_t f = 0;
  if (c.viscosity > 0.0f) f |= F_VISC;
  if (c.artificial_viscosity > 0.0f) f |= F_AV;
  if (c.surface_tension > 0.0f) f |= F_COHESION;
  if (c.wall_friction > 0.0f) f |= F_FRICTION;
  if (c.gamma != 1.0f) f |= F_TAIT;
  if (!w->mass_uniform) f |= F_MASS;
  if (!w->phase_uniform) f |= F_PHASE;
  if (!(P.hg2 <= P.hk2)) f |= F_WIDE_NB;
  if (c.boundary_particles && w->nghost && w->d_gtab) {
    f |= F_GHOST;
    P.gpos = w->d_gpos;
    P.gq = w->d_gq;
    P.gtab = w->d_gtab;
    P.gtab_mask = w->gtab_mask;
    P.nghost = w->nghost;
    P.gmass = std::max(c.particle_mass, kEps);
    P.rest0 = c.rest_density;
  }
  const AmbientConfig3Ffi& a = w->ambient;
  if (a.turbulence_enabled != 0 && a.turbulence_amplitude > 0.0f && w->scalar) {  // fluid3.rs:1090-1091
    f |= F_TURB;
    if (a.turbulence_divergence_free) f |= F_TURB_CURL;
    P.turb_amp = a.turbulence_amplitude;
    P.turb_freq = a.turbulence_frequency;
    P.turb_tscale = a.turbulence_time_scale;
    P.turb_seed = a.turbulence_seed;
    P.turb_oct = std::min<uint32_t>(std::max<uint32_t>(a.turbulence_octaves, 1u), 8u);
    P.clock = reinterpret_cast<const float*>(w->scalar + kClockWord3);
  }
  P.flags = f;
  P.nbodies = (uint32_t)w->bodies.size();
  P.uniform_phase = w->phase_value;
  if (w->precision == PHIENG_SPH_TOLERANCE) P.flags |= F_FAST;
  return P;
}

void enqueue_sort3(World3* w, const StepParams3& P, cudaStream_t st) {
  BucketSort bs;
  bs.count = w->count;
  bs.tilesum = w->tilesum;
  bs.done = w->scalar + 8;  // scan counters [8], [9]
  bs.tstate = w->tstate;
  bs.err = w->scalar + 12;
  bs.start = w->start;
  bs.key = w->key;
  bs.sid_prev = w->sid;
  bs.tkey = w->tkey;
  bs.tid = w->tid;
  enqueue_bucket_place(bs, w->n, P.grid.sentinel + 1, w->sid_perm_n == w->n, st);
  const bool m = (P.flags & F_MASS) != 0, ph = (P.flags & F_PHASE) != 0;
  k_fixup3<<<cdiv(w->n, 256), 256, 0, st>>>(w->tkey, w->tid, w->start, w->n, w->skey, w->sid, w->pos, w->vel, w->mass,
                                            w->phase, w->spos, w->svel, m ? w->smass : nullptr,
                                            ph ? w->sphase : nullptr);
  cudaMemsetAsync(w->count, 0, sizeof(uint32_t) * w->count_len, st);
}

void enqueue_density3(World3* w, const StepParams3& P, cudaStream_t st) {
  const bool m = (P.flags & F_MASS) != 0, ph = (P.flags & F_PHASE) != 0;
  const uint32_t g = cdiv(w->n, 256);
  const bool wide = (P.flags & F_WIDE_NB) != 0;
#define PHIENG_D3(M, PH)                                                                                     \
  do {                                                                                                       \
    if (wide)                                                                                                \
      k_density3<M, PH, true><<<g, 256, 0, st>>>(w->spos, w->skey, w->smass, w->sphase, w->n, w->start, P,  \
                                                 w->sdq, w->spres, w->nmask);                                \
    else                                                                                                     \
      k_density3<M, PH, false><<<g, 256, 0, st>>>(w->spos, w->skey, w->smass, w->sphase, w->n, w->start, P, \
                                                  w->sdq, w->spres, w->nmask);                               \
  } while (0)
  if (m && ph) PHIENG_D3(true, true);
  else if (m) PHIENG_D3(true, false);
  else if (ph) PHIENG_D3(false, true);
  else PHIENG_D3(false, false);
#undef PHIENG_D3
}

void enqueue_force3(World3* w, const StepParams3& P, float4* dbg, cudaStream_t st) {
  const bool m = (P.flags & F_MASS) != 0;
  const uint32_t g = cdiv(w->n, 128);  // 128-thread blocks: 286 -> 280 us at 1M (256, 5-block cap: 329 us)
  // XSPH on, artificial viscosity and cohesion off, h*h <= hk*hk: the
  // optional pair terms compiled out
  const bool plain = (P.flags & F_VISC) && !(P.flags & (F_AV | F_COHESION | F_WIDE_NB | F_TURB | F_GHOST));
  // tolerance mode: the plain pass with uniform mass runs pair3_fast
  const bool fast = plain && !m && (P.flags & F_FAST);
#define PHIENG_F3X(M, D, PL, FA)                                                                                    \
  k_force3<M, D, PL, FA><<<g, 128, 0, st>>>(w->spos, w->svel, w->sdq, w->skey, w->sid, w->smass, w->n, w->start, \
                                            P, w->dbodies, w->nmask, w->pos, w->vel, w->key, w->count, dbg)
#define PHIENG_F3(M, D, PL) PHIENG_F3X(M, D, PL, false)
  if (fast) {
    if (dbg) PHIENG_F3X(false, true, true, true);
    else PHIENG_F3X(false, false, true, true);
  } else if (dbg) {
    if (m) PHIENG_F3(true, true, false);
    else PHIENG_F3(false, true, false);
  } else if (plain) {
    if (m) PHIENG_F3(true, false, true);
    else PHIENG_F3(false, false, true);
  } else {
    if (m) PHIENG_F3(true, false, false);
    else PHIENG_F3(false, false, false);
  }
#undef PHIENG_F3
#undef PHIENG_F3X
}

void enqueue_substep3(World3* w, const StepParams3& P, cudaStream_t st) {
  if (w->profiling) cudaEventRecordWithFlags(w->ev[0], st, cudaEventRecordExternal);
  enqueue_sort3(w, P, st);
  if (w->profiling) cudaEventRecordWithFlags(w->ev[1], st, cudaEventRecordExternal);
  enqueue_density3(w, P, st);
  if ((P.flags & F_GHOST) && P.nghost) {
    if (P.flags & F_MASS)
      k_ghost_density3<true><<<cdiv(P.nghost, 256), 256, 0, st>>>(w->spos, w->smass, w->start, P);
    else
      k_ghost_density3<false><<<cdiv(P.nghost, 256), 256, 0, st>>>(w->spos, w->smass, w->start, P);
  }
  if (w->profiling) cudaEventRecordWithFlags(w->ev[2], st, cudaEventRecordExternal);
  enqueue_force3(w, P, nullptr, st);
  if (w->profiling) cudaEventRecordWithFlags(w->ev[3], st, cudaEventRecordExternal);
}

bool run_substep3(World3* w, const StepParams3& P) {
  std::string sig((const char*)&P, sizeof(P));
  sig.append((const char*)&w->n, sizeof(w->n));
  sig.push_back(w->profiling ? 'p' : '-');
  sig.push_back(w->sid_perm_n == w->n ? 's' : '-');
  if (!w->gexec || sig != w->gsig) {
    release_graph3(w);
    cudaGraph_t g = nullptr;
    if (!ok3(w, cudaStreamBeginCapture(w->own_stream, cudaStreamCaptureModeThreadLocal))) return false;
    enqueue_substep3(w, P, w->own_stream);
    cudaError_t r = cudaStreamEndCapture(w->own_stream, &g);
    if (!ok3(w, r)) return false;
    r = cudaGraphInstantiate(&w->gexec, g, 0);
    cudaGraphDestroy(g);
    if (!ok3(w, r)) {
      w->gexec = nullptr;
      return false;
    }
    w->gsig = sig;
  }
  if (!ok3(w, cudaGraphLaunch(w->gexec, w->stream))) return false;
  w->sid_perm_n = w->n;
  w->substeps++;
  w->host_valid = false;
  w->dp_dev = true;
  w->keys_valid = true;
  return true;
}

bool cfl_substeps3(World3* w, float dt, uint32_t* out) {
  const FluidConfig3Ffi& c = w->cfg;
  const uint32_t mx = std::max<uint32_t>(c.max_substeps, 1);
  *out = 1;
  if (c.cfl <= 0.0f || mx <= 1) return true;
  const float h = rmaxf(c.smoothing_length, kEps);
  const float rho0 = rmaxf(c.rest_density, kEps);
  const float c0 = (c.gamma == 1.0f) ? std::sqrt(rmaxf(c.stiffness, 0.0f))
                                     : std::sqrt(c.gamma * rmaxf(c.stiffness, 0.0f) * rho0);
  float vmax = 0.0f;
  if (w->host_valid) {
    for (uint32_t i = 0; i < w->n; i++) {
      const float4 v = w->h_vel[i];
      vmax = rmaxf(vmax, std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z));
    }
  } else {
    cudaMemsetAsync(w->scalar, 0, 4, w->stream);
    k_vmax3<<<std::min(cdiv(w->n, 256), 148u * 8u), 256, 0, w->stream>>>(w->vel, w->n, w->scalar);
    if (!ok3(w, cudaMemcpyAsync(w->h_pinned, w->scalar, 4, cudaMemcpyDeviceToHost, w->stream)) ||
        !ok3(w, cudaStreamSynchronize(w->stream)))
      return false;
    std::memcpy(&vmax, w->h_pinned, 4);
  }
  const float speed = c0 + vmax;
  if (!std::isfinite(speed) || speed <= kEps) return true;
  const float dt_max = c.cfl * h / speed;
  if (!std::isfinite(dt_max) || dt_max <= 0.0f) return true;
  const float q = std::ceil(dt / dt_max);
  int64_t k;
  if (q != q)
    k = 0;
  else if (q >= 9.2233720368547758e18f)
    k = INT64_MAX;
  else
    k = (int64_t)q;
  k = std::max<int64_t>(1, std::min<int64_t>(k, mx));
  *out = (uint32_t)k;
  return true;
}

void recompute_uniformity3(World3* w);

// One 3D substep with adaptive resolution (fluid3.rs:1008-1016), as the 2D
// one: sort and density, resample (one thread), one read of the new count,
// then the new set's keys and the whole substep body.
bool run_substep3_adaptive(World3* w, float dt) {
  if (w->dcap < resample_bound3(w->n)) {
    // an earlier CFL substep of this step grew the set: bring the state home
    // and upload it into buffers with room for this pass's output
    if (!ensure_host3(w)) return false;
    w->dev_valid = false;
    if (!prepare3(w)) return false;
  }
  const uint32_t c = w->dcap;
  if (w->rs_cap < c || !w->rs_pos) {
    cudaStreamSynchronize(w->stream);
    dfree3(w->rs_slot), dfree3(w->rs_absorbed), dfree3(w->rs_pos), dfree3(w->rs_vel), dfree3(w->rs_mass),
        dfree3(w->rs_phase);
    if (!dalloc3(w, w->rs_slot, c) || !dalloc3(w, w->rs_absorbed, c) || !dalloc3(w, w->rs_pos, c) ||
        !dalloc3(w, w->rs_vel, c) || !dalloc3(w, w->rs_mass, c) || !dalloc3(w, w->rs_phase, c))
      return false;
    w->rs_cap = c;
  }
  cudaStream_t st = w->stream;
  StepParams3 P = make_params3(w, dt);
  enqueue_sort3(w, P, st);
  w->sid_perm_n = w->n;
  enqueue_density3(w, P, st);
  const FluidConfig3Ffi& cf = w->cfg;
  const float rest = std::max(cf.rest_density, kEps);
  uint32_t* n_out = w->scalar + 18;
  if (w->n) {
    k_resample_prep3<<<cdiv(w->n, 256), 256, 0, st>>>(w->sid, w->n, w->rs_slot, w->mass, w->phase,
                                                       w->mass_uniform ? 1 : 0, P.mass, w->phase_uniform ? 1 : 0,
                                                       (uint8_t)P.uniform_phase);
    k_resample3<<<1, 1, 0, st>>>(w->n, w->pos, w->vel, w->mass, w->phase, w->sdq, w->sid, w->skey, w->rs_slot,
                                 w->start, P, cf.merge_density_ratio * rest, cf.split_density_ratio * rest,
                                 std::max(cf.particle_mass, kEps) * 0.125f, w->rs_absorbed, w->rs_pos, w->rs_vel,
                                 w->rs_mass, w->rs_phase, c, n_out);
  } else {
    cudaMemsetAsync(n_out, 0, 4, st);
  }
  if (!ok3(w, cudaMemcpyAsync(w->h_pinned, n_out, 4, cudaMemcpyDeviceToHost, st)) || !ok3(w, cudaStreamSynchronize(st)))
    return false;
  uint32_t n2;
  std::memcpy(&n2, w->h_pinned, 4);
  if (n2 > c) {
    w->error = PHIENG_SPH_E_CUDA;
    return false;
  }
  w->h_pos.resize(n2), w->h_vel.resize(n2), w->h_mass.resize(n2), w->h_phase.resize(n2);
  w->h_dens.resize(n2), w->h_pres.resize(n2);
  if (n2 && (!ok3(w, cudaMemcpyAsync(w->pos, w->rs_pos, sizeof(float4) * n2, cudaMemcpyDeviceToDevice, st)) ||
             !ok3(w, cudaMemcpyAsync(w->vel, w->rs_vel, sizeof(float4) * n2, cudaMemcpyDeviceToDevice, st)) ||
             !ok3(w, cudaMemcpyAsync(w->mass, w->rs_mass, sizeof(float) * n2, cudaMemcpyDeviceToDevice, st)) ||
             !ok3(w, cudaMemcpyAsync(w->phase, w->rs_phase, n2, cudaMemcpyDeviceToDevice, st)) ||
             !ok3(w, cudaMemcpyAsync(w->h_mass.data(), w->rs_mass, sizeof(float) * n2, cudaMemcpyDeviceToHost, st)) ||
             !ok3(w, cudaMemcpyAsync(w->h_phase.data(), w->rs_phase, n2, cudaMemcpyDeviceToHost, st)) ||
             !ok3(w, cudaStreamSynchronize(st))))
    return false;
  w->n = n2;
  recompute_uniformity3(w);
  w->aux_valid = true;
  w->host_valid = false;
  P = make_params3(w, dt);
  enqueue_keys3(w, st);
  w->sid_perm_n = 0;
  enqueue_substep3(w, P, st);
  if (!ok3(w, cudaGetLastError())) return false;
  w->sid_perm_n = w->n;
  w->substeps++;
  w->dp_dev = true;
  w->keys_valid = true;
  return true;
}

bool world_step3(World3* w, float dt) {
  if (w->cfg.enabled && w->n > 0 && dt > 0.0f) {
    if (w->cfg.adaptive_resolution && w->pos && w->dcap < std::max(resample_bound3(w->n), kMaxParticles3D)) {
      if (!ensure_host3(w)) return false;  // room for the splits: re-upload into larger buffers
      w->dev_valid = false;
    }
    if (!prepare3(w)) return false;
    if (w->cfg.boundary_particles && !refresh_ghosts3(w, w->bodies)) return false;
    uint32_t ns = 1;
    if (!cfl_substeps3(w, dt, &ns)) return false;
    const StepParams3 P = make_params3(w, dt / (float)ns);
    if (P.flags & F_TURB) {  // every CFL substep sees the step's start time (world.rs:2811)
      uint32_t bits;
      std::memcpy(&bits, &w->time, 4);
      enqueue_set_word(w->scalar + kClockWord3, bits, w->stream);
    }
    for (uint32_t k = 0; k < ns; k++)
      if (!(w->cfg.adaptive_resolution ? run_substep3_adaptive(w, dt / (float)ns) : run_substep3(w, P))) return false;
  }
  w->time += dt;
  return true;
}

void recompute_uniformity3(World3* w) {
  w->mass_uniform = w->phase_uniform = true;
  w->mass_value = rmaxf(w->cfg.phase_mass[0], 0.0f);
  w->phase_value = 0;
  if (w->n) {
    w->mass_value = w->h_mass[0];
    w->phase_value = std::min<uint32_t>(w->h_phase[0], 3);
  }
  for (uint32_t i = 1; i < w->n; i++) {
    if (w->h_mass[i] != w->mass_value) w->mass_uniform = false;
    if (std::min<uint32_t>(w->h_phase[i], 3) != w->phase_value) w->phase_uniform = false;
  }
}

uint32_t add_particles3(World3* w, const float* xyz, const uint8_t* phases, uint32_t count) {
  uint32_t n = std::min(count, kMaxAddPerCall);
  for (uint64_t i = 0; i < 3ull * n; i++)
    if (!std::isfinite(xyz[i])) return 0;
  const uint32_t room = w->cap > w->n ? w->cap - w->n : 0;
  n = std::min(n, room);
  if (n == 0) return 0;
  if (!ensure_host3(w) || !ensure_host_dp3(w)) return 0;
  for (uint32_t i = 0; i < n; i++) {
    const uint8_t ph = phases ? phases[i] : 0;
    const uint32_t k = std::min<uint32_t>(ph, 3);
    w->h_pos.push_back(make_float4(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], 0.0f));
    w->h_vel.push_back(make_float4(0.0f, 0.0f, 0.0f, 0.0f));
    w->h_dens.push_back(w->cfg.phase_rest_density[k]);
    w->h_pres.push_back(0.0f);
    w->h_mass.push_back(rmaxf(w->cfg.phase_mass[k], 0.0f));
    w->h_phase.push_back(ph);
  }
  w->n += n;
  recompute_uniformity3(w);
  w->dev_valid = w->aux_valid = w->plan_valid = w->keys_valid = false;
  return n;
}

// ---------------------------------------------------------------- the fluid phase with the engine's bodies
// Host restatements of the rotation arithmetic the device and the buoyancy
// samples use (f32, no contraction): q v q* as in qrot3, Mat3::from_quat,
// column-major products, RigidBody3::world_inv_inertia (body.rs:1328-1331).
void qrot_h(float qx, float qy, float qz, float qw, float vx, float vy, float vz, float& ox, float& oy, float& oz) {
  const float s = qw * qw - ((qx * qx + qy * qy) + qz * qz);
  const float d = ((vx * qx + vy * qy) + vz * qz) * 2.0f;
  const float w2 = qw * 2.0f;
  const float cx = qy * vz - qz * vy, cy = qz * vx - qx * vz, cz = qx * vy - qy * vx;
  ox = (vx * s + qx * d) + cx * w2;
  oy = (vy * s + qy * d) + cy * w2;
  oz = (vz * s + qz * d) + cz * w2;
}

void mat3_from_quat_h(float x, float y, float z, float w, float m[9]) {
  const float x2 = x + x, y2 = y + y, z2 = z + z;
  const float xx = x * x2, xy = x * y2, xz = x * z2, yy = y * y2, yz = y * z2, zz = z * z2;
  const float wx = w * x2, wy = w * y2, wz = w * z2;
  m[0] = 1.0f - (yy + zz), m[1] = xy + wz, m[2] = xz - wy;
  m[3] = xy - wz, m[4] = 1.0f - (xx + zz), m[5] = yz + wx;
  m[6] = xz + wy, m[7] = yz - wx, m[8] = 1.0f - (xx + yy);
}

void world_inv_inertia_h(const PhiengBody3& b, float out[9]) {
  float r[9], rt[9], t[9];
  mat3_from_quat_h(b.qx, b.qy, b.qz, b.qw, r);
  for (int j = 0; j < 3; j++)
    for (int i = 0; i < 3; i++) rt[3 * j + i] = r[3 * i + j];
  auto mul = [](const float* a, const float* c, float* o) {
    for (int j = 0; j < 3; j++)
      for (int i = 0; i < 3; i++) o[3 * j + i] = (a[i] * c[3 * j] + a[3 + i] * c[3 * j + 1]) + a[6 + i] * c[3 * j + 2];
  };
  mul(r, b.inv_inertia, t);
  mul(t, rt, out);
}

// Buoyancy surface samples of a dynamic body (fluid3.rs:371-467): 14 sphere
// directions, 4 per box face (each face's points at its fixed coordinate -he,
// as the reference writes them), two rings of 8 and the two poles of a
// capsule; none for hulls. Two float4 per sample: (point, area), (normal, 0).
// The ring angles' cosines and sines come from the C library, as f32::cos /
// f32::sin do.
void surface_samples3_h(const PhiengBody3& b, std::vector<float4>& out) {
  const float pi = 3.14159265358979323846f;
  auto push = [&](float lx, float ly, float lz, float nlx, float nly, float nlz, float area) {
    float x, y, z, nx, ny, nz;
    qrot_h(b.qx, b.qy, b.qz, b.qw, lx, ly, lz, x, y, z);
    qrot_h(b.qx, b.qy, b.qz, b.qw, nlx, nly, nlz, nx, ny, nz);
    out.push_back(make_float4(x + b.px, y + b.py, z + b.pz, area));
    out.push_back(make_float4(nx, ny, nz, 0.0f));
  };
  if (b.shape_tag == PHIENG_SHAPE3_SPHERE) {
    const float r = b.a;
    float dirs[14][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    const float sg[8][3] = {{1, 1, 1}, {1, 1, -1}, {1, -1, 1}, {1, -1, -1},
                            {-1, 1, 1}, {-1, 1, -1}, {-1, -1, 1}, {-1, -1, -1}};
    for (int k = 0; k < 8; k++) {  // normalize_or_zero: v * (1 / |v|)
      const float rcp = 1.0f / std::sqrt((sg[k][0] * sg[k][0] + sg[k][1] * sg[k][1]) + sg[k][2] * sg[k][2]);
      for (int a = 0; a < 3; a++) dirs[6 + k][a] = sg[k][a] * rcp;
    }
    const float area = 4.0f * pi * r * r / 14.0f;
    for (auto& d : dirs) push(d[0] * r, d[1] * r, d[2] * r, d[0], d[1], d[2], area);
  } else if (b.shape_tag == PHIENG_SHAPE3_BOX) {
    const float hx = b.a, hy = b.b, hz = b.c;
    const float area = 8.0f * (hx * hy + hy * hz + hz * hx) / 24.0f;
    struct Face {
      float n[3];
      float fixed;
      int axis;
    };
    const Face faces[6] = {{{0, 1, 0}, -hy, 0},  {{0, -1, 0}, -hy, 0}, {{1, 0, 0}, -hx, 1},
                           {{-1, 0, 0}, -hx, 1}, {{0, 0, 1}, -hz, 2},  {{0, 0, -1}, -hz, 2}};
    const float ts[4][2] = {{-0.75f, -0.75f}, {0.75f, -0.75f}, {-0.75f, 0.75f}, {0.75f, 0.75f}};
    for (const Face& f : faces)
      for (const auto& t : ts) {
        if (f.axis == 0) push(hx * t[0], f.fixed, hz * t[1], f.n[0], f.n[1], f.n[2], area);
        else if (f.axis == 1) push(f.fixed, hy * t[0], hz * t[1], f.n[0], f.n[1], f.n[2], area);
        else push(hx * t[0], hy * t[1], f.fixed, f.n[0], f.n[1], f.n[2], area);
      }
  } else if (b.shape_tag == PHIENG_SHAPE3_CAPSULE) {
    const float r = b.a, hl = b.b;
    const float side = 4.0f * pi * r * hl / 16.0f, cap = 2.0f * pi * r * r;
    for (float sy : {-hl * 0.5f, hl * 0.5f})
      for (int k = 0; k < 8; k++) {
        const float a = 2.0f * pi * (float)k / 8.0f;
        const float c = std::cos(a), sn = std::sin(a);
        push(c * r + 0.0f * sy, 0.0f * r + 1.0f * sy, sn * r + 0.0f * sy, c, 0.0f, sn, side);  // dir * r + Y * sy
      }
    for (float sg : {-1.0f, 1.0f}) {
      const float len = hl + r;
      push((0.0f * sg) * len, (1.0f * sg) * len, (0.0f * sg) * len, 0.0f * sg, 1.0f * sg, 0.0f * sg, cap);
    }
  }
}

struct HullIn {
  const float* xyz = nullptr;
  const uint32_t* first = nullptr;
  const uint32_t* count = nullptr;
};

bool identity_rotation(const PhiengBody3& b) { return b.qx == 0.0f && b.qy == 0.0f && b.qz == 0.0f && b.qw == 1.0f; }

bool ensure_body_buffers3(World3* w, uint32_t nb, uint32_t nsamples, uint32_t nhull) {
  auto grow = [&](auto*& p, uint32_t& cap, uint32_t need, uint32_t floor_) {
    if (need <= cap && p) return true;
    cudaStreamSynchronize(w->stream);
    dfree3(p);
    const uint32_t c = std::max(need, floor_);
    if (!dalloc3(w, p, c)) return false;
    cap = c;
    return true;
  };
  if (nb > w->qbody_cap || !w->d_qbodies) {
    cudaStreamSynchronize(w->stream);
    dfree3(w->d_qbodies), dfree3(w->d_dyn), dfree3(w->d_buoy);
    const uint32_t c = std::max<uint32_t>(16, nb);
    if (!dalloc3(w, w->d_qbodies, c) || !dalloc3(w, w->d_dyn, c) || !dalloc3(w, w->d_buoy, c)) return false;
    w->qbody_cap = c;
  }
  if (!grow(w->d_samples, w->sample_cap, 2 * nsamples, 64) || !grow(w->d_hullv, w->hull_cap, nhull, 64)) return false;
  if (w->n > w->dyn_pcap || !w->d_defer) {
    cudaStreamSynchronize(w->stream);
    dfree3(w->d_defer), dfree3(w->d_dcount), dfree3(w->d_dstart), dfree3(w->d_dtile), dfree3(w->d_list);
    dfree3(w->d_dq_id), dfree3(w->d_p_id);
    const uint32_t c = std::max<uint32_t>(1024, w->n);
    const uint32_t tiles = (c + 1 + kBucketScanTile - 1) / kBucketScanTile;
    const size_t len = (size_t)tiles * kBucketScanTile;
    if (!dalloc3(w, w->d_defer, c) || !dalloc3(w, w->d_dcount, len) || !dalloc3(w, w->d_dstart, len + 1) ||
        !dalloc3(w, w->d_dtile, tiles) || !dalloc3(w, w->d_list, c) || !dalloc3(w, w->d_dq_id, c) ||
        !dalloc3(w, w->d_p_id, c))
      return false;
    w->dyn_pcap = c;
  }
  return grow(w->d_count2, w->count2_cap, w->count_len, 1);
}

// The grid on the post-boundary positions for the buoyancy pass, from a copy
// of the bucket counts (the next substep's sort needs the originals), with
// the density pass's values carried into the new order.
void enqueue_resort3(World3* w, const StepParams3& P, cudaStream_t st) {
  const uint32_t g = cdiv(w->n, 256);
  k_dp_to_id3<<<g, 256, 0, st>>>(w->sdq, w->spres, w->sid, w->n, w->d_dq_id, w->d_p_id);
  cudaMemcpyAsync(w->d_count2, w->count, sizeof(uint32_t) * w->count_len, cudaMemcpyDeviceToDevice, st);
  BucketSort bs;
  bs.count = w->d_count2;
  bs.tilesum = w->tilesum;
  bs.done = w->scalar + 8;
  bs.tstate = w->tstate;
  bs.err = w->scalar + 12;
  bs.start = w->start;
  bs.key = w->key;
  bs.sid_prev = w->sid;
  bs.tkey = w->tkey;
  bs.tid = w->tid;
  enqueue_bucket_place(bs, w->n, P.grid.sentinel + 1, true, st);
  const bool m = (P.flags & F_MASS) != 0, ph = (P.flags & F_PHASE) != 0;
  k_fixup3<<<g, 256, 0, st>>>(w->tkey, w->tid, w->start, w->n, w->skey, w->sid, w->pos, w->vel, w->mass, w->phase,
                              w->spos, w->svel, m ? w->smass : nullptr, ph ? w->sphase : nullptr);
  k_dp_from_id3<<<g, 256, 0, st>>>(w->d_dq_id, w->d_p_id, w->sid, w->n, w->sdq, w->spres);
}

// FluidState3::step_fluid with the caller's bodies (fluid3.rs:591-607,
// 990-1213). Bodies are validated by the caller.
bool step_fluid_bodies3(World3* w, PhiengBody3* bodies, uint32_t nb, float dt, const HullIn& hin = HullIn()) {
  if (!w->cfg.enabled || w->n == 0 || !(dt > 0.0f)) return true;  // step_fluid guards (fluid3.rs:599-601)
  if (w->error != PHIENG_SPH_OK) return false;
  if (w->cfg.adaptive_resolution) {
    w->error = PHIENG_SPH_E_UNSUPPORTED;
    return false;
  }
  std::vector<DevBodyQ3> qb(nb);
  std::vector<DynBody3> dy(nb);
  std::vector<float4> samples, hullv;
  std::vector<uint32_t> buoy;
  std::vector<DevBody3> statics;  // ghost sources
  bool any_dyn = false, ghost_ok = true;
  const float pr = rmaxf(w->cfg.particle_radius, 0.0f);
  for (uint32_t k = 0; k < nb; k++) {
    const PhiengBody3& b = bodies[k];
    DevBodyQ3& d = qb[k];
    std::memset(&d, 0, sizeof(d));
    d.shape = (int32_t)b.shape_tag;
    d.px = b.px, d.py = b.py, d.pz = b.pz;
    d.qx = b.qx, d.qy = b.qy, d.qz = b.qz, d.qw = b.qw;
    d.a = b.a, d.b = b.b, d.c = b.c;
    d.dyn = (!b.is_static || b.vx != 0.0f || b.vy != 0.0f || b.vz != 0.0f) ? 1u : 0u;
    any_dyn = any_dyn || d.dyn;
    // world bounding box half extents around the position, the particle
    // radius included, padded by 1% (the rotation is unit within 1e-3)
    float m[9];
    mat3_from_quat_h(b.qx, b.qy, b.qz, b.qw, m);
    float he[3] = {b.a + pr, b.a + pr, b.a + pr};
    if (b.shape_tag == PHIENG_SHAPE3_BOX) he[1] = b.b + pr, he[2] = b.c + pr;
    if (b.shape_tag == PHIENG_SHAPE3_CAPSULE) he[1] = b.b + b.a + pr;
    float ext[3] = {0.0f, 0.0f, 0.0f};
    if (b.shape_tag == PHIENG_SHAPE3_SPHERE) {
      ext[0] = ext[1] = ext[2] = he[0];
    } else if (b.shape_tag == PHIENG_SHAPE3_HULL) {
      d.vfirst = (uint32_t)hullv.size();
      d.vcount = hin.count[k];
      for (uint32_t i = hin.first[k]; i < hin.first[k] + hin.count[k]; i++) {
        float x, y, z;
        qrot_h(b.qx, b.qy, b.qz, b.qw, hin.xyz[3 * (size_t)i], hin.xyz[3 * (size_t)i + 1], hin.xyz[3 * (size_t)i + 2],
               x, y, z);
        const float4 v = make_float4(x + b.px, y + b.py, z + b.pz, 0.0f);
        hullv.push_back(v);
        ext[0] = std::max(ext[0], std::fabs(v.x - b.px) + pr);
        ext[1] = std::max(ext[1], std::fabs(v.y - b.py) + pr);
        ext[2] = std::max(ext[2], std::fabs(v.z - b.pz) + pr);
      }
    } else {
      for (int i = 0; i < 3; i++)
        ext[i] = std::fabs(m[i]) * he[0] + std::fabs(m[3 + i]) * he[1] + std::fabs(m[6 + i]) * he[2];
    }
    d.ex = ext[0] * 1.01f + 1e-30f;
    d.ey = ext[1] * 1.01f + 1e-30f;
    d.ez = ext[2] * 1.01f + 1e-30f;
    DynBody3& y = dy[k];
    std::memset(&y, 0, sizeof(y));
    y.vx = b.vx, y.vy = b.vy, y.vz = b.vz, y.wx = b.wx, y.wy = b.wy, y.wz = b.wz;
    y.inv_mass = b.inv_mass;
    world_inv_inertia_h(b, y.iw);
    y.is_static = b.is_static ? 1u : 0u;
    y.sleeping = b.is_sleeping ? 1u : 0u;
    y.sample_first = (uint32_t)(samples.size() / 2);
    if (!b.is_static) surface_samples3_h(b, samples);
    y.sample_count = (uint32_t)(samples.size() / 2) - y.sample_first;
    if (y.sample_count) buoy.push_back(k);
    if (b.is_static && w->cfg.boundary_particles) {
      // ghosts are generated for static spheres, boxes and capsules at the
      // identity rotation (generate_ghosts3)
      if (b.shape_tag == PHIENG_SHAPE3_HULL || !identity_rotation(b)) ghost_ok = false;
      DevBody3 g;
      std::memset(&g, 0, sizeof(g));
      g.shape = (int32_t)b.shape_tag;
      g.px = b.px, g.py = b.py, g.pz = b.pz;
      g.a = b.a, g.b = b.b, g.c = b.c;
      statics.push_back(g);
    }
  }
  if (!ghost_ok) {
    w->error = PHIENG_SPH_E_UNSUPPORTED;
    return false;
  }
  if (!prepare3(w)) return false;
  if (w->cfg.boundary_particles && !refresh_ghosts3(w, statics)) return false;
  if (!ensure_body_buffers3(w, nb, (uint32_t)(samples.size() / 2), (uint32_t)hullv.size())) return false;
  cudaStream_t st = w->stream;
  if (nb && (!ok3(w, cudaMemcpyAsync(w->d_qbodies, qb.data(), sizeof(DevBodyQ3) * nb, cudaMemcpyHostToDevice, st)) ||
             !ok3(w, cudaMemcpyAsync(w->d_dyn, dy.data(), sizeof(DynBody3) * nb, cudaMemcpyHostToDevice, st))))
    return false;
  if (!buoy.empty() &&
      !ok3(w, cudaMemcpyAsync(w->d_buoy, buoy.data(), 4 * buoy.size(), cudaMemcpyHostToDevice, st)))
    return false;
  if (!samples.empty() && !ok3(w, cudaMemcpyAsync(w->d_samples, samples.data(), sizeof(float4) * samples.size(),
                                                  cudaMemcpyHostToDevice, st)))
    return false;
  if (!hullv.empty() &&
      !ok3(w, cudaMemcpyAsync(w->d_hullv, hullv.data(), sizeof(float4) * hullv.size(), cudaMemcpyHostToDevice, st)))
    return false;
  uint32_t ns = 1;
  if (!cfl_substeps3(w, dt, &ns)) return false;
  const float sub = dt / (float)ns;
  StepParams3 P = make_params3(w, sub);
  P.flags |= F_QBODIES;
  if (any_dyn) P.flags |= F_DYNAMIC;
  P.nbodies = nb;
  P.qbodies = w->d_qbodies;
  P.hullv = w->d_hullv;
  P.defer = w->d_defer;
  P.dcount = w->d_dcount;
  if (P.flags & F_TURB) {  // the world clock (world.rs:2811)
    uint32_t bits;
    std::memcpy(&bits, &w->time, 4);
    enqueue_set_word(w->scalar + kClockWord3, bits, st);
  }
  const float drag = rmaxf(w->cfg.drag, 0.0f);
  const size_t dlen = (size_t)((w->n + 1 + kBucketScanTile - 1) / kBucketScanTile) * kBucketScanTile;
  for (uint32_t k = 0; k < ns; k++) {
    enqueue_sort3(w, P, st);
    w->sid_perm_n = w->n;
    enqueue_density3(w, P, st);
    if ((P.flags & F_GHOST) && P.nghost) {
      if (P.flags & F_MASS)
        k_ghost_density3<true><<<cdiv(P.nghost, 256), 256, 0, st>>>(w->spos, w->smass, w->start, P);
      else
        k_ghost_density3<false><<<cdiv(P.nghost, 256), 256, 0, st>>>(w->spos, w->smass, w->start, P);
    }
    if (any_dyn) cudaMemsetAsync(w->d_dcount, 0, sizeof(uint32_t) * dlen, st);
    enqueue_force3(w, P, nullptr, st);
    if (any_dyn) {
      enqueue_flag_compact(w->d_dcount, w->n, w->d_dtile, w->scalar + 20, w->d_dstart, w->d_list, st);
      k_dynamic_walls3<<<1, 32, 0, st>>>(w->d_list, w->d_dstart + w->n, w->pos, w->vel, w->mass, w->key, w->count,
                                         w->d_dyn, P);
    }
    if (!buoy.empty()) {
      enqueue_resort3(w, P, st);
      k_buoyancy3<<<cdiv((uint32_t)buoy.size(), 32), 32, 0, st>>>(
          w->d_buoy, (uint32_t)buoy.size(), w->d_dyn, w->d_samples, w->spos, w->sdq, w->spres, w->smass, w->start, P,
          drag, sub, w->ambient.wind_x, w->ambient.wind_y, w->ambient.wind_z);
    }
    w->substeps++;
  }
  if (!ok3(w, cudaGetLastError())) return false;
  w->host_valid = false;
  w->dp_dev = true;
  w->keys_valid = true;
  if (nb) {
    if (!ok3(w, cudaMemcpyAsync(dy.data(), w->d_dyn, sizeof(DynBody3) * nb, cudaMemcpyDeviceToHost, st)) ||
        !ok3(w, cudaStreamSynchronize(st)))
      return false;
    for (uint32_t k = 0; k < nb; k++) {
      bodies[k].vx = dy[k].vx, bodies[k].vy = dy[k].vy, bodies[k].vz = dy[k].vz;
      bodies[k].wx = dy[k].wx, bodies[k].wy = dy[k].wy, bodies[k].wz = dy[k].wz;
      bodies[k].is_sleeping = dy[k].sleeping ? 1 : 0;
    }
  }
  return true;
}

// Fields a body of the fluid phase must have: a known shape with positive
// finite sizes (hulls: phieng_sph3_step_fluid_hull), finite transform and
// motion state, a rotation of norm 1 within 1e-3.
bool body3_valid(const PhiengBody3& b, bool hull_ok) {
  const float f[] = {b.px, b.py, b.pz, b.qx, b.qy, b.qz, b.qw, b.vx, b.vy, b.vz, b.wx, b.wy, b.wz, b.inv_mass};
  for (float x : f)
    if (!std::isfinite(x)) return false;
  for (float x : b.inv_inertia)
    if (!std::isfinite(x)) return false;
  const float n2 = ((b.qx * b.qx + b.qy * b.qy) + b.qz * b.qz) + b.qw * b.qw;
  if (!(std::fabs(n2 - 1.0f) <= 1e-3f)) return false;
  auto pos = [](float v) { return std::isfinite(v) && v > 0.0f; };
  switch (b.shape_tag) {
    case PHIENG_SHAPE3_SPHERE: return pos(b.a);
    case PHIENG_SHAPE3_BOX: return pos(b.a) && pos(b.b) && pos(b.c);
    case PHIENG_SHAPE3_CAPSULE: return pos(b.a) && pos(b.b);
    case PHIENG_SHAPE3_HULL: return hull_ok;
    default: return false;
  }
}

constexpr uint32_t kMaxCallBodies3 = 65536;
constexpr uint32_t kMaxHullVerts3 = 1u << 20;

}  // namespace

extern "C" {

World3* phieng_world3_new(void) { return new (std::nothrow) World3(); }

void phieng_world3_free(World3* w) {
  if (!w) return;
  if (w->device >= 0) {
    cudaStreamSynchronize(w->stream);
    release_graph3(w);
    free_particles3(w);
    dfree3(w->count), dfree3(w->start), dfree3(w->tilesum), dfree3(w->tstate), dfree3(w->scalar), dfree3(w->dbodies);
    dfree3(w->d_gpos), dfree3(w->d_gq), dfree3(w->d_gtab);
    dfree3(w->rs_slot), dfree3(w->rs_absorbed), dfree3(w->rs_pos), dfree3(w->rs_vel), dfree3(w->rs_mass),
        dfree3(w->rs_phase);
    dfree3(w->d_qbodies), dfree3(w->d_dyn), dfree3(w->d_buoy), dfree3(w->d_samples), dfree3(w->d_hullv);
    dfree3(w->d_defer), dfree3(w->d_dcount), dfree3(w->d_dstart), dfree3(w->d_dtile), dfree3(w->d_list);
    dfree3(w->d_dq_id), dfree3(w->d_p_id), dfree3(w->d_count2);
    for (auto& e : w->ev)
      if (e) cudaEventDestroy(e);
    if (w->h_pinned) cudaFreeHost(w->h_pinned);
    if (w->own_stream) cudaStreamDestroy(w->own_stream);
  }
  delete w;
}

void phieng_world3_step(World3* w, float dt) {
  if (!w || !std::isfinite(dt) || dt <= 0.0f) return;
  world_step3(w, std::min(dt, kMaxDt));
}

void phieng_world3_set_gravity(World3* w, float gx, float gy, float gz) {
  if (!w || !std::isfinite(gx) || !std::isfinite(gy) || !std::isfinite(gz)) return;
  w->gx = gx;
  w->gy = gy;
  w->gz = gz;
}

int32_t phieng_world3_set_time(World3* w, float t) {
  if (!w || !std::isfinite(t)) return 0;
  w->time = t;
  return 1;
}

int32_t phieng_world3_get_time(World3* w, float* out) {
  if (!w || !out) return 0;
  *out = w->time;
  return 1;
}

int32_t phieng_world3_body_count(World3* w) { return w ? (int32_t)w->bodies.size() : -1; }

uint32_t phieng_sph3_fluid_masses(World3* w, float* out, uint32_t max) {
  if (!w) return 0;
  for (uint32_t i = 0; out && i < std::min(w->n, max); i++) out[i] = w->h_mass[i];
  return w->n;
}

uint32_t phieng_sph3_ghosts(World3* w, float* xyz, uint32_t max, uint64_t* regens) {
  if (!w) return 0;
  if (regens) *regens = w->ghost_regens;
  const uint32_t n = (uint32_t)w->h_gpos.size();
  for (uint32_t i = 0; xyz && i < std::min(n, max); i++) {
    xyz[3 * i] = w->h_gpos[i].x;
    xyz[3 * i + 1] = w->h_gpos[i].y;
    xyz[3 * i + 2] = w->h_gpos[i].z;
  }
  return n;
}

int32_t phieng_world3_set_ambient_config(World3* w, const AmbientConfig3Ffi* cfg) {
  if (!w || !cfg) return 0;
  const AmbientConfig3Ffi& c = *cfg;
  // ambient3_from_ffi (ffi.rs:414-475): finite floats, non-negative
  // coefficients, octaves stored as min(v, 255)
  for (float v : {c.spring_ax, c.spring_ay, c.spring_az, c.spring_stiffness, c.spring_damping,
                  c.spring_max_displacement, c.drag_linear, c.drag_quadratic, c.air_density, c.drag_angular,
                  c.wind_x, c.wind_y, c.wind_z, c.turbulence_amplitude, c.turbulence_frequency,
                  c.turbulence_time_scale})
    if (!std::isfinite(v)) return 0;
  if (c.spring_stiffness < 0.0f || c.spring_damping < 0.0f || c.spring_max_displacement < 0.0f ||
      c.drag_linear < 0.0f || c.drag_quadratic < 0.0f || c.air_density < 0.0f || c.drag_angular < 0.0f ||
      c.turbulence_amplitude < 0.0f)
    return 0;
  AmbientConfig3Ffi a = c;
  a.spring_enabled = c.spring_enabled != 0;
  a.drag_enabled = c.drag_enabled != 0;
  a.turbulence_enabled = c.turbulence_enabled != 0;
  a.turbulence_divergence_free = c.turbulence_divergence_free != 0;
  a.turbulence_octaves = std::min<uint32_t>(c.turbulence_octaves, 255u);
  w->ambient = a;
  return 1;
}

int32_t phieng_world3_get_ambient_config(World3* w, AmbientConfig3Ffi* out) {
  if (!w || !out) return 0;
  *out = w->ambient;
  return 1;
}

int32_t phieng_world3_add_body(World3* w, float px, float py, float pz, uint32_t shape_tag, float a, float b, float c,
                               float density, uint8_t is_static, float friction, float restitution) {
  (void)friction;
  (void)restitution;
  if (!w || !std::isfinite(px) || !std::isfinite(py) || !std::isfinite(pz)) return -1;
  auto pos = [](float v) { return std::isfinite(v) && v > 0.0f; };
  DevBody3 bd;
  std::memset(&bd, 0, sizeof(bd));
  if (shape_tag == PHIENG_SHAPE3_SPHERE && pos(a)) {
    bd.shape = 0;
    bd.a = a;
  } else if (shape_tag == PHIENG_SHAPE3_BOX && pos(a) && pos(b) && pos(c)) {
    bd.shape = 1;
    bd.a = a;
    bd.b = b;
    bd.c = c;
  } else if (shape_tag == PHIENG_SHAPE3_CAPSULE && pos(a) && pos(b)) {
    bd.shape = 2;
    bd.a = a;
    bd.b = b;
  } else {
    return -1;
  }
  if (!pos(density)) return -1;
  if (!is_static) return -1;  // dynamic bodies are not part of this library
  bd.px = px;
  bd.py = py;
  bd.pz = pz;
  // world bounding box half extents of the (unrotated) body, padded by 0.1%
  const float ex = bd.a;
  const float ey = bd.shape == 0 ? bd.a : bd.shape == 1 ? bd.b : bd.b + bd.a;
  const float ez = bd.shape == 1 ? bd.c : bd.a;
  bd.ex = ex * 1.001f + 1e-30f;
  bd.ey = ey * 1.001f + 1e-30f;
  bd.ez = ez * 1.001f + 1e-30f;
  if (w->bodies.size() >= 0x7FFFFFFF) return -1;
  w->bodies.push_back(bd);
  w->bodies_dirty = true;
  return (int32_t)(w->bodies.size() - 1);
}

uint32_t phieng_world3_add_bodies(World3* w, const BodyDesc3D* descs, uint32_t n, int32_t* out_ids) {
  if (!w || !descs || !out_ids) return 0;
  n = std::min<uint32_t>(n, kMaxAddPerCall);
  uint32_t added = 0;
  for (uint32_t i = 0; i < n; i++) {
    const BodyDesc3D& d = descs[i];
    out_ids[i] = phieng_world3_add_body(w, d.pos_x, d.pos_y, d.pos_z, d.shape_tag, d.a, d.b, d.c, d.density,
                                        d.is_static, d.friction, d.restitution);
    if (out_ids[i] >= 0) added++;
  }
  return added;
}

int32_t phieng_world3_set_fluid_config(World3* w, const FluidConfig3Ffi* cfg) {
  if (!w || !cfg || !valid_config(*cfg)) return 0;
  if (w->device >= 0) cudaStreamSynchronize(w->stream);
  if (!ensure_host3(w)) return 0;
  w->cfg = *cfg;
  w->plan_valid = false;
  release_graph3(w);
  return 1;
}

int32_t phieng_world3_get_fluid_config(World3* w, FluidConfig3Ffi* out) {
  if (!w || !out) return 0;
  *out = w->cfg;
  return 1;
}

uint32_t phieng_world3_fluid_add(World3* w, const float* xyz, uint32_t count) {
  if (!w || !xyz) return 0;
  return add_particles3(w, xyz, nullptr, count);
}

uint32_t phieng_world3_fluid_add_phase(World3* w, const float* xyz, const uint8_t* phases, uint32_t count) {
  if (!w || !xyz || !phases) return 0;
  return add_particles3(w, xyz, phases, count);
}

uint32_t phieng_world3_fluid_count(const World3* w) { return w ? w->n : 0; }

int32_t phieng_world3_fluid_clear(World3* w) {
  if (!w) return 0;
  if (w->device >= 0) cudaStreamSynchronize(w->stream);
  w->n = 0;
  w->h_pos.clear(), w->h_vel.clear(), w->h_mass.clear(), w->h_phase.clear(), w->h_dens.clear(), w->h_pres.clear();
  w->dp_dev = false;
  recompute_uniformity3(w);
  w->host_valid = true;
  w->dev_valid = w->aux_valid = w->plan_valid = w->keys_valid = false;
  return 1;
}

uint32_t phieng_world3_fluid_get(const World3* cw, float* out, uint32_t max) {
  if (!cw || !out) return 0;
  World3* w = const_cast<World3*>(cw);
  const uint32_t n = std::min(max, w->n);
  if (n && !ensure_host3(w)) return 0;
  for (uint32_t i = 0; i < n; i++) {
    const float4 p = w->h_pos[i], v = w->h_vel[i];
    float* o = out + 6 * (size_t)i;
    o[0] = p.x, o[1] = p.y, o[2] = p.z, o[3] = v.x, o[4] = v.y, o[5] = v.z;
  }
  return n;
}

int64_t phieng_sph3_fluid_block_save(World3* w, uint32_t version, uint8_t* out, uint64_t cap) {
  if (!w || version == 0 || version > snap::kSchemaLatest) return -1;
  if (w->n && !ensure_host3(w)) return -1;
  std::vector<snap::Particle> ps(w->n);
  for (uint32_t i = 0; i < w->n; i++) {
    const float4 p = w->h_pos[i], v = w->h_vel[i];
    ps[i] = snap::Particle{p.x, p.y, p.z, v.x, v.y, v.z, w->h_mass[i], w->h_phase[i]};
  }
  std::vector<uint8_t> o;
  snap::encode(o, w->cfg, ps, 3, version);
  if (out && cap >= o.size()) std::memcpy(out, o.data(), o.size());
  return (int64_t)o.size();
}

int64_t phieng_sph3_fluid_block_load(World3* w, uint32_t version, const uint8_t* data, uint64_t len) {
  if (!w || !data || version == 0 || version > snap::kSchemaLatest) return -1;
  snap::Reader r(data, len);
  snap::Block b;
  if (!snap::decode(r, version, 3, w->cap, b)) return -2;
  if (w->device >= 0) cudaStreamSynchronize(w->stream);
  w->cfg = b.cfg;
  const uint32_t n = (uint32_t)b.particles.size();
  w->h_pos.resize(n);
  w->h_vel.resize(n);
  w->h_mass.resize(n);
  w->h_phase.resize(n);
  w->h_dens.assign(n, b.cfg.rest_density);  // density / pressure are recomputed by the next step
  w->h_pres.assign(n, 0.0f);
  for (uint32_t i = 0; i < n; i++) {
    const snap::Particle& q = b.particles[i];
    w->h_pos[i] = make_float4(q.x, q.y, q.z, 0.0f);
    w->h_vel[i] = make_float4(q.vx, q.vy, q.vz, 0.0f);
    w->h_mass[i] = q.mass;
    w->h_phase[i] = q.phase;
  }
  w->n = n;
  recompute_uniformity3(w);
  w->host_valid = true;
  w->dp_dev = false;
  w->dev_valid = w->aux_valid = w->plan_valid = w->keys_valid = false;
  release_graph3(w);
  return (int64_t)r.off;
}

// ---- extension ----
int32_t phieng_sph3_status(const World3* w, PhiengSphStatus* out) {
  if (!w || !out) return 0;
  std::memset(out, 0, sizeof(*out));
  out->error = w->error;
  out->particles = w->n;
  out->substeps = w->substeps;
  out->grid_log2_w = w->plan.log2w;
  out->grid_log2_h = w->plan.log2h;
  out->sort_passes = 1;
  out->grid_cx0 = w->plan.cx0;
  out->grid_cy0 = w->plan.cy0;
  out->grid_buckets = w->plan.nbuckets;
  return 1;
}

int32_t phieng_sph3_clear_error(World3* w) {
  if (!w) return 0;
  w->error = PHIENG_SPH_OK;
  return 1;
}

const char* phieng_sph3_error_string(const World3* w) { return error_text(w ? w->error : PHIENG_SPH_E_ARG); }

int32_t phieng_sph3_set_particle_cap(World3* w, uint32_t cap) {
  if (!w || cap == 0) return 0;
  w->cap = cap;
  return 1;
}

int32_t phieng_sph3_step_n(World3* w, float dt, uint32_t steps) {
  if (!w) return 0;
  if (!std::isfinite(dt) || dt <= 0.0f) return 1;
  const float d = std::min(dt, kMaxDt);
  for (uint32_t s = 0; s < steps; s++)
    if (!world_step3(w, d)) return 0;
  return 1;
}

int32_t phieng_sph3_set_stream(World3* w, void* stream) {
  if (!w) return 0;
  if (w->device >= 0) cudaStreamSynchronize(w->stream);
  w->stream = stream ? (cudaStream_t)stream : w->own_stream;
  w->user_stream = stream != nullptr;
  return 1;
}

int32_t phieng_sph3_sync(World3* w) {
  if (!w) return 0;
  if (w->device >= 0) {
    if (!ok3(w, cudaStreamSynchronize(w->stream)) ||
        !ok3(w, cudaMemcpy(w->h_pinned + 8, w->scalar + 12, 4, cudaMemcpyDeviceToHost)))
      return 0;
    if (w->h_pinned[8] != 0u && w->error == PHIENG_SPH_OK) w->error = PHIENG_SPH_E_CUDA;  // a scan wait gave up
  }
  return w->error == PHIENG_SPH_OK ? 1 : 0;
}

int32_t phieng_sph3_step_fluid(World3* w, PhiengBody3* bodies, uint32_t nbodies, float dt) {
  if (!w || (nbodies && !bodies) || nbodies > kMaxCallBodies3) return 0;
  for (uint32_t k = 0; k < nbodies; k++)
    if (!body3_valid(bodies[k], false)) return 0;
  return step_fluid_bodies3(w, bodies, nbodies, dt) ? 1 : 0;
}

int32_t phieng_sph3_step_fluid_hull(World3* w, PhiengBody3* bodies, uint32_t nbodies, const float* hull_xyz,
                                    const uint32_t* hull_first, const uint32_t* hull_count, uint32_t hull_nverts,
                                    float dt) {
  if (!w || (nbodies && !bodies) || nbodies > kMaxCallBodies3 || hull_nverts > kMaxHullVerts3) return 0;
  uint64_t total = 0;
  for (uint32_t k = 0; k < nbodies; k++) {
    const PhiengBody3& b = bodies[k];
    if (!body3_valid(b, true)) return 0;
    if (b.shape_tag != PHIENG_SHAPE3_HULL) continue;
    if (!hull_xyz || !hull_first || !hull_count) return 0;
    const uint64_t f = hull_first[k], c = hull_count[k];
    if (c < 1 || f + c > hull_nverts) return 0;
    for (uint64_t i = 3 * f; i < 3 * (f + c); i++)
      if (!std::isfinite(hull_xyz[i])) return 0;
    total += c;
  }
  if (total > kMaxHullVerts3) return 0;
  HullIn hin;
  hin.xyz = hull_xyz;
  hin.first = hull_first;
  hin.count = hull_count;
  return step_fluid_bodies3(w, bodies, nbodies, dt, hin) ? 1 : 0;
}

int32_t phieng_sph3_set_state(World3* w, const float* xyzv, uint32_t n) {
  if (!w || !xyzv || n > w->n) return 0;
  for (uint64_t i = 0; i < 6ull * n; i++)
    if (!std::isfinite(xyzv[i])) return 0;
  if (!ensure_host3(w) || !ensure_host_dp3(w)) return 0;
  for (uint32_t i = 0; i < n; i++) {
    const float* q = xyzv + 6 * (size_t)i;
    w->h_pos[i] = make_float4(q[0], q[1], q[2], 0.0f);
    w->h_vel[i] = make_float4(q[3], q[4], q[5], 0.0f);
  }
  w->dev_valid = false;
  w->keys_valid = false;
  w->plan_valid = false;
  return 1;
}

// Run the density pass (and, with fxyz, the force pass without integrating)
// on the current state; write density, pressure and force [fx, fy, fz] in
// insertion order (each output may be null). Returns the number written.
int32_t phieng_sph3_set_precision(World3* w, uint32_t mode) {
  if (!w || (mode != PHIENG_SPH_EXACT && mode != PHIENG_SPH_TOLERANCE)) return 0;
  if (mode == w->precision) return 1;
  if (w->device >= 0) cudaStreamSynchronize(w->stream);
  release_graph3(w);
  w->precision = mode;
  return 1;
}

uint32_t phieng_sph3_get_precision(const World3* w) { return w ? w->precision : PHIENG_SPH_EXACT; }

uint32_t phieng_sph3_debug_forces(World3* w, float* dens, float* pres, float* fxyz, uint32_t max) {
  if (!w) return 0;
  const uint32_t n = std::min(max, w->n);
  if (n == 0) return 0;
  if (!prepare3(w)) return 0;
  const StepParams3 P = make_params3(w, 0.0f);
  float4* dbg = nullptr;
  if (fxyz && !dalloc3(w, dbg, w->n)) return 0;
  enqueue_sort3(w, P, w->stream);
  enqueue_density3(w, P, w->stream);
  if (fxyz) enqueue_force3(w, P, dbg, w->stream);
  w->sid_perm_n = w->n;
  w->keys_valid = false;  // the sort consumed the bucket counts
  w->dp_dev = true;
  std::vector<float> f(fxyz ? 4 * (size_t)w->n : 0);
  bool ok = ok3(w, cudaGetLastError());
  if (ok && fxyz)
    ok = ok3(w, cudaMemcpyAsync(f.data(), dbg, sizeof(float4) * w->n, cudaMemcpyDeviceToHost, w->stream));
  ok = ok && ensure_host_dp3(w);
  cudaFree(dbg);
  if (!ok) return 0;
  if (dens) std::memcpy(dens, w->h_dens.data(), sizeof(float) * n);
  if (pres) std::memcpy(pres, w->h_pres.data(), sizeof(float) * n);
  if (fxyz)
    for (uint32_t i = 0; i < n; i++) {
      fxyz[3 * i] = f[4 * i];
      fxyz[3 * i + 1] = f[4 * i + 1];
      fxyz[3 * i + 2] = f[4 * i + 2];
    }
  return n;
}

// Density and pressure of every particle as the last substep's density pass
// left them (insertion order; rest density and 0 before the first step).
uint32_t phieng_sph3_get_density_pressure(World3* w, float* dens, float* pres, uint32_t max) {
  if (!w) return 0;
  const uint32_t n = std::min(max, w->n);
  if (n == 0) return 0;
  if (!ensure_host_dp3(w)) return 0;
  if (dens) std::memcpy(dens, w->h_dens.data(), sizeof(float) * n);
  if (pres) std::memcpy(pres, w->h_pres.data(), sizeof(float) * n);
  return n;
}

int32_t phieng_sph3_set_profiling(World3* w, int32_t on) {
  if (!w) return 0;
  if (on && !w->ev[0]) {
    if (!ensure_device3(w)) return 0;
    for (auto& e : w->ev)
      if (!ok3(w, cudaEventCreate(&e))) return 0;
  }
  w->profiling = on != 0;
  release_graph3(w);
  return 1;
}

uint32_t phieng_sph3_phase_times(World3* w, float* ms, uint32_t max) {
  if (!w || !ms || !w->profiling || !w->ev[0] || max == 0) return 0;
  if (!ok3(w, cudaEventSynchronize(w->ev[3]))) return 0;
  const uint32_t k = std::min<uint32_t>(max, 3);
  for (uint32_t i = 0; i < k; i++)
    if (cudaEventElapsedTime(&ms[i], w->ev[i], w->ev[i + 1]) != cudaSuccess) return 0;
  return k;
}

}  // extern "C"
