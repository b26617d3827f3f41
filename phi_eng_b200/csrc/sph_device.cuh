// Device-side definitions shared by the SPH kernels.
//
// Arithmetic contract: this translation unit is compiled with --fmad=false
// and IEEE division / square root (no fast-math), and every expression keeps
// the evaluation order of the reference (crates/dynamics/src/fluid.rs), so
// per-pair arithmetic is bit-identical to the reference's f32 arithmetic.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace phieng {

// crates/math/src/math.rs:3-4
constexpr float kEps = 1e-6f;
constexpr float kEpsSq = 1e-12f;

// Bucket grid. A particle's cell (cx, cy) = (floor(x/h), floor(y/h)) as
// saturating i32 (fluid.rs:350-356) maps to bucket
//   bx = (cx - cx0) mod W, by = (cy - cy0) mod H, key = base + by * W + bx,
// W = 2^log2w, H = 2^log2h, both >= 4. Particles with a non-finite position
// get key = sentinel (sorted last, never visited), as rebuild_grid skips
// them (fluid.rs:347-349). Cells that alias into one bucket are at least
// (W - 2) cells apart, so the distance test (d2 < h*h) rejects every aliased
// candidate and the per-particle visit order stays the reference's.
// A batch of independent scenes gives each scene its own bucket range
// [base, base + nbuckets) of one shared key space, so no scene ever sees
// another's particles; a single world has base 0 and sentinel = nbuckets.
struct GridPlan {
  int32_t cx0, cy0;
  uint32_t log2w, log2h;
  uint32_t maskw, maskh;
  uint32_t nbuckets;  // buckets of this scene (W * H)
  float hg;           // config.smoothing_length (the raw value rebuild_grid uses)
  uint32_t base;      // first key of this scene's buckets
  uint32_t sentinel;  // key of non-finite particles (= total buckets)
};

enum StepFlags : uint32_t {
  F_VISC = 1u << 0,      // XSPH (viscosity > 0)
  F_AV = 1u << 1,        // Monaghan artificial viscosity (alpha > 0)
  F_COHESION = 1u << 2,  // surface tension > 0
  F_FRICTION = 1u << 3,  // wall friction > 0
  F_TAIT = 1u << 4,      // gamma != 1
  F_MASS = 1u << 5,      // per-particle mass array (non-uniform)
  F_PHASE = 1u << 6,     // per-particle phase array (non-uniform rest density)
  F_DYNAMIC = 1u << 7,   // bodies with impulses or velocity: their contacts run in the ordered pass
  F_WIDE_NB = 1u << 8,   // h*h > max(h, EPS)^2 (h <= 0 from a snapshot): poly6 keeps its range test for neighbours
  F_TURB = 1u << 9,      // ambient turbulence on (enabled and amplitude > 0)
  F_TURB_CURL = 1u << 10,  // turbulence as divergence-free curl noise
  F_GHOST = 1u << 11,      // boundary ghost particles (boundary_particles)
  F_POLY = 1u << 12,       // polygon bodies among the launch's bodies
  F_FAST = 1u << 13,       // tolerance mode: the plain passes may run the reassociated kernels (sph_fast.cuh)
  F_QBODIES = 1u << 14,    // 3D: the boundary pass runs over the engine's bodies (rotations, reactions)
  F_WBOX = 1u << 15,       // StepParams::wbox holds every body's padded bounding box (at most kWallBoxes bodies)
};

// One cell of the boundary ghosts' hash grid: ghosts [start, start + count)
// of the cell-sorted ghost array lie in cell (cx, cy); count 0 = empty slot.
struct GhostCell {
  int32_t cx, cy;
  uint32_t start, count;
};

// Open-addressing slot of a ghost cell (linear probing from here).
__host__ __device__ inline uint32_t ghost_cell_hash(int32_t cx, int32_t cy, uint32_t mask) {
  uint32_t h = (uint32_t)cx * 0x9E3779B1u ^ ((uint32_t)cy * 0x85EBCA77u + 0x165667B1u);
  h ^= h >> 15;
  return h & mask;
}

// Bodies whose bounding boxes a launch can carry in its parameters.
constexpr uint32_t kWallBoxes = 4;

struct StepParams {
  GridPlan grid;
  float hg2;       // hg*hg: neighbour filter (fluid.rs:383)
  float hk;        // max(h, EPS): kernel support (fluid.rs:908)
  float hk2;       // hk*hk
  float c_poly6;   // 4/(PI*h2*h2*h2*h2), f32, as fluid.rs:272 evaluates it
  float c_spiky;   // -30/(PI*h*h*h*h*h), as fluid.rs:283
  float rho_cap;   // 3*max(rest_density, EPS) (fluid.rs:605)
  float stiffness;
  float gamma;
  float rest[4];   // phase_rest_density
  float mass;      // uniform particle mass when !F_MASS
  float visc;      // XSPH factor
  float vmax;      // max_velocity
  float dt;
  float gx, gy;
  float pr;        // max(particle_radius, 0)
  float pr_pad;    // pr padded by 0.1% (+1e-30) for the bounding-box reject
  float mu;        // clamp(wall_friction, 0, 1)
  float av_alpha;
  float c_s;       // sqrt(max(stiffness, 0))
  float surface_tension;
  uint32_t flags;
  uint32_t nbodies;
  uint32_t body_first;     // first of this scene's bodies in the body array
  uint32_t uniform_phase;  // phase used for every particle when !F_PHASE
  float wind_x, wind_y;  // ambient.drag.wind, against which the buoyancy drag acts (fluid.rs:1121-1124)
  const float2* poly;    // world-space vertices of the polygon bodies
  // boundary ghosts (F_GHOST, fluid.rs:617-818): cell-sorted positions, their
  // q = p / max(rho, EPS)^2 of the current substep, the cell table
  const float2* gpos;
  float* gq;
  const GhostCell* gtab;
  uint32_t gtab_mask, nghost;
  float gmass;  // particle_mass.max(EPS)
  float rest0;  // config rest_density (the ghosts' EOS reference)
  // ambient turbulence (F_TURB; TurbulenceConfig2, ambient.rs:108-126)
  float turb_amp, turb_freq, turb_tscale;
  uint32_t turb_seed, turb_oct;  // octaves already clamped to 1..8
  const float* clock;            // device word holding the world clock of the current step
  // F_WBOX: body k's bounding box as (px, py, ex + pr_pad, ey + pr_pad), the
  // values of the wall pass's reject test; unused slots never pass it
  float4 wbox[kWallBoxes];
};

// Per-launch scene access: a single world passes its parameters by value
// (constant bank); a batch reads each particle's scene row from a device
// table.
template <bool BATCH>
__device__ __forceinline__ const StepParams& scene_params(const StepParams& P0, const StepParams* __restrict__ ptab,
                                                          uint32_t scene) {
  if constexpr (BATCH)
    return ptab[scene];
  else
    return P0;
}

// Static body as the fluid sees it: shape 0 = circle (a = radius), 1 = box
// (a, b = half extents), 2 = polygon (vertices [vfirst, vfirst + vcount) of
// StepParams::poly, already in world space; a, b = their centroid); rotation
// columns x_axis = (xax, xay), y_axis = (yax, yay) (crates/math/src/math.rs:34-60).
struct DevBody {
  int32_t shape;
  float px, py;
  float xax, xay, yax, yay;
  float a, b;
  uint32_t vfirst, vcount;
  // half extents of the body's world-space bounding box, padded by 0.1%: a
  // particle farther than this plus its radius from the centre along x or
  // y cannot touch the body, so the exact test is skipped for it
  float ex, ey;
  // 1: a contact with this body reads or changes the body's velocity (a
  // dynamic body, or a static one given a velocity), so it is resolved in
  // particle order by the ordered pass instead of in parallel
  uint32_t dyn;
};

// A body's velocity state during one fluid phase (phieng_sph_step_fluid).
struct DynBody {
  float vx, vy, w;  // velocity, angular velocity
  float inv_mass, inv_inertia;
  uint32_t is_static, sleeping;
  uint32_t sample_first, sample_count;  // buoyancy surface samples (point, normal) and areas
};

constexpr uint32_t kNoDefer = 0xFFFFFFFFu;

__device__ __forceinline__ bool finitef(float v) { return isfinite(v); }

__device__ __forceinline__ uint32_t bucket_of_cell(int32_t cx, int32_t cy, const GridPlan& g) {
  uint32_t bx = ((uint32_t)cx - (uint32_t)g.cx0) & g.maskw;
  uint32_t by = ((uint32_t)cy - (uint32_t)g.cy0) & g.maskh;
  return g.base + ((by << g.log2w) | bx);
}

// cvt.rmi.s32.f32 = floor then saturating conversion with NaN -> 0, the
// semantics of `(x / h).floor() as i32` (fluid.rs:351-354).
__device__ __forceinline__ uint32_t bucket_key(float x, float y, const GridPlan& g) {
  if (!finitef(x) || !finitef(y)) return g.sentinel;
  int32_t cx = __float2int_rd(__fdiv_rn(x, g.hg));
  int32_t cy = __float2int_rd(__fdiv_rn(y, g.hg));
  return bucket_of_cell(cx, cy, g);
}

// poly6 (fluid.rs:265-273) with the constant factor precomputed in f32 by
// the same expression; (((c * t) * t) * t) keeps the reference order.
__device__ __forceinline__ float poly6(float r2, const StepParams& P) {
  if (r2 >= P.hk2 || r2 < 0.0f) return 0.0f;
  float t = __fsub_rn(P.hk2, r2);
  return __fmul_rn(__fmul_rn(__fmul_rn(P.c_poly6, t), t), t);
}

// poly6 of a neighbour (d2 < h*h, d2 >= 0 as a sum of squares): unless WIDE
// (h*h > hk*hk, F_WIDE_NB) the range test always passes and is skipped.
template <bool WIDE, class PP>
__device__ __forceinline__ float poly6_nb(float d2, const PP& P) {
  if (WIDE && (d2 >= P.hk2 || d2 < 0.0f)) return 0.0f;
  const float t = __fsub_rn(P.hk2, d2);
  return __fmul_rn(__fmul_rn(__fmul_rn(P.c_poly6, t), t), t);
}

// x^g rounded once to f32: for an integer g in [1, 64] by binary
// exponentiation in double (each product correctly rounded, so the result
// is the same on any IEEE machine), else via double pow. This is the
// correctly rounded f32 power except when x^g lies within a few double ulps
// of an f32 rounding boundary.
__device__ __forceinline__ float powf_cr(float x, float g) {
  if (g >= 1.0f && g <= 64.0f && g == floorf(g)) {
    unsigned e = (unsigned)g;
    double b = (double)x, r = 1.0;
    while (e) {
      if (e & 1u) r = __dmul_rn(r, b);
      e >>= 1;
      if (e) b = __dmul_rn(b, b);
    }
    return __double2float_rn(r);
  }
  return __double2float_rn(pow((double)x, (double)g));
}

// equation of state (fluid.rs:290-297)
template <class PP>
__device__ __forceinline__ float eos(float density, float rho0, const PP& P) {
  if (!(P.flags & F_TAIT)) {
    return fmaxf(__fmul_rn(P.stiffness, __fsub_rn(density, rho0)), 0.0f);
  }
  float r0 = fmaxf(rho0, kEps);
  float ratio = __fdiv_rn(density, r0);
  float pw = powf_cr(ratio, P.gamma);
  return fmaxf(__fmul_rn(__fmul_rn(P.stiffness, r0), __fsub_rn(pw, 1.0f)), 0.0f);
}

// Particle vs body (fluid.rs:463-533, circle and box branches). Returns
// false when separated. With cp: the contact point on the body surface
// (circle: position + normal * radius; box: transform_point(clamped)).
// ---- polygon walls: fluid.rs:518-530 with crates/collision/src/sat.rs ----
// glam 0.29 Vec2::normalize_or_zero: v * (1 / |v|) when that reciprocal is
// finite and positive, else zero.
__device__ __forceinline__ void normalize_or_zero2(float x, float y, float& ox, float& oy) {
  const float rcp = __fdiv_rn(1.0f, __fsqrt_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y))));
  if (isfinite(rcp) && rcp > 0.0f) {
    ox = __fmul_rn(x, rcp);
    oy = __fmul_rn(y, rcp);
  } else {
    ox = 0.0f;
    oy = 0.0f;
  }
}

// project_polygon (sat.rs:88-99): min / max of axis . v, folded from
// (f32::MAX, f32::MIN) with f32::min / max (a NaN loses).
__device__ __forceinline__ void project_poly(const float2* __restrict__ v, uint32_t n, float ax, float ay, float& mn,
                                             float& mx) {
  mn = 3.40282347e38f;
  mx = -3.40282347e38f;
  for (uint32_t i = 0; i < n; i++) {
    const float2 p = v[i];
    const float d = __fadd_rn(__fmul_rn(ax, p.x), __fmul_rn(ay, p.y));
    mn = fminf(mn, d);
    mx = fmaxf(mx, d);
  }
}

// point_in_polygon (sat.rs:203-220): even-odd crossing test.
__device__ __forceinline__ bool point_in_poly(float px, float py, const float2* __restrict__ v, uint32_t n) {
  bool inside = false;
  uint32_t j = n - 1;
  for (uint32_t i = 0; i < n; i++) {
    const float2 a = v[i], b = v[j];
    if (((a.y > py) != (b.y > py)) &&
        (px < __fadd_rn(__fdiv_rn(__fmul_rn(__fsub_rn(b.x, a.x), __fsub_rn(py, a.y)), __fsub_rn(b.y, a.y)), a.x)))
      inside = !inside;
    j = i;
  }
  return inside;
}

// Edge i's unit normal (-e.y, e.x) of a polygon, false for an edge shorter
// than sqrt(EPS_SQ) (sat.rs:112-116).
__device__ __forceinline__ bool poly_edge_normal(const float2* __restrict__ v, uint32_t n, uint32_t i, float& nx,
                                                 float& ny) {
  const float2 a = v[i], b = v[i + 1 == n ? 0 : i + 1];
  const float ex = __fsub_rn(b.x, a.x), ey = __fsub_rn(b.y, a.y);
  if (__fadd_rn(__fmul_rn(ex, ex), __fmul_rn(ey, ey)) < kEpsSq) return false;
  normalize_or_zero2(-ey, ex, nx, ny);
  return true;
}

// sat_circle_polygon (sat.rs:104-200): the edge-normal axes (least overlap
// wins), the closest-vertex axis (can only separate), and for a centre
// inside the polygon the closest edge (largest signed distance). Returns the
// axis (orientation undefined) and the penetration, or false.
__device__ __forceinline__ bool sat_circle_poly(float cx, float cy, float r, const float2* __restrict__ v, uint32_t n,
                                                float& axx, float& axy, float& pen) {
  if (n < 3 || r <= 0.0f) return false;
  float best = 3.40282347e38f, bx = 0.0f, by = 0.0f;
  for (uint32_t i = 0; i < n; i++) {
    float nx, ny;
    if (!poly_edge_normal(v, n, i, nx, ny)) continue;
    float mn, mx;
    project_poly(v, n, nx, ny, mn, mx);
    const float cp = __fadd_rn(__fmul_rn(nx, cx), __fmul_rn(ny, cy));
    const float lo = __fsub_rn(cp, r), hi = __fadd_rn(cp, r);
    if (mx < lo || hi < mn) return false;
    const float ov = __fsub_rn(fminf(mx, hi), fmaxf(mn, lo));
    if (ov < best) {
      best = ov;
      bx = nx;
      by = ny;
    }
  }
  {
    float2 cl = v[0];
    float dx = __fsub_rn(cx, cl.x), dy = __fsub_rn(cy, cl.y);
    float bd = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
    for (uint32_t i = 1; i < n; i++) {
      const float2 q = v[i];
      const float ex = __fsub_rn(cx, q.x), ey = __fsub_rn(cy, q.y);
      const float d = __fadd_rn(__fmul_rn(ex, ex), __fmul_rn(ey, ey));
      if (d < bd) {
        bd = d;
        cl = q;
      }
    }
    dx = __fsub_rn(cx, cl.x);
    dy = __fsub_rn(cy, cl.y);
    if (__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)) >= kEpsSq) {
      float ux, uy;
      normalize_or_zero2(dx, dy, ux, uy);
      if (!(ux == 0.0f && uy == 0.0f)) {
        float mn, mx;
        project_poly(v, n, ux, uy, mn, mx);
        const float cp = __fadd_rn(__fmul_rn(ux, cx), __fmul_rn(uy, cy));
        if (mx < __fsub_rn(cp, r) || __fadd_rn(cp, r) < mn) return false;
      }
    }
  }
  if (point_in_poly(cx, cy, v, n)) {
    float bd = -3.40282347e38f, cnx = 0.0f, cny = 0.0f;
    for (uint32_t i = 0; i < n; i++) {
      float nx, ny;
      if (!poly_edge_normal(v, n, i, nx, ny)) continue;
      const float2 q = v[i];
      const float dist = __fadd_rn(__fmul_rn(nx, __fsub_rn(q.x, cx)), __fmul_rn(ny, __fsub_rn(q.y, cy)));
      if (dist > bd) {
        bd = dist;
        cnx = nx;
        cny = ny;
      }
    }
    if (cnx == 0.0f && cny == 0.0f) return false;
    axx = -cnx;
    axy = -cny;
    pen = __fsub_rn(r, bd);
    return true;
  }
  if (bx == 0.0f && by == 0.0f) return false;
  axx = bx;
  axy = by;
  pen = best;
  return true;
}

// POLY = false compiles the polygon branch out: launches without polygon
// bodies (F_POLY clear) keep the registers of the circle / box tests alone.
template <bool POLY = true>
__device__ __forceinline__ bool collide(float px, float py, float pr, const DevBody& b, float& nx,
                                        float& ny, float& depth, float2* cp = nullptr,
                                        const float2* __restrict__ poly = nullptr) {
  if (POLY && b.shape == 2) {
    // fluid.rs:518-530: SAT on the world-space vertices, the axis oriented
    // from the vertex centroid towards the particle, contact point
    // particle - normal * pr
    float ax, ay, pen;
    if (!sat_circle_poly(px, py, pr, poly + b.vfirst, b.vcount, ax, ay, pen)) return false;
    if (__fadd_rn(__fmul_rn(__fsub_rn(px, b.a), ax), __fmul_rn(__fsub_rn(py, b.b), ay)) < 0.0f) {
      ax = -ax;
      ay = -ay;
    }
    nx = ax;
    ny = ay;
    depth = pen;
    if (cp) *cp = make_float2(__fsub_rn(px, __fmul_rn(ax, pr)), __fsub_rn(py, __fmul_rn(ay, pr)));
    return true;
  }
  if (b.shape == 0) {
    float dx = __fsub_rn(px, b.px);
    float dy = __fsub_rn(py, b.py);
    float dist = __fsqrt_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)));
    float rr = __fadd_rn(b.a, pr);
    if (dist >= rr) return false;
    if (dist > kEps) {
      nx = __fdiv_rn(dx, dist);
      ny = __fdiv_rn(dy, dist);
    } else {
      nx = 1.0f;
      ny = 0.0f;
    }
    depth = __fsub_rn(rr, dist);
    if (cp) *cp = make_float2(__fadd_rn(b.px, __fmul_rn(nx, b.a)), __fadd_rn(b.py, __fmul_rn(ny, b.a)));
    return true;
  }
  float rx = __fsub_rn(px, b.px);
  float ry = __fsub_rn(py, b.py);
  // fluid.rs:483-489 literally: x_axis.x*rel.x + y_axis.x*rel.y, ...
  float lx = __fadd_rn(__fmul_rn(b.xax, rx), __fmul_rn(b.yax, ry));
  float ly = __fadd_rn(__fmul_rn(b.xay, rx), __fmul_rn(b.yay, ry));
  float hx = b.a, hy = b.b;
  // f32::clamp: NaN passes through
  float cxl = lx;
  if (cxl < -hx) cxl = -hx;
  if (cxl > hx) cxl = hx;
  float cyl = ly;
  if (cyl < -hy) cyl = -hy;
  if (cyl > hy) cyl = hy;
  float ddx = __fsub_rn(lx, cxl);
  float ddy = __fsub_rn(ly, cyl);
  float l2 = __fadd_rn(__fmul_rn(ddx, ddx), __fmul_rn(ddy, ddy));
  float lnx, lny;
  if (l2 > kEpsSq) {
    float dist = __fsqrt_rn(l2);
    if (dist >= pr) return false;
    lnx = __fdiv_rn(ddx, dist);
    lny = __fdiv_rn(ddy, dist);
    depth = __fsub_rn(pr, dist);
  } else {
    float dxp = __fsub_rn(hx, fabsf(lx));
    float dyp = __fsub_rn(hy, fabsf(ly));
    // signum().copysign(1.0) is +1 (a NaN stays a positive NaN): the eject
    // normal is always +x or +y in the box frame (fluid.rs:504-516).
    if (dxp < dyp) {
      lnx = (lx != lx) ? fabsf(lx) : 1.0f;
      lny = 0.0f;
      depth = __fadd_rn(pr, dxp);
    } else {
      lnx = 0.0f;
      lny = (ly != ly) ? fabsf(ly) : 1.0f;
      depth = __fadd_rn(pr, dyp);
    }
  }
  // glam Mat2 * Vec2 = x_axis * v.x + y_axis * v.y
  nx = __fadd_rn(__fmul_rn(b.xax, lnx), __fmul_rn(b.yax, lny));
  ny = __fadd_rn(__fmul_rn(b.xay, lnx), __fmul_rn(b.yay, lny));
  if (cp)
    *cp = make_float2(__fadd_rn(__fadd_rn(__fmul_rn(b.xax, cxl), __fmul_rn(b.yax, cyl)), b.px),
                      __fadd_rn(__fadd_rn(__fmul_rn(b.xay, cxl), __fmul_rn(b.yay, cyl)), b.py));
  return true;
}

// Boundary response for one particle against every body in order
// (fluid.rs:1056-1094). Statics take no impulse (body.rs:675-687) and have
// zero velocity, which the no-slip branch reads. Returns kNoDefer, or the
// index of the first body marked dyn that the particle touches: the state is
// then left as it was before that body, for the ordered pass to resume.
template <bool POLY = true>
__device__ __forceinline__ uint32_t walls(float& x, float& y, float& vx, float& vy,
                                          const DevBody* __restrict__ bodies, const StepParams& P) {
  if (P.flags & F_WBOX) {
    // the reject test below for every body at once, from the launch
    // parameters: a particle it rejects for every body touches none, and
    // nothing moves it between bodies, so the loop would change nothing
    bool near = false;
#pragma unroll
    for (uint32_t k = 0; k < kWallBoxes; k++) {
      const float4 wb = P.wbox[k];
      near = near || !(fabsf(x - wb.x) > wb.z || fabsf(y - wb.y) > wb.w);
    }
    if (!near) return kNoDefer;
  }
  for (uint32_t k = 0; k < P.nbodies; k++) {
    const DevBody* bp = bodies + P.body_first + k;
    // bounding-box reject first: only the centre and the padded extents are read
    if (fabsf(x - __ldg(&bp->px)) > __ldg(&bp->ex) + P.pr_pad || fabsf(y - __ldg(&bp->py)) > __ldg(&bp->ey) + P.pr_pad)
      continue;
    const DevBody b = *bp;
    float nx, ny, depth;
    if (!collide<POLY>(x, y, P.pr, b, nx, ny, depth, nullptr, P.poly)) continue;
    if (depth <= 0.0f) continue;
    if (b.dyn) return k;
    x = __fadd_rn(x, __fmul_rn(nx, depth));
    y = __fadd_rn(y, __fmul_rn(ny, depth));
    float vn = __fadd_rn(__fmul_rn(vx, nx), __fmul_rn(vy, ny));
    if (vn < 0.0f) {
      vx = __fsub_rn(vx, __fmul_rn(nx, vn));
      vy = __fsub_rn(vy, __fmul_rn(ny, vn));
      if (P.flags & F_FRICTION) {
        float vtx = vx, vty = vy;
        float wvx = 0.0f, wvy = 0.0f;
        float wdot = __fadd_rn(__fmul_rn(wvx, nx), __fmul_rn(wvy, ny));
        float wtx = __fsub_rn(wvx, __fmul_rn(nx, wdot));
        float wty = __fsub_rn(wvy, __fmul_rn(ny, wdot));
        float dvx = __fmul_rn(__fsub_rn(wtx, vtx), P.mu);
        float dvy = __fmul_rn(__fsub_rn(wty, vty), P.mu);
        vx = __fadd_rn(vx, dvx);
        vy = __fadd_rn(vy, dvy);
      }
    }
  }
  return kNoDefer;
}

// RigidBody2::apply_impulse (body.rs:675-687): statics ignore it; a
// dynamic body wakes, v += J * inv_mass, w += (r x J) * inv_inertia.
__device__ __forceinline__ void apply_impulse(DynBody& d, float bpx, float bpy, float jx, float jy, float qx,
                                              float qy) {
  if (d.is_static) return;
  d.sleeping = 0;
  d.vx = __fadd_rn(d.vx, __fmul_rn(jx, d.inv_mass));
  d.vy = __fadd_rn(d.vy, __fmul_rn(jy, d.inv_mass));
  const float rx = __fsub_rn(qx, bpx), ry = __fsub_rn(qy, bpy);
  const float torque = __fsub_rn(__fmul_rn(rx, jy), __fmul_rn(ry, jx));
  d.w = __fadd_rn(d.w, __fmul_rn(torque, d.inv_inertia));
}

// The full body loop of one particle from body k0 on, with the reactions on
// the bodies (fluid.rs:1056-1094): push out, remove the approach velocity,
// impulse n * (vn * m) on the body, then the no-slip pull toward the body's
// tangential velocity and its reaction -dv * m. Run in particle order.
__device__ __forceinline__ void walls_ordered(float& x, float& y, float& vx, float& vy, float m, uint32_t k0,
                                              const DevBody* __restrict__ bodies, DynBody* __restrict__ dyn,
                                              const StepParams& P) {
  for (uint32_t k = k0; k < P.nbodies; k++) {
    const DevBody b = bodies[P.body_first + k];
    if (fabsf(x - b.px) > b.ex + P.pr_pad || fabsf(y - b.py) > b.ey + P.pr_pad) continue;
    float nx, ny, depth;
    float2 cp;
    if (!collide(x, y, P.pr, b, nx, ny, depth, &cp, P.poly)) continue;
    if (depth <= 0.0f) continue;
    x = __fadd_rn(x, __fmul_rn(nx, depth));
    y = __fadd_rn(y, __fmul_rn(ny, depth));
    const float vn = __fadd_rn(__fmul_rn(vx, nx), __fmul_rn(vy, ny));
    if (vn < 0.0f) {
      vx = __fsub_rn(vx, __fmul_rn(nx, vn));
      vy = __fsub_rn(vy, __fmul_rn(ny, vn));
      if (!b.dyn) {
        // a plain wall: no reaction, zero velocity
        if (P.flags & F_FRICTION) {
          const float wdot = __fadd_rn(__fmul_rn(0.0f, nx), __fmul_rn(0.0f, ny));
          const float wtx = __fsub_rn(0.0f, __fmul_rn(nx, wdot));
          const float wty = __fsub_rn(0.0f, __fmul_rn(ny, wdot));
          vx = __fadd_rn(vx, __fmul_rn(__fsub_rn(wtx, vx), P.mu));
          vy = __fadd_rn(vy, __fmul_rn(__fsub_rn(wty, vy), P.mu));
        }
        continue;
      }
      DynBody& d = dyn[k];
      if (!d.is_static) d.sleeping = 0;
      const float vm = __fmul_rn(vn, m);
      apply_impulse(d, b.px, b.py, __fmul_rn(nx, vm), __fmul_rn(ny, vm), cp.x, cp.y);
      if (P.flags & F_FRICTION) {
        const float vtx = vx, vty = vy;
        const float wvx = d.vx, wvy = d.vy;
        const float wdot = __fadd_rn(__fmul_rn(wvx, nx), __fmul_rn(wvy, ny));
        const float wtx = __fsub_rn(wvx, __fmul_rn(nx, wdot));
        const float wty = __fsub_rn(wvy, __fmul_rn(ny, wdot));
        const float dvx = __fmul_rn(__fsub_rn(wtx, vtx), P.mu);
        const float dvy = __fmul_rn(__fsub_rn(wty, vty), P.mu);
        vx = __fadd_rn(vx, dvx);
        vy = __fadd_rn(vy, dvy);
        apply_impulse(d, b.px, b.py, __fmul_rn(-dvx, m), __fmul_rn(-dvy, m), cp.x, cp.y);
      }
    }
  }
}

// ---------------------------------------------------------------- closure features
// Neighbour aggregates of one particle for the closure network, accumulated
// over the same neighbour pairs and in the same order as the pressure force
// (j != i, the reference's visit order). Per pair, with delta = x_i - x_j,
// grad = spiky_grad(delta), w = poly6(|delta|^2), V_j = m_j / rho_j and
// dv = v_j - v_i:
//   pressure force   P -= grad * (m_j * (q_i + q_j)),  q = p / rho^2
//   divergence       D += V_j * (dv . grad)
//   curl (z)         C += V_j * (dv.x grad.y - dv.y grad.x)
//   kernel moments   S += V_j w, M1 += V_j w dv, M2 += V_j w (dv.x^2, dv.y^2)
//   pressure mean    Q += V_j w p_j,  p_j = (q_j rho_j) rho_j
struct FeatAcc {
  float px = 0.0f, py = 0.0f, div = 0.0f, curl = 0.0f;
  float wsum = 0.0f, m1x = 0.0f, m1y = 0.0f, m2xx = 0.0f, m2yy = 0.0f, pw = 0.0f;
  uint32_t cnt = 0;
};

// vol = V_j = m_j / rho_j and pj = (q_j rho_j) rho_j come precomputed per
// particle (the density pass's closure factors). PXY: accumulate the pressure
// sum P here; a caller whose force sum has no other terms (no artificial
// viscosity, no cohesion) takes P from it instead, which is the same sum of
// the same products in the same order.
template <bool PXY>
__device__ __forceinline__ void feat_pair(FeatAcc& a, float gxx, float gyy, float w, float vol, float pj, float m_j,
                                          float q_i, float q_j, float dvx, float dvy) {
  if constexpr (PXY) {
    const float mt = __fmul_rn(m_j, __fadd_rn(q_i, q_j));
    a.px = __fsub_rn(a.px, __fmul_rn(gxx, mt));
    a.py = __fsub_rn(a.py, __fmul_rn(gyy, mt));
  }
  a.div = __fadd_rn(a.div, __fmul_rn(vol, __fadd_rn(__fmul_rn(dvx, gxx), __fmul_rn(dvy, gyy))));
  a.curl = __fadd_rn(a.curl, __fmul_rn(vol, __fsub_rn(__fmul_rn(dvx, gyy), __fmul_rn(dvy, gxx))));
  const float ww = __fmul_rn(vol, w);
  a.wsum = __fadd_rn(a.wsum, ww);
  const float wx = __fmul_rn(ww, dvx), wy = __fmul_rn(ww, dvy);
  a.m1x = __fadd_rn(a.m1x, wx);
  a.m1y = __fadd_rn(a.m1y, wy);
  a.m2xx = __fadd_rn(a.m2xx, __fmul_rn(wx, dvx));
  a.m2yy = __fadd_rn(a.m2yy, __fmul_rn(wy, dvy));
  a.pw = __fadd_rn(a.pw, __fmul_rn(ww, pj));
  a.cnt++;
}

// Nearest static body within 3h: signed distance to its surface (negative
// inside, from the box's local frame as collide() builds it) and the
// outward normal in world axes. d is returned in units of h, clamped to
// [-1, 3]; the normal is zero when no body is that close. A body whose
// padded bounding box is farther than 3h along x or y cannot be nearer than
// 3h and is skipped.
__device__ __forceinline__ void wall_feature(float x, float y, const DevBody* __restrict__ bodies,
                                             const StepParams& P, float& fd, float& fnx, float& fny) {
  const float lim = __fmul_rn(3.0f, P.hk);
  float best = lim, bnx = 0.0f, bny = 0.0f;
  for (uint32_t k = 0; k < P.nbodies; k++) {
    const DevBody b = bodies[P.body_first + k];
    if (b.shape == 2) continue;  // polygons (fluid-phase bodies only) are not part of the feature
    if (fabsf(__fsub_rn(x, b.px)) > __fadd_rn(b.ex, lim) || fabsf(__fsub_rn(y, b.py)) > __fadd_rn(b.ey, lim)) continue;
    float d, nx, ny;
    if (b.shape == 0) {
      const float dx = __fsub_rn(x, b.px), dy = __fsub_rn(y, b.py);
      const float dist = __fsqrt_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)));
      d = __fsub_rn(dist, b.a);
      if (dist > kEps) {
        nx = __fdiv_rn(dx, dist);
        ny = __fdiv_rn(dy, dist);
      } else {
        nx = 1.0f;
        ny = 0.0f;
      }
    } else {
      const float rx = __fsub_rn(x, b.px), ry = __fsub_rn(y, b.py);
      const float lx = __fadd_rn(__fmul_rn(b.xax, rx), __fmul_rn(b.yax, ry));
      const float ly = __fadd_rn(__fmul_rn(b.xay, rx), __fmul_rn(b.yay, ry));
      const float qx = __fsub_rn(fabsf(lx), b.a), qy = __fsub_rn(fabsf(ly), b.b);
      float lnx, lny;
      if (qx > 0.0f || qy > 0.0f) {
        const float ox = fmaxf(qx, 0.0f), oy = fmaxf(qy, 0.0f);
        d = __fsqrt_rn(__fadd_rn(__fmul_rn(ox, ox), __fmul_rn(oy, oy)));
        lnx = __fdiv_rn(copysignf(ox, lx), d);
        lny = __fdiv_rn(copysignf(oy, ly), d);
      } else if (qx >= qy) {
        d = qx;
        lnx = copysignf(1.0f, lx);
        lny = 0.0f;
      } else {
        d = qy;
        lnx = 0.0f;
        lny = copysignf(1.0f, ly);
      }
      nx = __fadd_rn(__fmul_rn(b.xax, lnx), __fmul_rn(b.yax, lny));
      ny = __fadd_rn(__fmul_rn(b.xay, lnx), __fmul_rn(b.yay, lny));
    }
    if (d < best) {
      best = d;
      bnx = nx;
      bny = ny;
    }
  }
  fd = __fdiv_rn(fmaxf(best, -P.hk), P.hk);
  fnx = bnx;
  fny = bny;
}

// The 16 closure inputs of one particle for a coarse step of P.dt:
//   0 rho/rho0 - 1          1 p / (k rho0)          2 D dt       3 C dt
//   4 neighbours / 16       5 wall distance / h     6, 7 wall normal
//   8, 9 M1/S (dt/h)        10, 12 M2/S (dt/h)^2 (xx, yy)
//   11 (p - Q/S) / (k rho0) (pressure deviation from the neighbour mean:
//      near zero for a smooth pressure field, large for particle-scale noise)
//   13, 14 (P / rho) dt^2/h (pressure displacement over the step)
//   15 |v| dt / h
__device__ __forceinline__ void feat_finish(const FeatAcc& a, float dens, float rho_i, float p, float r0, float vx,
                                            float vy, float wd, float wnx, float wny, const StepParams& P,
                                            float (&f)[16]) {
  const float dt = P.dt;
  const float ih = __fdiv_rn(1.0f, P.hk);
  const float s1 = __fmul_rn(dt, ih);
  const float s2 = __fmul_rn(s1, s1);
  const float s3 = __fmul_rn(__fmul_rn(dt, dt), ih);
  const float rr = fmaxf(r0, kEps);
  const float kr = __fmul_rn(P.stiffness, rr);
  f[0] = __fsub_rn(__fdiv_rn(dens, rr), 1.0f);
  f[1] = kr > 0.0f ? __fdiv_rn(p, kr) : 0.0f;
  f[2] = __fmul_rn(a.div, dt);
  f[3] = __fmul_rn(a.curl, dt);
  f[4] = __fmul_rn((float)a.cnt, 0.0625f);
  f[5] = wd;
  f[6] = wnx;
  f[7] = wny;
  const float iw = a.wsum > 0.0f ? __fdiv_rn(1.0f, a.wsum) : 0.0f;
  f[8] = __fmul_rn(__fmul_rn(a.m1x, iw), s1);
  f[9] = __fmul_rn(__fmul_rn(a.m1y, iw), s1);
  f[10] = __fmul_rn(__fmul_rn(a.m2xx, iw), s2);
  f[11] = kr > 0.0f ? __fdiv_rn(__fsub_rn(p, __fmul_rn(a.pw, iw)), kr) : 0.0f;
  f[12] = __fmul_rn(__fmul_rn(a.m2yy, iw), s2);
  f[13] = __fmul_rn(__fdiv_rn(a.px, rho_i), s3);
  f[14] = __fmul_rn(__fdiv_rn(a.py, rho_i), s3);
  f[15] = __fmul_rn(__fsqrt_rn(__fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy))), s1);
}

}  // namespace phieng
