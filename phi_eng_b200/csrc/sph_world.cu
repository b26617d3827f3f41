// World2 and the C ABI of libphieng_sph.so (include/phieng_sph.h).
//
// The world mirrors the slice of the reference's World2 that the fluid step
// reads (crates/dynamics/src/world.rs: gravity, time, static bodies, the
// FluidState2) and keeps the particle state resident on the GPU. Host
// mirrors of the state exist only to serve the copy-in / copy-out entry
// points; a validity flag on each side says which copy is current.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/phieng_sph.h"
#include "sph_kernels.h"
#include "sph_mlp_host.h"
#include "sph_host.h"
#include "sph_snapshot.h"

using namespace phieng;

namespace {
using namespace phieng::host;
constexpr uint32_t kMaxParticles2D = 4096;  // MAX_PARTICLES_2D (fluid.rs:30)

// Most particles one resample pass (fluid.rs:826-893) can leave from n: every
// particle is kept or split in two, and a split only happens while the output
// holds fewer than MAX_PARTICLES_2D - 1 particles, so at most
// MAX_PARTICLES_2D / 2 particles split. The output is a Vec in the reference
// and has no cap of its own.
inline uint32_t resample_bound(uint32_t n) { return n + std::min(n, kMaxParticles2D / 2); }
constexpr uint32_t kClockWord = 16;         // scalar word holding the step's world clock (turbulence)

// AmbientConfig2::default (ambient.rs): springs, drag and turbulence off, air
// density 1, turbulence frequency 1, time scale 1, 3 octaves.
AmbientConfig2Ffi default_ambient() {
  AmbientConfig2Ffi a;
  std::memset(&a, 0, sizeof(a));
  a.air_density = 1.0f;
  a.turbulence_frequency = 1.0f;
  a.turbulence_time_scale = 1.0f;
  a.turbulence_octaves = 3;
  return a;
}
}  // namespace

struct World2 {
  FluidConfig2Ffi cfg = default_config();
  AmbientConfig2Ffi ambient = default_ambient();
  float gx = 0.0f, gy = -9.81f;  // World2::new (world.rs:338)
  float time = 0.0f;
  std::vector<DevBody> bodies;
  bool bodies_dirty = true;
  uint32_t cap = kMaxParticles2D;

  // particles (host mirror); mass and phase are fixed at insertion
  uint32_t n = 0;
  std::vector<float4, PinnedAlloc<float4>> h_state;  // (x, y, vx, vy) by id
  // bounding box of the finite host positions, kept while particles are
  // added so the first grid plan needs no pass over a large state
  bool bbox_valid = true;
  float bx0 = INFINITY, bx1 = -INFINITY, by0 = INFINITY, by1 = -INFINITY;
  std::vector<float> h_mass;
  std::vector<uint8_t> h_phase;
  std::vector<float> h_dens, h_pres;
  bool mass_uniform = true;
  float mass_value = 0.0f;
  bool phase_uniform = true;
  uint32_t phase_value = 0;

  bool host_state_valid = true;
  bool dev_state_valid = false;
  bool dev_aux_valid = false;
  bool dp_on_device = false;
  bool keys_valid = false;   // key[] and the bucket counts match the state
  bool plan_valid = false;
  bool plan_locked = false;  // set by phieng_sph_set_grid: no automatic replan
  uint32_t sid_perm_n = 0;   // d.sid is a permutation of [0, sid_perm_n)
  GridPlan plan{};

  int device = -1;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  bool user_stream = false;
  FluidBufs d;
  float* d_tmp = nullptr;
  size_t d_tmp_bytes = 0;
  unsigned int* h_pinned = nullptr;

  cudaGraphExec_t gexec = nullptr;
  std::string gsig;

  // phase timing: events recorded between the phases of every substep
  bool profiling = false;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};

  int32_t error = PHIENG_SPH_OK;
  uint64_t substeps = 0;

  // Batch of independent scenes (empty for an ordinary world): scene k owns
  // particles [first, first + count) and bodies [body_first, +nbodies), and
  // has its own config, gravity and bucket grid; w->plan then spans all
  // scenes' buckets.
  struct Scene {
    uint32_t first = 0, count = 0;
    FluidConfig2Ffi cfg;
    float gx = 0.0f, gy = -9.81f;
    uint32_t body_first = 0, nbodies = 0;
    bool mass_uniform = true, phase_uniform = true;
    float mass_value = 0.0f;
    uint32_t phase_value = 0;
    GridPlan plan{};
  };
  std::vector<Scene> scenes;
  StepParams* d_ptab = nullptr;
  uint32_t* d_pscene = nullptr;
  uint32_t* d_sscene = nullptr;
  uint32_t batch_cap = 0;
  bool is_batch() const { return !scenes.empty(); }

  // x-slab rank world (phieng_sph_slab_*): slots, exchange buffers and the
  // free-slot stack [own_cap] + words [kSlabWords] (d_slab)
  bool slab = false;
  SlabPlan slab_plan{};
  uint32_t* d_slab = nullptr;
  uint32_t slab_cap = 0;

  // learned closure (phieng_sph_set_closure / phieng_sph_closure_step)
  PhiengMlp* closure = nullptr;
  uint32_t closure_ratio = 4;
  float closure_threshold = 0.03f;
  uint32_t closure_criterion = 0;
  float4* d_save = nullptr;     // pre-step state of the last coarse step (id order)
  float* d_rho_prev = nullptr;  // pre-step density (id order)
  float4* d_block_save = nullptr;  // state at the start of an optimistic block of coarse steps
  float2* d_svp = nullptr;         // sorted closure factors of the last closure density pass
  uint32_t closure_cap = 0;
  cudaGraphExec_t cexec = nullptr;
  std::string csig;

  // bodies of the last phieng_sph_step_fluid call and their buffers
  DynBufs dynb;
  DevBody* d_cbodies = nullptr;
  uint32_t cbody_cap = 0, sample_cap = 0, dyn_pcap = 0, count2_cap = 0;
  float2* d_poly = nullptr;  // world-space polygon vertices of the last fluid-phase call
  uint32_t poly_cap = 0;
  // boundary ghosts (boundary_particles): regenerated when their inputs change
  std::string ghost_sig;
  std::vector<float2> h_gpos;  // host copy of the device ghosts (cell-grouped order)
  uint64_t ghost_regens = 0;   // boundary_regens (fluid.rs:207)
  uint32_t nghost = 0, ghost_cap = 0, gtab_mask = 0, gtab_cap = 0;
  float2* d_gpos = nullptr;
  float* d_gq = nullptr;
  GhostCell* d_gtab = nullptr;
  // adaptive resolution scratch (capacity = d.cap when allocated)
  ResampleBufs rs;
  uint32_t rs_cap = 0;

  // launch tuning (phieng_sph_set_tuning)
  float buckets_per_particle = 2.0f;
  // arithmetic of the plain density / force passes (phieng_sph_set_precision)
  uint32_t precision = PHIENG_SPH_EXACT;
};

namespace {

void set_error(World2* w, int32_t e, const char* what) {
  if (w->error == PHIENG_SPH_OK) {
    w->error = e;
    std::fprintf(stderr, "phieng_sph: %s (%s)\n", error_text(e), what ? what : "");
  }
}

bool cuda_ok(World2* w, cudaError_t r, const char* what) {
  if (r == cudaSuccess) return true;
  cudaGetLastError();
  if (w->error == PHIENG_SPH_OK) {
    w->error = PHIENG_SPH_E_CUDA;
    std::fprintf(stderr, "phieng_sph: %s failed: %s\n", what, cudaGetErrorString(r));
  }
  return false;
}

// A look-back wait of the scan that gave up leaves a sticky device flag
// (a wrong grid order): read it where the host synchronises anyway.
bool scan_flag_ok(World2* w) {
  if (w->device < 0 || !w->d.scalar) return true;
  if (!cuda_ok(w, cudaMemcpyAsync(w->h_pinned + 8, w->d.scan_err, 4, cudaMemcpyDeviceToHost, w->stream), "flag") ||
      !cuda_ok(w, cudaStreamSynchronize(w->stream), "sync"))
    return false;
  if (w->h_pinned[8] != 0u) {
    set_error(w, PHIENG_SPH_E_CUDA, "a bounded device wait gave up (bucket scan or tensor core)");
    return false;
  }
  return true;
}

template <class T>
void dfree(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

void free_particle_buffers(FluidBufs& d) {
  dfree(d.order);  // order tags do not survive a reallocation
  dfree(d.state);
  dfree(d.mass);
  dfree(d.phase);
  dfree(d.key);
  dfree(d.tkey);
  dfree(d.tid);
  dfree(d.skey);
  dfree(d.sid);
  dfree(d.spos);
  dfree(d.svel);
  dfree(d.smass);
  dfree(d.sphase);
  dfree(d.sdq);
  dfree(d.spres);
  dfree(d.nmask);
  d.cap = 0;
}

void release_graph(World2* w) {
  if (w->gexec) cudaGraphExecDestroy(w->gexec);
  w->gexec = nullptr;
  w->gsig.clear();
  if (w->cexec) cudaGraphExecDestroy(w->cexec);
  w->cexec = nullptr;
  w->csig.clear();
}

bool ensure_device(World2* w) {
  if (w->device >= 0) return true;
  int count = 0;
  cudaError_t r = cudaGetDeviceCount(&count);
  if (r != cudaSuccess || count == 0) {
    cudaGetLastError();
    set_error(w, PHIENG_SPH_E_NO_DEVICE, "cudaGetDeviceCount");
    return false;
  }
  int dev = 0;
  if (!cuda_ok(w, cudaGetDevice(&dev), "cudaGetDevice")) return false;
  if (!cuda_ok(w, cudaStreamCreateWithFlags(&w->own_stream, cudaStreamNonBlocking), "cudaStreamCreate"))
    return false;
  if (!w->user_stream) w->stream = w->own_stream;
  if (!cuda_ok(w, cudaMalloc(&w->d.scalar, 128), "cudaMalloc(scalar)")) return false;
  if (!cuda_ok(w, cudaMemset(w->d.scalar, 0, 128), "cudaMemset(scalar)")) return false;
  w->d.done = w->d.scalar + 8;       // scan counters [8], [9]
  w->d.scan_err = w->d.scalar + 12;  // set when a scan's look-back wait or a tensor-core wait gave up
  if (!cuda_ok(w, cudaMallocHost(&w->h_pinned, 64), "cudaMallocHost")) return false;
  w->device = dev;
  return true;
}

template <class T>
bool dalloc(World2* w, T*& p, size_t count) {
  return cuda_ok(w, cudaMalloc(&p, sizeof(T) * std::max<size_t>(count, 1)), "cudaMalloc");
}

bool ensure_capacity(World2* w, uint32_t need) {
  FluidBufs& d = w->d;
  if (need <= d.cap && d.state) return true;
  cudaStreamSynchronize(w->stream);
  free_particle_buffers(d);
  release_graph(w);
  uint32_t c = std::max<uint32_t>(need, 1024);
  bool ok = dalloc(w, d.state, c) && dalloc(w, d.mass, c) && dalloc(w, d.phase, c) && dalloc(w, d.key, c) &&
            dalloc(w, d.tkey, c) && dalloc(w, d.tid, c) &&
            dalloc(w, d.skey, c) && dalloc(w, d.sid, c) && dalloc(w, d.spos, c) && dalloc(w, d.svel, c) &&
            dalloc(w, d.smass, c) && dalloc(w, d.sphase, c) && dalloc(w, d.sdq, c) && dalloc(w, d.spres, c) &&
            dalloc(w, d.nmask, 3 * (size_t)c);
  if (ok && w->is_batch()) {
    dfree(w->d_pscene);
    dfree(w->d_sscene);
    dfree(w->d_ptab);
    ok = dalloc(w, w->d_pscene, c) && dalloc(w, w->d_sscene, c) && dalloc(w, w->d_ptab, w->scenes.size());
    d.batch.ptab = w->d_ptab;
    d.batch.pscene = w->d_pscene;
    d.batch.sscene = w->d_sscene;
  }
  if (!ok) {
    free_particle_buffers(d);
    return false;
  }
  d.cap = c;
  w->dev_state_valid = false;
  w->dev_aux_valid = false;
  w->dp_on_device = false;
  w->keys_valid = false;
  w->sid_perm_n = 0;
  return true;
}

bool ensure_tmp(World2* w, size_t bytes) {
  if (bytes <= w->d_tmp_bytes && w->d_tmp) return true;
  dfree(w->d_tmp);
  w->d_tmp_bytes = 0;
  if (!cuda_ok(w, cudaMalloc(&w->d_tmp, bytes), "cudaMalloc(tmp)")) return false;
  w->d_tmp_bytes = bytes;
  return true;
}

// Download the particle state if the device copy is the current one.
bool ensure_host_state(World2* w) {
  if (w->host_state_valid) return true;
  if (!cuda_ok(w, cudaMemcpyAsync(w->h_state.data(), w->d.state, sizeof(float4) * w->n, cudaMemcpyDeviceToHost,
                                  w->stream),
               "download state"))
    return false;
  if (!cuda_ok(w, cudaStreamSynchronize(w->stream), "sync")) return false;
  if (!scan_flag_ok(w)) return false;
  w->host_state_valid = true;
  w->bbox_valid = false;
  return true;
}

bool ensure_host_dp(World2* w) {
  if (!w->dp_on_device) return true;
  if (w->n == 0) {
    w->dp_on_device = false;
    return true;
  }
  if (!ensure_tmp(w, sizeof(float) * 2 * (size_t)w->n)) return false;
  enqueue_unsort_dp(w->d, w->n, w->d_tmp, w->d_tmp + w->n, w->stream);
  if (!cuda_ok(w, cudaGetLastError(), "unsort")) return false;
  cudaMemcpyAsync(w->h_dens.data(), w->d_tmp, sizeof(float) * w->n, cudaMemcpyDeviceToHost, w->stream);
  cudaMemcpyAsync(w->h_pres.data(), w->d_tmp + w->n, sizeof(float) * w->n, cudaMemcpyDeviceToHost, w->stream);
  if (!cuda_ok(w, cudaStreamSynchronize(w->stream), "sync")) return false;
  w->dp_on_device = false;
  return true;
}

// Bucket grid from the particle bounding box (host copy must be current).
// Bucket grid covering the cells of n particles (with a margin), ~2 buckets
// per particle at most.
GridPlan plan_cells(int64_t x0, int64_t x1, int64_t y0, int64_t y1, uint32_t n, float hg,
                    float buckets_per_particle);

GridPlan plan_for(const float4* st, uint32_t n, float hg, float buckets_per_particle) {
  int64_t x0 = INT64_MAX, x1 = INT64_MIN, y0 = INT64_MAX, y1 = INT64_MIN;
  for (uint32_t i = 0; i < n; i++) {
    float4 s = st[i];
    if (!std::isfinite(s.x) || !std::isfinite(s.y)) continue;
    int32_t cx = sat_floor_i32(s.x / hg), cy = sat_floor_i32(s.y / hg);
    x0 = std::min<int64_t>(x0, cx);
    x1 = std::max<int64_t>(x1, cx);
    y0 = std::min<int64_t>(y0, cy);
    y1 = std::max<int64_t>(y1, cy);
  }
  return plan_cells(x0, x1, y0, y1, n, hg, buckets_per_particle);
}

// The plan from the cell bounds of the particles (x0 > x1: none).
GridPlan plan_cells(int64_t x0, int64_t x1, int64_t y0, int64_t y1, uint32_t n, float hg,
                    float buckets_per_particle) {
  if (x0 > x1) x0 = x1 = y0 = y1 = 0;
  const int64_t sx = x1 - x0 + 1, sy = y1 - y0 + 1;
  const int64_t mx = std::max<int64_t>(2, sx / 8), my = std::max<int64_t>(2, sy / 8);
  uint32_t W = std::max<uint32_t>(4, next_pow2((uint64_t)(sx + 2 * mx)));
  uint32_t H = std::max<uint32_t>(4, next_pow2((uint64_t)(sy + 2 * my)));
  // bucket budget: buckets_per_particle (2 by default) per particle, rounded
  // up to a power of two; each bucket costs ~20 B of count / scan /
  // range-table traffic per substep, fewer buckets alias more cells into one
  const uint64_t want = (uint64_t)std::ceil((double)buckets_per_particle * (double)std::max<uint32_t>(n, 1));
  const uint64_t budget = std::min<uint64_t>(1ull << 24, std::max<uint64_t>(1ull << 12, next_pow2(want)));
  while ((uint64_t)W * H > budget) {
    if (W >= H && W > 4)
      W >>= 1;
    else if (H > 4)
      H >>= 1;
    else
      break;
  }
  GridPlan g;
  g.log2w = log2u(W);
  g.log2h = log2u(H);
  g.maskw = W - 1;
  g.maskh = H - 1;
  g.nbuckets = W * H;
  g.base = 0;
  g.sentinel = g.nbuckets;
  g.cx0 = (int32_t)std::max<int64_t>(INT32_MIN, x0 - mx);
  g.cy0 = (int32_t)std::max<int64_t>(INT32_MIN, y0 - my);
  g.hg = hg;
  return g;
}

void plan_grid(World2* w) {
  if (w->is_batch()) {
    // one bucket range per scene, laid end to end
    uint64_t base = 0;
    for (auto& sc : w->scenes) {
      GridPlan g = plan_for(w->h_state.data() + sc.first, sc.count, sc.cfg.smoothing_length, w->buckets_per_particle);
      g.base = (uint32_t)base;
      base += g.nbuckets;
      sc.plan = g;
    }
    for (auto& sc : w->scenes) sc.plan.sentinel = (uint32_t)base;
    GridPlan all{};
    all.nbuckets = (uint32_t)base;
    all.sentinel = (uint32_t)base;
    all.base = 0;
    all.hg = w->scenes[0].cfg.smoothing_length;
    w->plan = all;
  } else if (w->bbox_valid && w->cfg.smoothing_length > 0.0f) {
    // floor(x / h) is monotonic in x for h > 0: the bounding box's cells
    // bound every particle's cell
    const float hg = w->cfg.smoothing_length;
    if (w->n == 0 || !(w->bx0 <= w->bx1))
      w->plan = plan_cells(1, 0, 1, 0, w->n, hg, w->buckets_per_particle);
    else
      w->plan = plan_cells(sat_floor_i32(w->bx0 / hg), sat_floor_i32(w->bx1 / hg), sat_floor_i32(w->by0 / hg),
                           sat_floor_i32(w->by1 / hg), w->n, hg, w->buckets_per_particle);
  } else {
    w->plan = plan_for(w->h_state.data(), w->n, w->cfg.smoothing_length, w->buckets_per_particle);
  }
  w->plan_valid = true;
  w->keys_valid = false;
}

// Bucket-grid arrays: counts (padded to whole scan tiles), the range table
// and the scan tile sums.
// Bucket arrays for up to nbuckets buckets (+ the sentinel), zeroed.
bool alloc_range(World2* w, uint32_t nbuckets) {
  FluidBufs& d = w->d;
  const uint32_t tiles = (nbuckets + 1 + kBucketScanTile - 1) / kBucketScanTile;
  cudaStreamSynchronize(w->stream);
  dfree(d.count);
  dfree(d.start);
  dfree(d.tilesum);
  dfree(d.tstate);
  d.range_cap = 0;
  release_graph(w);
  const uint32_t len = tiles * kBucketScanTile;
  if (!dalloc(w, d.count, len) || !dalloc(w, d.start, (size_t)len + 1) || !dalloc(w, d.tilesum, tiles) ||
      !dalloc(w, d.tstate, tiles))
    return false;
  if (!cuda_ok(w, cudaMemsetAsync(d.count, 0, sizeof(uint32_t) * len, w->stream), "memset") ||
      !cuda_ok(w, cudaMemsetAsync(d.tstate, 0, sizeof(unsigned long long) * tiles, w->stream), "memset"))
    return false;
  d.range_cap = nbuckets;
  d.count_len = len;
  w->keys_valid = false;
  return true;
}

bool ensure_range(World2* w) {
  FluidBufs& d = w->d;
  const uint32_t m = w->plan.sentinel + 1;  // buckets + the non-finite sentinel
  const uint32_t tiles = (m + kBucketScanTile - 1) / kBucketScanTile;
  if (d.count && d.range_cap >= w->plan.sentinel) {
    d.count_len = tiles * kBucketScanTile;
    return true;
  }
  if (!alloc_range(w, w->plan.sentinel)) return false;
  d.count_len = tiles * kBucketScanTile;
  return true;
}

bool ensure_bodies(World2* w) {
  if (!w->bodies_dirty) return true;
  FluidBufs& d = w->d;
  uint32_t nb = (uint32_t)w->bodies.size();
  if (nb > d.bodies_cap || !d.bodies) {
    cudaStreamSynchronize(w->stream);
    dfree(d.bodies);
    release_graph(w);
    uint32_t c = std::max<uint32_t>(16, nb);
    if (!dalloc(w, d.bodies, c)) return false;
    d.bodies_cap = c;
  }
  if (nb && !cuda_ok(w, cudaMemcpyAsync(d.bodies, w->bodies.data(), sizeof(DevBody) * nb, cudaMemcpyHostToDevice,
                                        w->stream),
                     "upload bodies"))
    return false;
  w->bodies_dirty = false;
  return true;
}

bool upload_scene_table(World2* w, float dt);

// Everything a substep needs: device, buffers, current state on the device,
// a bucket grid, the bodies and valid keys.
bool prepare(World2* w) {
  if (w->error != PHIENG_SPH_OK) return false;
  if (!ensure_device(w)) return false;
  if (!w->dev_state_valid) {
    // adaptive resolution: room for what a resample pass can output
    if (!ensure_capacity(w, w->cfg.adaptive_resolution ? std::max(resample_bound(w->n), kMaxParticles2D) : w->n))
      return false;
    if (!w->plan_valid) plan_grid(w);
    if (w->n && !cuda_ok(w, cudaMemcpyAsync(w->d.state, w->h_state.data(), sizeof(float4) * w->n,
                                            cudaMemcpyHostToDevice, w->stream),
                         "upload state"))
      return false;
    if (w->is_batch()) {
      std::vector<uint32_t> ps(w->n);
      for (uint32_t k = 0; k < w->scenes.size(); k++)
        for (uint32_t i = 0; i < w->scenes[k].count; i++) ps[w->scenes[k].first + i] = k;
      if (!cuda_ok(w, cudaMemcpyAsync(w->d_pscene, ps.data(), 4ull * w->n, cudaMemcpyHostToDevice, w->stream),
                   "upload scene ids"))
        return false;
    }
    w->dev_state_valid = true;
    w->keys_valid = false;
  }
  if (!w->dev_aux_valid && (!w->mass_uniform || !w->phase_uniform) && w->n) {
    cudaMemcpyAsync(w->d.mass, w->h_mass.data(), sizeof(float) * w->n, cudaMemcpyHostToDevice, w->stream);
    cudaMemcpyAsync(w->d.phase, w->h_phase.data(), w->n, cudaMemcpyHostToDevice, w->stream);
    w->dev_aux_valid = true;
  }
  if (!w->plan_valid) {
    if (!ensure_host_state(w)) return false;
    plan_grid(w);
  }
  if (!ensure_range(w)) return false;
  if (!ensure_bodies(w)) return false;
  if (!w->keys_valid) {
    if (w->is_batch() && !upload_scene_table(w, 0.0f)) return false;  // the keys read each scene's grid
    enqueue_keys(w->d, w->n, w->plan, w->stream);
    w->keys_valid = true;
  }
  return cuda_ok(w, cudaGetLastError(), "prepare");
}

StepParams make_params_for(const FluidConfig2Ffi& c, float gx, float gy, bool mass_uniform, float mass_value,
                           bool phase_uniform, uint32_t phase_value, const GridPlan& plan, uint32_t body_first,
                           uint32_t nbodies, float dt) {
  StepParams P;
  std::memset(&P, 0, sizeof(P));
  P.grid = plan;
  const float hg = c.smoothing_length;
  P.hg2 = hg * hg;
  const float h = rmaxf(hg, kEps);  // substep's h (fluid.rs:908)
  P.hk = h;
  const float h2 = h * h;
  P.hk2 = h2;
  const float pi = 3.14159265358979323846f;  // std::f32::consts::PI
  P.c_poly6 = 4.0f / (pi * h2 * h2 * h2 * h2);
  P.c_spiky = -30.0f / (pi * h * h * h * h * h);
  P.rho_cap = 3.0f * rmaxf(c.rest_density, kEps);
  P.stiffness = c.stiffness;
  P.gamma = c.gamma;
  for (int k = 0; k < 4; k++) P.rest[k] = c.phase_rest_density[k];
  P.mass = mass_value;
  P.visc = c.viscosity;
  P.vmax = c.max_velocity;
  P.dt = dt;
  P.gx = gx;
  P.gy = gy;
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
  if (!mass_uniform) f |= F_MASS;
  if (!phase_uniform) f |= F_PHASE;
  if (!(P.hg2 <= P.hk2)) f |= F_WIDE_NB;
  P.flags = f;
  P.nbodies = nbodies;
  P.body_first = body_first;
  P.uniform_phase = phase_value;
  return P;
}

// The launch's copy of the wall pass's bounding-box reject (F_WBOX), for
// the P.nbodies bodies at `bodies` (the array the kernels read from
// P.body_first on): each box is the test's (px, py, ex + pr_pad, ey + pr_pad),
// summed in f32 as the device sums it; unused slots hold an extent of -1,
// which every finite position exceeds.
void set_wall_boxes(StepParams& P, const DevBody* bodies) {
  if (P.nbodies > kWallBoxes || (P.nbodies && !bodies)) return;
  for (uint32_t k = 0; k < kWallBoxes; k++)
    P.wbox[k] = k < P.nbodies ? make_float4(bodies[k].px, bodies[k].py, bodies[k].ex + P.pr_pad, bodies[k].ey + P.pr_pad)
                              : make_float4(0.0f, 0.0f, -1.0f, -1.0f);
  P.flags |= F_WBOX;
}

// Ambient turbulence of a single world (fluid.rs:1001-1002: on when enabled
// with a positive amplitude). The kernels read the step's clock from a device
// word (set_clock), so cached graphs stay valid as the clock advances.
void apply_ambient(const World2* w, StepParams& P) {
  const AmbientConfig2Ffi& a = w->ambient;
  P.wind_x = a.wind_x;  // read by the buoyancy drag whether or not drag is enabled (fluid.rs:1124)
  P.wind_y = a.wind_y;
  if (!(a.turbulence_enabled != 0 && a.turbulence_amplitude > 0.0f) || !w->d.scalar) return;
  P.flags |= F_TURB;
  if (a.turbulence_divergence_free) P.flags |= F_TURB_CURL;
  P.turb_amp = a.turbulence_amplitude;
  P.turb_freq = a.turbulence_frequency;
  P.turb_tscale = a.turbulence_time_scale;
  P.turb_seed = a.turbulence_seed;
  P.turb_oct = std::min<uint32_t>(std::max<uint32_t>(a.turbulence_octaves, 1u), 8u);  // (octaves as u32).clamp(1, 8)
  P.clock = reinterpret_cast<const float*>(w->d.scalar + kClockWord);
}

void apply_ghosts(const World2* w, StepParams& P);  // boundary ghosts, below

// The clock the next substeps' turbulence reads (the world time at the start
// of the step, fluid.rs:1009 with world.rs:848), in stream order.
void set_clock(World2* w, const StepParams& P, float t) {
  if (P.flags & F_TURB) {
    uint32_t bits;
    std::memcpy(&bits, &t, 4);
    enqueue_set_word(w->d.scalar + kClockWord, bits, w->stream);
  }
}

StepParams make_params(const World2* w, float dt) {
  if (!w->is_batch()) {
    StepParams P = make_params_for(w->cfg, w->gx, w->gy, w->mass_uniform, w->mass_value, w->phase_uniform,
                                   w->phase_value, w->plan, 0, (uint32_t)w->bodies.size(), dt);
    set_wall_boxes(P, w->bodies.data());
    apply_ambient(w, P);
    apply_ghosts(w, P);
    if (w->precision == PHIENG_SPH_TOLERANCE) P.flags |= F_FAST;
    return P;
  }
  // batch: the kernels read each scene's row of the device table; the launch
  // parameters carry the union of the per-particle array flags and the
  // global key range
  StepParams P = make_params_for(w->scenes[0].cfg, 0.0f, 0.0f, true, 0.0f, true, 0, w->plan, 0, 0, dt);
  for (const auto& sc : w->scenes) {
    if (!sc.mass_uniform) P.flags |= F_MASS;
    if (!sc.phase_uniform) P.flags |= F_PHASE;
    const float hg = sc.cfg.smoothing_length, hk = rmaxf(hg, kEps);
    if (!(hg * hg <= hk * hk)) P.flags |= F_WIDE_NB;
  }
  if (w->precision == PHIENG_SPH_TOLERANCE) {
    // the tolerance-mode kernels take a batch only if every scene has the
    // plain flag set (XSPH on; no artificial viscosity, cohesion, per-particle
    // mass or phase, h > 0): the launch's own flags are scene 0's
    bool all_plain = true;
    for (const auto& sc : w->scenes) {
      const uint32_t f = make_params_for(sc.cfg, sc.gx, sc.gy, sc.mass_uniform, sc.mass_value, sc.phase_uniform,
                                         sc.phase_value, sc.plan, sc.body_first, sc.nbodies, dt)
                             .flags;
      all_plain = all_plain && (f & F_VISC) && !(f & (F_AV | F_COHESION | F_WIDE_NB | F_MASS | F_PHASE));
    }
    if (all_plain) P.flags |= F_FAST;
  }
  return P;
}

// Per-scene parameter rows of a batch for substeps of length dt.
bool upload_scene_table(World2* w, float dt) {
  std::vector<StepParams> tab;
  tab.reserve(w->scenes.size());
  for (const auto& sc : w->scenes) {
    tab.push_back(make_params_for(sc.cfg, sc.gx, sc.gy, sc.mass_uniform, sc.mass_value, sc.phase_uniform,
                                  sc.phase_value, sc.plan, sc.body_first, sc.nbodies, dt));
    set_wall_boxes(tab.back(), w->bodies.data() + sc.body_first);
  }
  return cuda_ok(w, cudaMemcpyAsync(w->d_ptab, tab.data(), sizeof(StepParams) * tab.size(), cudaMemcpyHostToDevice,
                                    w->stream),
                 "upload scene table");
}

void enqueue_substep_body(World2* w, const StepParams& P, cudaStream_t st) {
  if (w->profiling) cudaEventRecordWithFlags(w->ev[0], st, cudaEventRecordExternal);
  enqueue_sort_and_ranges(w->d, w->n, P, w->sid_perm_n == w->n, st);
  if (w->profiling) cudaEventRecordWithFlags(w->ev[1], st, cudaEventRecordExternal);
  enqueue_density(w->d, w->n, P, st);
  enqueue_ghost_density(w->d, P, st);
  if (w->profiling) cudaEventRecordWithFlags(w->ev[2], st, cudaEventRecordExternal);
  enqueue_force_integrate(w->d, w->n, P, nullptr, st);
  if (w->profiling) cudaEventRecordWithFlags(w->ev[3], st, cudaEventRecordExternal);
}

// One substep, replayed from a cached CUDA graph while the launch
// parameters stay the same.
bool run_substep(World2* w, const StepParams& P) {
  // Buffer reallocations release the graph, so the parameters and the
  // particle count identify it.
  std::string sig((const char*)&P, sizeof(P));
  sig.append((const char*)&w->n, sizeof(w->n));
  sig.push_back(w->profiling ? 'p' : '-');
  sig.push_back(w->sid_perm_n == w->n ? 's' : '-');
  if (!w->gexec || sig != w->gsig) {
    release_graph(w);
    cudaGraph_t g = nullptr;
    if (!cuda_ok(w, cudaStreamBeginCapture(w->own_stream, cudaStreamCaptureModeThreadLocal), "begin capture"))
      return false;
    enqueue_substep_body(w, P, w->own_stream);
    cudaError_t r = cudaStreamEndCapture(w->own_stream, &g);
    if (!cuda_ok(w, r, "end capture")) return false;
    r = cudaGraphInstantiate(&w->gexec, g, 0);
    cudaGraphDestroy(g);
    if (!cuda_ok(w, r, "graph instantiate")) {
      w->gexec = nullptr;
      return false;
    }
    w->gsig = sig;
  }
  if (!cuda_ok(w, cudaGraphLaunch(w->gexec, w->stream), "graph launch")) return false;
  w->sid_perm_n = w->n;
  w->substeps++;
  w->host_state_valid = false;
  w->dp_on_device = true;
  w->keys_valid = true;
  return true;
}

// cfl_substeps (fluid.rs:562-588); vmax from the current state.
bool cfl_substeps(World2* w, float dt, uint32_t* out) {
  const FluidConfig2Ffi& c = w->cfg;
  uint32_t mx = std::max<uint32_t>(c.max_substeps, 1);
  *out = 1;
  if (c.cfl <= 0.0f || mx <= 1) return true;
  const float h = rmaxf(c.smoothing_length, kEps);
  const float rho0 = rmaxf(c.rest_density, kEps);
  const float c0 = (c.gamma == 1.0f) ? std::sqrt(rmaxf(c.stiffness, 0.0f))
                                     : std::sqrt(c.gamma * rmaxf(c.stiffness, 0.0f) * rho0);
  float vmax = 0.0f;
  if (w->host_state_valid) {
    for (uint32_t i = 0; i < w->n; i++) {
      float4 s = w->h_state[i];
      vmax = rmaxf(vmax, std::sqrt(s.z * s.z + s.w * s.w));
    }
  } else {
    enqueue_vmax(w->d, w->n, w->stream);
    if (!cuda_ok(w, cudaMemcpyAsync(w->h_pinned, w->d.scalar, 4, cudaMemcpyDeviceToHost, w->stream), "vmax"))
      return false;
    if (!cuda_ok(w, cudaStreamSynchronize(w->stream), "sync")) return false;
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

// Features the closure and feature passes do not take: adaptive resolution
// and boundary ghosts; the fluid phase takes ghosts (ghosts_ok), the world
// step both (world_ok).
bool unsupported(World2* w, bool ghosts_ok = false, bool world_ok = false) {
  if ((w->cfg.adaptive_resolution && !world_ok) || (w->cfg.boundary_particles && !ghosts_ok)) {
    set_error(w, PHIENG_SPH_E_UNSUPPORTED, "step");
    return true;
  }
  return false;
}

// ---- boundary ghosts (fluid.rs:617-818) ----
// A static body as the ghost generator reads it.
struct GhostSource {
  int shape;  // 0 circle, 1 box, 2 polygon
  float px, py, xax, xay, yax, yay, a, b;
  const float* verts = nullptr;  // polygon: local vertices (x, y pairs)
  uint32_t nverts = 0;
};

constexpr size_t kMaxGhosts = 1u << 22;

// f32 -> usize / i32 as Rust's `as` (truncate, saturate, NaN -> 0).
uint64_t as_usize(float v) {
  if (!(v > 0.0f)) return 0;
  if (v >= 1.8446744e19f) return UINT64_MAX;
  return (uint64_t)v;
}
int32_t as_i32(float v) {
  if (v != v) return 0;
  if (v <= -2147483648.0f) return INT32_MIN;
  if (v >= 2147483648.0f) return INT32_MAX;
  return (int32_t)v;
}

// refresh_boundaries (fluid.rs:665-741) at spacing max(h * 0.5, EPS): circles
// n = ceil(2 pi r / s) points at angles 2 pi k / n; boxes 4 edges (bottom,
// top, left, right) of ceil(2 extent / s) points at (k + 0.5) / n; polygons
// each edge of length >= EPS at (k + 0.5) / n; every point moved by the
// body's transform (rotation * local + position). false past kMaxGhosts.
bool generate_ghosts(const std::vector<GhostSource>& src, float hk, std::vector<float2>& out) {
  const float spacing = std::max(hk * 0.5f, kEps);
  const float pi = 3.14159265358979323846f;
  out.clear();
  auto push = [&](const GhostSource& b, float lx, float ly) {
    out.push_back(make_float2((b.xax * lx + b.yax * ly) + b.px, (b.xay * lx + b.yay * ly) + b.py));
  };
  for (const GhostSource& b : src) {
    if (b.shape == 0) {
      const uint64_t n = std::max<uint64_t>(as_usize(std::ceil((2.0f * pi * b.a) / spacing)), 1);
      if (n > kMaxGhosts || out.size() + n > kMaxGhosts) return false;
      for (uint64_t k = 0; k < n; k++) {
        const float ang = 2.0f * pi * (float)k / (float)n;
        push(b, std::cos(ang) * b.a, std::sin(ang) * b.a);
      }
    } else if (b.shape == 1) {
      const float hx = b.a, hy = b.b;
      // (origin, tangent) of the bottom, top, left and right edges
      const float edges[4][4] = {{-hx, -hy, 0.0f, 1.0f}, {-hx, hy, 0.0f, 1.0f}, {-hx, -hy, 1.0f, 0.0f},
                                 {hx, -hy, 1.0f, 0.0f}};
      for (const auto& e : edges) {
        const float extent = e[2] == 1.0f ? hx : hy;
        const uint64_t n = std::max<uint64_t>(as_usize(std::ceil((2.0f * extent) / spacing)), 1);
        if (n > kMaxGhosts || out.size() + n > kMaxGhosts) return false;
        for (uint64_t k = 0; k < n; k++) {
          const float t = ((float)k + 0.5f) / (float)n;
          const float sc = 2.0f * extent * t;
          push(b, e[0] + e[2] * sc, e[1] + e[3] * sc);
        }
      }
    } else {
      for (uint32_t e = 0; e < b.nverts; e++) {
        const uint32_t f = (e + 1) % b.nverts;
        const float ax = b.verts[2 * e], ay = b.verts[2 * e + 1];
        const float ex = b.verts[2 * f] - ax, ey = b.verts[2 * f + 1] - ay;
        const float len = std::sqrt(ex * ex + ey * ey);
        if (len < kEps) continue;
        const uint64_t n = std::max<uint64_t>(as_usize(std::ceil(len / spacing)), 1);
        if (n > kMaxGhosts || out.size() + n > kMaxGhosts) return false;
        for (uint64_t k = 0; k < n; k++) {
          const float t = ((float)k + 0.5f) / (float)n;
          push(b, ax + ex * t, ay + ey * t);
        }
      }
    }
  }
  return true;
}

// Make the device ghosts current for these static bodies (regenerated when
// the inputs of boundary_fingerprint change, fluid.rs:614-660, 929-936):
// positions grouped by cell (floor(p / hk), rebuild_boundary_grid,
// fluid.rs:744-756; generation order within a cell; non-finite ghosts are in
// no cell and are dropped), and the open-addressing cell table.
bool refresh_ghosts(World2* w, const std::vector<GhostSource>& src) {
  const FluidConfig2Ffi& c = w->cfg;
  std::string sig;
  auto add = [&](const void* p, size_t n) { sig.append((const char*)p, n); };
  add(&c.smoothing_length, 4);
  add(&c.particle_mass, 4);
  add(&c.rest_density, 4);
  for (const GhostSource& b : src) {
    add(&b.shape, 4);
    add(&b.px, 4 * 8);
    add(&b.nverts, 4);
    if (b.nverts) add(b.verts, 8 * (size_t)b.nverts);
  }
  if (sig == w->ghost_sig && w->d_gtab) return true;
  const float hk = std::max(c.smoothing_length, kEps);
  std::vector<float2> raw;
  if (!generate_ghosts(src, hk, raw)) {
    set_error(w, PHIENG_SPH_E_ARG, "too many boundary ghosts");
    return false;
  }
  // group by cell, keeping generation order inside each cell
  std::vector<std::pair<int64_t, uint32_t>> order;  // (cell key, generation index)
  std::vector<std::pair<int32_t, int32_t>> cell_of(raw.size());
  for (uint32_t i = 0; i < raw.size(); i++) {
    const float2 g = raw[i];
    if (!std::isfinite(g.x) || !std::isfinite(g.y)) continue;
    const int32_t cx = as_i32(std::floor(g.x / hk)), cy = as_i32(std::floor(g.y / hk));
    cell_of[i] = {cx, cy};
    order.push_back({((int64_t)cx << 32) | (uint32_t)cy, i});
  }
  std::stable_sort(order.begin(), order.end(),
                   [](const std::pair<int64_t, uint32_t>& x, const std::pair<int64_t, uint32_t>& y) {
                     return x.first < y.first;
                   });
  std::vector<float2> gpos(order.size());
  std::vector<GhostCell> cells;
  for (size_t k = 0; k < order.size(); k++) {
    gpos[k] = raw[order[k].second];
    const auto cc = cell_of[order[k].second];
    if (cells.empty() || cells.back().cx != cc.first || cells.back().cy != cc.second)
      cells.push_back({cc.first, cc.second, (uint32_t)k, 0});
    cells.back().count++;
  }
  uint32_t tsize = 16;
  while (tsize < 2 * cells.size()) tsize <<= 1;
  std::vector<GhostCell> tab(tsize, GhostCell{0, 0, 0, 0});
  for (const GhostCell& gc : cells) {
    uint32_t slot = ghost_cell_hash(gc.cx, gc.cy, tsize - 1);
    while (tab[slot].count != 0) slot = (slot + 1) & (tsize - 1);
    tab[slot] = gc;
  }
  const uint32_t ng = (uint32_t)gpos.size();
  if (ng > w->ghost_cap) {
    cudaStreamSynchronize(w->stream);
    dfree(w->d_gpos), dfree(w->d_gq);
    if (!dalloc(w, w->d_gpos, std::max<uint32_t>(ng, 64)) || !dalloc(w, w->d_gq, std::max<uint32_t>(ng, 64)))
      return false;
    w->ghost_cap = std::max<uint32_t>(ng, 64);
  }
  if (tsize > w->gtab_cap) {
    cudaStreamSynchronize(w->stream);
    dfree(w->d_gtab);
    if (!dalloc(w, w->d_gtab, tsize)) return false;
    w->gtab_cap = tsize;
  }
  if ((ng && !cuda_ok(w, cudaMemcpyAsync(w->d_gpos, gpos.data(), sizeof(float2) * ng, cudaMemcpyHostToDevice,
                                          w->stream), "upload ghosts")) ||
      !cuda_ok(w, cudaMemcpyAsync(w->d_gtab, tab.data(), sizeof(GhostCell) * tsize, cudaMemcpyHostToDevice, w->stream),
               "upload ghost cells") ||
      !cuda_ok(w, cudaStreamSynchronize(w->stream), "sync"))  // the host vectors go out of scope
    return false;
  w->nghost = ng;
  w->gtab_mask = tsize - 1;
  w->ghost_sig = sig;
  w->h_gpos = std::move(gpos);
  w->ghost_regens++;
  return true;
}

// The world's static bodies as ghost sources (all of them are static).
std::vector<GhostSource> world_ghost_sources(const World2* w) {
  std::vector<GhostSource> v;
  for (const DevBody& b : w->bodies) {
    GhostSource g;
    g.shape = b.shape;
    g.px = b.px, g.py = b.py, g.xax = b.xax, g.xay = b.xay, g.yax = b.yax, g.yay = b.yay, g.a = b.a, g.b = b.b;
    v.push_back(g);
  }
  return v;
}

void apply_ghosts(const World2* w, StepParams& P) {
  if (!w->cfg.boundary_particles || w->nghost == 0 || !w->d_gtab) return;
  P.flags |= F_GHOST;
  P.gpos = w->d_gpos;
  P.gq = w->d_gq;
  P.gtab = w->d_gtab;
  P.gtab_mask = w->gtab_mask;
  P.nghost = w->nghost;
  P.gmass = std::max(w->cfg.particle_mass, kEps);
  P.rest0 = w->cfg.rest_density;
}

void recompute_uniformity(World2* w);

// One substep with adaptive resolution (fluid.rs:909-920): sort and density,
// resample, then the new particle set's sort and density and the rest of the
// substep. The count changes mid-substep, so it runs as plain launches with
// one read of the new count; the host mirrors of mass and phase follow the
// device, and the uniform-mass shortcut ends once masses differ.
bool ensure_resample_buffers(World2* w) {
  const uint32_t c = w->d.cap;
  if (w->rs_cap >= c && w->rs.state) return true;
  ResampleBufs& r = w->rs;
  cudaStreamSynchronize(w->stream);
  dfree(r.slot_of), dfree(r.absorbed), dfree(r.state), dfree(r.mass), dfree(r.phase);
  if (!dalloc(w, r.slot_of, c) || !dalloc(w, r.absorbed, c) || !dalloc(w, r.state, c) || !dalloc(w, r.mass, c) ||
      !dalloc(w, r.phase, c))
    return false;
  r.n_out = w->d.scalar + 18;
  r.cap = c;
  w->rs_cap = c;
  return true;
}

bool run_substep_adaptive(World2* w, float dt) {
  if (w->d.cap < resample_bound(w->n)) {
    // an earlier CFL substep of this step grew the set: bring the state home
    // and upload it into buffers with room for this pass's output
    if (!ensure_host_state(w)) return false;
    w->dev_state_valid = false;
    if (!prepare(w)) return false;
  }
  if (!ensure_resample_buffers(w)) return false;
  cudaStream_t st = w->stream;
  StepParams P = make_params(w, dt);
  enqueue_sort_and_ranges(w->d, w->n, P, w->sid_perm_n == w->n, st);
  w->sid_perm_n = w->n;
  enqueue_density(w->d, w->n, P, st);
  const FluidConfig2Ffi& c = w->cfg;
  const float rest = std::max(c.rest_density, kEps);
  enqueue_resample(w->d, w->n, P, w->rs, c.merge_density_ratio * rest, c.split_density_ratio * rest,
                   std::max(c.particle_mass, kEps) * 0.125f, w->mass_uniform, w->phase_uniform, st);
  if (!cuda_ok(w, cudaMemcpyAsync(w->h_pinned, w->rs.n_out, 4, cudaMemcpyDeviceToHost, st), "resample count") ||
      !cuda_ok(w, cudaStreamSynchronize(st), "sync"))
    return false;
  uint32_t n2;
  std::memcpy(&n2, w->h_pinned, 4);
  if (n2 > w->d.cap) {  // the kernel stopped at the buffer's end (cannot happen with resample_bound)
    set_error(w, PHIENG_SPH_E_CUDA, "resample output exceeds the particle buffers");
    return false;
  }
  w->h_state.resize(n2);
  w->h_mass.resize(n2);
  w->h_phase.resize(n2);
  w->h_dens.resize(n2);
  w->h_pres.resize(n2);
  if (n2 &&
      (!cuda_ok(w, cudaMemcpyAsync(w->d.state, w->rs.state, sizeof(float4) * n2, cudaMemcpyDeviceToDevice, st),
                "resample state") ||
       !cuda_ok(w, cudaMemcpyAsync(w->d.mass, w->rs.mass, sizeof(float) * n2, cudaMemcpyDeviceToDevice, st),
                "resample mass") ||
       !cuda_ok(w, cudaMemcpyAsync(w->d.phase, w->rs.phase, n2, cudaMemcpyDeviceToDevice, st), "resample phase") ||
       !cuda_ok(w, cudaMemcpyAsync(w->h_mass.data(), w->rs.mass, sizeof(float) * n2, cudaMemcpyDeviceToHost, st),
                "resample mass down") ||
       !cuda_ok(w, cudaMemcpyAsync(w->h_phase.data(), w->rs.phase, n2, cudaMemcpyDeviceToHost, st),
                "resample phase down") ||
       !cuda_ok(w, cudaStreamSynchronize(st), "sync")))
    return false;
  w->n = n2;
  recompute_uniformity(w);
  w->dev_aux_valid = true;
  w->host_state_valid = false;
  w->bbox_valid = false;
  // the second density pass on the resampled set, then the rest
  P = make_params(w, dt);
  enqueue_keys(w->d, w->n, w->plan, st);
  enqueue_sort_and_ranges(w->d, w->n, P, false, st);
  w->sid_perm_n = w->n;
  enqueue_density(w->d, w->n, P, st);
  enqueue_ghost_density(w->d, P, st);
  enqueue_force_integrate(w->d, w->n, P, nullptr, st);
  if (!cuda_ok(w, cudaGetLastError(), "adaptive substep")) return false;
  w->substeps++;
  w->dp_on_device = true;
  w->keys_valid = true;
  return true;
}

// World2::step (world.rs:706-732) restricted to the fluid phase (1b).
bool world_step(World2* w, float dt) {
  if (w->is_batch()) {
    // every scene advances one substep of dt (batches take no CFL substeps)
    if (w->n > 0 && dt > 0.0f) {
      if (!prepare(w)) return false;
      if (!upload_scene_table(w, dt)) return false;
      if (!run_substep(w, make_params(w, dt))) return false;
    }
    w->time += dt;
    return true;
  }
  if (w->cfg.enabled && w->n > 0 && dt > 0.0f) {  // step_fluid guards (fluid.rs:550-552)
    if (unsupported(w, true, true)) return false;
    if (w->cfg.adaptive_resolution && w->d.state && w->d.cap < std::max(resample_bound(w->n), kMaxParticles2D)) {
      // room for the splits: bring the state home and upload it into larger buffers
      if (!ensure_host_state(w)) return false;
      w->dev_state_valid = false;
    }
    if (!prepare(w)) return false;
    if (w->cfg.boundary_particles && !refresh_ghosts(w, world_ghost_sources(w))) return false;
    uint32_t ns = 1;
    if (!cfl_substeps(w, dt, &ns)) return false;
    const float sub = dt / (float)ns;
    const StepParams P = make_params(w, sub);
    set_clock(w, P, w->time);  // every CFL substep sees the step's start time
    for (uint32_t k = 0; k < ns; k++)
      if (!(w->cfg.adaptive_resolution ? run_substep_adaptive(w, sub) : run_substep(w, P))) return false;
  }
  w->time += dt;
  return true;
}


// ---------------------------------------------------------------- bodies that react
// FluidState2::step_fluid (fluid.rs:541-557) with the caller's bodies: the
// fluid phase of World2::step_inner (world.rs:843-849), where the engine
// passes its rigid bodies and keeps the updated velocities.
constexpr uint32_t kMaxCallBodies = 65536;

bool ensure_dyn_buffers(World2* w, uint32_t nb, uint32_t ns) {
  DynBufs& y = w->dynb;
  if (nb > w->cbody_cap) {
    cudaStreamSynchronize(w->stream);
    dfree(w->d_cbodies), dfree(y.dyn), dfree(y.buoy);
    const uint32_t c = std::max<uint32_t>(16, nb);
    if (!dalloc(w, w->d_cbodies, c) || !dalloc(w, y.dyn, c) || !dalloc(w, y.buoy, c)) return false;
    w->cbody_cap = c;
  }
  if (ns > w->sample_cap) {
    cudaStreamSynchronize(w->stream);
    dfree(y.samples), dfree(y.areas);
    const uint32_t c = std::max<uint32_t>(64, ns);
    if (!dalloc(w, y.samples, c) || !dalloc(w, y.areas, c)) return false;
    w->sample_cap = c;
  }
  if (w->n > w->dyn_pcap || !w->d.defer) {
    cudaStreamSynchronize(w->stream);
    dfree(w->d.defer), dfree(w->d.dcount), dfree(y.dstart), dfree(y.dtile), dfree(y.list), dfree(y.dq_id),
        dfree(y.p_id);
    const uint32_t c = std::max<uint32_t>(1024, w->n);
    const uint32_t tiles = (c + 1 + kBucketScanTile - 1) / kBucketScanTile;
    const size_t len = (size_t)tiles * kBucketScanTile;
    if (!dalloc(w, w->d.defer, c) || !dalloc(w, w->d.dcount, len) || !dalloc(w, y.dstart, len + 1) ||
        !dalloc(w, y.dtile, tiles) || !dalloc(w, y.list, c) || !dalloc(w, y.dq_id, c) || !dalloc(w, y.p_id, c))
      return false;
    w->dyn_pcap = c;
  }
  if (w->d.count_len > w->count2_cap) {
    cudaStreamSynchronize(w->stream);
    dfree(y.count2);
    if (!dalloc(w, y.count2, w->d.count_len)) return false;
    w->count2_cap = w->d.count_len;
  }
  y.dcount = w->d.dcount;
  y.done = w->d.scalar + 10;
  return true;
}

// Surface samples of a dynamic body for buoyancy (fluid.rs:417-458): circles
// 12 perimeter points, boxes 4 per edge; (point, outward normal) in world
// axes and the sample's area. The angles' cosines and sines come from the C
// library, as f32::cos / f32::sin do.
void surface_samples(const PhiengBody2& b, std::vector<float4>& pts, std::vector<float>& areas) {
  if (b.shape_tag == PHIENG_SHAPE_POLYGON) return;  // impulse-coupled only (fluid.rs:415-418)
  const float pi = 3.14159265358979323846f;
  auto rot = [&](float x, float y, float& ox, float& oy) {  // glam Mat2 * Vec2
    ox = b.xax * x + b.yax * y;
    oy = b.xay * x + b.yay * y;
  };
  if (b.shape_tag == PHIENG_SHAPE_CIRCLE) {
    const int n = 12;
    const float r = b.a;
    const float area = 2.0f * pi * r / (float)n;
    for (int k = 0; k < n; k++) {
      const float a = 2.0f * pi * (float)k / (float)n;
      const float c = std::cos(a), sn = std::sin(a);
      float qx, qy, nx, ny;
      rot(c * r, sn * r, qx, qy);
      rot(c, sn, nx, ny);
      pts.push_back(make_float4(qx + b.px, qy + b.py, nx, ny));
      areas.push_back(area);
    }
  } else if (b.shape_tag == PHIENG_SHAPE_BOX) {
    const float hx = b.a, hy = b.b;
    const float perimeter = 4.0f * (hx + hy);
    const float area = perimeter / 16.0f;
    struct Edge {
      float nx, ny, ox, oy;
      bool along_x;
    };
    const Edge edges[4] = {{0.0f, -1.0f, -hx, -hy, true},
                           {0.0f, 1.0f, -hx, hy, true},
                           {-1.0f, 0.0f, -hx, -hy, false},
                           {1.0f, 0.0f, hx, -hy, false}};
    for (const Edge& e : edges) {
      for (int k = 0; k < 4; k++) {
        const float t = ((float)k + 0.5f) / 4.0f;
        const float extent = e.along_x ? hx : hy;
        const float sc = 2.0f * extent * t;
        const float tx = e.along_x ? 1.0f : 0.0f, ty = e.along_x ? 0.0f : 1.0f;  // Vec2::X / Vec2::Y
        const float lx = e.ox + tx * sc, ly = e.oy + ty * sc;
        float qx, qy, nx, ny;
        rot(lx, ly, qx, qy);
        rot(e.nx, e.ny, nx, ny);
        pts.push_back(make_float4(qx + b.px, qy + b.py, nx, ny));
        areas.push_back(area);
      }
    }
  }
}

bool body_valid(const PhiengBody2& b) {
  if (b.shape_tag != PHIENG_SHAPE_CIRCLE && b.shape_tag != PHIENG_SHAPE_BOX) return false;
  const float v[] = {b.a, b.b, b.px, b.py, b.xax, b.xay, b.yax, b.yay, b.vx, b.vy, b.w, b.inv_mass, b.inv_inertia};
  for (float x : v)
    if (!std::isfinite(x)) return false;
  return b.a > 0.0f && (b.shape_tag == PHIENG_SHAPE_CIRCLE || b.b > 0.0f);
}

DevBody dev_body(const PhiengBody2& b) {
  DevBody d;
  std::memset(&d, 0, sizeof(d));
  d.shape = b.shape_tag == PHIENG_SHAPE_CIRCLE ? 0 : 1;
  d.px = b.px;
  d.py = b.py;
  d.xax = b.xax;
  d.xay = b.xay;
  d.yax = b.yax;
  d.yay = b.yay;
  d.a = b.a;
  d.b = b.b;
  if (d.shape == 0) {
    d.ex = d.ey = b.a * 1.001f + 1e-30f;
  } else {
    // the box test maps rel to x_axis.x*rel.x + y_axis.x*rel.y, ... (fluid.rs:483-489),
    // i.e. the box sits at R^T: both candidate extents for a rotation, none
    // for a matrix that is not one
    const float det = b.xax * b.yay - b.yax * b.xay;
    const float c0 = b.xax * b.xax + b.xay * b.xay, c1 = b.yax * b.yax + b.yay * b.yay;
    if (std::fabs(det - 1.0f) > 1e-3f || std::fabs(c0 - 1.0f) > 1e-3f || std::fabs(c1 - 1.0f) > 1e-3f) {
      d.ex = d.ey = INFINITY;
    } else {
      const float ax = std::fabs(b.xax), ay = std::fabs(b.xay), bx = std::fabs(b.yax), by = std::fabs(b.yay);
      d.ex = std::max(ax * b.a + bx * b.b, ax * b.a + ay * b.b) * 1.001f + 1e-30f;
      d.ey = std::max(ay * b.a + by * b.b, bx * b.a + by * b.b) * 1.001f + 1e-30f;
    }
  }
  d.dyn = (!b.is_static || b.vx != 0.0f || b.vy != 0.0f) ? 1u : 0u;
  return d;
}

// Polygon vertices of one call (validated by the caller): local vertices
// moved by each polygon body's transform (Transform2::transform_point,
// math.rs:58-60: rotation * v + position, glam Mat2 * Vec2 = x_axis * v.x +
// y_axis * v.y), as fluid.rs:519-523 builds poly_scratch for every test.
struct PolyIn {
  const float* xy = nullptr;
  const uint32_t* first = nullptr;
  const uint32_t* count = nullptr;
};

bool step_fluid_bodies(World2* w, PhiengBody2* bodies, uint32_t nb, float dt, const PolyIn& pin = PolyIn()) {
  if (!w->cfg.enabled || w->n == 0 || dt <= 0.0f) return true;  // step_fluid guards (fluid.rs:550-552)
  if (unsupported(w, true)) return false;
  if (!prepare(w)) return false;
  if (w->cfg.boundary_particles) {  // ghosts of the call's static bodies (fluid.rs:929-936)
    std::vector<GhostSource> src;
    for (uint32_t k = 0; k < nb; k++) {
      const PhiengBody2& b = bodies[k];
      if (!b.is_static) continue;
      GhostSource g;
      g.shape = b.shape_tag == PHIENG_SHAPE_CIRCLE ? 0 : b.shape_tag == PHIENG_SHAPE_POLYGON ? 2 : 1;
      g.px = b.px, g.py = b.py, g.xax = b.xax, g.xay = b.xay, g.yax = b.yax, g.yay = b.yay, g.a = b.a, g.b = b.b;
      if (g.shape == 2) {
        g.verts = pin.xy + 2 * (size_t)pin.first[k];
        g.nverts = pin.count[k];
      }
      src.push_back(g);
    }
    if (!refresh_ghosts(w, src)) return false;
  }
  std::vector<float2> wv;  // world-space polygon vertices
  std::vector<DevBody> db(nb);
  std::vector<DynBody> dy(nb);
  std::vector<float4> pts;
  std::vector<float> areas;
  std::vector<uint32_t> buoy;
  bool any_dyn = false;
  for (uint32_t k = 0; k < nb; k++) {
    const PhiengBody2& b = bodies[k];
    db[k] = dev_body(b);
    if (b.shape_tag == PHIENG_SHAPE_POLYGON) {
      DevBody& d = db[k];
      d.shape = 2;
      d.vfirst = (uint32_t)wv.size();
      d.vcount = pin.count[k];
      float sx = 0.0f, sy = 0.0f;  // polygon_centroid (sat.rs:77-83): fold from zero, then / len
      for (uint32_t i = 0; i < pin.count[k]; i++) {
        const float lx = pin.xy[2 * ((size_t)pin.first[k] + i)], ly = pin.xy[2 * ((size_t)pin.first[k] + i) + 1];
        const float2 v = make_float2((b.xax * lx + b.yax * ly) + b.px, (b.xay * lx + b.yay * ly) + b.py);
        wv.push_back(v);
        sx = sx + v.x;
        sy = sy + v.y;
      }
      d.a = sx / (float)pin.count[k];
      d.b = sy / (float)pin.count[k];
      d.ex = d.ey = INFINITY;  // no bounding-box reject for polygons
    }
    any_dyn = any_dyn || db[k].dyn;
    DynBody& d = dy[k];
    d.vx = b.vx;
    d.vy = b.vy;
    d.w = b.w;
    d.inv_mass = b.inv_mass;
    d.inv_inertia = b.inv_inertia;
    d.is_static = b.is_static ? 1u : 0u;
    d.sleeping = b.is_sleeping ? 1u : 0u;
    d.sample_first = (uint32_t)pts.size();
    if (!b.is_static) surface_samples(b, pts, areas);
    d.sample_count = (uint32_t)pts.size() - d.sample_first;
    if (d.sample_count) buoy.push_back(k);
  }
  if (!ensure_dyn_buffers(w, nb, (uint32_t)pts.size())) return false;
  if (wv.size() > w->poly_cap) {
    cudaStreamSynchronize(w->stream);
    dfree(w->d_poly);
    const uint32_t c = std::max<uint32_t>(64, (uint32_t)wv.size());
    if (!dalloc(w, w->d_poly, c)) return false;
    w->poly_cap = c;
  }
  if (!wv.empty() && !cuda_ok(w, cudaMemcpyAsync(w->d_poly, wv.data(), sizeof(float2) * wv.size(),
                                                  cudaMemcpyHostToDevice, w->stream),
                              "upload polygon vertices"))
    return false;
  DynBufs y = w->dynb;
  y.nbuoy = (uint32_t)buoy.size();
  cudaStream_t st = w->stream;
  if (nb && (!cuda_ok(w, cudaMemcpyAsync(w->d_cbodies, db.data(), sizeof(DevBody) * nb, cudaMemcpyHostToDevice, st),
                      "upload bodies") ||
             !cuda_ok(w, cudaMemcpyAsync(y.dyn, dy.data(), sizeof(DynBody) * nb, cudaMemcpyHostToDevice, st),
                      "upload body state") ||
             !cuda_ok(w, cudaMemcpyAsync(y.buoy, buoy.data(), 4 * buoy.size(), cudaMemcpyHostToDevice, st),
                      "upload body list")))
    return false;
  if (!pts.empty() &&
      (!cuda_ok(w, cudaMemcpyAsync(y.samples, pts.data(), sizeof(float4) * pts.size(), cudaMemcpyHostToDevice, st),
                "upload samples") ||
       !cuda_ok(w, cudaMemcpyAsync(y.areas, areas.data(), 4 * areas.size(), cudaMemcpyHostToDevice, st),
                "upload sample areas")))
    return false;
  uint32_t ns = 1;
  if (!cfl_substeps(w, dt, &ns)) return false;
  const float sub = dt / (float)ns;
  StepParams P = make_params_for(w->cfg, w->gx, w->gy, w->mass_uniform, w->mass_value, w->phase_uniform,
                                 w->phase_value, w->plan, 0, nb, sub);
  set_wall_boxes(P, db.data());
  if (any_dyn) P.flags |= F_DYNAMIC;
  if (!wv.empty()) P.flags |= F_POLY;
  P.poly = w->d_poly;
  apply_ambient(w, P);
  apply_ghosts(w, P);
  set_clock(w, P, w->time);
  FluidBufs dB = w->d;
  dB.bodies = w->d_cbodies;
  const float drag = rmaxf(w->cfg.drag, 0.0f);
  const size_t dlen = (size_t)((w->n + 1 + kBucketScanTile - 1) / kBucketScanTile) * kBucketScanTile;
  for (uint32_t k = 0; k < ns; k++) {
    enqueue_sort_and_ranges(dB, w->n, P, w->sid_perm_n == w->n, st);
    w->sid_perm_n = w->n;
    enqueue_density(dB, w->n, P, st);
    enqueue_ghost_density(dB, P, st);
    if (any_dyn) cudaMemsetAsync(dB.dcount, 0, sizeof(uint32_t) * dlen, st);
    enqueue_force_integrate(dB, w->n, P, nullptr, st);
    if (any_dyn) enqueue_dynamic_walls(dB, y, w->n, P, st);
    if (y.nbuoy) enqueue_buoyancy(dB, y, w->n, P, drag, sub, st);
    w->substeps++;
  }
  if (!cuda_ok(w, cudaGetLastError(), "step_fluid")) return false;
  w->host_state_valid = false;
  w->dp_on_device = true;
  w->keys_valid = true;
  if (nb) {
    if (!cuda_ok(w, cudaMemcpyAsync(dy.data(), y.dyn, sizeof(DynBody) * nb, cudaMemcpyDeviceToHost, st),
                 "download body state") ||
        !cuda_ok(w, cudaStreamSynchronize(st), "sync"))
      return false;
    for (uint32_t k = 0; k < nb; k++) {
      bodies[k].vx = dy[k].vx;
      bodies[k].vy = dy[k].vy;
      bodies[k].w = dy[k].w;
      bodies[k].is_sleeping = dy[k].sleeping ? 1 : 0;
    }
  }
  return true;
}

// ---------------------------------------------------------------- learned closure
bool ensure_closure_buffers(World2* w) {
  if (w->closure_cap >= w->d.cap && w->d_save) return true;
  dfree(w->d_save);
  dfree(w->d_rho_prev);
  dfree(w->d_block_save);
  dfree(w->d_svp);
  w->closure_cap = 0;
  if (!dalloc(w, w->d_save, w->d.cap) || !dalloc(w, w->d_rho_prev, w->d.cap) ||
      !dalloc(w, w->d_block_save, w->d.cap) || !dalloc(w, w->d_svp, w->d.cap))
    return false;
  w->closure_cap = w->d.cap;
  release_graph(w);
  return true;
}

// Sort + density of the current state with parameters P (the state and its
// keys / bucket counts are current). Leaves the counts consumed. svp: also
// the closure factors (closure passes).
void enqueue_sort_density(World2* w, const StepParams& P, float2* svp = nullptr) {
  enqueue_sort_and_ranges(w->d, w->n, P, w->sid_perm_n == w->n, w->stream);
  enqueue_density(w->d, w->n, P, w->stream, svp);
  w->sid_perm_n = w->n;
  w->dp_on_device = true;
}

// One coarse step from a sorted state with its density: closure force pass,
// then sort + density of the new state and the density check into
// scalar[4]; replayed from a cached graph.
bool run_coarse(World2* w, const StepParams& P, const MlpDev& mlp, const ClosureIO& io) {
  std::string sig((const char*)&P, sizeof(P));
  sig.append((const char*)&w->n, sizeof(w->n));
  sig.append((const char*)&mlp, sizeof(mlp));
  sig.append((const char*)&io, sizeof(io));
  if (!w->cexec || sig != w->csig) {
    if (w->cexec) cudaGraphExecDestroy(w->cexec);
    w->cexec = nullptr;
    cudaGraph_t g = nullptr;
    if (!cuda_ok(w, cudaStreamBeginCapture(w->own_stream, cudaStreamCaptureModeThreadLocal), "begin capture"))
      return false;
    enqueue_closure_force(w->d, w->n, P, mlp, io, w->own_stream);
    enqueue_sort_and_ranges(w->d, w->n, P, true, w->own_stream);
    enqueue_density(w->d, w->n, P, w->own_stream, w->d_svp);
    enqueue_closure_check(w->d, w->n, P, io.rho_prev, w->d.scalar + 4, w->own_stream);
    cudaError_t r = cudaStreamEndCapture(w->own_stream, &g);
    if (!cuda_ok(w, r, "end capture")) return false;
    r = cudaGraphInstantiate(&w->cexec, g, 0);
    cudaGraphDestroy(g);
    if (!cuda_ok(w, r, "graph instantiate")) {
      w->cexec = nullptr;
      return false;
    }
    w->csig = sig;
  }
  return cuda_ok(w, cudaGraphLaunch(w->cexec, w->stream), "graph launch");
}

void recompute_uniformity(World2* w) {
  w->mass_uniform = true;
  w->phase_uniform = true;
  if (w->n == 0) {
    w->mass_value = 0.0f;
    w->phase_value = 0;
    return;
  }
  uint32_t m0;
  std::memcpy(&m0, &w->h_mass[0], 4);
  w->mass_value = w->h_mass[0];
  w->phase_value = std::min<uint32_t>(w->h_phase[0], 3);
  for (uint32_t i = 1; i < w->n; i++) {
    uint32_t mi;
    std::memcpy(&mi, &w->h_mass[i], 4);
    if (mi != m0) w->mass_uniform = false;
    if (std::min<uint32_t>(w->h_phase[i], 3) != w->phase_value) w->phase_uniform = false;
  }
}

// add_particles_phase (fluid.rs:241-257) behind the FFI checks (ffi.rs:2486-2539).
uint32_t add_particles(World2* w, const float* xy, const uint8_t* phases, uint32_t count) {
  uint32_t n = std::min(count, kMaxAddPerCall);
  for (uint64_t i = 0; i < 2ull * n; i++)
    if (!std::isfinite(xy[i])) return 0;
  uint32_t room = w->cap > w->n ? w->cap - w->n : 0;
  n = std::min(n, room);
  if (n == 0) return 0;
  if (!ensure_host_state(w) || !ensure_host_dp(w)) return 0;
  for (uint32_t i = 0; i < n; i++) {
    uint8_t ph = phases ? phases[i] : 0;
    uint32_t k = std::min<uint32_t>(ph, 3);
    w->h_state.push_back(make_float4(xy[2 * i], xy[2 * i + 1], 0.0f, 0.0f));
    w->bx0 = std::min(w->bx0, xy[2 * i]);
    w->bx1 = std::max(w->bx1, xy[2 * i]);
    w->by0 = std::min(w->by0, xy[2 * i + 1]);
    w->by1 = std::max(w->by1, xy[2 * i + 1]);
    w->h_dens.push_back(w->cfg.phase_rest_density[k]);
    w->h_pres.push_back(0.0f);
    w->h_mass.push_back(rmaxf(w->cfg.phase_mass[k], 0.0f));
    w->h_phase.push_back(ph);
  }
  w->n += n;
  recompute_uniformity(w);
  w->dev_state_valid = false;
  w->dev_aux_valid = false;
  if (!w->plan_locked) w->plan_valid = false;
  w->keys_valid = false;
  return n;
}

}  // namespace

// =====================================================================
// C ABI
// =====================================================================
extern "C" {

World2* phieng_world_new(void) { return new (std::nothrow) World2(); }

void phieng_world_free(World2* w) {
  if (!w) return;
  if (w->device >= 0) {
    cudaStreamSynchronize(w->stream);
    release_graph(w);
    free_particle_buffers(w->d);
    dfree(w->d.bodies);
    dfree(w->d.scalar);
    dfree(w->d.count);
    dfree(w->d.start);
    dfree(w->d.tilesum);
    dfree(w->d.tstate);
    dfree(w->d_tmp);
    dfree(w->d_slab);
    dfree(w->d_pscene);
    dfree(w->d_sscene);
    dfree(w->d_ptab);
    dfree(w->d_save);
    dfree(w->d_rho_prev);
    dfree(w->d_block_save);
    dfree(w->d_svp);
    dfree(w->d_cbodies);
    dfree(w->d_poly);
    dfree(w->d_gpos);
    dfree(w->d_gq);
    dfree(w->d_gtab);
    dfree(w->rs.slot_of), dfree(w->rs.absorbed), dfree(w->rs.state), dfree(w->rs.mass), dfree(w->rs.phase);
    dfree(w->dynb.dyn);
    dfree(w->dynb.samples);
    dfree(w->dynb.areas);
    dfree(w->dynb.buoy);
    dfree(w->d.defer);
    dfree(w->d.dcount);
    dfree(w->dynb.dstart);
    dfree(w->dynb.dtile);
    dfree(w->dynb.list);
    dfree(w->dynb.dq_id);
    dfree(w->dynb.p_id);
    dfree(w->dynb.count2);
    if (w->cexec) cudaGraphExecDestroy(w->cexec);
    for (auto& e : w->ev)
      if (e) cudaEventDestroy(e);
    if (w->h_pinned) cudaFreeHost(w->h_pinned);
    if (w->own_stream) cudaStreamDestroy(w->own_stream);
  }
  delete w;
}

void phieng_world_step(World2* w, float dt) {
  if (!w || !std::isfinite(dt) || dt <= 0.0f) return;
  world_step(w, std::min(dt, kMaxDt));
}

void phieng_world_set_gravity(World2* w, float gx, float gy) {
  if (!w || w->is_batch() || !std::isfinite(gx) || !std::isfinite(gy)) return;
  w->gx = gx;
  w->gy = gy;
}

int32_t phieng_world_set_time(World2* w, float t) {
  if (!w || !std::isfinite(t)) return 0;
  w->time = t;
  return 1;
}

int32_t phieng_world_get_time(World2* w, float* out) {
  if (!w || !out) return 0;
  *out = w->time;
  return 1;
}

int32_t phieng_world_set_ambient_config(World2* w, const AmbientConfig2Ffi* cfg) {
  if (!w || !cfg) return 0;
  const AmbientConfig2Ffi& c = *cfg;
  // ambient2_from_ffi (ffi.rs:328-386): finite floats, non-negative
  // coefficients, octaves stored as min(v, 255)
  for (float v : {c.spring_ax, c.spring_ay, c.spring_stiffness, c.spring_damping, c.spring_max_displacement,
                  c.drag_linear, c.drag_quadratic, c.air_density, c.drag_angular, c.wind_x, c.wind_y,
                  c.turbulence_amplitude, c.turbulence_frequency, c.turbulence_time_scale})
    if (!std::isfinite(v)) return 0;
  if (c.spring_stiffness < 0.0f || c.spring_damping < 0.0f || c.spring_max_displacement < 0.0f ||
      c.drag_linear < 0.0f || c.drag_quadratic < 0.0f || c.air_density < 0.0f || c.drag_angular < 0.0f ||
      c.turbulence_amplitude < 0.0f)
    return 0;
  AmbientConfig2Ffi a = c;
  a.spring_enabled = c.spring_enabled != 0;
  a.drag_enabled = c.drag_enabled != 0;
  a.turbulence_enabled = c.turbulence_enabled != 0;
  a.turbulence_divergence_free = c.turbulence_divergence_free != 0;
  a.turbulence_octaves = std::min<uint32_t>(c.turbulence_octaves, 255u);
  w->ambient = a;
  return 1;
}

int32_t phieng_world_get_ambient_config(World2* w, AmbientConfig2Ffi* out) {
  if (!w || !out) return 0;
  *out = w->ambient;
  return 1;
}

uint32_t phieng_sph_fluid_masses(World2* w, float* out, uint32_t max) {
  if (!w) return 0;
  for (uint32_t i = 0; out && i < std::min(w->n, max); i++) out[i] = w->h_mass[i];
  return w->n;
}

uint32_t phieng_sph_ghosts(World2* w, float* xy, uint32_t max, uint64_t* regens) {
  if (!w) return 0;
  if (regens) *regens = w->ghost_regens;
  const uint32_t n = (uint32_t)w->h_gpos.size();
  if (xy)
    for (uint32_t i = 0; i < std::min(n, max); i++) {
      xy[2 * i] = w->h_gpos[i].x;
      xy[2 * i + 1] = w->h_gpos[i].y;
    }
  return n;
}

int32_t phieng_world_body_count(World2* w) {
  if (!w) return -1;
  return (int32_t)w->bodies.size();
}

int32_t phieng_world_add_body(World2* w, float px, float py, uint32_t shape_tag, float a, float b, float density,
                              uint8_t is_static, float friction, float restitution) {
  (void)friction;
  (void)restitution;
  if (!w || w->is_batch() || !std::isfinite(px) || !std::isfinite(py)) return -1;
  DevBody bd;
  std::memset(&bd, 0, sizeof(bd));
  auto pos = [](float v) { return std::isfinite(v) && v > 0.0f; };
  if (shape_tag == PHIENG_SHAPE_CIRCLE && pos(a)) {
    bd.shape = 0;
    bd.a = a;
  } else if (shape_tag == PHIENG_SHAPE_BOX && pos(a) && pos(b)) {
    bd.shape = 1;
    bd.a = a;
    bd.b = b;
  } else {
    return -1;
  }
  if (!pos(density)) return -1;
  if (!is_static) return -1;  // dynamic bodies are not part of this library
  bd.px = px;
  bd.py = py;
  // Transform2::from_position_angle(p, 0.0) (ffi.rs:1184): Mat2::from_angle(0)
  // = columns (cos, sin), (-sin, cos) = (1, 0), (-0, 1).
  bd.xax = 1.0f;
  bd.xay = 0.0f;
  bd.yax = -0.0f;
  bd.yay = 1.0f;
  {
    // world bounding box of the (unrotated) body, padded by 0.1%
    const float ha = bd.a, hb = bd.shape == 0 ? bd.a : bd.b;
    bd.ex = (std::fabs(bd.xax) * ha + std::fabs(bd.yax) * hb) * 1.001f + 1e-30f;
    bd.ey = (std::fabs(bd.xay) * ha + std::fabs(bd.yay) * hb) * 1.001f + 1e-30f;
  }
  if (w->bodies.size() >= 0x7FFFFFFF) return -1;
  w->bodies.push_back(bd);
  w->bodies_dirty = true;
  return (int32_t)(w->bodies.size() - 1);
}

uint32_t phieng_world_add_bodies(World2* w, const BodyDesc2D* descs, uint32_t n, int32_t* out_ids) {
  if (!w || !descs || !out_ids) return 0;
  n = std::min<uint32_t>(n, 1000000u);
  uint32_t added = 0;
  for (uint32_t i = 0; i < n; i++) {
    const BodyDesc2D& d = descs[i];
    out_ids[i] = phieng_world_add_body(w, d.pos_x, d.pos_y, d.shape_tag, d.a, d.b, d.density, d.is_static,
                                       d.friction, d.restitution);
    if (out_ids[i] >= 0) added++;
  }
  return added;
}

int32_t phieng_sph_reserve(World2* w, uint32_t n) {
  if (!w || w->is_batch()) return 0;
  if (w->error != PHIENG_SPH_OK || !ensure_device(w)) return 0;
  n = std::max(n, w->n);
  if (!ensure_capacity(w, n)) return 0;
  // the bucket arrays for the largest grid a plan for n particles can take
  // (plan_cells: a power of two of buckets_per_particle * n, 2^12 .. 2^24)
  const uint64_t want = (uint64_t)std::ceil((double)w->buckets_per_particle * (double)std::max<uint32_t>(n, 1));
  const uint32_t budget = (uint32_t)std::min<uint64_t>(1ull << 24, std::max<uint64_t>(1ull << 12, next_pow2(want)));
  if (w->d.count && w->d.range_cap >= budget) return 1;
  return alloc_range(w, budget) ? 1 : 0;
}

int32_t phieng_sph_step_fluid(World2* w, PhiengBody2* bodies, uint32_t nbodies, float dt) {
  if (!w || w->is_batch() || (nbodies && !bodies) || nbodies > kMaxCallBodies) return 0;
  for (uint32_t k = 0; k < nbodies; k++)
    if (!body_valid(bodies[k])) return 0;
  return step_fluid_bodies(w, bodies, nbodies, dt) ? 1 : 0;
}

constexpr uint32_t kMaxPolyVerts = 1u << 20;

int32_t phieng_sph_step_fluid_poly(World2* w, PhiengBody2* bodies, uint32_t nbodies, const float* poly_xy,
                                   const uint32_t* poly_first, const uint32_t* poly_count, uint32_t poly_nverts,
                                   float dt) {
  if (!w || w->is_batch() || (nbodies && !bodies) || nbodies > kMaxCallBodies || poly_nverts > kMaxPolyVerts)
    return 0;
  uint64_t total = 0;
  for (uint32_t k = 0; k < nbodies; k++) {
    const PhiengBody2& b = bodies[k];
    if (b.shape_tag != PHIENG_SHAPE_POLYGON) {
      if (!body_valid(b)) return 0;
      continue;
    }
    if (!poly_xy || !poly_first || !poly_count) return 0;
    const float t[] = {b.px, b.py, b.xax, b.xay, b.yax, b.yay, b.vx, b.vy, b.w, b.inv_mass, b.inv_inertia};
    for (float x : t)
      if (!std::isfinite(x)) return 0;
    const uint64_t f = poly_first[k], c = poly_count[k];
    if (c < 3 || f + c > poly_nverts) return 0;
    for (uint64_t i = 2 * f; i < 2 * (f + c); i++)
      if (!std::isfinite(poly_xy[i])) return 0;
    total += c;
  }
  if (total > kMaxPolyVerts) return 0;
  PolyIn pin;
  pin.xy = poly_xy;
  pin.first = poly_first;
  pin.count = poly_count;
  return step_fluid_bodies(w, bodies, nbodies, dt, pin) ? 1 : 0;
}

int32_t phieng_world_set_fluid_config(World2* w, const FluidConfig2Ffi* cfg) {
  if (!w || !cfg || w->is_batch()) return 0;
  if (!valid_config(*cfg)) return 0;
  FluidConfig2Ffi c = *cfg;
  c.adaptive_resolution = c.adaptive_resolution ? 1 : 0;
  c.boundary_particles = c.boundary_particles ? 1 : 0;
  c.enabled = c.enabled ? 1 : 0;
  bool regrid = c.smoothing_length != w->cfg.smoothing_length;
  w->cfg = c;
  if (regrid) {
    if (w->plan_locked) w->plan.hg = c.smoothing_length;
    else w->plan_valid = false;
    w->keys_valid = false;
  }
  return 1;
}

int64_t phieng_sph_fluid_block_save(World2* w, uint32_t version, uint8_t* out, uint64_t cap) {
  if (!w || w->is_batch() || version == 0 || version > snap::kSchemaLatest) return -1;
  if (w->n && !ensure_host_state(w)) return -1;
  std::vector<snap::Particle> ps(w->n);
  for (uint32_t i = 0; i < w->n; i++) {
    const float4 q = w->h_state[i];
    ps[i] = snap::Particle{q.x, q.y, 0.0f, q.z, q.w, 0.0f, w->h_mass[i], w->h_phase[i]};
  }
  std::vector<uint8_t> o;
  snap::encode(o, w->cfg, ps, 2, version);
  if (out && cap >= o.size()) std::memcpy(out, o.data(), o.size());
  return (int64_t)o.size();
}

int64_t phieng_sph_fluid_block_load(World2* w, uint32_t version, const uint8_t* data, uint64_t len) {
  if (!w || w->is_batch() || !data || version == 0 || version > snap::kSchemaLatest) return -1;
  snap::Reader r(data, len);
  snap::Block b;
  if (!snap::decode(r, version, 2, w->cap, b)) return -2;
  if (w->device >= 0) cudaStreamSynchronize(w->stream);
  const bool regrid = b.cfg.smoothing_length != w->cfg.smoothing_length;
  w->cfg = b.cfg;
  const uint32_t n = (uint32_t)b.particles.size();
  w->h_state.resize(n);
  w->h_mass.resize(n);
  w->h_phase.resize(n);
  w->h_dens.assign(n, b.cfg.rest_density);  // density / pressure are recomputed by the next step
  w->h_pres.assign(n, 0.0f);
  for (uint32_t i = 0; i < n; i++) {
    const snap::Particle& q = b.particles[i];
    w->h_state[i] = make_float4(q.x, q.y, q.vx, q.vy);
    w->bbox_valid = false;
    w->h_mass[i] = q.mass;
    w->h_phase[i] = q.phase;
  }
  w->n = n;
  recompute_uniformity(w);
  w->host_state_valid = true;
  w->dev_state_valid = false;
  w->dev_aux_valid = false;
  w->dp_on_device = false;
  if (w->plan_locked) {
    if (regrid) w->plan.hg = b.cfg.smoothing_length;
  } else {
    w->plan_valid = false;
  }
  w->keys_valid = false;
  return (int64_t)r.off;
}

int32_t phieng_world_get_fluid_config(World2* w, FluidConfig2Ffi* out) {
  if (!w || !out) return 0;
  *out = w->cfg;
  return 1;
}

uint32_t phieng_world_fluid_add(World2* w, const float* positions, uint32_t count) {
  if (!w || !positions || w->is_batch()) return 0;
  return add_particles(w, positions, nullptr, count);
}

uint32_t phieng_world_fluid_add_phase(World2* w, const float* positions, const uint8_t* phases, uint32_t count) {
  if (!w || !positions || !phases || w->is_batch()) return 0;
  return add_particles(w, positions, phases, count);
}

uint32_t phieng_world_fluid_count(const World2* w) {
  if (!w) return 0;
  return w->n;
}

int32_t phieng_world_fluid_clear(World2* w) {
  if (!w || w->is_batch()) return 0;
  if (w->device >= 0) cudaStreamSynchronize(w->stream);
  w->n = 0;
  w->h_state.clear();
  w->bbox_valid = true;
  w->bx0 = w->by0 = INFINITY;
  w->bx1 = w->by1 = -INFINITY;
  w->h_mass.clear();
  w->h_phase.clear();
  w->h_dens.clear();
  w->h_pres.clear();
  recompute_uniformity(w);
  w->host_state_valid = true;
  w->dev_state_valid = false;
  w->dev_aux_valid = false;
  w->dp_on_device = false;
  w->plan_valid = false;
  w->keys_valid = false;
  return 1;
}

uint32_t phieng_world_fluid_get(const World2* cw, float* out, uint32_t max) {
  if (!cw || !out) return 0;
  World2* w = const_cast<World2*>(cw);
  uint32_t n = std::min(max, w->n);
  if (n == 0) return 0;
  if (!w->host_state_valid) {
    // straight from the device into the caller's buffer (a DMA when it is
    // page-locked)
    if (w->device < 0) return 0;
    if (!cuda_ok(w, cudaMemcpyAsync(out, w->d.state, sizeof(float4) * n, cudaMemcpyDeviceToHost, w->stream),
                 "download state") ||
        !cuda_ok(w, cudaStreamSynchronize(w->stream), "sync") || !scan_flag_ok(w))
      return 0;
    return n;
  }
  std::memcpy(out, w->h_state.data(), sizeof(float4) * n);
  return n;
}

// ---------------------------------------------------------------- extension
int32_t phieng_sph_status(const World2* w, PhiengSphStatus* out) {
  if (!w || !out) return 0;
  std::memset(out, 0, sizeof(*out));
  out->error = w->error;
  out->particles = w->n;
  out->substeps = w->substeps;
  out->grid_log2_w = w->plan_valid ? w->plan.log2w : 0;
  out->grid_log2_h = w->plan_valid ? w->plan.log2h : 0;
  out->sort_passes = w->plan_valid ? 1 : 0;
  out->grid_cx0 = w->plan_valid ? w->plan.cx0 : 0;
  out->grid_cy0 = w->plan_valid ? w->plan.cy0 : 0;
  out->grid_buckets = w->plan_valid ? w->plan.sentinel : 0;
  return 1;
}

int32_t phieng_sph_clear_error(World2* w) {
  if (!w) return 0;
  w->error = PHIENG_SPH_OK;
  return 1;
}

const char* phieng_sph_error_string(const World2* w) { return error_text(w ? w->error : PHIENG_SPH_E_ARG); }

int32_t phieng_sph_set_particle_cap(World2* w, uint32_t cap) {
  if (!w || cap == 0) return 0;
  w->cap = cap;
  return 1;
}

int32_t phieng_sph_step_n(World2* w, float dt, uint32_t steps) {
  if (!w) return 0;
  if (!std::isfinite(dt) || dt <= 0.0f) return 1;
  const float d = std::min(dt, kMaxDt);
  for (uint32_t s = 0; s < steps; s++)
    if (!world_step(w, d)) return 0;
  return 1;
}

int32_t phieng_sph_set_stream(World2* w, void* stream) {
  if (!w) return 0;
  if (w->device >= 0) cudaStreamSynchronize(w->stream);
  if (stream) {
    w->stream = (cudaStream_t)stream;
    w->user_stream = true;
  } else {
    w->stream = w->own_stream;
    w->user_stream = false;
  }
  return 1;
}

int32_t phieng_sph_sync(World2* w) {
  if (!w) return 0;
  if (w->device < 0) return w->error == PHIENG_SPH_OK ? 1 : 0;
  if (!cuda_ok(w, cudaStreamSynchronize(w->stream), "sync")) return 0;
  if (!scan_flag_ok(w)) return 0;
  return w->error == PHIENG_SPH_OK ? 1 : 0;
}

int32_t phieng_sph_set_state(World2* w, const float* xyvv, uint32_t n) {
  if (!w || !xyvv || n > w->n) return 0;
  for (uint64_t i = 0; i < 4ull * n; i++)
    if (!std::isfinite(xyvv[i])) return 0;
  if (!ensure_host_state(w)) return 0;
  std::memcpy(w->h_state.data(), xyvv, sizeof(float4) * n);
  w->bbox_valid = false;
  w->dev_state_valid = false;
  w->keys_valid = false;
  if (!w->plan_locked) w->plan_valid = false;
  return 1;
}

uint32_t phieng_sph_get_density_pressure(const World2* cw, float* dens, float* pres, uint32_t max) {
  if (!cw) return 0;
  World2* w = const_cast<World2*>(cw);
  uint32_t n = std::min(max, w->n);
  if (n == 0) return 0;
  if (!ensure_host_dp(w)) return 0;
  if (dens) std::memcpy(dens, w->h_dens.data(), sizeof(float) * n);
  if (pres) std::memcpy(pres, w->h_pres.data(), sizeof(float) * n);
  return n;
}

int32_t phieng_sph_replan(World2* w) {
  if (!w) return 0;
  if (!ensure_host_state(w)) return 0;
  w->plan_locked = false;
  plan_grid(w);
  return 1;
}

int32_t phieng_sph_set_grid(World2* w, uint32_t log2w, uint32_t log2h, int32_t cx0, int32_t cy0) {
  if (!w || w->is_batch() || log2w < 2 || log2h < 2 || log2w + log2h > 24) return 0;
  GridPlan g;
  g.log2w = log2w;
  g.log2h = log2h;
  g.maskw = (1u << log2w) - 1u;
  g.maskh = (1u << log2h) - 1u;
  g.nbuckets = 1u << (log2w + log2h);
  g.base = 0;
  g.sentinel = g.nbuckets;
  g.cx0 = cx0;
  g.cy0 = cy0;
  g.hg = w->cfg.smoothing_length;
  w->plan = g;
  w->plan_valid = true;
  w->plan_locked = true;
  w->keys_valid = false;
  return 1;
}

int32_t phieng_sph_set_profiling(World2* w, int32_t on) {
  if (!w) return 0;
  if (on && !w->ev[0]) {
    if (!ensure_device(w)) return 0;
    for (auto& e : w->ev)
      if (!cuda_ok(w, cudaEventCreate(&e), "cudaEventCreate")) return 0;
  }
  if (w->device >= 0) cudaStreamSynchronize(w->stream);
  w->profiling = on != 0;
  release_graph(w);
  return 1;
}

uint32_t phieng_sph_phase_times(World2* w, float* ms, uint32_t max) {
  if (!w || !ms || !w->profiling || w->substeps == 0) return 0;
  if (!cuda_ok(w, cudaStreamSynchronize(w->stream), "sync")) return 0;
  uint32_t k = 0;
  for (; k < 3 && k < max; k++)
    if (!cuda_ok(w, cudaEventElapsedTime(&ms[k], w->ev[k], w->ev[k + 1]), "cudaEventElapsedTime")) return 0;
  return k;
}

int32_t phieng_sph_front_metrics(World2* w, float* out) {
  if (!w || !out) return 0;
  out[0] = -INFINITY;
  out[1] = 0.0f;
  if (w->n == 0) return 1;
  if (w->host_state_valid) {
    for (uint32_t i = 0; i < w->n; i++) {
      float4 s = w->h_state[i];
      out[0] = rmaxf(out[0], s.x);
      out[1] = rmaxf(out[1], std::sqrt(s.z * s.z + s.w * s.w));
    }
    return 1;
  }
  if (w->device < 0) return 0;
  enqueue_front_metrics(w->d, w->n, w->stream);
  if (!cuda_ok(w, cudaMemcpyAsync(w->h_pinned, w->d.scalar + 2, 8, cudaMemcpyDeviceToHost, w->stream), "metrics"))
    return 0;
  if (!cuda_ok(w, cudaStreamSynchronize(w->stream), "sync")) return 0;
  unsigned int bx = w->h_pinned[0], bv = w->h_pinned[1];
  unsigned int ux = (bx & 0x80000000u) ? (bx & 0x7FFFFFFFu) : ~bx;  // undo the order-preserving map
  if (bx == 0u) {
    out[0] = -INFINITY;
  } else {
    std::memcpy(&out[0], &ux, 4);
  }
  std::memcpy(&out[1], &bv, 4);
  return 1;
}

int32_t phieng_sph_front_metrics_async(World2* w, uint32_t* raw) {
  if (!w || !raw) return 0;
  if (w->n == 0) {
    raw[0] = 0u;
    raw[1] = 0u;
    return 1;
  }
  if (w->host_state_valid) {
    float m[2];
    if (!phieng_sph_front_metrics(w, m)) return 0;
    uint32_t bx, bv;
    std::memcpy(&bx, &m[0], 4);
    std::memcpy(&bv, &m[1], 4);
    raw[0] = (bx & 0x80000000u) ? ~bx : (bx | 0x80000000u);  // the device reduction's order-preserving map
    raw[1] = bv;
    return 1;
  }
  if (w->device < 0) return 0;
  enqueue_front_metrics(w->d, w->n, w->stream);
  return cuda_ok(w, cudaMemcpyAsync(raw, w->d.scalar + 2, 8, cudaMemcpyDeviceToHost, w->stream), "metrics") ? 1 : 0;
}

void phieng_sph_front_metrics_decode(const uint32_t* raw, float* out) {
  if (!raw || !out) return;
  const uint32_t bx = raw[0], bv = raw[1];
  if (bx == 0u) {
    out[0] = -INFINITY;
  } else {
    const uint32_t ux = (bx & 0x80000000u) ? (bx & 0x7FFFFFFFu) : ~bx;
    std::memcpy(&out[0], &ux, 4);
  }
  std::memcpy(&out[1], &bv, 4);
}

int32_t phieng_sph_set_tuning(World2* w, const PhiengSphTuning* t) {
  if (!w || !t) return 0;
  auto ok_block = [](uint32_t b) { return b == 64 || b == 128 || b == 256; };
  if (!ok_block(t->density_block) || !ok_block(t->force_block) || !(t->buckets_per_particle >= 0.125f) ||
      !(t->buckets_per_particle <= 16.0f) || t->stage > 7u)
    return 0;
  if (w->device >= 0) cudaStreamSynchronize(w->stream);
  release_graph(w);
  w->d.block_density = t->density_block;
  w->d.block_force = t->force_block;
  w->d.stage = t->stage;
  if (w->buckets_per_particle != t->buckets_per_particle) {
    w->buckets_per_particle = t->buckets_per_particle;
    if (!w->plan_locked) {
      if (!ensure_host_state(w)) return 0;
      plan_grid(w);
    }
  }
  return 1;
}

int32_t phieng_sph_get_tuning(const World2* w, PhiengSphTuning* t) {
  if (!w || !t) return 0;
  t->density_block = w->d.block_density;
  t->force_block = w->d.block_force;
  t->buckets_per_particle = w->buckets_per_particle;
  t->stage = w->d.stage;
  return 1;
}

int32_t phieng_sph_set_precision(World2* w, uint32_t mode) {
  if (!w || (mode != PHIENG_SPH_EXACT && mode != PHIENG_SPH_TOLERANCE)) return 0;
  if (mode == w->precision) return 1;
  if (w->device >= 0) cudaStreamSynchronize(w->stream);
  release_graph(w);
  w->precision = mode;
  return 1;
}

uint32_t phieng_sph_get_precision(const World2* w) { return w ? w->precision : PHIENG_SPH_EXACT; }

int32_t phieng_sph_set_order(World2* w, const uint32_t* tags, uint32_t n) {
  if (!w || w->is_batch() || !tags || n == 0 || n != w->n) return 0;
  if (!prepare(w)) return 0;
  if (!w->d.order && !dalloc(w, w->d.order, w->d.cap)) return 0;
  if (!cuda_ok(w, cudaMemcpyAsync(w->d.order, tags, sizeof(uint32_t) * n, cudaMemcpyDefault, w->stream),
               "order tags"))
    return 0;
  release_graph(w);  // the captured sort reads the tag array
  return 1;
}

int32_t phieng_sph_slab_setup(World2* w, int32_t lo, int32_t hi, uint32_t neighbours, uint32_t own_cap,
                              uint32_t halo_cap, void* send_left, void* send_right, const void* recv_left,
                              const void* recv_right) {
  if (!w || w->is_batch() || !w->d.order || hi <= lo || halo_cap == 0 || neighbours > 3u ||
      (uint64_t)own_cap + 4ull * halo_cap != w->n)
    return 0;
  // a slab between two neighbours spans at least two halo bands
  if (neighbours == 3u && (int64_t)hi - (int64_t)lo < 2 * kSlabHaloColumns) return 0;
  if ((neighbours & 1u) && (!send_left || !recv_left)) return 0;
  if ((neighbours & 2u) && (!send_right || !recv_right)) return 0;
  // one substep per world step (the ranks agree on the substep count), and
  // none of the passes that change the particle set or add particles
  if ((w->cfg.cfl > 0.0f && w->cfg.max_substeps > 1) || w->cfg.adaptive_resolution || w->cfg.boundary_particles)
    return 0;
  if (!prepare(w)) return 0;  // keys and bucket counts of the current slots
  if (w->slab_cap < own_cap + kSlabWords) {
    cudaStreamSynchronize(w->stream);
    dfree(w->d_slab);
    w->slab_cap = 0;
    if (!dalloc(w, w->d_slab, (size_t)own_cap + kSlabWords)) return 0;
    w->slab_cap = own_cap + kSlabWords;
  }
  SlabPlan& sp = w->slab_plan;
  sp.lo = lo;
  sp.hi = hi;
  sp.has_left = neighbours & 1u;
  sp.has_right = (neighbours >> 1) & 1u;
  sp.h = w->cfg.smoothing_length;
  sp.own_cap = own_cap;
  sp.halo_cap = halo_cap;
  sp.send[0] = sp.has_left ? static_cast<unsigned char*>(send_left) : nullptr;
  sp.send[1] = sp.has_right ? static_cast<unsigned char*>(send_right) : nullptr;
  sp.recv[0] = sp.has_left ? static_cast<const unsigned char*>(recv_left) : nullptr;
  sp.recv[1] = sp.has_right ? static_cast<const unsigned char*>(recv_right) : nullptr;
  sp.free_stack = w->d_slab;
  sp.words = w->d_slab + own_cap;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, w->device);
  sp.pack_blocks = 4u * (uint32_t)std::max(sms, 1);
  enqueue_slab_init(w->d, sp, w->stream);
  w->slab = true;
  return cuda_ok(w, cudaGetLastError(), "slab setup") ? 1 : 0;
}

int32_t phieng_sph_slab_pack(World2* w, uint32_t phase) {
  if (!w || !w->slab || phase > 1 || !w->d.order) return 0;
  if (!prepare(w)) return 0;
  enqueue_slab_pack(w->d, w->slab_plan, w->plan, phase, w->stream);
  return cuda_ok(w, cudaGetLastError(), "slab pack") ? 1 : 0;
}

int32_t phieng_sph_slab_unpack(World2* w, uint32_t phase) {
  if (!w || !w->slab || phase > 1 || !w->d.order) return 0;
  if (!prepare(w)) return 0;
  enqueue_slab_unpack(w->d, w->slab_plan, w->plan, phase, w->stream);
  w->host_state_valid = false;
  w->dp_on_device = false;
  return cuda_ok(w, cudaGetLastError(), "slab unpack") ? 1 : 0;
}

int32_t phieng_sph_slab_vmax(World2* w, float* out) {
  if (!w || !w->slab || !out) return 0;
  if (!prepare(w)) return 0;
  FluidBufs b = w->d;
  b.scalar = reinterpret_cast<unsigned int*>(out);
  enqueue_vmax(b, w->slab_plan.own_cap, w->stream);
  return cuda_ok(w, cudaGetLastError(), "slab vmax") ? 1 : 0;
}

int32_t phieng_sph_slab_status(World2* w) {
  if (!w || !w->slab) return 0;
  uint32_t e = 1;
  if (!cuda_ok(w, cudaMemcpyAsync(&e, w->slab_plan.words + 1, 4, cudaMemcpyDeviceToHost, w->stream), "slab status") ||
      !cuda_ok(w, cudaStreamSynchronize(w->stream), "sync"))
    return 0;
  return e == 0 ? 1 : 0;
}

uint32_t phieng_sph_slab_owned(World2* w, float* state, uint32_t* tags, uint32_t max) {
  if (!w || !w->slab || !state || !tags) return 0;
  const uint32_t oc = w->slab_plan.own_cap;
  std::vector<float4> st(oc);
  std::vector<uint32_t> tg(oc);
  if (oc && (!cuda_ok(w, cudaMemcpyAsync(st.data(), w->d.state, sizeof(float4) * oc, cudaMemcpyDeviceToHost,
                                          w->stream),
                      "slab owned") ||
             !cuda_ok(w, cudaMemcpyAsync(tg.data(), w->d.order, 4ull * oc, cudaMemcpyDeviceToHost, w->stream),
                      "slab owned") ||
             !cuda_ok(w, cudaStreamSynchronize(w->stream), "sync")))
    return 0;
  uint32_t k = 0;
  for (uint32_t i = 0; i < oc; i++) {
    if (tg[i] == kSlabFree) continue;
    if (k < max) {
      std::memcpy(state + 4ull * k, &st[i], sizeof(float4));
      tags[k] = tg[i];
    }
    k++;
  }
  return k;
}

int32_t phieng_sph_load_state_device(World2* w, const float* src, uint32_t n) {
  if (!w || w->is_batch() || (n && !src) || n > w->cap) return 0;
  if (!ensure_device(w)) return 0;
  cudaStreamSynchronize(w->stream);
  w->n = n;
  w->h_state.resize(n);
  w->h_dens.assign(n, w->cfg.phase_rest_density[0]);
  w->h_pres.assign(n, 0.0f);
  w->h_mass.assign(n, rmaxf(w->cfg.phase_mass[0], 0.0f));
  w->h_phase.assign(n, 0);
  recompute_uniformity(w);
  if (n && !ensure_capacity(w, n)) return 0;
  if (n && !cuda_ok(w, cudaMemcpyAsync(w->d.state, src, sizeof(float4) * n, cudaMemcpyDeviceToDevice, w->stream),
                    "load state"))
    return 0;
  w->dev_state_valid = true;
  w->host_state_valid = n == 0;
  w->dev_aux_valid = false;
  w->dp_on_device = false;
  w->keys_valid = false;  // the bucket grid stays: any grid is exact
  return 1;
}

uint32_t phieng_sph_get_state_device(World2* w, float* dst, uint32_t max) {
  if (!w || !dst) return 0;
  const uint32_t n = std::min(max, w->n);
  if (n == 0) return 0;
  if (!prepare(w)) return 0;
  if (!cuda_ok(w, cudaMemcpyAsync(dst, w->d.state, sizeof(float4) * n, cudaMemcpyDeviceToDevice, w->stream),
               "get state"))
    return 0;
  return n;
}

int32_t phieng_sph_set_state_device(World2* w, const float* src, uint32_t n) {
  if (!w || !src || n != w->n) return 0;
  if (n == 0) return 1;
  if (!prepare(w)) return 0;
  if (!cuda_ok(w, cudaMemcpyAsync(w->d.state, src, sizeof(float4) * n, cudaMemcpyDeviceToDevice, w->stream),
               "set state"))
    return 0;
  w->host_state_valid = false;
  w->dp_on_device = false;
  w->keys_valid = false;  // the bucket grid stays: any grid is exact, it only affects speed
  return 1;
}

int32_t phieng_sph_features(World2* w, float dt, float* feat) {
  if (!w || !feat || !std::isfinite(dt) || dt <= 0.0f) return 0;
  if (w->n == 0) return 1;
  if (!w->is_batch() && unsupported(w)) return 0;
  if (!prepare(w)) return 0;
  if (w->is_batch() && !upload_scene_table(w, dt)) return 0;
  if (!ensure_closure_buffers(w)) return 0;
  const StepParams P = make_params(w, dt);
  enqueue_sort_density(w, P, w->d_svp);
  enqueue_closure_features(w->d, w->n, P, feat, w->d_svp, w->stream);
  w->keys_valid = false;  // the sort consumed the bucket counts
  return cuda_ok(w, cudaGetLastError(), "features") ? 1 : 0;
}

int32_t phieng_sph_set_closure(World2* w, PhiengMlp* mlp, uint32_t ratio, float threshold, uint32_t criterion) {
  if (!w || ratio < 1 || !(threshold >= 0.0f) || criterion > PHIENG_CLOSURE_GROWTH) return 0;
  if (mlp && phieng_mlp_status(mlp) != PHIENG_SPH_OK) return 0;
  w->closure = mlp;
  w->closure_ratio = ratio;
  w->closure_threshold = threshold;
  w->closure_criterion = criterion;
  return 1;
}

int32_t phieng_sph_closure_step(World2* w, float dt_fine, uint32_t coarse_steps, PhiengClosureStats* stats) {
  if (!w || !w->closure || !std::isfinite(dt_fine) || dt_fine <= 0.0f) return 0;
  const float dtc = dt_fine * (float)w->closure_ratio;
  const bool batch = w->is_batch();
  if ((!batch && !w->cfg.enabled) || w->n == 0 || coarse_steps == 0) {
    w->time += dtc * (float)coarse_steps;
    return 1;
  }
  if (!batch && unsupported(w)) return 0;
  if (!prepare(w)) return 0;
  if (!ensure_closure_buffers(w)) return 0;
  // a batch reads each scene's step length from its parameter table
  if (batch && !upload_scene_table(w, dtc)) return 0;
  const StepParams Pc = make_params(w, dtc);
  const StepParams Pf = make_params(w, dt_fine);
  const MlpDev mlp = phieng_mlp_dev(w->closure);
  ClosureIO io;
  io.save = w->d_save;
  io.rho_prev = w->d_rho_prev;
  io.svp = w->d_svp;
  io.err = w->d.scan_err;  // tolerance mode: the tensor-core waits of the fused pass report here
  enqueue_sort_density(w, Pc, w->d_svp);
  // Coarse steps run in optimistic blocks: kBlock steps back to back with the
  // checks folded on the device and one read of their maxima. If every step
  // passes, the block stands exactly as step-by-step acceptance would have
  // left it; otherwise the block's start is restored and its steps are taken
  // one at a time with the per-step check and fallback, so the result is the
  // same as that of the per-step rule in every case.
  constexpr uint32_t kBlock = 8;
  float* acc = reinterpret_cast<float*>(w->d.scalar + 13);
  uint32_t k = 0;
  while (k < coarse_steps) {
    const uint32_t nb = std::min(kBlock, coarse_steps - k);
    if (nb > 1) {
      if (!cuda_ok(w, cudaMemcpyAsync(w->d_block_save, w->d.state, sizeof(float4) * w->n, cudaMemcpyDeviceToDevice,
                                      w->stream),
                   "block save"))
        return 0;
      enqueue_check_fold(w->d.scalar + 4, acc, true, w->stream);
      float tb = w->time;
      for (uint32_t b = 0; b < nb; b++) {
        set_clock(w, Pc, tb);
        tb += dtc;
        if (!run_coarse(w, Pc, mlp, io)) return 0;
        w->sid_perm_n = w->n;
        enqueue_check_fold(w->d.scalar + 4, acc, false, w->stream);
      }
      if (!cuda_ok(w, cudaMemcpyAsync(w->h_pinned, w->d.scalar + 4, 12 * sizeof(unsigned int), cudaMemcpyDeviceToHost,
                                      w->stream),
                   "check") ||
          !cuda_ok(w, cudaStreamSynchronize(w->stream), "sync"))
        return 0;
      float last[3], mx[3];
      std::memcpy(last, w->h_pinned, 12);
      std::memcpy(mx, w->h_pinned + 9, 12);  // scalar[13..15]
      const int c = (int)w->closure_criterion;
      const float chk = c == PHIENG_CLOSURE_JUMP ? mx[0] : c == PHIENG_CLOSURE_COMPRESSION ? mx[1] : mx[2];
      w->host_state_valid = false;
      if (chk <= w->closure_threshold) {
        if (stats) {
          stats->coarse_steps += nb;
          stats->accepted += nb;
          stats->last_check = c == PHIENG_CLOSURE_JUMP          ? last[0]
                              : c == PHIENG_CLOSURE_COMPRESSION ? last[1]
                                                                : last[1] - last[2];
          stats->max_check = std::max(stats->max_check, chk);
        }
        w->substeps += nb;
        for (uint32_t b = 0; b < nb; b++) w->time += dtc;
        k += nb;
        continue;
      }
      // a step of the block failed: back to its start, then step by step
      if (!cuda_ok(w, cudaMemcpyAsync(w->d.state, w->d_block_save, sizeof(float4) * w->n, cudaMemcpyDeviceToDevice,
                                      w->stream),
                   "block restore"))
        return 0;
      w->keys_valid = false;
      if (!prepare(w)) return 0;
      enqueue_sort_density(w, Pc, w->d_svp);
    }
    const uint32_t kend = k + nb;
    for (; k < kend; k++) {
      set_clock(w, Pc, w->time);
      if (!run_coarse(w, Pc, mlp, io)) return 0;
      w->sid_perm_n = w->n;
      if (!cuda_ok(w, cudaMemcpyAsync(w->h_pinned, w->d.scalar + 4, 12, cudaMemcpyDeviceToHost, w->stream), "check") ||
          !cuda_ok(w, cudaStreamSynchronize(w->stream), "sync"))
        return 0;
      float v[3];
      std::memcpy(v, w->h_pinned, 12);
      const float chk = w->closure_criterion == PHIENG_CLOSURE_JUMP          ? v[0]
                        : w->closure_criterion == PHIENG_CLOSURE_COMPRESSION ? v[1]
                                                                             : v[1] - v[2];
      if (stats) {
        stats->coarse_steps++;
        stats->last_check = chk;
        stats->max_check = std::max(stats->max_check, chk);
      }
      w->host_state_valid = false;
      if (chk <= w->closure_threshold) {
        if (stats) stats->accepted++;
        w->substeps++;
      } else {
        // undo the coarse step, take ratio plain substeps instead
        if (stats) stats->fallbacks++;
        if (!cuda_ok(w, cudaMemcpyAsync(w->d.state, w->d_save, sizeof(float4) * w->n, cudaMemcpyDeviceToDevice,
                                        w->stream),
                     "restore"))
          return 0;
        w->keys_valid = false;
        if (!prepare(w)) return 0;
        if (batch && !upload_scene_table(w, dt_fine)) return 0;
        float tf = w->time;
        for (uint32_t r = 0; r < w->closure_ratio; r++) {
          set_clock(w, Pf, tf);
          tf += dt_fine;
          if (!run_substep(w, Pf)) return 0;
        }
        if (batch && !upload_scene_table(w, dtc)) return 0;
        if (k + 1 < coarse_steps) enqueue_sort_density(w, Pc, w->d_svp);
      }
      w->time += dtc;
    }
  }
  w->keys_valid = false;  // the last sort consumed the bucket counts
  return cuda_ok(w, cudaGetLastError(), "closure step") ? 1 : 0;
}

int32_t phieng_sph_debug_scan_timeout(World2* w) {
  if (!w || !prepare(w)) return 0;
  const uint32_t m = w->plan.sentinel + 1;
  // at least two look-back blocks
  if ((m + kBucketScanTile * kBucketScanSuper - 1) / (kBucketScanTile * kBucketScanSuper) < 2) return 0;
  enqueue_scan_silent_tile(w->d, m, w->stream);
  if (!cuda_ok(w, cudaGetLastError(), "scan")) return 0;
  w->keys_valid = false;  // the counts became cursors
  return scan_flag_ok(w) ? 1 : 0;
}

uint32_t phieng_sph_debug_sorted(World2* w, uint32_t* ids, uint32_t* keys, uint32_t max) {
  if (!w || w->n == 0 || w->is_batch()) return 0;
  if (!ensure_host_dp(w)) return 0;  // the re-sort below invalidates the sorted density
  if (!prepare(w)) return 0;
  const StepParams P = make_params(w, 0.0f);
  enqueue_keys(w->d, w->n, w->plan, w->stream);
  enqueue_sort_and_ranges(w->d, w->n, P, false, w->stream);
  w->sid_perm_n = w->n;
  w->keys_valid = false;  // the sort consumed the bucket counts
  uint32_t n = std::min(max, w->n);
  if (ids) cudaMemcpyAsync(ids, w->d.sid, 4ull * n, cudaMemcpyDeviceToHost, w->stream);
  if (keys) cudaMemcpyAsync(keys, w->d.skey, 4ull * n, cudaMemcpyDeviceToHost, w->stream);
  if (!cuda_ok(w, cudaStreamSynchronize(w->stream), "debug_sorted")) return 0;
  return w->n;
}

uint32_t phieng_sph_debug_neighbors(World2* w, uint32_t* counts, uint32_t* lists, uint32_t max_per, uint32_t max) {
  if (!w || !counts || !lists || w->n == 0 || max < w->n || w->is_batch()) return 0;
  if (!ensure_host_dp(w)) return 0;
  if (!prepare(w)) return 0;
  const StepParams P = make_params(w, 0.0f);
  enqueue_keys(w->d, w->n, w->plan, w->stream);
  enqueue_sort_and_ranges(w->d, w->n, P, false, w->stream);
  w->sid_perm_n = w->n;
  w->keys_valid = false;  // the sort consumed the bucket counts
  size_t bytes = 4ull * w->n * (1 + (size_t)max_per);
  if (!ensure_tmp(w, bytes)) return 0;
  uint32_t* dc = (uint32_t*)w->d_tmp;
  uint32_t* dl = dc + w->n;
  enqueue_debug_neighbors(w->d, w->n, P, dc, dl, max_per, w->stream);
  cudaMemcpyAsync(counts, dc, 4ull * w->n, cudaMemcpyDeviceToHost, w->stream);
  cudaMemcpyAsync(lists, dl, 4ull * w->n * max_per, cudaMemcpyDeviceToHost, w->stream);
  if (!cuda_ok(w, cudaStreamSynchronize(w->stream), "debug_neighbors")) return 0;
  return w->n;
}

uint32_t phieng_sph_debug_forces(World2* w, float* fxy, uint32_t max) {
  if (!w || !fxy || w->n == 0 || max < w->n || w->is_batch()) return 0;
  if (!ensure_host_dp(w)) return 0;
  if (!prepare(w)) return 0;
  const StepParams P = make_params(w, 0.0f);
  enqueue_keys(w->d, w->n, w->plan, w->stream);
  enqueue_sort_and_ranges(w->d, w->n, P, false, w->stream);
  w->sid_perm_n = w->n;
  w->keys_valid = false;  // the sort consumed the bucket counts
  enqueue_density(w->d, w->n, P, w->stream);
  if (!ensure_tmp(w, sizeof(float2) * (size_t)w->n)) return 0;
  enqueue_force_integrate(w->d, w->n, P, (float2*)w->d_tmp, w->stream);
  cudaMemcpyAsync(fxy, w->d_tmp, sizeof(float2) * w->n, cudaMemcpyDeviceToHost, w->stream);
  if (!cuda_ok(w, cudaStreamSynchronize(w->stream), "debug_forces")) return 0;
  w->dp_on_device = true;
  return w->n;
}

// ---------------------------------------------------------------- batches
World2* phieng_sph_batch_new(World2* const* worlds, uint32_t count) {
  if (!worlds || count == 0) return nullptr;
  for (uint32_t k = 0; k < count; k++) {
    World2* src = worlds[k];
    if (!src || src->is_batch()) return nullptr;
    const FluidConfig2Ffi& c = src->cfg;
    if (!c.enabled || c.adaptive_resolution || c.boundary_particles || (c.cfl > 0.0f && c.max_substeps > 1))
      return nullptr;
    if (!ensure_host_state(src) || !ensure_host_dp(src)) return nullptr;
  }
  World2* b = new (std::nothrow) World2();
  if (!b) return nullptr;
  uint64_t total = 0;
  for (uint32_t k = 0; k < count; k++) total += worlds[k]->n;
  if (total > 0xFFFFFFFFull) {
    delete b;
    return nullptr;
  }
  b->n = (uint32_t)total;
  b->cap = b->n;
  b->cfg = worlds[0]->cfg;
  b->h_state.reserve(b->n);
  for (uint32_t k = 0; k < count; k++) {
    World2* src = worlds[k];
    World2::Scene sc;
    sc.first = (uint32_t)b->h_state.size();
    sc.count = src->n;
    sc.cfg = src->cfg;
    sc.gx = src->gx;
    sc.gy = src->gy;
    sc.body_first = (uint32_t)b->bodies.size();
    sc.nbodies = (uint32_t)src->bodies.size();
    sc.mass_uniform = src->mass_uniform;
    sc.mass_value = src->mass_value;
    sc.phase_uniform = src->phase_uniform;
    sc.phase_value = src->phase_value;
    b->h_state.insert(b->h_state.end(), src->h_state.begin(), src->h_state.end());
    b->h_mass.insert(b->h_mass.end(), src->h_mass.begin(), src->h_mass.end());
    b->h_phase.insert(b->h_phase.end(), src->h_phase.begin(), src->h_phase.end());
    b->h_dens.insert(b->h_dens.end(), src->h_dens.begin(), src->h_dens.end());
    b->h_pres.insert(b->h_pres.end(), src->h_pres.begin(), src->h_pres.end());
    b->bodies.insert(b->bodies.end(), src->bodies.begin(), src->bodies.end());
    b->scenes.push_back(sc);
  }
  // the per-particle mass / phase arrays are uploaded when any scene needs them
  b->mass_uniform = b->phase_uniform = true;
  for (const auto& sc : b->scenes) {
    b->mass_uniform = b->mass_uniform && sc.mass_uniform;
    b->phase_uniform = b->phase_uniform && sc.phase_uniform;
  }
  return b;
}

uint32_t phieng_sph_batch_scenes(const World2* b) {
  if (!b) return 0;
  return (uint32_t)b->scenes.size();
}

int32_t phieng_sph_batch_scene_range(const World2* b, uint32_t scene, uint32_t* first, uint32_t* count) {
  if (!b || scene >= b->scenes.size() || !first || !count) return 0;
  *first = b->scenes[scene].first;
  *count = b->scenes[scene].count;
  return 1;
}

int32_t phieng_sph_batch_store(World2* b, World2* const* worlds, uint32_t count) {
  if (!b || !b->is_batch() || !worlds || count != b->scenes.size()) return 0;
  for (uint32_t k = 0; k < count; k++)
    if (!worlds[k] || worlds[k]->is_batch() || worlds[k]->n != b->scenes[k].count) return 0;
  if (!ensure_host_state(b) || !ensure_host_dp(b)) return 0;
  for (uint32_t k = 0; k < count; k++) {
    World2* dst = worlds[k];
    const World2::Scene& sc = b->scenes[k];
    if (!ensure_host_state(dst) || !ensure_host_dp(dst)) return 0;
    std::copy(b->h_state.begin() + sc.first, b->h_state.begin() + sc.first + sc.count, dst->h_state.begin());
    dst->bbox_valid = false;
    std::copy(b->h_dens.begin() + sc.first, b->h_dens.begin() + sc.first + sc.count, dst->h_dens.begin());
    std::copy(b->h_pres.begin() + sc.first, b->h_pres.begin() + sc.first + sc.count, dst->h_pres.begin());
    dst->dev_state_valid = false;
    dst->keys_valid = false;
    if (!dst->plan_locked) dst->plan_valid = false;
  }
  return 1;
}

}  // extern "C"
