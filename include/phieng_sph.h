/*
 * phieng_sph.h — C ABI of the B200 SPH fluid library (libphieng_sph.so).
 *
 * The first block re-exports the PhiEng engine's 2D world/fluid entry points
 * with identical signatures and semantics, so a host that drives the
 * reference through its C ABI (crates/engine/src/ffi.rs) can link this
 * library instead for the fluid step. Each declaration cites the reference
 * entry point it replaces. The second block (phieng_sph_*) is additive.
 *
 * World model: the world owns a set of static rigid bodies (walls: boxes and
 * circles) and an SPH fluid whose particle state lives on the GPU. Every
 * entry point tolerates null pointers (no-op / error code), never aborts,
 * and copies caller buffers in or out; no allocation crosses the boundary.
 * Stepping is asynchronous on the world's CUDA stream; every call that
 * returns particle data synchronises that stream first, so observable
 * semantics are synchronous, like the reference's.
 *
 * Not supported by this library (the call fails cleanly instead):
 *  - dynamic bodies (phieng_world_add_body with is_static = 0 returns -1);
 *  - adaptive resolution and boundary ghost particles (the config is
 *    accepted as the reference accepts it, but phieng_world_step then
 *    leaves the world unchanged and phieng_sph_status reports
 *    PHIENG_SPH_E_UNSUPPORTED).
 */
#ifndef PHIENG_SPH_H
#define PHIENG_SPH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Opaque world handle (reference: Box<World2>, ffi.rs:51-54). */
typedef struct World2 World2;

/* Shape tags (ffi.rs:26-28). */
#define PHIENG_SHAPE_CIRCLE 0u
#define PHIENG_SHAPE_BOX 1u
/* Shape2::Polygon (body.rs): accepted by phieng_sph_step_fluid_poly only
 * (the reference's add_body takes circles and boxes). */
#define PHIENG_SHAPE_POLYGON 2u

/* 2D SPH fluid config, #[repr(C)] mirror of FluidConfig2Ffi (ffi.rs:712-739).
 * Rust `bool` fields are one byte (0 or 1). Size 112, align 4. */
typedef struct FluidConfig2Ffi {
  float particle_mass;        /* 0   */
  float rest_density;         /* 4   */
  float smoothing_length;     /* 8   */
  float stiffness;            /* 12  */
  float gamma;                /* 16  */
  float artificial_viscosity; /* 20  */
  float surface_tension;      /* 24  */
  float cfl;                  /* 28  */
  uint32_t max_substeps;      /* 32  */
  uint8_t adaptive_resolution;/* 36  */
  float split_density_ratio;  /* 40  */
  float merge_density_ratio;  /* 44  */
  uint8_t boundary_particles; /* 48  */
  float viscosity;            /* 52  */
  float drag;                 /* 56  */
  float wall_friction;        /* 60  */
  uint8_t phase_count;        /* 64  */
  float phase_rest_density[4];/* 68  */
  float phase_mass[4];        /* 84  */
  float max_velocity;         /* 100 */
  float particle_radius;      /* 104 */
  uint8_t enabled;            /* 108 */
} FluidConfig2Ffi;

#ifdef __cplusplus
static_assert(sizeof(FluidConfig2Ffi) == 112, "FluidConfig2Ffi must match ffi.rs:712-739");
static_assert(offsetof(FluidConfig2Ffi, max_substeps) == 32, "layout");
static_assert(offsetof(FluidConfig2Ffi, split_density_ratio) == 40, "layout");
static_assert(offsetof(FluidConfig2Ffi, viscosity) == 52, "layout");
static_assert(offsetof(FluidConfig2Ffi, phase_count) == 64, "layout");
static_assert(offsetof(FluidConfig2Ffi, phase_rest_density) == 68, "layout");
static_assert(offsetof(FluidConfig2Ffi, phase_mass) == 84, "layout");
static_assert(offsetof(FluidConfig2Ffi, enabled) == 108, "layout");
#endif

/* 2D ambient-force config, #[repr(C)] mirror of AmbientConfig2Ffi
 * (ffi.rs:231-276): spring / drag / wind act on rigid bodies only and are
 * kept for the round trip; the fluid reads the turbulence fields
 * (fluid.rs:1001-1019). Flags are u32 (0 = off). Size 80, align 4. */
typedef struct AmbientConfig2Ffi {
  uint32_t spring_enabled;            /* 0  */
  float spring_ax, spring_ay;         /* 4  */
  float spring_stiffness;             /* 12 */
  float spring_damping;               /* 16 */
  float spring_max_displacement;      /* 20 */
  uint32_t drag_enabled;              /* 24 */
  float drag_linear;                  /* 28 */
  float drag_quadratic;               /* 32 */
  float air_density;                  /* 36 */
  float drag_angular;                 /* 40 */
  float wind_x, wind_y;               /* 44 */
  uint32_t turbulence_enabled;        /* 52 */
  float turbulence_amplitude;         /* 56 */
  float turbulence_frequency;         /* 60 */
  float turbulence_time_scale;        /* 64 */
  uint32_t turbulence_seed;           /* 68 */
  uint32_t turbulence_octaves;        /* 72: stored as min(v, 255); the noise clamps to 1..8 */
  uint32_t turbulence_divergence_free;/* 76 */
} AmbientConfig2Ffi;

#ifdef __cplusplus
static_assert(sizeof(AmbientConfig2Ffi) == 80, "AmbientConfig2Ffi must match ffi.rs:231-276");
static_assert(offsetof(AmbientConfig2Ffi, turbulence_enabled) == 52, "layout");
#endif

/* ---------------- reference entry points (ffi.rs) ---------------- */

/* ffi.rs:51 phieng_world_new — never returns null. No GPU work happens here;
 * device memory is acquired on first use. */
World2* phieng_world_new(void);

/* ffi.rs:62 phieng_world_free — null is a no-op. */
void phieng_world_free(World2* world);

/* ffi.rs:76 phieng_world_step — null, non-finite or non-positive dt is a
 * no-op; dt is clamped to <= 1/15 s. Runs ceil-CFL fluid substeps
 * (fluid.rs:541-588) on the GPU and advances the world clock. */
void phieng_world_step(World2* world, float dt);

/* ffi.rs:89 phieng_world_set_gravity — non-finite components are ignored. */
void phieng_world_set_gravity(World2* world, float gx, float gy);

/* ffi.rs:1067 / 1079 world clock. 1 ok, 0 null or non-finite. */
int32_t phieng_world_set_time(World2* world, float t);
int32_t phieng_world_get_time(World2* world, float* out);

/* ffi.rs:512 phieng_world_set_ambient_config — 1 ok; 0 for a null world or
 * config, a non-finite float, or a negative spring stiffness / damping / max
 * displacement, drag coefficient, air density or turbulence amplitude (world
 * unchanged). Turbulence (enabled and amplitude > 0) adds the reference's
 * value-noise acceleration to every particle in the integrate, sampled at
 * the world clock of the step's start. */
int32_t phieng_world_set_ambient_config(World2* world, const AmbientConfig2Ffi* cfg);

/* ffi.rs:533 phieng_world_get_ambient_config — 1 ok, 0 for null world / out.
 * A new world holds the reference's defaults (ambient.rs: everything off,
 * air density 1, turbulence frequency 1, time scale 1, 3 octaves). */
int32_t phieng_world_get_ambient_config(World2* world, AmbientConfig2Ffi* out);

/* ffi.rs:1123 body count, -1 for null. */
int32_t phieng_world_body_count(World2* world);

/* ffi.rs:1159 phieng_world_add_body — shape_tag PHIENG_SHAPE_CIRCLE
 * (a = radius) or PHIENG_SHAPE_BOX (a, b = half extents), unrotated.
 * Returns the body id, or -1 on invalid input. Static bodies only: a
 * dynamic body (is_static == 0) returns -1 here. friction and restitution
 * are accepted and sanitised as the reference does; the fluid does not
 * read them. */
int32_t phieng_world_add_body(World2* world, float pos_x, float pos_y, uint32_t shape_tag, float a,
                              float b, float density, uint8_t is_static, float friction,
                              float restitution);

/* ffi.rs:1209-1227 BodyDesc2D: blittable body descriptor for
 * phieng_world_add_bodies (36 bytes; is_static is one byte + 3 pad bytes). */
typedef struct BodyDesc2D {
  float pos_x, pos_y;
  uint32_t shape_tag;
  float a, b;
  float density;
  uint8_t is_static;
  uint8_t _pad[3];
  float friction, restitution;
} BodyDesc2D;
#ifdef __cplusplus
static_assert(sizeof(BodyDesc2D) == 36, "BodyDesc2D must match ffi.rs:1209-1227");
#endif

/* ffi.rs:1242 phieng_world_add_bodies — n descriptors validated and added
 * exactly like phieng_world_add_body; out_ids[i] = new id or -1 (rejected,
 * including dynamic bodies here). Returns the number added; 0 for null
 * world / descs / out_ids. n capped at 1,000,000. Non-atomic, as the
 * reference. */
uint32_t phieng_world_add_bodies(World2* world, const BodyDesc2D* descs, uint32_t n, int32_t* out_ids);

/* ffi.rs:999 / 1017 fluid config. set: 1 ok, 0 null or invalid (the
 * validation of fluid2_from_ffi, ffi.rs:773-855; world unchanged on
 * reject). get: 1 ok, 0 null. */
int32_t phieng_world_set_fluid_config(World2* world, const FluidConfig2Ffi* cfg);
int32_t phieng_world_get_fluid_config(World2* world, FluidConfig2Ffi* out);

/* ffi.rs:2486 phieng_world_fluid_add — interleaved [x0,y0,x1,y1,...]; count
 * capped at 1,000,000 per call and by the fluid's particle cap (4096 by
 * default, as MAX_PARTICLES_2D, fluid.rs:30; see phieng_sph_set_particle_cap).
 * Any non-finite input adds nothing (returns 0). Returns the number added. */
uint32_t phieng_world_fluid_add(World2* world, const float* positions, uint32_t count);

/* ffi.rs:2515 phieng_world_fluid_add_phase — as fluid_add, with a phase
 * (0..=3, clamped for the mass/rest-density lookup) per particle. */
uint32_t phieng_world_fluid_add_phase(World2* world, const float* positions, const uint8_t* phases,
                                      uint32_t count);

/* ffi.rs:2546 particle count (0 for null). */
uint32_t phieng_world_fluid_count(const World2* world);

/* ffi.rs:2559 remove all particles; 1 ok, 0 null. */
int32_t phieng_world_fluid_clear(World2* world);

/* ffi.rs:2575 copy out up to `max` quads [x, y, vx, vy] in insertion order;
 * returns the number written (0 on null). Synchronises the world stream. */
uint32_t phieng_world_fluid_get(const World2* world, float* out, uint32_t max);

/* ---------------- extension (no reference counterpart) ---------------- */

/* Error codes reported by phieng_sph_status().error. */
#define PHIENG_SPH_OK 0
#define PHIENG_SPH_E_NO_DEVICE 1   /* no usable CUDA device */
#define PHIENG_SPH_E_CUDA 2        /* a CUDA call failed */
#define PHIENG_SPH_E_UNSUPPORTED 3 /* config enables a feature this library lacks */
#define PHIENG_SPH_E_ARG 4         /* invalid argument */
#define PHIENG_SPH_E_TOO_LARGE 5   /* more particles than phieng_sph_density_noalloc holds */

typedef struct PhiengSphStatus {
  int32_t error;          /* last error (sticky until phieng_sph_clear_error) */
  uint32_t particles;     /* particle count */
  uint64_t substeps;      /* fluid substeps run since creation */
  uint32_t grid_log2_w;   /* bucket grid: columns = 1 << grid_log2_w */
  uint32_t grid_log2_h;   /* rows = 1 << grid_log2_h */
  uint32_t sort_passes;   /* passes of the bucket sort per substep (1) */
  int32_t grid_cx0;       /* bucket grid origin cell: bucket = ((cy - grid_cy0) mod H) * W */
  int32_t grid_cy0;       /*   + ((cx - grid_cx0) mod W), cx = floor(x / h) as i32 */
  uint32_t grid_buckets;  /* buckets of all scenes (a batch has one grid per scene) */
} PhiengSphStatus;

/* Fill *out; 1 ok, 0 null. Does not synchronise. */
int32_t phieng_sph_status(const World2* world, PhiengSphStatus* out);
/* Reset the sticky error; 1 ok, 0 null. */
int32_t phieng_sph_clear_error(World2* world);
/* Human-readable text for the last error (static storage; never null). */
const char* phieng_sph_error_string(const World2* world);

/* Raise (or lower) the fluid's particle cap (default 4096). Particles beyond
 * a lowered cap are kept. 1 ok, 0 null or cap == 0. */
int32_t phieng_sph_set_particle_cap(World2* world, uint32_t cap);

/* Run `steps` world steps of `dt` each (the same as calling
 * phieng_world_step `steps` times) without host round trips; replays a
 * captured CUDA graph when the CFL substep count is fixed. 1 ok, 0 error. */
int32_t phieng_sph_step_n(World2* world, float dt, uint32_t steps);

/* Bind the world to a caller CUDA stream (cudaStream_t passed as void*;
 * null selects the world's own stream). 1 ok, 0 null world. */
int32_t phieng_sph_set_stream(World2* world, void* stream);
/* Block until the world's queued GPU work is done. 1 ok, 0 error. */
int32_t phieng_sph_sync(World2* world);

/* Overwrite position and velocity of the first n particles from quads
 * [x, y, vx, vy] (n <= count). Non-finite input is rejected. 1 ok, 0 error. */
int32_t phieng_sph_set_state(World2* world, const float* xyvv, uint32_t n);

/* Copy out density and pressure of the last substep (insertion order; either
 * pointer may be null). Returns the number written. Synchronises. */
uint32_t phieng_sph_get_density_pressure(const World2* world, float* density, float* pressure,
                                         uint32_t max);

/* Recompute the bucket grid from the current particle bounding box. */
int32_t phieng_sph_replan(World2* world);

/* Fix the bucket grid: 2^log2w x 2^log2h buckets (log2w, log2h >= 2,
 * log2w + log2h <= 24) with origin cell (cx0, cy0). Cells farther apart than
 * the grid share buckets; results are unchanged, only the work grows. Stays
 * in force until phieng_sph_replan. 1 ok, 0 invalid. */
int32_t phieng_sph_set_grid(World2* world, uint32_t log2w, uint32_t log2h, int32_t cx0, int32_t cy0);

/* max_i x_i and max_i |v_i| over the fluid (the per-step readings of the
 * reference's fluid_dam example, fluid_dam.rs:46-52) into out[0], out[1];
 * reduced on the GPU, 8 bytes copied back. 1 ok, 0 error. Synchronises. */
int32_t phieng_sph_front_metrics(World2* world, float* out);
/* The same reduction without waiting: enqueues it and an 8-byte copy of its
 * raw result into raw[0..1] (host memory, page-locked for the copy to be
 * asynchronous) on the world's stream, and returns at once. raw must stay
 * valid until the stream has passed the copy (phieng_sph_sync, or any call
 * that synchronises: phieng_world_fluid_get). A host that reads a metric
 * every step can so keep the GPU busy with the next steps meanwhile.
 * phieng_sph_front_metrics_decode turns raw into (max x, max |v|). 1 ok,
 * 0 error. No counterpart in the reference. */
int32_t phieng_sph_front_metrics_async(World2* world, uint32_t* raw);
void phieng_sph_front_metrics_decode(const uint32_t* raw, float* out);

/* Record CUDA events between the substep phases (sort + ranges, density,
 * force + integrate) of every following substep. 1 ok, 0 error. */
int32_t phieng_sph_set_profiling(World2* world, int32_t on);
/* Milliseconds of each phase of the most recent substep (3 values);
 * returns the count written, 0 if profiling is off. Synchronises. */
uint32_t phieng_sph_phase_times(World2* world, float* ms, uint32_t max);

/* Density and pressure of n particles (phase 0) at the positions xy
 * (device memory, interleaved [x0, y0, x1, y1, ...]) into density[n] and
 * pressure[n] (device memory, input order), computed as one density pass of
 * the fluid step under cfg, on `stream` (a cudaStream_t; null = legacy
 * default stream). No counterpart in the reference: it exists for callers
 * that must not allocate GPU memory while they run, such as a game engine's
 * simulation thread, where cudaMalloc can synchronise the device and stall
 * the frame, or a host that reserves all its GPU memory up front. It
 * allocates nothing: all scratch lives in one fixed device array of about
 * 6 MiB inside this library (held on every GPU that loads it until exit),
 * which limits n to 65536 (more returns PHIENG_SPH_E_TOO_LARGE). The first
 * call on a device resolves that array's address; make it before any stream
 * capture. The address is kept per device for the life of the process: after
 * cudaDeviceReset the process must be restarted before the next call. Calls
 * share the array, so calls whose GPU work overlaps race: order them on the
 * device. Every call blocks the calling thread once, until `stream` has
 * finished the particles' bounding-box pass (a 20-byte read-back that sizes
 * the bucket grid); the remaining work is queued on `stream` when it returns.
 * Every particle is phase 0 (cfg's phase_rest_density[0] and phase_mass[0]).
 * Returns PHIENG_SPH_OK or an error code. */
int32_t phieng_sph_density_noalloc(const float* xy, uint32_t n, const FluidConfig2Ffi* cfg, float* density,
                                   float* pressure, void* stream);

/* ---- batches of independent scenes ----
 * A batch is a World2 holding copies of `count` worlds (particles, static
 * bodies, fluid config, gravity) as independent scenes that advance together:
 * phieng_world_step(batch, dt) runs one fluid substep of dt in every scene
 * (one CUDA graph for the whole batch; each scene's results are those of
 * stepping that world alone). Scenes may differ in size, walls, gravity and
 * config; CFL substepping is not available in a batch. phieng_world_fluid_get
 * returns all particles in scene order; particle-adding, clearing, config,
 * gravity and body calls fail on a batch. Returns null if any world is null,
 * is itself a batch, uses CFL substeps or an unsupported feature. */
World2* phieng_sph_batch_new(World2* const* worlds, uint32_t count);
uint32_t phieng_sph_batch_scenes(const World2* batch);
/* Particle range [first, first + count) of one scene. 1 ok, 0 invalid. */
int32_t phieng_sph_batch_scene_range(const World2* batch, uint32_t scene, uint32_t* first, uint32_t* count);
/* Copy every scene's particle state (and density / pressure) back into the
 * worlds it came from (same order and sizes). 1 ok, 0 invalid. */
int32_t phieng_sph_batch_store(World2* batch, World2* const* worlds, uint32_t count);

/* ---- launch tuning (additive) ----
 * Launch shapes that change speed, never results (the neighbour visit order
 * and every sum stay the same). phi_eng_b200/autotune.py picks them per GPU
 * and workload. */
typedef struct PhiengSphTuning {
  uint32_t density_block;     /* threads per block of the density pass: 64, 128, 256 (default 256) */
  uint32_t force_block;       /* threads per block of the force pass: 64, 128, 256 (default 256) */
  float buckets_per_particle; /* bucket-grid budget per particle, 0.125..16 (default 2) */
  uint32_t stage;             /* tolerance mode: bit 0 = the density pass stages its neighbour rows in
                                 shared memory, bit 1 = the force pass does, bit 2 = the force pass
                                 reassigns each block's particles to its lanes by neighbour count
                                 (ignored with bit 1); 0..7, default 0; no effect on results */
} PhiengSphTuning;

/* 1 ok, 0 null or out of range (world unchanged). Replans the bucket grid
 * unless phieng_sph_set_grid fixed it. */
int32_t phieng_sph_set_tuning(World2* world, const PhiengSphTuning* tuning);
int32_t phieng_sph_get_tuning(const World2* world, PhiengSphTuning* out);

/* ---- arithmetic mode of the density and force passes (additive) ----
 * EXACT (default): every pair term in the reference's f32 expression order
 * with IEEE division and square root (fluid.rs:265-297, 592-611, 942-1050):
 * bit-identical to the reference's arithmetic in the Jacobi integrate order.
 * TOLERANCE: for the plain flag set (uniform mass and phase, XSPH on, no
 * artificial viscosity, cohesion, turbulence, ghosts or polygons) the force
 * and XSPH sums are reassociated with fused multiply-adds, one approximate
 * reciprocal square root and one approximate reciprocal per neighbour pair;
 * the density pass stays exact (bit-identical). Neighbour sets, sort
 * order and visit order stay exact and runs stay bit-reproducible; from
 * identical state, density agrees with the exact mode within 1e-5 and force
 * within 1e-4 of their RMS. Other flag sets run the exact passes in either
 * mode. */
#define PHIENG_SPH_EXACT 0u
#define PHIENG_SPH_TOLERANCE 1u
/* 1 ok, 0 null or an unknown mode (world unchanged). */
int32_t phieng_sph_set_precision(World2* world, uint32_t mode);
uint32_t phieng_sph_get_precision(const World2* world);

/* ---- device-resident state (additive; callers that keep data on the GPU) ----
 * Pointers are CUDA device pointers on the world's device; the copies are
 * ordered on the world's stream. */

/* Copy up to max particles' [x, y, vx, vy] (insertion order) into dst.
 * Returns the count copied. */
uint32_t phieng_sph_get_state_device(World2* world, float* dst, uint32_t max);
/* Overwrite the state of all n = fluid_count particles from src. 1 ok, 0 on
 * a count mismatch or null. Works on batches. */
int32_t phieng_sph_set_state_device(World2* world, const float* src, uint32_t n);
/* Replace every particle by n phase-0 particles whose [x, y, vx, vy] come
 * from src (device); n <= the particle cap. 1 ok, 0 otherwise. */
int32_t phieng_sph_load_state_device(World2* world, const float* src, uint32_t n);

/* ---- x-slab decomposition of one scene over ranks (additive) ----
 * A rank world holds own_cap owned slots, then 2 halo_cap halo slots for the
 * left side and 2 halo_cap for the right (n = own_cap + 4 halo_cap, loaded
 * with phieng_sph_load_state_device); an unused slot holds [NaN, NaN, 0, 0]
 * and the order tag PHIENG_SPH_SLAB_FREE. Once before the first step the
 * host calls pack(0), moves each send buffer to the neighbour's receive
 * buffer (point-to-point, whole buffers: the count travels inside) and calls
 * unpack(0); then every substep is phieng_world_step, pack(1), the same
 * exchange, unpack(1): one exchange per substep carries the particles that
 * left the slab and the halo of those that stayed. Everything is ordered on
 * the world's stream and nothing is read on the host, so with NCCL on that
 * stream a substep never synchronises. The owned particles' results are
 * bit-identical to the single-domain step's. Global ids are below 2^31 - 1;
 * a particle moves less than one cell column per substep. */
#define PHIENG_SPH_SLAB_FREE 0xFFFFFFFFu
/* Bytes of one exchange buffer for halo_cap rows: header (count, overflow
 * flag, 2 x 0; uint32), float [halo_cap][4] states, uint32 [halo_cap] tags. */
#define PHIENG_SPH_SLAB_BUFFER_BYTES(halo_cap) (16u + 20u * (uint32_t)(halo_cap))
/* Per-particle order tags (n = fluid_count values; host or device memory):
 * each cell's particles are visited in ascending tag instead of ascending
 * index. Tags of finite particles must be distinct; with the global ids of
 * the single domain, a world that holds any subset of its particles in any
 * order visits neighbours in the single domain's order. Cleared when the
 * particle buffers are reallocated. 1 ok, 0 otherwise. */
int32_t phieng_sph_set_order(World2* world, const uint32_t* tags, uint32_t n);
/* Make the world a slab rank: owned cell columns [lo, hi) (column =
 * floor(x / smoothing_length)), neighbours bit 0 = left rank exists, bit 1 =
 * right (with both, hi - lo >= 4); device buffers of
 * PHIENG_SPH_SLAB_BUFFER_BYTES(halo_cap) each (a side without a neighbour
 * may pass null). Requires order tags, one substep per step (cfl 0 or
 * max_substeps 1), no adaptive resolution or ghosts. Owned slots whose tag is
 * PHIENG_SPH_SLAB_FREE form the free-slot stack. */
int32_t phieng_sph_slab_setup(World2* world, int32_t lo, int32_t hi, uint32_t neighbours, uint32_t own_cap,
                              uint32_t halo_cap, void* send_left, void* send_right, const void* recv_left,
                              const void* recv_right);
/* phase 1 (after a step): owned particles whose column left [lo, hi) into
 * that side's send buffer as migrants (their slots freed), the others within
 * two cell columns of a shared edge as halo; phase 0 (before the first step):
 * the halo only. */
int32_t phieng_sph_slab_pack(World2* world, uint32_t phase);
/* After the exchange: received migrants into free owned slots, each side's
 * halo (its received halo rows and this rank's own migrants to that side)
 * into the halo slots, the others emptied. A buffer that overflowed or a
 * full owned region sets the slab error that phieng_sph_slab_status
 * reports. */
int32_t phieng_sph_slab_unpack(World2* world, uint32_t phase);
/* *out (device float) = max |v| over the owned particles (for the ranks'
 * all-reduce of the CFL substep count). */
int32_t phieng_sph_slab_vmax(World2* world, float* out);
/* Synchronise; 1 if no exchange overflowed since set-up, else 0. */
int32_t phieng_sph_slab_status(World2* world);
/* Synchronise; the owned particles' [x, y, vx, vy] and tags (host buffers,
 * up to max rows, slot order). Returns the number of owned particles. */
uint32_t phieng_sph_slab_owned(World2* world, float* state, uint32_t* tags, uint32_t max);

/* ---- learned closure (additive; no reference counterpart) ----
 * A per-particle network 16 -> 64 -> 64 -> 2 (SiLU, BF16 weights on the
 * tensor cores, FP32 accumulate) predicts the displacement correction that
 * lets one substep of ratio * dt_fine track ratio plain substeps of dt_fine.
 * Parameters: one flat FP32 vector of PHIENG_MLP_PARAMS values,
 *   W1[64][16] | b1[64] | W2[64][64] | b2[64] | W3[2][64] | b3[2]
 * (W[out][in]), and PHIENG_MLP_NORM normalisation values
 *   mu[16] | isd[16] | out_scale[2]
 * (input x_hat = (x - mu) * isd; output = network * out_scale, in units of
 * the smoothing length). */
#define PHIENG_MLP_PARAMS 5378u
#define PHIENG_MLP_NORM 34u
#define PHIENG_MLP_FEATURES 16u

typedef struct PhiengMlp PhiengMlp;

/* New network on the current CUDA device: hidden layers U(-1/sqrt(fan_in),
 * 1/sqrt(fan_in)) from SplitMix64(seed), output layer zero, identity
 * normalisation. Never null; check phieng_mlp_status. */
PhiengMlp* phieng_mlp_new(uint64_t seed);
void phieng_mlp_free(PhiengMlp* mlp);
/* PHIENG_SPH_OK or the first error. */
int32_t phieng_mlp_status(const PhiengMlp* mlp);
/* Stream for the network's work (null: its own stream). */
int32_t phieng_mlp_set_stream(PhiengMlp* mlp, void* stream);
/* Host copies of the parameters / normalisation (either may be null). */
int32_t phieng_mlp_get_params(PhiengMlp* mlp, float* params, float* norm);
/* Load parameters and normalisation; resets the Adam state and step count. */
int32_t phieng_mlp_set_params(PhiengMlp* mlp, const float* params, const float* norm);
/* Adam steps taken since the last set_params. */
uint32_t phieng_mlp_step_count(PhiengMlp* mlp);
/* y[n][2] = network(x[n][16]) (device pointers), asynchronous. */
int32_t phieng_mlp_forward(PhiengMlp* mlp, const float* x, uint32_t n, float* y);
/* The same forward pass on the 5th-generation tensor cores (tcgen05.mma
 * with TMEM accumulators, 128 particles per CTA), same layer numerics:
 * results agree with phieng_mlp_forward within the network's tolerance,
 * not bit for bit (the tensor core's accumulation order differs).
 * Asynchronous; its waits for the tensor core are bounded, and one that
 * runs out is reported by phieng_mlp_check_waits. */
int32_t phieng_mlp_forward_tc(PhiengMlp* mlp, const float* x, uint32_t n, float* y);
/* Synchronise the network's stream; 1 if no bounded wait of a tcgen05 kernel
 * ran out since creation, else 0 (and the network reports
 * PHIENG_SPH_E_CUDA). */
int32_t phieng_mlp_check_waits(PhiengMlp* mlp);
/* Loss and gradient (host buffers, PHIENG_MLP_PARAMS values) of the minibatch
 * that training step `iter` with `seed` would draw from the npairs pairs
 * (x[npairs][16], t[npairs][2], device); batch a multiple of 128. */
int32_t phieng_mlp_grad(PhiengMlp* mlp, const float* x, const float* t, uint32_t npairs, uint32_t batch,
                        uint64_t seed, uint32_t iter, float* grad, float* loss);
/* iters Adam steps (beta 0.9 / 0.999, eps 1e-8, learning rate lr) on
 * minibatches of `batch` pairs; loss_hist (host, iters values) may be null. */
int32_t phieng_mlp_train(PhiengMlp* mlp, const float* x, const float* t, uint32_t npairs, uint32_t batch,
                         uint32_t iters, float lr, uint64_t seed, float* loss_hist);
/* Data-parallel training, one rank's share of an iteration (asynchronous on
 * the network's stream; x, t, grad on the device): grad[PHIENG_MLP_PARAMS + 1]
 * = the gradient over samples [first, first + batch) of the total-sample
 * minibatch that Adam step phieng_mlp_step_count() draws with `seed` (the
 * sampling of phieng_mlp_train; each sample's dL/dy carries 1 / total), then
 * those samples' sum of squared errors. Summed over ranks whose slices tile
 * [0, total) (an all-reduce), it is the minibatch gradient, and the loss is
 * the last entry / (2 total). batch a multiple of 128, first + batch <= total. */
int32_t phieng_mlp_shard_grad(PhiengMlp* mlp, const float* x, const float* t, uint32_t npairs, uint32_t first,
                              uint32_t batch, uint32_t total, uint64_t seed, float* grad);
/* One Adam step (as phieng_mlp_train's) from a device gradient laid out as
 * phieng_mlp_shard_grad writes it; asynchronous. Ranks that apply the same
 * all-reduced gradient keep bit-identical parameters. */
int32_t phieng_mlp_apply_grad(PhiengMlp* mlp, const float* grad, float lr);
/* Tensor-core path of phieng_mlp_grad / phieng_mlp_train (default
 * PHIENG_MLP_TCGEN05). Both draw the
 * same minibatches and round at the same points (BF16 / FP16 operands, f32
 * accumulation); their gradients agree within the network's tolerance, not
 * bit for bit (different accumulation order). Each is bit-reproducible.
 *   PHIENG_MLP_TCGEN05   5th-generation tensor cores: per 128-sample round
 *                        the forward layers, dH1 = dZ2 W2 and one weight-
 *                        gradient GEMM (both hidden layers' weights and
 *                        biases, accumulated in TMEM over the CTA's rounds)
 *                        as tcgen05.mma chains; bounded waits, reported
 *                        like phieng_mlp_check_waits (the call returns 0)
 *   PHIENG_MLP_MMA_SYNC  warp-level mma.sync m16n8k16 tiles */
#define PHIENG_MLP_TCGEN05 0
#define PHIENG_MLP_MMA_SYNC 1
int32_t phieng_mlp_set_train_engine(PhiengMlp* mlp, int32_t engine);
/* The current training path (-1 for a null network). */
int32_t phieng_mlp_get_train_engine(const PhiengMlp* mlp);
/* Network of the tolerance-mode coarse pass of phieng_sph_closure_step
 * (PHIENG_SPH_TOLERANCE worlds with the plain flag set): PHIENG_MLP_MMA_SYNC
 * (default: 256-particle blocks, warp-level mma.sync tiles; 132 us per
 * coarse pass at 2^20 particles on B200) or PHIENG_MLP_TCGEN05 (one
 * persistent pass, 128-particle tiles through the tcgen05 tensor cores; 167
 * us: each tile's three dependent MMA round trips are latency-bound). The
 * same numerics; results agree within the network's tolerance. The exact
 * mode's coarse pass always uses mma.sync. */
int32_t phieng_mlp_set_closure_engine(PhiengMlp* mlp, int32_t engine);
int32_t phieng_mlp_get_closure_engine(const PhiengMlp* mlp);
/* The pair indices of one minibatch (device idx[batch]). */
int32_t phieng_mlp_sample_indices(uint32_t npairs, uint32_t batch, uint64_t seed, uint32_t iter, uint32_t* idx,
                                  void* stream);
/* Add uniform noise in [-amp, amp] to x and y of every particle of a [n][4]
 * device state (deterministic in seed): perturbed states for training pairs. */
int32_t phieng_mlp_perturb(float* state, uint32_t n, float amp, uint64_t seed, void* stream);
/* Training targets per particle from two [n][4] states (device): mode 0
 * (x_fine - x_coarse) * inv_h, mode 1 (v_fine - v_coarse) * dt * inv_h,
 * mode 2 their mean (dt = the coarse step). */
int32_t phieng_mlp_targets(const float* fine, const float* coarse, uint32_t n, float inv_h, float dt, uint32_t mode,
                           float* out, void* stream);

/* Closure inputs of every particle at the current state for a substep of dt
 * (device feat[n][16], insertion order). The state is unchanged. */
int32_t phieng_sph_features(World2* world, float dt, float* feat);

#define PHIENG_CLOSURE_JUMP 0u        /* max_i (rho_i after - rho_i before) / rho0 */
#define PHIENG_CLOSURE_COMPRESSION 1u /* max_i rho_i after / rho0 - 1 */
#define PHIENG_CLOSURE_GROWTH 2u      /* (max_i rho_i after - max_i rho_i before) / rho0 */

/* Attach a network (null detaches) for phieng_sph_closure_step: each coarse
 * step is one substep of ratio * dt_fine with the network's correction; a
 * coarse step whose density check exceeds threshold is undone and replaced
 * by ratio plain substeps of dt_fine. The world keeps the pointer. */
int32_t phieng_sph_set_closure(World2* world, PhiengMlp* mlp, uint32_t ratio, float threshold, uint32_t criterion);

typedef struct PhiengClosureStats {
  uint32_t coarse_steps; /* coarse steps attempted */
  uint32_t accepted;     /* kept */
  uint32_t fallbacks;    /* replaced by plain substeps */
  uint32_t reserved;
  float last_check;      /* density check of the last coarse step */
  float max_check;       /* largest check seen */
} PhiengClosureStats;

/* Advance by `coarse_steps` x ratio x dt_fine (no CFL substeps; on a batch
 * every scene advances and the check and fallback act on the whole batch).
 * stats (may be null) accumulates. 1 ok, 0 on error. */
int32_t phieng_sph_closure_step(World2* world, float dt_fine, uint32_t coarse_steps, PhiengClosureStats* stats);

/* ---- diagnostics used by the parity tests ---- */

/* Run the density + force passes of one substep on the current state without
 * integrating; write per-particle force [fx, fy] (insertion order, the
 * scratch forces of fluid.rs:942-997) and refresh density/pressure.
 * Returns the number written. */
uint32_t phieng_sph_debug_forces(World2* world, float* fxy, uint32_t max);

/* Run one bucket scan in which the first tile never publishes its prefix
 * (the grid must span at least two look-back blocks of the bucket scan,
 * i.e. more than 4096 buckets): the other blocks' bounded
 * look-back waits run out, the device flag is set and read back, and the
 * world reports PHIENG_SPH_E_CUDA. Returns 1 if no wait ran out (then the
 * bound failed to trigger), 0 otherwise. Test hook for the bounded waits. */
int32_t phieng_sph_debug_scan_timeout(World2* world);

/* Rebuild the grid from the current state and write the sorted order:
 * ids[s] = particle id at sorted slot s, keys[s] = its bucket key (either may
 * be null). Returns n. */
uint32_t phieng_sph_debug_sorted(World2* world, uint32_t* ids, uint32_t* keys, uint32_t max);

/* Rebuild the grid and write each particle's neighbour list in visit order
 * (fluid.rs:368-386): counts[i] (total found) and lists[i*max_per + k] for
 * k < min(counts[i], max_per). Returns n. */
uint32_t phieng_sph_debug_neighbors(World2* world, uint32_t* counts, uint32_t* lists,
                                    uint32_t max_per, uint32_t max);

/* Particle masses by id (set at insertion; merges and splits of adaptive
 * resolution change them). Returns the particle count; writes up to max. */
uint32_t phieng_sph_fluid_masses(World2* world, float* out, uint32_t max);

/* Boundary ghosts (FluidConfig2Ffi.boundary_particles, fluid.rs:617-818):
 * the count of the last generated set, and up to max positions (x, y pairs,
 * grouped by grid cell, generation order inside a cell) into xy (may be
 * null); *regens (may be null) = how many times they were generated
 * (boundary_regens: once per change of the static bodies or of h, mass, rest
 * density). 0 for a null world. */
uint32_t phieng_sph_ghosts(World2* world, float* xy, uint32_t max, uint64_t* regens);

/* Allocate the device arrays for n particles now (as std::vector::reserve),
 * and the bucket arrays of the largest grid a plan for n particles can use,
 * so the first step allocates nothing. 1 ok, 0 for a null world, a batch, no
 * device or an allocation error. */
int32_t phieng_sph_reserve(World2* world, uint32_t n);

/* ---- the fluid phase with the engine's rigid bodies (two-way coupling) ----
 * A rigid body as the fluid phase sees it (RigidBody2, body.rs:560-700):
 * shape, transform, velocity and inverse mass / inertia. 60 bytes. */
typedef struct PhiengBody2 {
  uint32_t shape_tag;        /* PHIENG_SHAPE_CIRCLE (a = radius), PHIENG_SHAPE_BOX (a, b = half extents) or
                                PHIENG_SHAPE_POLYGON (phieng_sph_step_fluid_poly) */
  float a, b;
  float px, py;              /* transform.position */
  float xax, xay, yax, yay;  /* transform.rotation columns x_axis, y_axis */
  float vx, vy, w;           /* velocity, angular velocity: updated for dynamic bodies */
  float inv_mass, inv_inertia;
  uint8_t is_static;         /* statics take no reaction */
  uint8_t is_sleeping;       /* cleared when the fluid pushes or floats the body */
  uint8_t _pad[2];
} PhiengBody2;
#ifdef __cplusplus
static_assert(sizeof(PhiengBody2) == 60, "PhiengBody2 layout");
#endif

/* FluidState2::step_fluid(bodies, gravity, ambient, time, dt) (fluid.rs:541-557),
 * the fluid phase of World2::step_inner (world.rs:843-849): CFL substeps of
 * the world's fluid against `bodies` in their order (in place of the world's
 * own static bodies), with the reactions of fluid.rs:1056-1094 (impulse
 * n * (vn * m) and the no-slip reaction on each body, applied in particle
 * order) and the buoyancy + drag pass of fluid.rs:1103-1135 on dynamic
 * circles and boxes; vx, vy, w and is_sleeping of `bodies` are updated in
 * place. The world's ambient config applies as World2::step_inner passes
 * it: turbulence at the world clock (phieng_world_set_time), the wind in the
 * buoyancy drag (fluid.rs:1121-1124). Does not advance the world clock and
 * does not clamp dt (the caller's World2::step does both).
 * 1 ok; 0 for a null world, a batch, a body with an unknown shape or a
 * non-finite field, more than 65536 bodies, or an error (phieng_sph_status). */
int32_t phieng_sph_step_fluid(World2* world, PhiengBody2* bodies, uint32_t nbodies, float dt);

/* phieng_sph_step_fluid with polygon bodies as well: a body with shape_tag
 * PHIENG_SHAPE_POLYGON (a, b unused) has poly_count[k] >= 3 vertices in its
 * own frame at poly_xy[2 * poly_first[k] ...] (Shape2::Polygon; the arrays
 * are indexed by body and read for polygons only). The fluid tests it as
 * fluid.rs:518-530 does: the vertices moved by the body's transform, SAT
 * circle-polygon (collision/src/sat.rs:104-200), the axis oriented from the
 * vertex centroid to the particle, contact point particle - normal * r.
 * Polygons are impulse-coupled only, as in the reference: no buoyancy
 * samples (fluid.rs:415-418). Each particle tests every polygon (a non-convex
 * polygon's SAT can report a contact outside its bounding box, so no box
 * reject applies). 0 also for a polygon with fewer than 3 vertices, a vertex
 * range outside poly_nverts or a non-finite vertex. */
int32_t phieng_sph_step_fluid_poly(World2* world, PhiengBody2* bodies, uint32_t nbodies, const float* poly_xy,
                                   const uint32_t* poly_first, const uint32_t* poly_count, uint32_t poly_nverts,
                                   float dt);

/* ---- snapshot fluid block (crates/dynamics/src/snapshot.rs) ----
 * The fluid section of the reference's binary world snapshot: config, then
 * per particle position, velocity, mass and phase, little-endian, in the
 * layout of encode_fluid2 (snapshot.rs:6478) for schema `version` (1 ..
 * PHIENG_SNAPSHOT_SCHEMA; schema 5 and later carry the EOS / CFL / phase
 * fields). A host that writes or reads world snapshots splices this block
 * where the reference's encode_world2 / decode place the fluid. */
#define PHIENG_SNAPSHOT_SCHEMA 17u

/* Encode the world's fluid. Returns the block size in bytes and writes it to
 * out when out is not null and cap >= the size; -1 for a null world, a batch
 * or an unknown version. */
int64_t phieng_sph_fluid_block_save(World2* world, uint32_t version, uint8_t* out, uint64_t cap);
/* Replace the world's fluid config and particles by a decoded block with the
 * rules of the reference's load (apply_fluid2, snapshot.rs:4471): finite
 * config scalars and particle values, at most the particle cap (4096 by
 * default), a single phase resets the phase tables, mass = stored mass if
 * positive else particle_mass, density = rest_density and pressure = 0 until
 * the next step. Continuing to step after a save and a load is bit-identical
 * to never having saved. Returns the bytes consumed; -1 for null / bad
 * version; -2 for a malformed block (the world is then unchanged). */
int64_t phieng_sph_fluid_block_load(World2* world, uint32_t version, const uint8_t* data, uint64_t len);

/* ======================================================================
 * 3D SPH world (crates/dynamics/src/fluid3.rs behind ffi.rs:3199-3885).
 * The fluid step of World3 with static sphere / box / capsule walls; the
 * other World3 subsystems (rigid dynamics, joints, queries) are not part
 * of this library.
 * ====================================================================== */

/* Opaque 3D world handle (reference: Box<World3>, ffi.rs:3199). */
typedef struct World3 World3;

/* 3D shape tags (ffi.rs:3192-3195). */
#define PHIENG_SHAPE3_SPHERE 0u
#define PHIENG_SHAPE3_BOX 1u
#define PHIENG_SHAPE3_CAPSULE 2u

/* FluidConfig3Ffi (ffi.rs:744-767) has the fields, layout, defaults
 * (fluid3.rs:108-135) and validation (fluid3_from_ffi, ffi.rs:857) of
 * the 2D config. */
typedef FluidConfig2Ffi FluidConfig3Ffi;

/* ffi.rs:3199 / 3209: create / destroy (free(NULL) is a no-op). Gravity
 * starts at (0, -9.81, 0), the clock at 0. */
World3* phieng_world3_new(void);
void phieng_world3_free(World3* world);

/* ffi.rs:3221: advance by min(dt, 1/15); ignored for null, non-finite or
 * dt <= 0. The fluid phase runs its CFL substeps; the clock advances by dt. */
void phieng_world3_step(World3* world, float dt);

/* ffi.rs:3234: gravity (ignored when any component is non-finite). */
void phieng_world3_set_gravity(World3* world, float gx, float gy, float gz);

/* ffi.rs:1091 / 1106: clock. 1 ok, 0 null or non-finite. */
int32_t phieng_world3_set_time(World3* world, float t);
int32_t phieng_world3_get_time(World3* world, float* out);

/* ffi.rs:3387: number of bodies, -1 for null. */
int32_t phieng_world3_body_count(World3* world);

/* 3D ambient-force config, #[repr(C)] mirror of AmbientConfig3Ffi
 * (ffi.rs:278-326): as AmbientConfig2Ffi with 3D anchor and wind. Size 88,
 * align 4. */
typedef struct AmbientConfig3Ffi {
  uint32_t spring_enabled;                 /* 0  */
  float spring_ax, spring_ay, spring_az;   /* 4  */
  float spring_stiffness;                  /* 16 */
  float spring_damping;                    /* 20 */
  float spring_max_displacement;           /* 24 */
  uint32_t drag_enabled;                   /* 28 */
  float drag_linear;                       /* 32 */
  float drag_quadratic;                    /* 36 */
  float air_density;                       /* 40 */
  float drag_angular;                      /* 44 */
  float wind_x, wind_y, wind_z;            /* 48 */
  uint32_t turbulence_enabled;             /* 60 */
  float turbulence_amplitude;              /* 64 */
  float turbulence_frequency;              /* 68 */
  float turbulence_time_scale;             /* 72 */
  uint32_t turbulence_seed;                /* 76 */
  uint32_t turbulence_octaves;             /* 80 */
  uint32_t turbulence_divergence_free;     /* 84 */
} AmbientConfig3Ffi;

#ifdef __cplusplus
static_assert(sizeof(AmbientConfig3Ffi) == 88, "AmbientConfig3Ffi must match ffi.rs:278-326");
static_assert(offsetof(AmbientConfig3Ffi, turbulence_enabled) == 60, "layout");
#endif

/* 3D boundary ghosts (fluid3.rs:719-922), as phieng_sph_ghosts: count,
 * up to max (x, y, z) triples (cell-grouped), generation count. */
uint32_t phieng_sph3_ghosts(World3* world, float* xyz, uint32_t max, uint64_t* regens);

/* 3D particle masses by id (adaptive resolution changes them), as
 * phieng_sph_fluid_masses. */
uint32_t phieng_sph3_fluid_masses(World3* world, float* out, uint32_t max);

/* ffi.rs:549 / 568 phieng_world3_set/get_ambient_config — as the 2D pair
 * (ambient3_from_ffi, ffi.rs:414-475); turbulence acts on the 3D fluid
 * (fluid3.rs:1090-1108). */
int32_t phieng_world3_set_ambient_config(World3* world, const AmbientConfig3Ffi* cfg);
int32_t phieng_world3_get_ambient_config(World3* world, AmbientConfig3Ffi* out);

/* ffi.rs:3703 phieng_world3_add_body — PHIENG_SHAPE3_SPHERE (a = radius),
 * PHIENG_SHAPE3_BOX (a, b, c = half extents), PHIENG_SHAPE3_CAPSULE (a =
 * radius, b = half length along y); at (pos_x, pos_y, pos_z) with the
 * identity rotation. Returns the body id or -1 on invalid input. Static
 * bodies only: is_static == 0 returns -1 here. */
int32_t phieng_world3_add_body(World3* world, float pos_x, float pos_y, float pos_z, uint32_t shape_tag,
                               float a, float b, float c, float density, uint8_t is_static, float friction,
                               float restitution);

/* ffi.rs:3767-3786 BodyDesc3D (44 bytes). */
typedef struct BodyDesc3D {
  float pos_x, pos_y, pos_z;
  uint32_t shape_tag;
  float a, b, c;
  float density;
  uint8_t is_static;
  uint8_t _pad[3];
  float friction, restitution;
} BodyDesc3D;
#ifdef __cplusplus
static_assert(sizeof(BodyDesc3D) == 44, "BodyDesc3D must match ffi.rs:3767-3786");
#endif

/* ffi.rs:3801 phieng_world3_add_bodies — each descriptor as
 * phieng_world3_add_body; out_ids[i] = id or -1. Returns the number added,
 * 0 for null world / descs / out_ids; n capped at 1,000,000. */
uint32_t phieng_world3_add_bodies(World3* world, const BodyDesc3D* descs, uint32_t n, int32_t* out_ids);

/* ffi.rs:1032 / 1050: fluid config. set: 1 ok, 0 null or invalid (world
 * unchanged). get: 1 ok, 0 null. */
int32_t phieng_world3_set_fluid_config(World3* world, const FluidConfig3Ffi* cfg);
int32_t phieng_world3_get_fluid_config(World3* world, FluidConfig3Ffi* out);

/* ffi.rs:3579 / 3609: add `count` particles from xyz triples (phase 0, or
 * the given phases); 0 when any of the first min(count, 1e6) triples is
 * non-finite or a pointer is null; at most 4096 particles in total (the
 * reference's MAX_PARTICLES_3D; phieng_sph3_set_particle_cap raises it).
 * Returns the number added. */
uint32_t phieng_world3_fluid_add(World3* world, const float* positions, uint32_t count);
uint32_t phieng_world3_fluid_add_phase(World3* world, const float* positions, const uint8_t* phases,
                                       uint32_t count);

/* ffi.rs:3643 / 3656 / 3672: count, clear (1 ok, 0 null), and state out as
 * [x, y, z, vx, vy, vz] sextuples (returns the number written). */
uint32_t phieng_world3_fluid_count(const World3* world);
int32_t phieng_world3_fluid_clear(World3* world);
uint32_t phieng_world3_fluid_get(const World3* world, float* out, uint32_t max);

/* The 3D fluid block (encode_fluid3 / apply_fluid3, snapshot.rs:6662,
 * :4545): as the 2D one with z components. */
int64_t phieng_sph3_fluid_block_save(World3* world, uint32_t version, uint8_t* out, uint64_t cap);
int64_t phieng_sph3_fluid_block_load(World3* world, uint32_t version, const uint8_t* data, uint64_t len);

/* ---- the 3D fluid phase with the engine's rigid bodies (two-way coupling) ----
 * A rigid body as the 3D fluid phase sees it (RigidBody3, body.rs:902-956):
 * shape, transform (position and unit-quaternion rotation), velocity,
 * angular velocity (world frame), inverse mass and the body-frame inverse
 * inertia tensor. 112 bytes. */
#define PHIENG_SHAPE3_HULL 3u /* Shape3::ConvexHull / ConvexMesh vertices (phieng_sph3_step_fluid_hull only) */
typedef struct PhiengBody3 {
  uint32_t shape_tag;       /* PHIENG_SHAPE3_SPHERE (a = radius), _BOX (a, b, c = half extents), _CAPSULE (a =
                               radius, b = half length along the body's y axis) or _HULL */
  float a, b, c;
  float px, py, pz;         /* transform.position */
  float qx, qy, qz, qw;     /* transform.rotation */
  float vx, vy, vz;         /* velocity: updated for dynamic bodies */
  float wx, wy, wz;         /* angular velocity: updated for dynamic bodies */
  float inv_mass;
  float inv_inertia[9];     /* body-frame inverse inertia (glam Mat3, column-major: x_axis, y_axis, z_axis) */
  uint8_t is_static;        /* statics take no reaction */
  uint8_t is_sleeping;      /* cleared when the fluid pushes or floats the body */
  uint8_t _pad[2];
} PhiengBody3;
#ifdef __cplusplus
static_assert(sizeof(PhiengBody3) == 112, "PhiengBody3 layout");
#endif

/* FluidState3::step_fluid(bodies, gravity, ambient, time, dt)
 * (fluid3.rs:591-607), the fluid phase of World3::step (world.rs:2805-2812):
 * CFL substeps of the world's 3D fluid against `bodies` in their order (in
 * place of the world's own static bodies). Per substep (fluid3.rs:990-1214):
 * sort, density, ghosts, force and integrate, then the boundary pass of
 * fluid3.rs:1140-1178 in particle order (push-out, approach velocity removed,
 * impulse n * (vn * m) on a dynamic body, the no-slip pull toward the body's
 * velocity and its reaction -dv * m; RigidBody3::apply_impulse with the
 * world-frame inverse inertia R I^-1 R^T, body.rs:1324-1361), then the
 * buoyancy + drag pass of fluid3.rs:1180-1213 over the surface samples of
 * dynamic spheres (14), boxes (24) and capsules (18) (fluid3.rs:371-467:
 * pressure sampled on the re-sorted grid, force -n (p A) - v_rel (drag A
 * |v_rel|) against the ambient wind, RigidBody3::apply_force). vx .. wz and
 * is_sleeping of `bodies` are updated in place; the transforms are the
 * caller's (the host engine integrates them). Turbulence uses the world
 * clock (phieng_world3_set_time). Does not advance the clock.
 * 1 ok; 0 for a null world, a body with an unknown shape, a non-finite
 * field or a rotation whose norm is not 1 within 1e-3, more than 65536
 * bodies, adaptive resolution on, boundary particles on with a static body
 * that is rotated (its ghosts are generated for the identity rotation
 * only), or an error (phieng_sph3_status). */
int32_t phieng_sph3_step_fluid(World3* world, PhiengBody3* bodies, uint32_t nbodies, float dt);

/* phieng_sph3_step_fluid with convex hulls as well: a body with shape_tag
 * PHIENG_SHAPE3_HULL (a, b, c unused) has hull_count[k] >= 1 vertices in its
 * own frame at hull_xyz[3 * hull_first[k] ...] (the arrays are indexed by
 * body and read for hulls only). A particle tests a hull as fluid3.rs:568-585
 * does: the nearest vertex sphere of radius particle_radius among the
 * vertices moved by the body's transform (the first of equal depths), contact
 * point the vertex. Hulls are impulse-coupled only: no buoyancy samples
 * (fluid3.rs:464). 0 also for a hull with no vertex, a vertex range outside
 * hull_nverts or a non-finite vertex. */
int32_t phieng_sph3_step_fluid_hull(World3* world, PhiengBody3* bodies, uint32_t nbodies, const float* hull_xyz,
                                    const uint32_t* hull_first, const uint32_t* hull_count, uint32_t hull_nverts,
                                    float dt);

/* ---- 3D extensions (no reference counterpart) ---- */

/* As phieng_sph_status (grid_log2_h holds log2 of the rows; depth is not
 * reported). 1 ok, 0 null. */
int32_t phieng_sph3_status(const World3* world, PhiengSphStatus* out);
/* Reset the sticky error (1 ok, 0 null) / its text (never null). */
int32_t phieng_sph3_clear_error(World3* world);
const char* phieng_sph3_error_string(const World3* world);
/* Particle cap in place of 4096 (for workloads past the reference's limit). */
int32_t phieng_sph3_set_particle_cap(World3* world, uint32_t cap);
/* `steps` x phieng_world3_step(dt) without synchronising. 1 ok, 0 error. */
int32_t phieng_sph3_step_n(World3* world, float dt, uint32_t steps);
/* Launch on this CUDA stream (NULL: the library's own). */
int32_t phieng_sph3_set_stream(World3* world, void* stream);
/* Wait for the world's stream; 1 ok, 0 on a (sticky) error. */
int32_t phieng_sph3_sync(World3* world);
/* Overwrite the first n particles' state from [x, y, z, vx, vy, vz]
 * sextuples (non-finite values rejected). 1 ok, 0 bad input. */
int32_t phieng_sph3_set_state(World3* world, const float* xyzv, uint32_t n);
/* Density and pressure as the last substep's density pass left them
 * (fluid3.rs:639-658; insertion order). Returns the number written. */
uint32_t phieng_sph3_get_density_pressure(World3* world, float* density, float* pressure, uint32_t max);
/* Density + pressure (and, with fxyz, the pressure force of the next
 * substep, fluid3.rs:1040-1086) of the current state, insertion order. */
uint32_t phieng_sph3_debug_forces(World3* world, float* density, float* pressure, float* fxyz, uint32_t max);
/* Arithmetic mode of the 3D step, as phieng_sph_set_precision's: in
 * PHIENG_SPH_TOLERANCE the plain force pass (XSPH on, no artificial
 * viscosity, cohesion, ghosts or turbulence, uniform mass) reassociates its
 * pair terms (one approximate reciprocal square root and one approximate
 * reciprocal per pair, fused multiply-adds); the density pass, the neighbour
 * sets and the visit order stay exact, and runs stay bit-reproducible. 1 ok,
 * 0 for a null world or an unknown mode. */
int32_t phieng_sph3_set_precision(World3* world, uint32_t mode);
uint32_t phieng_sph3_get_precision(const World3* world);
/* CUDA-event times of the sort, density and force passes of the last
 * substep (after phieng_sph3_set_profiling(world, 1)). */
int32_t phieng_sph3_set_profiling(World3* world, int32_t on);
uint32_t phieng_sph3_phase_times(World3* world, float* ms, uint32_t max);

#ifdef __cplusplus
}
#endif

#endif /* PHIENG_SPH_H */
