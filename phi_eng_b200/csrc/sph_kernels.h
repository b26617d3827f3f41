// Host-side interface of the SPH kernel chain (sph_kernels.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "sph_device.cuh"
#include "sph_mlp.cuh"

namespace phieng {


// A batch of independent scenes advanced together: per-scene parameters and
// each particle's scene (ptab == nullptr: a single world).
struct BatchTab {
  const StepParams* ptab = nullptr;  // [scenes] device table
  const uint32_t* pscene = nullptr;  // id order: scene of each particle
  uint32_t* sscene = nullptr;        // sorted order (gathered by the sort)
};

// Device arrays of one fluid. "id order" = insertion order (the reference's
// particle index); "sorted order" = (bucket key, id) order of the last sort.
struct FluidBufs {
  uint32_t cap = 0;          // particle capacity of every per-particle array
  float4* state = nullptr;   // id order: (x, y, vx, vy)
  float* mass = nullptr;     // id order (used when F_MASS)
  uint8_t* phase = nullptr;  // id order (used when F_PHASE)
  uint32_t* key = nullptr;   // id order: bucket key for the next sort
  uint32_t* tkey = nullptr;  // placed (key, id) before the in-bucket rank
  uint32_t* tid = nullptr;
  uint32_t* skey = nullptr;  // sorted keys
  uint32_t* sid = nullptr;   // sorted slot -> particle id
  float2* spos = nullptr;    // sorted (x, y)
  float2* svel = nullptr;    // sorted (vx, vy)
  float* smass = nullptr;    // sorted mass (F_MASS)
  uint8_t* sphase = nullptr; // sorted phase (F_PHASE)
  float2* sdq = nullptr;     // sorted (density, pressure / max(density,EPS)^2)
  float* spres = nullptr;    // sorted pressure
  uint32_t* nmask = nullptr; // [3][cap] per-row neighbour masks written by K5, read by K6
  // per id: the tag that orders a bucket's particles (null: the id itself).
  // Tags of finite particles are distinct; the x-slab decomposition sets the
  // global ids, so a rank world visits its neighbours in the single domain's
  // order whatever slot a particle occupies. With tags, the non-finite
  // sentinel bucket keeps its placement order (nothing visits it).
  uint32_t* order = nullptr;
  // per bucket grid (sized by the number of buckets B)
  uint32_t* count = nullptr;    // particles per bucket, then the placement cursor
  uint32_t count_len = 0;       // B + 1 rounded up to the scan tile
  uint32_t* start = nullptr;    // bucket b holds sorted slots [start[b], start[b+1])
  uint32_t* tilesum = nullptr;  // scan tile sums / offsets
  uint32_t range_cap = 0;       // buckets the arrays above can hold
  uint32_t* done = nullptr;     // scan counters (two words, zero between scans)
  // single-pass scan: per-tile (flag, value) states, zero between scans, and a
  // sticky flag set when a look-back wait gave up (null: the two-kernel scan)
  unsigned long long* tstate = nullptr;
  uint32_t* scan_err = nullptr;
  BatchTab batch;
  DevBody* bodies = nullptr;
  uint32_t bodies_cap = 0;
  // bodies that react (F_DYNAMIC): per id, the body index the ordered pass
  // resumes from, and 1 / 0 = deferred or not (padded to a scan tile)
  uint32_t* defer = nullptr;
  uint32_t* dcount = nullptr;
  unsigned int* scalar = nullptr;  // small device scratch (vmax etc.)
  // launch shapes (autotuned; results do not depend on them)
  uint32_t block_density = 256;  // threads per block of K5: 64, 128 or 256
  uint32_t block_force = 256;    // threads per block of K6: 64, 128 or 256
  // tolerance-mode passes: bit 0 = K5 stages its neighbour rows in shared
  // memory, bit 1 = K6 does, bit 2 = K6 reassigns each block's particles to
  // its lanes by neighbour count (not with bit 1). Results do not depend on
  // them.
  uint32_t stage = 0;
};

// Scan tile of the bucket counts; count arrays are padded to a multiple.
constexpr uint32_t kBucketScanTile = 4096;
// Scan tiles per block of the single-pass (look-back) scan. One tile per
// 256-thread block measured fastest on B200 for 2^20 buckets (9.7 us against
// 12.0 us for four tiles per 1024-thread block and 13.9 us for four tiles
// per 256-thread block): the shorter look-back chain of bigger blocks does
// not make up for the SMs they leave idle.
constexpr uint32_t kBucketScanSuper = 1;

// K1: bucket key of every particle from its position (id order), and the
// bucket counts the next sort starts from.
void enqueue_keys(const FluidBufs& b, uint32_t n, const GridPlan& g, cudaStream_t st);

// K2+K3+K4: counting sort of the particles by bucket key, ranked by id
// inside each bucket (final order = (key, id)); fills the bucket range table
// and gathers the particle state into sorted order.
// by_slot: b.sid holds a permutation of [0, n) (the previous sort), walked
// for locality; otherwise particles are placed in id order.
void enqueue_sort_and_ranges(const FluidBufs& b, uint32_t n, const StepParams& P, bool by_slot, cudaStream_t st);

// The dimension-independent part of the bucket sort: scan the bucket counts
// of keys [0, m) into the start table (count becomes the placement cursor),
// then give every particle a slot inside its bucket (tkey / tid; the in-bucket
// rank by id and the gather are the caller's). by_slot: sid_prev holds the
// previous sort's order (walked for locality), else ids are taken in order.
struct BucketSort {
  uint32_t* count = nullptr;
  uint32_t* tilesum = nullptr;
  uint32_t* done = nullptr;
  unsigned long long* tstate = nullptr;  // single-pass scan when set (see FluidBufs)
  uint32_t* err = nullptr;
  uint32_t* start = nullptr;
  const uint32_t* key = nullptr;
  const uint32_t* sid_prev = nullptr;
  uint32_t* tkey = nullptr;
  uint32_t* tid = nullptr;
};
void enqueue_bucket_place(const BucketSort& bs, uint32_t n, uint32_t m, bool by_slot, cudaStream_t st);

// Adaptive resolution scratch: inverse sort permutation, merge flags, the
// resampled particles (cap rows; a pass over n particles writes at most
// n + min(n, 2048)) and their count (cap + 1 if the output would not fit).
struct ResampleBufs {
  uint32_t* slot_of = nullptr;
  uint8_t* absorbed = nullptr;
  float4* state = nullptr;
  float* mass = nullptr;
  uint8_t* phase = nullptr;
  uint32_t cap = 0;
  uint32_t* n_out = nullptr;
};

// resample (fluid.rs:826-893) after a sort and density pass: merges and
// splits into r.state / r.mass / r.phase (id order), the new count into
// *r.n_out. Overwrites b.mass / b.phase with per-particle values when they
// were uniform, and the merged particles' velocity and mass in b.
void enqueue_resample(const FluidBufs& b, uint32_t n, const StepParams& P, const ResampleBufs& r, float merge_hi,
                      float split_lo, float min_mass, bool mass_uniform, bool phase_uniform, cudaStream_t st);

// Boundary ghosts' density / pressure from the fluid of the current sort
// (after K5, before K6); no-op unless P has F_GHOST.
void enqueue_ghost_density(const FluidBufs& b, const StepParams& P, cudaStream_t st);

// K5: density + EOS in sorted order. svp (optional, sorted order): also
// (m / max(density, EPS), q max(density, EPS)^2) per particle, the
// neighbour factors of the closure feature sums.
void enqueue_density(const FluidBufs& b, uint32_t n, const StepParams& P, cudaStream_t st, float2* svp = nullptr);

// K6: pressure force + XSPH + integrate + walls; writes state and next keys
// in id order. With dbg_force != nullptr it only writes the forces (id
// order) and leaves the state untouched.
void enqueue_force_integrate(const FluidBufs& b, uint32_t n, const StepParams& P, float2* dbg_force,
                             cudaStream_t st);

// Closure pass buffers: features (id order, 16 per particle) for the
// features mode; pre-step state and density (id order) kept by the closure
// step.
struct ClosureIO {
  float* feat = nullptr;
  float4* save = nullptr;
  float* rho_prev = nullptr;
  const float2* svp = nullptr;  // K5's closure factors of the current sort (required)
  uint32_t* err = nullptr;       // sticky flag: a tensor-core wait of the tolerance-mode pass ran out
};

// Closure features of every particle for a coarse step of P.dt (after the
// sort and density of the current state); state untouched.
void enqueue_closure_features(const FluidBufs& b, uint32_t n, const StepParams& P, float* feat, const float2* svp,
                              cudaStream_t st);

// Coarse step with the closure network: K6 + features + network + corrected
// integrate. Writes the new state, next keys and counts like K6, plus the
// pre-step state (io.save) and density (io.rho_prev).
void enqueue_closure_force(const FluidBufs& b, uint32_t n, const StepParams& P, const MlpDev& mlp,
                           const ClosureIO& io, cudaStream_t st);

// Density checks after the coarse step's new state was sorted and its density
// computed, into out[0..2] (zeroed first): largest per-particle increase over
// the step, largest compression after it, largest compression before it
// (relative to the rest density, float bits).
void enqueue_closure_check(const FluidBufs& b, uint32_t n, const StepParams& P, const float* rho_prev,
                           unsigned int* out, cudaStream_t st);

// Device buffers of a fluid phase with bodies that react (phieng_sph_step_fluid).
struct DynBufs {
  DynBody* dyn = nullptr;        // [bodies] velocity state, updated in place
  float4* samples = nullptr;     // buoyancy surface samples: point (x, y), outward normal (z, w)
  float* areas = nullptr;        // their areas
  uint32_t* buoy = nullptr;      // indices of the dynamic bodies with samples
  uint32_t nbuoy = 0;
  uint32_t* dcount = nullptr;    // = FluidBufs::dcount
  uint32_t* dstart = nullptr;    // exclusive prefix of dcount; dstart[n] = deferred count
  uint32_t* dtile = nullptr;     // scan tile sums
  uint32_t* done = nullptr;      // scan blocks finished (zero between scans)
  uint32_t* list = nullptr;      // deferred ids in id order
  float2* dq_id = nullptr;       // density pass values by id
  float* p_id = nullptr;
  uint32_t* count2 = nullptr;    // copy of the bucket counts for the buoyancy sort
};

// Ordered compaction of flagged ids: flags[0, n) hold 0 / 1 and are zero up
// to the next whole scan tile past n; start becomes their exclusive prefix
// (start[n] = the flagged count) and list[0, start[n]) the flagged ids in
// ascending order. done: a zeroed device word (left zero).
void enqueue_flag_compact(uint32_t* flags, uint32_t n, uint32_t* tile, uint32_t* done, uint32_t* start,
                          uint32_t* list, cudaStream_t st);

// After K6 with F_DYNAMIC: finish the body loop of the deferred particles in
// particle order with the bodies' reactions, and their keys / counts.
void enqueue_dynamic_walls(const FluidBufs& b, const DynBufs& y, uint32_t n, const StepParams& P, cudaStream_t st);

// Buoyancy + drag of the dynamic bodies (fluid.rs:1103-1135): re-sort on the
// new positions, then each body's samples in order. Leaves the sorted arrays
// and the density-pass values in the new order and the bucket counts intact.
void enqueue_buoyancy(const FluidBufs& b, const DynBufs& y, uint32_t n, const StepParams& P, float drag, float dt,
                      cudaStream_t st);

// One bucket scan in which tile 0 never publishes its prefix: every other
// tile's look-back wait runs out, sets b.scan_err and ends (the test of the
// bounded waits). Leaves the bucket ranges wrong.
void enqueue_scan_silent_tile(const FluidBufs& b, uint32_t m, cudaStream_t st);

// Fold one coarse step's checks (out[0..2] of enqueue_closure_check) into
// the block maxima acc[0..2] (jump, compression, growth), or reset them.
void enqueue_check_fold(const unsigned int* out, float* acc, bool reset, cudaStream_t st);

// *p = v, in stream order (the value travels as a launch argument, so the
// host may reuse its copy at once): the world clock word read by the
// turbulence term of cached step graphs.
void enqueue_set_word(unsigned int* p, uint32_t v, cudaStream_t st);

// Scatter the sorted density / pressure back to id order.
void enqueue_unsort_dp(const FluidBufs& b, uint32_t n, float* dens, float* pres, cudaStream_t st);

// Neighbour lists in visit order (id order), for the parity tests.
void enqueue_debug_neighbors(const FluidBufs& b, uint32_t n, const StepParams& P, uint32_t* counts,
                             uint32_t* lists, uint32_t max_per, cudaStream_t st);

// max_i |v_i| (f32::max semantics, NaN ignored) as float bits in b.scalar[0].
void enqueue_vmax(const FluidBufs& b, uint32_t n, cudaStream_t st);

// b.scalar[2] = order-preserving bits of max_i x_i, b.scalar[3] = bits of max_i |v_i|.
void enqueue_front_metrics(const FluidBufs& b, uint32_t n, cudaStream_t st);

// ---------------------------------------------------------------- x-slab ranks
// A rank world of the x-slab decomposition holds own_cap owned slots, then
// 2 * halo_cap halo slots for the left side and 2 * halo_cap for the right;
// an unused slot holds (NaN, NaN, 0, 0) with order tag kSlabFree (its key is
// the sentinel, so no walk visits it). Exchange buffers (one per direction)
// are 16 + 20 * halo_cap bytes: uint32 header [count, overflow, 0, 0], then
// float4 rows [halo_cap], then uint32 tags [halo_cap] (a migrant's tag
// carries kSlabMigrant); the host moves them between neighbours without
// reading them. Global ids (the tags) are below 2^31 - 1.
constexpr uint32_t kSlabFree = 0xFFFFFFFFu;
constexpr uint32_t kSlabMigrant = 0x80000000u;
constexpr int32_t kSlabHaloColumns = 2;
constexpr uint32_t kSlabWords = 8;

struct SlabPlan {
  int32_t lo = 0, hi = 0;             // owned cell columns [lo, hi)
  uint32_t has_left = 0, has_right = 0;
  float h = 1.0f;                     // cell width (config smoothing_length)
  uint32_t own_cap = 0, halo_cap = 0;
  uint32_t pack_blocks = 592;         // grid of the pack (4 blocks per SM)
  unsigned char* send[2] = {nullptr, nullptr};        // to the left (0) / right (1) neighbour
  const unsigned char* recv[2] = {nullptr, nullptr};  // from the left / right neighbour
  uint32_t* free_stack = nullptr;     // [own_cap] owned slots not in use
  // [0] free slots on the stack, [1] error (sticky), [2] pack blocks done,
  // [4], [5] rows appended to send[0] / send[1] by the running pack
  uint32_t* words = nullptr;
};

constexpr size_t slab_buffer_bytes(uint32_t cap) { return 16 + 20 * (size_t)cap; }

// Stack of the owned slots whose tag is kSlabFree, zeroed counters (set-up).
void enqueue_slab_init(const FluidBufs& b, const SlabPlan& sp, cudaStream_t st);
// After the rank's step (phase 1): migrants (owned particles whose column
// left the slab; their slots become free) and the halo of the others (within
// kSlabHaloColumns of a shared edge) into that side's send buffer. phase 0,
// before the first step: the halo only.
void enqueue_slab_pack(const FluidBufs& b, const SlabPlan& sp, const GridPlan& g, uint32_t phase, cudaStream_t st);
// After the exchange: received migrants into free owned slots, each side's
// halo (received halo rows and this rank's own migrants to that side) into
// its halo slots, the rest of them emptied. Keys and bucket counts follow
// every replaced slot; an overflowing buffer or a full owned region sets
// words[1].
void enqueue_slab_unpack(const FluidBufs& b, const SlabPlan& sp, const GridPlan& g, uint32_t phase, cudaStream_t st);

}  // namespace phieng
