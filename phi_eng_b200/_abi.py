"""ctypes binding of the C ABI in include/phieng_sph.h (libphieng_sph.so).

The library is built in-tree by ``phi_eng_b200.build`` (nvcc, sm_100a). There
is no fallback: if the shared object is missing or fails to load, importing
the product API raises, so nothing can silently run a CPU path instead.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# PHIENG_SPH_LIBRARY names another build of the same library (same ABI)
LIB_PATH = os.environ.get("PHIENG_SPH_LIBRARY") or os.path.join(HERE, "libphieng_sph.so")

SHAPE_CIRCLE = 0
SHAPE_BOX = 1
SHAPE_POLYGON = 2  # phieng_sph_step_fluid_poly only
SHAPE3_SPHERE = 0
SHAPE3_BOX = 1
SHAPE3_CAPSULE = 2
SHAPE3_HULL = 3  # phieng_sph3_step_fluid_hull only
MAX_PARTICLES_3D = 4096
SNAPSHOT_SCHEMA = 17

OK = 0
E_NO_DEVICE = 1
E_CUDA = 2
E_UNSUPPORTED = 3
E_ARG = 4
E_TOO_LARGE = 5
NOALLOC_MAX_PARTICLES = 65536


class FluidConfig2Ffi(C.Structure):
    """#[repr(C)] FluidConfig2Ffi (crates/engine/src/ffi.rs:712-739), 112 bytes."""

    _fields_ = [
        ("particle_mass", C.c_float),
        ("rest_density", C.c_float),
        ("smoothing_length", C.c_float),
        ("stiffness", C.c_float),
        ("gamma", C.c_float),
        ("artificial_viscosity", C.c_float),
        ("surface_tension", C.c_float),
        ("cfl", C.c_float),
        ("max_substeps", C.c_uint32),
        ("adaptive_resolution", C.c_uint8),
        ("split_density_ratio", C.c_float),
        ("merge_density_ratio", C.c_float),
        ("boundary_particles", C.c_uint8),
        ("viscosity", C.c_float),
        ("drag", C.c_float),
        ("wall_friction", C.c_float),
        ("phase_count", C.c_uint8),
        ("phase_rest_density", C.c_float * 4),
        ("phase_mass", C.c_float * 4),
        ("max_velocity", C.c_float),
        ("particle_radius", C.c_float),
        ("enabled", C.c_uint8),
    ]


assert C.sizeof(FluidConfig2Ffi) == 112


def default_config() -> FluidConfig2Ffi:
    """FluidConfig2::default() (crates/dynamics/src/fluid.rs:142-169)."""
    c = FluidConfig2Ffi()
    c.particle_mass = 0.0625
    c.rest_density = 1.0
    c.smoothing_length = 0.5
    c.stiffness = 100.0
    c.gamma = 1.0
    c.artificial_viscosity = 0.0
    c.surface_tension = 0.0
    c.cfl = 0.0
    c.max_substeps = 1
    c.adaptive_resolution = 0
    c.split_density_ratio = 0.5
    c.merge_density_ratio = 1.6
    c.boundary_particles = 0
    c.viscosity = 0.3
    c.drag = 4.0
    c.wall_friction = 0.0
    c.phase_count = 1
    for k in range(4):
        c.phase_rest_density[k] = 1.0
        c.phase_mass[k] = 0.0625
    c.max_velocity = 30.0
    c.particle_radius = 0.125
    c.enabled = 1
    return c


class AmbientConfig2Ffi(C.Structure):
    """#[repr(C)] AmbientConfig2Ffi (crates/engine/src/ffi.rs:231-276), 80 bytes."""

    _fields_ = [
        ("spring_enabled", C.c_uint32),
        ("spring_ax", C.c_float),
        ("spring_ay", C.c_float),
        ("spring_stiffness", C.c_float),
        ("spring_damping", C.c_float),
        ("spring_max_displacement", C.c_float),
        ("drag_enabled", C.c_uint32),
        ("drag_linear", C.c_float),
        ("drag_quadratic", C.c_float),
        ("air_density", C.c_float),
        ("drag_angular", C.c_float),
        ("wind_x", C.c_float),
        ("wind_y", C.c_float),
        ("turbulence_enabled", C.c_uint32),
        ("turbulence_amplitude", C.c_float),
        ("turbulence_frequency", C.c_float),
        ("turbulence_time_scale", C.c_float),
        ("turbulence_seed", C.c_uint32),
        ("turbulence_octaves", C.c_uint32),
        ("turbulence_divergence_free", C.c_uint32),
    ]


class AmbientConfig3Ffi(C.Structure):
    """#[repr(C)] AmbientConfig3Ffi (crates/engine/src/ffi.rs:278-326), 88 bytes."""

    _fields_ = [
        ("spring_enabled", C.c_uint32),
        ("spring_ax", C.c_float),
        ("spring_ay", C.c_float),
        ("spring_az", C.c_float),
        ("spring_stiffness", C.c_float),
        ("spring_damping", C.c_float),
        ("spring_max_displacement", C.c_float),
        ("drag_enabled", C.c_uint32),
        ("drag_linear", C.c_float),
        ("drag_quadratic", C.c_float),
        ("air_density", C.c_float),
        ("drag_angular", C.c_float),
        ("wind_x", C.c_float),
        ("wind_y", C.c_float),
        ("wind_z", C.c_float),
        ("turbulence_enabled", C.c_uint32),
        ("turbulence_amplitude", C.c_float),
        ("turbulence_frequency", C.c_float),
        ("turbulence_time_scale", C.c_float),
        ("turbulence_seed", C.c_uint32),
        ("turbulence_octaves", C.c_uint32),
        ("turbulence_divergence_free", C.c_uint32),
    ]


def default_ambient3() -> AmbientConfig3Ffi:
    """AmbientConfig3::default (crates/dynamics/src/ambient.rs)."""
    a = AmbientConfig3Ffi()
    a.air_density = 1.0
    a.turbulence_frequency = 1.0
    a.turbulence_time_scale = 1.0
    a.turbulence_octaves = 3
    return a


def default_ambient() -> AmbientConfig2Ffi:
    """AmbientConfig2::default (crates/dynamics/src/ambient.rs)."""
    a = AmbientConfig2Ffi()
    a.air_density = 1.0
    a.turbulence_frequency = 1.0
    a.turbulence_time_scale = 1.0
    a.turbulence_octaves = 3
    return a


class BodyDesc2D(C.Structure):
    """#[repr(C)] BodyDesc2D (crates/engine/src/ffi.rs:1209-1227), 36 bytes."""

    _fields_ = [
        ("pos_x", C.c_float),
        ("pos_y", C.c_float),
        ("shape_tag", C.c_uint32),
        ("a", C.c_float),
        ("b", C.c_float),
        ("density", C.c_float),
        ("is_static", C.c_uint8),
        ("_pad", C.c_uint8 * 3),
        ("friction", C.c_float),
        ("restitution", C.c_float),
    ]


assert C.sizeof(BodyDesc2D) == 36


class BodyDesc3D(C.Structure):
    """#[repr(C)] BodyDesc3D (crates/engine/src/ffi.rs:3767-3786), 44 bytes."""

    _fields_ = [
        ("pos_x", C.c_float),
        ("pos_y", C.c_float),
        ("pos_z", C.c_float),
        ("shape_tag", C.c_uint32),
        ("a", C.c_float),
        ("b", C.c_float),
        ("c", C.c_float),
        ("density", C.c_float),
        ("is_static", C.c_uint8),
        ("_pad", C.c_uint8 * 3),
        ("friction", C.c_float),
        ("restitution", C.c_float),
    ]


assert C.sizeof(BodyDesc3D) == 44

class PhiengBody2(C.Structure):
    """A rigid body as the fluid phase sees it (phieng_sph_step_fluid), 60 bytes."""

    _fields_ = [
        ("shape_tag", C.c_uint32),
        ("a", C.c_float),
        ("b", C.c_float),
        ("px", C.c_float),
        ("py", C.c_float),
        ("xax", C.c_float),
        ("xay", C.c_float),
        ("yax", C.c_float),
        ("yay", C.c_float),
        ("vx", C.c_float),
        ("vy", C.c_float),
        ("w", C.c_float),
        ("inv_mass", C.c_float),
        ("inv_inertia", C.c_float),
        ("is_static", C.c_uint8),
        ("is_sleeping", C.c_uint8),
        ("_pad", C.c_uint8 * 2),
    ]


assert C.sizeof(PhiengBody2) == 60


class PhiengBody3(C.Structure):
    """A rigid body as the 3D fluid phase sees it (phieng_sph3_step_fluid), 112 bytes."""

    _fields_ = [
        ("shape_tag", C.c_uint32),
        ("a", C.c_float),
        ("b", C.c_float),
        ("c", C.c_float),
        ("px", C.c_float),
        ("py", C.c_float),
        ("pz", C.c_float),
        ("qx", C.c_float),
        ("qy", C.c_float),
        ("qz", C.c_float),
        ("qw", C.c_float),
        ("vx", C.c_float),
        ("vy", C.c_float),
        ("vz", C.c_float),
        ("wx", C.c_float),
        ("wy", C.c_float),
        ("wz", C.c_float),
        ("inv_mass", C.c_float),
        ("inv_inertia", C.c_float * 9),
        ("is_static", C.c_uint8),
        ("is_sleeping", C.c_uint8),
        ("_pad", C.c_uint8 * 2),
    ]


assert C.sizeof(PhiengBody3) == 112

# FluidConfig3Ffi (ffi.rs:744-767) has the 2D config's fields and layout.
FluidConfig3Ffi = FluidConfig2Ffi


class PhiengSphStatus(C.Structure):
    _fields_ = [
        ("error", C.c_int32),
        ("particles", C.c_uint32),
        ("substeps", C.c_uint64),
        ("grid_log2_w", C.c_uint32),
        ("grid_log2_h", C.c_uint32),
        ("sort_passes", C.c_uint32),
        ("grid_cx0", C.c_int32),
        ("grid_cy0", C.c_int32),
        ("grid_buckets", C.c_uint32),
    ]


class PhiengClosureStats(C.Structure):
    _fields_ = [
        ("coarse_steps", C.c_uint32),
        ("accepted", C.c_uint32),
        ("fallbacks", C.c_uint32),
        ("reserved", C.c_uint32),
        ("last_check", C.c_float),
        ("max_check", C.c_float),
    ]


class PhiengSphTuning(C.Structure):
    _fields_ = [
        ("density_block", C.c_uint32),
        ("force_block", C.c_uint32),
        ("buckets_per_particle", C.c_float),
        ("stage", C.c_uint32),
    ]


EXACT = 0  # PHIENG_SPH_EXACT: the reference's f32 arithmetic, bit for bit
TOLERANCE = 1  # PHIENG_SPH_TOLERANCE: reassociated plain passes, within the stated tolerances
MLP_TCGEN05 = 0  # PHIENG_MLP_TCGEN05: training GEMMs on the 5th-generation tensor cores
MLP_MMA_SYNC = 1  # PHIENG_MLP_MMA_SYNC: training GEMMs on warp-level mma.sync tiles

MLP_PARAMS = 5378
MLP_NORM = 34
MLP_FEATURES = 16
CLOSURE_JUMP = 0
CLOSURE_COMPRESSION = 1
CLOSURE_GROWTH = 2

_P = C.c_void_p
_F = C.POINTER(C.c_float)
_U32P = C.POINTER(C.c_uint32)
_U8P = C.POINTER(C.c_uint8)

# name -> (restype, argtypes); the exact set declared in include/phieng_sph.h
SIGNATURES = {
    "phieng_world_new": (_P, []),
    "phieng_world_free": (None, [_P]),
    "phieng_world_step": (None, [_P, C.c_float]),
    "phieng_world_set_gravity": (None, [_P, C.c_float, C.c_float]),
    "phieng_world_set_time": (C.c_int32, [_P, C.c_float]),
    "phieng_world_get_time": (C.c_int32, [_P, _F]),
    "phieng_world_body_count": (C.c_int32, [_P]),
    "phieng_sph_ghosts": (C.c_uint32, [_P, _F, C.c_uint32, C.POINTER(C.c_uint64)]),
    "phieng_sph_fluid_masses": (C.c_uint32, [_P, _F, C.c_uint32]),
    "phieng_world_set_ambient_config": (C.c_int32, [_P, C.POINTER(AmbientConfig2Ffi)]),
    "phieng_world_get_ambient_config": (C.c_int32, [_P, C.POINTER(AmbientConfig2Ffi)]),
    "phieng_world_add_body": (
        C.c_int32,
        [_P, C.c_float, C.c_float, C.c_uint32, C.c_float, C.c_float, C.c_float, C.c_uint8,
         C.c_float, C.c_float],
    ),
    "phieng_world_add_bodies": (C.c_uint32, [_P, C.POINTER(BodyDesc2D), C.c_uint32, C.POINTER(C.c_int32)]),
    "phieng_world_set_fluid_config": (C.c_int32, [_P, C.POINTER(FluidConfig2Ffi)]),
    "phieng_world_get_fluid_config": (C.c_int32, [_P, C.POINTER(FluidConfig2Ffi)]),
    "phieng_world_fluid_add": (C.c_uint32, [_P, _F, C.c_uint32]),
    "phieng_world_fluid_add_phase": (C.c_uint32, [_P, _F, _U8P, C.c_uint32]),
    "phieng_world_fluid_count": (C.c_uint32, [_P]),
    "phieng_world_fluid_clear": (C.c_int32, [_P]),
    "phieng_world_fluid_get": (C.c_uint32, [_P, _F, C.c_uint32]),
    "phieng_sph_status": (C.c_int32, [_P, C.POINTER(PhiengSphStatus)]),
    "phieng_sph_clear_error": (C.c_int32, [_P]),
    "phieng_sph_error_string": (C.c_char_p, [_P]),
    "phieng_sph_set_particle_cap": (C.c_int32, [_P, C.c_uint32]),
    "phieng_sph_step_n": (C.c_int32, [_P, C.c_float, C.c_uint32]),
    "phieng_sph_set_stream": (C.c_int32, [_P, _P]),
    "phieng_sph_sync": (C.c_int32, [_P]),
    "phieng_sph_set_state": (C.c_int32, [_P, _F, C.c_uint32]),
    "phieng_sph_get_density_pressure": (C.c_uint32, [_P, _F, _F, C.c_uint32]),
    "phieng_sph_replan": (C.c_int32, [_P]),
    "phieng_sph_set_grid": (C.c_int32, [_P, C.c_uint32, C.c_uint32, C.c_int32, C.c_int32]),
    "phieng_sph_front_metrics": (C.c_int32, [_P, _F]),
    "phieng_sph_front_metrics_async": (C.c_int32, [_P, _P]),
    "phieng_sph_front_metrics_decode": (None, [_P, _P]),
    "phieng_sph_set_profiling": (C.c_int32, [_P, C.c_int32]),
    "phieng_sph_phase_times": (C.c_uint32, [_P, _F, C.c_uint32]),
    "phieng_sph_batch_new": (_P, [C.POINTER(_P), C.c_uint32]),
    "phieng_sph_batch_scenes": (C.c_uint32, [_P]),
    "phieng_sph_batch_scene_range": (C.c_int32, [_P, C.c_uint32, _U32P, _U32P]),
    "phieng_sph_batch_store": (C.c_int32, [_P, C.POINTER(_P), C.c_uint32]),
    "phieng_sph_density_noalloc": (C.c_int32, [_P, C.c_uint32, C.POINTER(FluidConfig2Ffi), _P, _P, _P]),
    "phieng_sph_set_tuning": (C.c_int32, [_P, C.POINTER(PhiengSphTuning)]),
    "phieng_sph_get_tuning": (C.c_int32, [_P, C.POINTER(PhiengSphTuning)]),
    "phieng_sph_set_precision": (C.c_int32, [_P, C.c_uint32]),
    "phieng_sph_get_precision": (C.c_uint32, [_P]),
    "phieng_sph_get_state_device": (C.c_uint32, [_P, _P, C.c_uint32]),
    "phieng_sph_set_state_device": (C.c_int32, [_P, _P, C.c_uint32]),
    "phieng_sph_load_state_device": (C.c_int32, [_P, _P, C.c_uint32]),
    "phieng_sph_set_order": (C.c_int32, [_P, _P, C.c_uint32]),
    "phieng_sph_slab_setup": (C.c_int32, [_P, C.c_int32, C.c_int32, C.c_uint32, C.c_uint32, C.c_uint32, _P, _P, _P,
                                          _P]),
    "phieng_sph_slab_pack": (C.c_int32, [_P, C.c_uint32]),
    "phieng_sph_slab_unpack": (C.c_int32, [_P, C.c_uint32]),
    "phieng_sph_slab_vmax": (C.c_int32, [_P, _P]),
    "phieng_sph_slab_status": (C.c_int32, [_P]),
    "phieng_sph_slab_owned": (C.c_uint32, [_P, _P, _P, C.c_uint32]),
    "phieng_mlp_new": (_P, [C.c_uint64]),
    "phieng_mlp_free": (None, [_P]),
    "phieng_mlp_status": (C.c_int32, [_P]),
    "phieng_mlp_set_stream": (C.c_int32, [_P, _P]),
    "phieng_mlp_get_params": (C.c_int32, [_P, _F, _F]),
    "phieng_mlp_set_params": (C.c_int32, [_P, _F, _F]),
    "phieng_mlp_step_count": (C.c_uint32, [_P]),
    "phieng_mlp_forward": (C.c_int32, [_P, _P, C.c_uint32, _P]),
    "phieng_mlp_forward_tc": (C.c_int32, [_P, _P, C.c_uint32, _P]),
    "phieng_mlp_check_waits": (C.c_int32, [_P]),
    "phieng_mlp_set_train_engine": (C.c_int32, [_P, C.c_int32]),
    "phieng_mlp_set_closure_engine": (C.c_int32, [_P, C.c_int32]),
    "phieng_mlp_get_closure_engine": (C.c_int32, [_P]),
    "phieng_mlp_shard_grad": (C.c_int32, [_P, _P, _P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64,
                                          _P]),
    "phieng_mlp_apply_grad": (C.c_int32, [_P, _P, C.c_float]),
    "phieng_mlp_get_train_engine": (C.c_int32, [_P]),
    "phieng_mlp_grad": (C.c_int32, [_P, _P, _P, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32, _F, _F]),
    "phieng_mlp_train": (C.c_int32, [_P, _P, _P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_float, C.c_uint64, _F]),
    "phieng_mlp_sample_indices": (C.c_int32, [C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32, _P, _P]),
    "phieng_mlp_targets": (C.c_int32, [_P, _P, C.c_uint32, C.c_float, C.c_float, C.c_uint32, _P, _P]),
    "phieng_mlp_perturb": (C.c_int32, [_P, C.c_uint32, C.c_float, C.c_uint64, _P]),
    "phieng_sph_features": (C.c_int32, [_P, C.c_float, _P]),
    "phieng_sph_set_closure": (C.c_int32, [_P, _P, C.c_uint32, C.c_float, C.c_uint32]),
    "phieng_sph_closure_step": (C.c_int32, [_P, C.c_float, C.c_uint32, C.POINTER(PhiengClosureStats)]),
    "phieng_sph_debug_forces": (C.c_uint32, [_P, _F, C.c_uint32]),
    "phieng_sph_debug_scan_timeout": (C.c_int32, [_P]),
    "phieng_sph_debug_sorted": (C.c_uint32, [_P, _U32P, _U32P, C.c_uint32]),
    "phieng_sph_debug_neighbors": (C.c_uint32, [_P, _U32P, _U32P, C.c_uint32, C.c_uint32]),
    "phieng_sph_reserve": (C.c_int32, [_P, C.c_uint32]),
    "phieng_sph_step_fluid": (C.c_int32, [_P, C.POINTER(PhiengBody2), C.c_uint32, C.c_float]),
    "phieng_sph_step_fluid_poly": (
        C.c_int32,
        [_P, C.POINTER(PhiengBody2), C.c_uint32, _F, _U32P, _U32P, C.c_uint32, C.c_float],
    ),
    "phieng_sph_fluid_block_save": (C.c_int64, [_P, C.c_uint32, _U8P, C.c_uint64]),
    "phieng_sph_fluid_block_load": (C.c_int64, [_P, C.c_uint32, _U8P, C.c_uint64]),
    "phieng_sph3_fluid_block_save": (C.c_int64, [_P, C.c_uint32, _U8P, C.c_uint64]),
    "phieng_sph3_fluid_block_load": (C.c_int64, [_P, C.c_uint32, _U8P, C.c_uint64]),
    "phieng_world3_new": (_P, []),
    "phieng_world3_free": (None, [_P]),
    "phieng_world3_step": (None, [_P, C.c_float]),
    "phieng_world3_set_gravity": (None, [_P, C.c_float, C.c_float, C.c_float]),
    "phieng_world3_set_time": (C.c_int32, [_P, C.c_float]),
    "phieng_world3_get_time": (C.c_int32, [_P, _F]),
    "phieng_world3_body_count": (C.c_int32, [_P]),
    "phieng_world3_set_ambient_config": (C.c_int32, [_P, C.POINTER(AmbientConfig3Ffi)]),
    "phieng_sph3_ghosts": (C.c_uint32, [_P, _F, C.c_uint32, C.POINTER(C.c_uint64)]),
    "phieng_sph3_fluid_masses": (C.c_uint32, [_P, _F, C.c_uint32]),
    "phieng_world3_get_ambient_config": (C.c_int32, [_P, C.POINTER(AmbientConfig3Ffi)]),
    "phieng_world3_add_body": (
        C.c_int32,
        [_P, C.c_float, C.c_float, C.c_float, C.c_uint32, C.c_float, C.c_float, C.c_float, C.c_float,
         C.c_uint8, C.c_float, C.c_float],
    ),
    "phieng_world3_add_bodies": (C.c_uint32, [_P, C.POINTER(BodyDesc3D), C.c_uint32, C.POINTER(C.c_int32)]),
    "phieng_world3_set_fluid_config": (C.c_int32, [_P, C.POINTER(FluidConfig2Ffi)]),
    "phieng_world3_get_fluid_config": (C.c_int32, [_P, C.POINTER(FluidConfig2Ffi)]),
    "phieng_world3_fluid_add": (C.c_uint32, [_P, _F, C.c_uint32]),
    "phieng_world3_fluid_add_phase": (C.c_uint32, [_P, _F, _U8P, C.c_uint32]),
    "phieng_world3_fluid_count": (C.c_uint32, [_P]),
    "phieng_world3_fluid_clear": (C.c_int32, [_P]),
    "phieng_world3_fluid_get": (C.c_uint32, [_P, _F, C.c_uint32]),
    "phieng_sph3_status": (C.c_int32, [_P, C.POINTER(PhiengSphStatus)]),
    "phieng_sph3_clear_error": (C.c_int32, [_P]),
    "phieng_sph3_error_string": (C.c_char_p, [_P]),
    "phieng_sph3_set_particle_cap": (C.c_int32, [_P, C.c_uint32]),
    "phieng_sph3_step_n": (C.c_int32, [_P, C.c_float, C.c_uint32]),
    "phieng_sph3_set_stream": (C.c_int32, [_P, _P]),
    "phieng_sph3_sync": (C.c_int32, [_P]),
    "phieng_sph3_set_state": (C.c_int32, [_P, _F, C.c_uint32]),
    "phieng_sph3_get_density_pressure": (C.c_uint32, [_P, _F, _F, C.c_uint32]),
    "phieng_sph3_debug_forces": (C.c_uint32, [_P, _F, _F, _F, C.c_uint32]),
    "phieng_sph3_set_precision": (C.c_int32, [_P, C.c_uint32]),
    "phieng_sph3_step_fluid": (C.c_int32, [_P, C.POINTER(PhiengBody3), C.c_uint32, C.c_float]),
    "phieng_sph3_step_fluid_hull": (
        C.c_int32,
        [_P, C.POINTER(PhiengBody3), C.c_uint32, C.POINTER(C.c_float), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
         C.c_uint32, C.c_float]),
    "phieng_sph3_get_precision": (C.c_uint32, [_P]),
    "phieng_sph3_set_profiling": (C.c_int32, [_P, C.c_int32]),
    "phieng_sph3_phase_times": (C.c_uint32, [_P, _F, C.c_uint32]),
}

_lib = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load libphieng_sph.so and bind every declared symbol; raise if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            f"{path} is missing: build it with `python -m phi_eng_b200.build` "
            "(the SPH step has no CPU fallback)"
        )
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
