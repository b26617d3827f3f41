"""C ABI surface of libphieng_sph.so, on the CPU (no kernel launches).

Restates the reference's FFI tests (crates/engine/src/ffi.rs): config
round trip and validation (fluid_config_roundtrip, :5720), particle
add/count/get/clear with null tolerance and atomic non-finite rejection
(test_ffi_fluid_roundtrip, :7255). None of these calls needs a GPU: the world
acquires the device lazily on the first step.
"""
import ctypes as C
import os
import re

import numpy as np
import pytest

from phi_eng_b200 import _abi
from phi_eng_b200._abi import FluidConfig2Ffi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
F = C.POINTER(C.c_float)


@pytest.fixture(scope="module")
def lib():
    return _abi.load()


def fp(a):
    return a.ctypes.data_as(F)


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "phieng_sph.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(phieng_(?:world3?|sph3?|mlp)_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_exactly_the_bound_symbols(lib):
    assert header_symbols() == sorted(_abi.SIGNATURES)


def test_library_exports_every_declared_symbol(lib):
    for name in header_symbols():
        assert hasattr(lib, name), name


def test_config_layout_matches_ffi_rs():
    assert C.sizeof(FluidConfig2Ffi) == 112
    off = {f[0]: getattr(FluidConfig2Ffi, f[0]).offset for f in FluidConfig2Ffi._fields_}
    assert off["max_substeps"] == 32 and off["adaptive_resolution"] == 36
    assert off["split_density_ratio"] == 40 and off["boundary_particles"] == 48
    assert off["viscosity"] == 52 and off["phase_count"] == 64
    assert off["phase_rest_density"] == 68 and off["phase_mass"] == 84
    assert off["max_velocity"] == 100 and off["particle_radius"] == 104 and off["enabled"] == 108


def roundtrip_cfg():
    c = FluidConfig2Ffi()
    c.particle_mass = 0.125
    c.rest_density = 2.0
    c.smoothing_length = 0.75
    c.stiffness = 200.0
    c.gamma = 7.0
    c.artificial_viscosity = 0.1
    c.surface_tension = 0.05
    c.cfl = 0.4
    c.max_substeps = 4
    c.adaptive_resolution = 1
    c.split_density_ratio = 0.4
    c.merge_density_ratio = 1.8
    c.boundary_particles = 1
    c.viscosity = 0.15
    c.drag = 2.0
    c.wall_friction = 0.3
    c.phase_count = 2
    for k, v in enumerate([1.0, 2.0, 1.0, 1.0]):
        c.phase_rest_density[k] = v
    for k, v in enumerate([0.125, 0.25, 0.125, 0.125]):
        c.phase_mass[k] = v
    c.max_velocity = 50.0
    c.particle_radius = 0.25
    c.enabled = 1
    return c


def clone(c, **kw):
    d = FluidConfig2Ffi()
    C.memmove(C.byref(d), C.byref(c), C.sizeof(c))
    for k, v in kw.items():
        if isinstance(v, list):
            arr = getattr(d, k)
            for i, x in enumerate(v):
                arr[i] = x
        else:
            setattr(d, k, v)
    return d


# ffi.rs:5720 fluid_config_roundtrip
def test_fluid_config_roundtrip(lib):
    w = lib.phieng_world_new()
    cfg = roundtrip_cfg()
    assert lib.phieng_world_set_fluid_config(w, C.byref(cfg)) == 1
    out = FluidConfig2Ffi()
    assert lib.phieng_world_get_fluid_config(w, C.byref(out)) == 1
    assert out.particle_mass == 0.125 and out.rest_density == 2.0 and out.smoothing_length == 0.75
    assert out.gamma == 7.0 and np.float32(out.cfl) == np.float32(0.4) and out.max_substeps == 4
    assert out.adaptive_resolution and out.boundary_particles
    assert out.phase_count == 2 and out.phase_rest_density[1] == 2.0 and out.phase_mass[1] == 0.25
    assert out.max_velocity == 50.0
    assert lib.phieng_world_set_fluid_config(None, C.byref(cfg)) == 0
    assert lib.phieng_world_get_fluid_config(w, None) == 0
    bad = [
        clone(cfg, particle_mass=-1.0),
        clone(cfg, rest_density=0.0),
        clone(cfg, gamma=0.5),
        clone(cfg, phase_count=0),
        clone(cfg, phase_count=5),
        clone(cfg, max_substeps=0),
        clone(cfg, cfl=1.5),
        clone(cfg, artificial_viscosity=3.0),
        clone(cfg, wall_friction=2.0),
        clone(cfg, phase_rest_density=[0.0, 1.0, 1.0, 1.0]),
        clone(cfg, smoothing_length=float("nan")),
        clone(cfg, viscosity=1.5),
        clone(cfg, merge_density_ratio=1.0),
        clone(cfg, phase_mass=[1.0, 1.0, 1.0, -1.0]),
        clone(cfg, particle_radius=-0.1),
    ]
    for b in bad:
        assert lib.phieng_world_set_fluid_config(w, C.byref(b)) == 0
    after = FluidConfig2Ffi()
    assert lib.phieng_world_get_fluid_config(w, C.byref(after)) == 1
    assert after.particle_mass == 0.125 and after.phase_count == 2
    pts = np.array([0.0, 0.0, 1.0, 0.0, 2.0, 0.0], np.float32)
    phases = np.array([0, 1, 0], np.uint8)
    P8 = C.POINTER(C.c_uint8)
    assert lib.phieng_world_fluid_add_phase(w, fp(pts), phases.ctypes.data_as(P8), 3) == 3
    assert lib.phieng_world_fluid_count(w) == 3
    assert lib.phieng_world_fluid_add_phase(None, fp(pts), phases.ctypes.data_as(P8), 3) == 0
    assert lib.phieng_world_fluid_add_phase(w, None, phases.ctypes.data_as(P8), 3) == 0
    assert lib.phieng_world_fluid_add_phase(w, fp(pts), None, 3) == 0
    lib.phieng_world_free(w)


# ffi.rs:7255 test_ffi_fluid_roundtrip
def test_ffi_fluid_roundtrip(lib):
    assert lib.phieng_world_fluid_add(None, None, 0) == 0
    assert lib.phieng_world_fluid_count(None) == 0
    assert lib.phieng_world_fluid_clear(None) == 0
    assert lib.phieng_world_fluid_get(None, None, 0) == 0
    w = lib.phieng_world_new()
    pts = np.array([0.0, 0.0, 0.25, 0.0, 0.0, 0.25], np.float32)
    assert lib.phieng_world_fluid_add(w, fp(pts), 3) == 3
    assert lib.phieng_world_fluid_count(w) == 3
    bad = np.array([0.0, np.nan], np.float32)
    assert lib.phieng_world_fluid_add(w, fp(bad), 1) == 0
    assert lib.phieng_world_fluid_count(w) == 3
    out = np.zeros(8, np.float32)
    assert lib.phieng_world_fluid_get(w, fp(out), 2) == 2
    assert (out[0], out[1], out[4], out[5]) == (0.0, 0.0, 0.25, 0.0)
    assert lib.phieng_world_fluid_clear(w) == 1
    assert lib.phieng_world_fluid_count(w) == 0
    lib.phieng_world_free(w)


def test_particle_cap_and_per_call_limit(lib):
    w = lib.phieng_world_new()
    pts = np.zeros((5000, 2), np.float32)
    pts[:, 0] = np.arange(5000, dtype=np.float32)
    # MAX_PARTICLES_2D = 4096 (fluid.rs:30): the excess is dropped
    assert lib.phieng_world_fluid_add(w, fp(pts), 5000) == 4096
    assert lib.phieng_world_fluid_add(w, fp(pts), 10) == 0
    assert lib.phieng_sph_set_particle_cap(w, 10000) == 1
    assert lib.phieng_world_fluid_add(w, fp(pts), 5000) == 5000
    assert lib.phieng_world_fluid_count(w) == 9096
    assert lib.phieng_sph_set_particle_cap(w, 0) == 0
    lib.phieng_world_free(w)


def test_add_body_validation(lib):
    w = lib.phieng_world_new()
    assert lib.phieng_world_add_body(None, 0, 0, 1, 1, 1, 1, 1, 0.4, 0.1) == -1
    assert lib.phieng_world_add_body(w, 0, 0, 1, 1.0, 0.5, 1.0, 1, 0.4, 0.1) == 0
    assert lib.phieng_world_add_body(w, 1, 1, 0, 0.5, 0.0, 1.0, 1, -3.0, 9.0) == 1  # material sanitised
    assert lib.phieng_world_add_body(w, np.nan, 0, 1, 1, 1, 1, 1, 0.4, 0.1) == -1
    assert lib.phieng_world_add_body(w, 0, 0, 1, -1.0, 1.0, 1, 1, 0.4, 0.1) == -1
    assert lib.phieng_world_add_body(w, 0, 0, 0, 0.0, 0.0, 1, 1, 0.4, 0.1) == -1
    assert lib.phieng_world_add_body(w, 0, 0, 7, 1.0, 1.0, 1, 1, 0.4, 0.1) == -1
    assert lib.phieng_world_add_body(w, 0, 0, 1, 1.0, 1.0, 0.0, 1, 0.4, 0.1) == -1
    assert lib.phieng_world_add_body(w, 0, 0, 1, 1.0, 1.0, 1.0, 0, 0.4, 0.1) == -1  # dynamic: unsupported
    assert lib.phieng_world_body_count(w) == 2
    assert lib.phieng_world_body_count(None) == -1
    lib.phieng_world_free(w)


def test_world_clock_and_gravity(lib):
    w = lib.phieng_world_new()
    t = C.c_float()
    assert lib.phieng_world_get_time(w, C.byref(t)) == 1 and t.value == 0.0
    assert lib.phieng_world_set_time(w, 2.5) == 1
    assert lib.phieng_world_set_time(w, float("inf")) == 0
    assert lib.phieng_world_get_time(w, C.byref(t)) == 1 and t.value == 2.5
    assert lib.phieng_world_get_time(None, C.byref(t)) == 0
    lib.phieng_world_set_gravity(w, 1.0, 2.0)
    lib.phieng_world_set_gravity(w, float("nan"), 2.0)  # ignored
    lib.phieng_world_set_gravity(None, 1.0, 2.0)
    # stepping an empty world advances the clock and touches no GPU
    lib.phieng_world_step(w, 0.5)
    lib.phieng_world_step(w, -1.0)
    lib.phieng_world_step(w, float("nan"))
    assert lib.phieng_world_get_time(w, C.byref(t)) == 1 and t.value == np.float32(2.5) + np.float32(1.0 / 15.0)
    lib.phieng_world_step(None, 0.1)
    lib.phieng_world_free(w)
    lib.phieng_world_free(None)


def test_set_state_rejects_nonfinite(lib):
    w = lib.phieng_world_new()
    pts = np.array([0.0, 0.0, 1.0, 0.0], np.float32)
    assert lib.phieng_world_fluid_add(w, fp(pts), 2) == 2
    good = np.array([[1, 2, 3, 4], [5, 6, 7, 8]], np.float32)
    assert lib.phieng_sph_set_state(w, fp(good), 2) == 1
    bad = good.copy()
    bad[1, 3] = np.inf
    assert lib.phieng_sph_set_state(w, fp(bad), 2) == 0
    assert lib.phieng_sph_set_state(w, fp(good), 3) == 0
    out = np.zeros((2, 4), np.float32)
    assert lib.phieng_world_fluid_get(w, fp(out), 2) == 2
    assert np.array_equal(out, good)
    d = np.zeros(2, np.float32)
    p = np.zeros(2, np.float32)
    assert lib.phieng_sph_get_density_pressure(w, fp(d), fp(p), 2) == 2
    assert (d == 1.0).all() and (p == 0.0).all()  # rest density, zero pressure at insertion
    lib.phieng_world_free(w)


def test_python_mirror_without_gpu():
    from phi_eng_b200.world import Box, World2

    w = World2()
    w.add_static_body((2.0, -1.0), Box(3.0, 0.5))
    assert w.body_count() == 1
    assert w.fluid.add_particles(np.array([[0, 0], [0.25, 0]], np.float32)) == 2
    assert len(w.fluid) == 2
    assert w.fluid.particles.shape == (2, 4)
    w.close()


# ffi.rs:1242 phieng_world_add_bodies: bulk add with per-descriptor rejection
def test_add_bodies_bulk(lib):
    D = _abi.BodyDesc2D
    descs = (D * 5)(
        D(0.0, -1.0, 1, 5.0, 0.5, 1.0, 1, (0, 0, 0), 0.4, 0.1),          # box, ok
        D(1.0, 2.0, 0, 0.3, 0.0, 1.0, 1, (0, 0, 0), 0.4, 0.1),           # circle, ok
        D(float("nan"), 0.0, 1, 1.0, 1.0, 1.0, 1, (0, 0, 0), 0.4, 0.1),  # non-finite position
        D(0.0, 0.0, 7, 1.0, 1.0, 1.0, 1, (0, 0, 0), 0.4, 0.1),           # unknown shape
        D(0.0, 0.0, 1, 1.0, 1.0, 1.0, 0, (0, 0, 0), 0.4, 0.1),           # dynamic: unsupported here
    )
    ids = (C.c_int32 * 5)()
    w = lib.phieng_world_new()
    assert lib.phieng_world_add_bodies(w, descs, 5, ids) == 2
    assert list(ids) == [0, 1, -1, -1, -1]
    assert lib.phieng_world_body_count(w) == 2
    assert lib.phieng_world_add_bodies(None, descs, 5, ids) == 0
    assert lib.phieng_world_add_bodies(w, None, 5, ids) == 0
    assert lib.phieng_world_add_bodies(w, descs, 5, None) == 0
    assert C.sizeof(_abi.BodyDesc2D) == 36 and _abi.BodyDesc2D.friction.offset == 28
    lib.phieng_world_free(w)


def _has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def test_reserve_and_read_into_host_paths(lib):
    """phieng_sph_reserve needs a device (loud failure without one); the host
    mirror read-back works without one."""
    from phi_eng_b200.world import World2

    w = World2()
    pts = np.array([[0.0, 0.0], [0.25, 0.0], [0.5, 0.25]], np.float32)
    assert w.fluid.add_particles(pts) == 3
    out = np.full((3, 4), np.nan, np.float32)
    assert w.fluid.read_into(out) == 3
    assert (out[:, :2] == pts).all() and (out[:, 2:] == 0).all()
    with pytest.raises(ValueError):
        w.fluid.read_into(np.zeros((3, 2), np.float32))
    if not _has_gpu():
        assert lib.phieng_sph_reserve(w._h, 1000) == 0
        assert w.status().error == _abi.E_NO_DEVICE
    w.close()
    assert lib.phieng_sph_reserve(None, 10) == 0
