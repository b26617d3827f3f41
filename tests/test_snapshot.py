"""Snapshot fluid block (crates/dynamics/src/snapshot.rs) of the GPU worlds.

The block layout is restated here independently of the library, from
encode_fluid_config2 / encode_fluid2 (snapshot.rs:6337-6491) and the 3D pair
(:6527-6677), and the load rules from apply_fluid2/3 (:4471-4612). CPU tests
cover the bytes, round trips, old schemas, the single-phase reset and hostile
input; GPU tests repeat the reference's continuation check
(test_snapshot_fluid_roundtrip_2d, snapshot.rs:8680-8715): stepping on after a
save and a load is bit-identical to never having saved.
"""
import ctypes as C
import struct

import numpy as np
import pytest

from phi_eng_b200 import _abi
from phi_eng_b200._abi import default_config

U8P = C.POINTER(C.c_uint8)
F = C.POINTER(C.c_float)


@pytest.fixture(scope="module")
def lib():
    return _abi.load()


def fp(a):
    return a.ctypes.data_as(F)


def save(lib, w, version=17, dim=2):
    fn = lib.phieng_sph_fluid_block_save if dim == 2 else lib.phieng_sph3_fluid_block_save
    n = fn(w, version, None, 0)
    assert n > 0
    buf = (C.c_uint8 * n)()
    assert fn(w, version, buf, n) == n
    return bytes(buf)


def load(lib, w, data, version=17, dim=2):
    fn = lib.phieng_sph_fluid_block_load if dim == 2 else lib.phieng_sph3_fluid_block_load
    buf = (C.c_uint8 * max(len(data), 1)).from_buffer_copy(data if data else b"\0")
    return fn(w, version, buf, len(data))


def parse_block(data, version=17, dim=2):
    """Independent decoder of the block (snapshot.rs:6384-6525)."""
    off = 0

    def take(fmt):
        nonlocal off
        v = struct.unpack_from("<" + fmt, data, off)
        off += struct.calcsize("<" + fmt)
        return v if len(v) > 1 else v[0]

    c = {}
    c["particle_mass"], c["rest_density"], c["smoothing_length"], c["stiffness"] = take("4f")
    if version >= 5:
        c["gamma"], c["artificial_viscosity"], c["surface_tension"], c["cfl"] = take("4f")
        c["max_substeps"] = take("I")
        c["adaptive_resolution"] = take("B")
        c["split"], c["merge"] = take("2f")
        c["boundary_particles"] = take("B")
        c["wall_friction"] = take("f")
        c["phase_count"] = take("B")
        c["phase_rest_density"] = take("4f")
        c["phase_mass"] = take("4f")
    c["viscosity"], c["drag"], c["max_velocity"], c["particle_radius"] = take("4f")
    c["enabled"] = take("B")
    n = take("I")
    ps = []
    for _ in range(n):
        pos = take("3f" if dim == 3 else "2f")
        vel = take("3f" if dim == 3 else "2f")
        if version >= 5:
            mass = take("f")
            phase = take("B")
        else:
            mass, phase = 0.0, 0
        ps.append((pos, vel, mass, phase))
    return c, ps, off


def world2(lib, pts, cfg=None, phases=None):
    w = lib.phieng_world_new()
    lib.phieng_world_add_body(w, 0.0, -1.0, _abi.SHAPE_BOX, 10.0, 0.5, 1.0, 1, 0.5, 0.0)
    if cfg is not None:
        assert lib.phieng_world_set_fluid_config(w, C.byref(cfg)) == 1
    p = np.ascontiguousarray(pts, np.float32)
    if phases is None:
        assert lib.phieng_world_fluid_add(w, fp(p.ravel()), len(p)) == len(p)
    else:
        ph = np.ascontiguousarray(phases, np.uint8)
        assert lib.phieng_world_fluid_add_phase(w, fp(p.ravel()), ph.ctypes.data_as(U8P), len(p)) == len(p)
    return w


def state2(lib, w):
    n = lib.phieng_world_fluid_count(w)
    out = np.zeros((n, 4), np.float32)
    assert lib.phieng_world_fluid_get(w, fp(out), n) == n
    return out


def grid_pts(nx=4, ny=3, s=0.25):
    return np.array([(ix * s, iy * s) for iy in range(ny) for ix in range(nx)], np.float32)


def test_block_bytes_follow_the_layout(lib):
    c = default_config()
    c.gamma = 7.0
    c.artificial_viscosity = 1.2
    c.surface_tension = 0.7
    c.wall_friction = 0.4
    c.phase_count = 2
    c.phase_rest_density[1] = 2.0
    c.phase_mass[1] = 0.125
    pts = grid_pts()
    phases = np.arange(12) % 2
    w = world2(lib, pts, c, phases)
    data = save(lib, w)
    cfg, ps, used = parse_block(data)
    assert used == len(data) == 4 * 4 + 4 * 4 + 4 + 1 + 8 + 1 + 4 + 1 + 32 + 16 + 1 + 4 + 12 * 21
    assert cfg["gamma"] == 7.0 and cfg["wall_friction"] == np.float32(0.4)
    assert cfg["phase_count"] == 2 and cfg["phase_rest_density"][1] == 2.0 and cfg["phase_mass"][1] == 0.125
    assert cfg["enabled"] == 1 and cfg["max_substeps"] == 1
    for i, (pos, vel, mass, phase) in enumerate(ps):
        assert pos == tuple(pts[i]) and vel == (0.0, 0.0)
        assert phase == phases[i] and mass == (0.125 if phases[i] else 0.0625)
    lib.phieng_world_free(w)


def test_single_phase_writes_defaults_and_load_resets_tables(lib):
    """phase_count 1 writes count 1, [1.0; 4], [particle_mass; 4]; a load
    therefore resets the phase tables (apply_fluid2, snapshot.rs:4507-4518)."""
    c = default_config()
    c.rest_density = 1000.0
    c.particle_mass = 0.0625 * 1000
    for k in range(4):
        c.phase_rest_density[k] = 1000.0
        c.phase_mass[k] = 62.5
    w = world2(lib, grid_pts(), c)
    data = save(lib, w)
    cfg, ps, _ = parse_block(data)
    assert cfg["phase_count"] == 1 and cfg["phase_rest_density"] == (1.0,) * 4 and cfg["phase_mass"] == (62.5,) * 4
    w2 = lib.phieng_world_new()
    assert load(lib, w2, data) == len(data)
    out = _abi.FluidConfig2Ffi()
    lib.phieng_world_get_fluid_config(w2, C.byref(out))
    assert list(out.phase_rest_density) == [1.0] * 4 and list(out.phase_mass) == [62.5] * 4
    assert out.rest_density == 1000.0
    d = np.zeros(12, np.float32)
    p = np.ones(12, np.float32)
    lib.phieng_sph_get_density_pressure(w2, fp(d), fp(p), 12)
    assert (d == 1000.0).all() and (p == 0.0).all()  # rest_density until the next step
    lib.phieng_world_free(w)
    lib.phieng_world_free(w2)


@pytest.mark.parametrize("version", [17, 5, 4, 1])
def test_roundtrip_bytes_and_state(lib, version):
    c = default_config()
    c.phase_count = 3
    c.phase_mass[2] = 0.25
    pts = grid_pts(5, 4)
    phases = np.arange(20) % 3
    w = world2(lib, pts, c, phases)
    data = save(lib, w, version)
    w2 = lib.phieng_world_new()
    assert load(lib, w2, data + b"trailing", version) == len(data)
    assert save(lib, w2, version) == data
    np.testing.assert_array_equal(state2(lib, w2), state2(lib, w))
    if version < 5:
        out = _abi.FluidConfig2Ffi()
        lib.phieng_world_get_fluid_config(w2, C.byref(out))
        assert out.gamma == 1.0 and out.max_substeps == 1 and out.phase_count == 1
        assert np.float32(out.split_density_ratio) == np.float32(0.5)
        assert np.float32(out.merge_density_ratio) == np.float32(1.6)
        cfg, ps, _ = parse_block(data, version)
        assert all(len(p) == 4 for p in ps)
    lib.phieng_world_free(w)
    lib.phieng_world_free(w2)


def test_hostile_blocks_are_rejected_and_leave_the_world(lib):
    w = world2(lib, grid_pts())
    good = save(lib, w)
    w2 = world2(lib, grid_pts(2, 2) + 5.0)
    before = state2(lib, w2)
    # every truncation
    for k in range(len(good)):
        assert load(lib, w2, good[:k]) == -2, k
    # enabled flag other than 0 / 1
    cfg, _, _ = parse_block(good)
    en_off = len(good) - 4 - 12 * 21 - 1
    bad = bytearray(good)
    bad[en_off] = 2
    assert load(lib, w2, bytes(bad)) == -2
    # a non-finite particle value and a non-finite config scalar
    bad = bytearray(good)
    struct.pack_into("<f", bad, en_off + 5 + 21 * 3 + 4, float("nan"))
    assert load(lib, w2, bytes(bad)) == -2
    bad = bytearray(good)
    struct.pack_into("<f", bad, 8, float("inf"))  # smoothing_length
    assert load(lib, w2, bytes(bad)) == -2
    # more particles than the cap (MAX_PARTICLES_2D = 4096)
    bad = bytearray(good)
    struct.pack_into("<I", bad, en_off + 1, 4097)
    assert load(lib, w2, bytes(bad)) == -2
    np.testing.assert_array_equal(state2(lib, w2), before)
    assert lib.phieng_world_fluid_count(w2) == 4
    # argument errors
    assert lib.phieng_sph_fluid_block_save(None, 17, None, 0) == -1
    assert lib.phieng_sph_fluid_block_save(w, 0, None, 0) == -1
    assert lib.phieng_sph_fluid_block_save(w, 18, None, 0) == -1
    assert load(lib, w2, good, version=0) == -1
    lib.phieng_world_free(w)
    lib.phieng_world_free(w2)


def test_stored_mass_rules(lib):
    """mass = stored mass if positive, else max(particle_mass, 0)."""
    w = world2(lib, grid_pts(2, 1))
    data = bytearray(save(lib, w))
    n_off = len(data) - 2 * 21
    struct.pack_into("<f", data, n_off + 16, 0.0)  # first particle's mass
    struct.pack_into("<f", data, n_off + 21 + 16, 0.5)
    w2 = lib.phieng_world_new()
    assert load(lib, w2, bytes(data)) == len(data)
    _, ps, _ = parse_block(save(lib, w2))
    assert ps[0][2] == np.float32(0.0625) and ps[1][2] == 0.5
    lib.phieng_world_free(w)
    lib.phieng_world_free(w2)


def world3(lib, pts, cfg=None):
    w = lib.phieng_world3_new()
    lib.phieng_world3_add_body(w, 0.0, -1.0, 0.0, 1, 10.0, 0.5, 10.0, 1.0, 1, 0.5, 0.0)
    if cfg is not None:
        assert lib.phieng_world3_set_fluid_config(w, C.byref(cfg)) == 1
    p = np.ascontiguousarray(pts, np.float32)
    assert lib.phieng_world3_fluid_add(w, fp(p.ravel()), len(p)) == len(p)
    return w


def state3(lib, w):
    n = lib.phieng_world3_fluid_count(w)
    out = np.zeros((n, 6), np.float32)
    assert lib.phieng_world3_fluid_get(w, fp(out), n) == n
    return out


def pts3():
    return np.array([(ix * 0.25, iy * 0.25, iz * 0.25) for iz in range(2) for iy in range(2) for ix in range(3)],
                    np.float32)


def test_block3_layout_and_roundtrip(lib):
    w = world3(lib, pts3())
    data = save(lib, w, dim=3)
    cfg, ps, used = parse_block(data, dim=3)
    assert used == len(data) and len(ps) == 12 and len(data) - 12 * 29 == 104
    assert ps[5][0] == tuple(pts3()[5])
    w2 = lib.phieng_world3_new()
    assert load(lib, w2, data, dim=3) == len(data)
    np.testing.assert_array_equal(state3(lib, w2), state3(lib, w))
    assert save(lib, w2, dim=3) == data
    for k in (0, 50, len(data) - 1):
        assert load(lib, w2, data[:k], dim=3) == -2
    lib.phieng_world3_free(w)
    lib.phieng_world3_free(w2)


# ---- GPU: exact continuation ----------------------------------------------

@pytest.mark.gpu
def test_continuation_after_reload_2d(lib):
    """snapshot.rs:8680-8715 on the GPU world: 60 steps, save, load into a
    fresh world with the same walls, 60 more steps on both: bit-identical."""
    c = default_config()
    c.gamma = 7.0
    c.stiffness = 15.0
    c.artificial_viscosity = 1.2
    c.surface_tension = 0.7
    c.wall_friction = 0.4
    w = world2(lib, grid_pts(), c)
    for _ in range(60):
        lib.phieng_world_step(w, 1 / 60)
    data = save(lib, w)
    w2 = lib.phieng_world_new()
    lib.phieng_world_add_body(w2, 0.0, -1.0, _abi.SHAPE_BOX, 10.0, 0.5, 1.0, 1, 0.5, 0.0)
    assert load(lib, w2, data) == len(data)
    np.testing.assert_array_equal(state2(lib, w2), state2(lib, w))
    for _ in range(60):
        lib.phieng_world_step(w, 1 / 60)
        lib.phieng_world_step(w2, 1 / 60)
    a, b = state2(lib, w), state2(lib, w2)
    assert (a.view(np.uint32) == b.view(np.uint32)).all()
    lib.phieng_world_free(w)
    lib.phieng_world_free(w2)


@pytest.mark.gpu
def test_continuation_after_reload_3d(lib):
    w = world3(lib, pts3())
    for _ in range(40):
        lib.phieng_world3_step(w, 1 / 60)
    data = save(lib, w, dim=3)
    w2 = lib.phieng_world3_new()
    lib.phieng_world3_add_body(w2, 0.0, -1.0, 0.0, 1, 10.0, 0.5, 10.0, 1.0, 1, 0.5, 0.0)
    assert load(lib, w2, data, dim=3) == len(data)
    for _ in range(40):
        lib.phieng_world3_step(w, 1 / 60)
        lib.phieng_world3_step(w2, 1 / 60)
    a, b = state3(lib, w), state3(lib, w2)
    assert (a.view(np.uint32) == b.view(np.uint32)).all()
    lib.phieng_world3_free(w)
    lib.phieng_world3_free(w2)


@pytest.mark.gpu
def test_negative_smoothing_length_from_a_block(lib):
    """A block may carry h <= 0 (the load checks finiteness only). The
    kernels then keep poly6's range test for neighbours (h*h > max(h, EPS)^2);
    the step stays bit-exact with the oracle fed the same config."""
    from oracle.oracle import JACOBI, OracleWorld

    w = world2(lib, grid_pts(6, 4))
    data = bytearray(save(lib, w))
    struct.pack_into("<f", data, 8, -0.5)  # smoothing_length
    w2 = lib.phieng_world_new()
    lib.phieng_world_add_body(w2, 0.0, -1.0, _abi.SHAPE_BOX, 10.0, 0.5, 1.0, 1, 0.5, 0.0)
    assert load(lib, w2, bytes(data)) == len(data)
    cfg = _abi.FluidConfig2Ffi()
    lib.phieng_world_get_fluid_config(w2, C.byref(cfg))
    assert cfg.smoothing_length == -0.5
    o = OracleWorld()
    o.set_config(cfg)
    o.add_box(0.0, -1.0, 10.0, 0.5)
    o.add_particles(grid_pts(6, 4))
    for _ in range(20):
        o.step(1 / 60, JACOBI)
        lib.phieng_world_step(w2, 1 / 60)
    a, b = o.state(), state2(lib, w2)
    assert (a.view(np.uint32) == b.view(np.uint32)).all()
    lib.phieng_world_free(w)
    lib.phieng_world_free(w2)
