"""Ambient turbulence in the fluid integrate (fluid.rs:1001-1019) with the
engine's value noise (crates/dynamics/src/noise.rs).

CPU: the C ABI's ambient config (phieng_world_set/get_ambient_config,
ffi.rs:512-545, validation as ambient2_from_ffi, ffi.rs:328-386), the
oracle's noise against the reference's own noise tests (noise.rs:229-300),
and the reference's determinism test on the oracle
(test_fluid_turbulence_deterministic, fluid.rs:1497-1516).
GPU: the world step with turbulence bit for bit against the oracle's Jacobi
integrate, both noise modes, over many steps (the clock advances every step).
"""
import ctypes as C
import math

import numpy as np
import pytest

import sims
from oracle import oracle as orc
from phi_eng_b200 import _abi


@pytest.fixture(scope="module")
def lib():
    return _abi.load()


# ---------------------------------------------------------------- C ABI (no GPU work)
def test_ambient_struct_layout():
    assert C.sizeof(_abi.AmbientConfig2Ffi) == 80
    assert _abi.AmbientConfig2Ffi.turbulence_enabled.offset == 52
    assert _abi.AmbientConfig2Ffi.turbulence_divergence_free.offset == 76


def test_ambient_defaults_and_roundtrip(lib):
    w = lib.phieng_world_new()
    try:
        a = _abi.AmbientConfig2Ffi()
        assert lib.phieng_world_get_ambient_config(w, C.byref(a)) == 1
        d = _abi.default_ambient()
        for name, _ in _abi.AmbientConfig2Ffi._fields_:
            assert getattr(a, name) == getattr(d, name), name
        a.turbulence_enabled = 7  # any non-zero flag reads back as 1
        a.turbulence_amplitude = 5.0
        a.turbulence_frequency = 0.5
        a.turbulence_seed = 0xFFFFFFFF
        a.turbulence_octaves = 1000  # stored as min(v, 255)
        a.turbulence_divergence_free = 1
        a.wind_x = -3.0
        assert lib.phieng_world_set_ambient_config(w, C.byref(a)) == 1
        b = _abi.AmbientConfig2Ffi()
        assert lib.phieng_world_get_ambient_config(w, C.byref(b)) == 1
        assert (b.turbulence_enabled, b.turbulence_amplitude, b.turbulence_frequency) == (1, 5.0, 0.5)
        assert (b.turbulence_seed, b.turbulence_octaves, b.turbulence_divergence_free) == (0xFFFFFFFF, 255, 1)
        assert b.wind_x == -3.0 and b.air_density == 1.0
    finally:
        lib.phieng_world_free(w)


@pytest.mark.parametrize("field,value", [
    ("turbulence_amplitude", -1.0), ("turbulence_amplitude", math.nan), ("turbulence_frequency", math.inf),
    ("turbulence_time_scale", -math.inf), ("spring_stiffness", -1.0), ("drag_linear", -0.5),
    ("air_density", -1.0), ("wind_y", math.nan), ("spring_max_displacement", -2.0)])
def test_ambient_rejects_invalid_and_keeps_world(lib, field, value):
    w = lib.phieng_world_new()
    try:
        a = _abi.default_ambient()
        a.turbulence_amplitude = 2.0
        assert lib.phieng_world_set_ambient_config(w, C.byref(a)) == 1
        bad = _abi.default_ambient()
        setattr(bad, field, value)
        assert lib.phieng_world_set_ambient_config(w, C.byref(bad)) == 0
        b = _abi.AmbientConfig2Ffi()
        lib.phieng_world_get_ambient_config(w, C.byref(b))
        assert b.turbulence_amplitude == 2.0  # unchanged
        # negative frequency / time scale are finite and accepted, as the reference
        ok = _abi.default_ambient()
        ok.turbulence_frequency = -1.0
        ok.turbulence_time_scale = -2.0
        assert lib.phieng_world_set_ambient_config(w, C.byref(ok)) == 1
    finally:
        lib.phieng_world_free(w)


def test_ambient_null_arguments(lib):
    a = _abi.default_ambient()
    assert lib.phieng_world_set_ambient_config(None, C.byref(a)) == 0
    assert lib.phieng_world_get_ambient_config(None, C.byref(a)) == 0
    w = lib.phieng_world_new()
    try:
        assert lib.phieng_world_set_ambient_config(w, None) == 0
        assert lib.phieng_world_get_ambient_config(w, None) == 0
    finally:
        lib.phieng_world_free(w)


# ---------------------------------------------------------------- oracle noise (noise.rs tests)
def test_value_noise_range():  # noise.rs:229-239
    for i in range(50):
        n = orc.noise2("value", np.float32(i * 0.37), np.float32(i * -0.53), seed=0x1234)
        assert 0.0 <= n < 1.0


def test_noise_deterministic():  # noise.rs:241-250
    a = orc.noise2("fbm", 1.25, -2.5, 3.0, 99, 4)
    b = orc.noise2("fbm", 1.25, -2.5, 3.0, 99, 4)
    assert np.float32(a).view(np.uint32) == np.float32(b).view(np.uint32)


def test_noise_lipschitz_and_continuity():  # noise.rs:252-265
    base = orc.noise2("fbm", 1.0, 1.0, 0.0, 5, 3)
    for k in range(1, 9):
        eps = np.float32(k) * np.float32(1e-3)
        assert abs(orc.noise2("fbm", np.float32(1.0) + eps, 1.0, 0.0, 5, 3) - base) < 0.5


def test_noise_time_continuity():  # noise.rs:267-272
    a = orc.noise2("fbm", 0.5, 0.5, 10.0, 3, 3)
    b = orc.noise2("fbm", 0.5, 0.5, 10.0001, 3, 3)
    assert abs(a - b) < 0.01


def test_noise_bounded():  # noise.rs:274-282
    for i in range(200):
        x = np.float32(np.float32(i) * np.float32(0.11) - np.float32(5.0))
        y = np.float32(np.float32(i) * np.float32(-0.07) + np.float32(3.0))
        n = orc.noise2("fbm", x, y, np.float32(i) * np.float32(0.05), i, 5)
        assert abs(n) <= 1.0 + 1e-5


def test_curl_divergence_free():  # noise.rs:284-300
    e = np.float32(1e-3)
    for i in range(20):
        x = np.float32(i) * np.float32(0.3)
        y = np.float32(i) * np.float32(0.21)
        dvx = (orc.noise2("curl", x + e, y, 0.0, 11, 3)[0] - orc.noise2("curl", x - e, y, 0.0, 11, 3)[0]) / (2 * e)
        dvy = (orc.noise2("curl", x, y + e, 0.0, 11, 3)[1] - orc.noise2("curl", x, y - e, 0.0, 11, 3)[1]) / (2 * e)
        assert abs(dvx + dvy) < 1.0


def test_octaves_clamped():
    # fbm_2 clamps octaves to 1..=8 (noise.rs:161): 0 acts as 1, 200 as 8
    assert orc.noise2("fbm", 0.7, 0.2, 1.5, 3, 0) == orc.noise2("fbm", 0.7, 0.2, 1.5, 3, 1)
    assert orc.noise2("fbm", 0.7, 0.2, 1.5, 3, 200) == orc.noise2("fbm", 0.7, 0.2, 1.5, 3, 8)


# ---------------------------------------------------------------- the reference's fluid test
REF_TURB = dict(amplitude=5.0, frequency=0.5, seed=7, octaves=3)  # fluid.rs:1503-1507


def ref_scene(sim, turb=None, divergence_free=False):
    sims.tank(sim)
    sims.lattice(sim, 0.0, 0.0, 6, 8, 0.25)
    if turb:
        sim.set_turbulence(**turb, divergence_free=divergence_free)
    return sim


class _OracleTurb(sims.OracleSim):
    def set_turbulence(self, **kw):
        self.w.set_turbulence(**kw)


class _GpuTurb(sims.GpuSim):
    def set_turbulence(self, **kw):
        self.w.set_turbulence(**kw)


@pytest.mark.parametrize("curl", [False, True])
def test_fluid_turbulence_deterministic_oracle(curl):
    """test_fluid_turbulence_deterministic (fluid.rs:1497-1516) on the oracle
    (the reference's in-place order): two runs agree bit for bit, and the
    field does move the fluid."""
    def run(turb):
        s = ref_scene(_OracleTurb(orc.REF_SEQ), turb, curl)
        s.step(1.0 / 60.0, 120)
        return s.state()

    a, b, c = run(REF_TURB), run(REF_TURB), run(None)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert np.isfinite(a).all()
    assert not np.array_equal(a, c)


# ---------------------------------------------------------------- GPU vs oracle
def _compare(gpu, ora, what):
    g, o = gpu.state(), ora.state()
    assert g.shape == o.shape
    bad = np.nonzero(g.view(np.uint32) != o.view(np.uint32))
    assert bad[0].size == 0, f"{what}: {bad[0].size} words differ, first particle {bad[0][:1]}"


@pytest.mark.gpu
@pytest.mark.parametrize("curl", [False, True])
def test_turbulence_matches_oracle_ref_scene(curl):
    """The reference's turbulence scene, 120 world steps of 1/60: the GPU step
    equals the oracle's Jacobi integrate bit for bit at every 20th step."""
    gpu = ref_scene(_GpuTurb(), REF_TURB, curl)
    ora = ref_scene(_OracleTurb(orc.JACOBI), REF_TURB, curl)
    for k in range(6):
        gpu.step(1.0 / 60.0, 20)
        ora.step(1.0 / 60.0, 20)
        _compare(gpu, ora, f"step {20 * (k + 1)}")
    # and the field is on: without it the state differs
    plain = ref_scene(_GpuTurb())
    plain.step(1.0 / 60.0, 120)
    assert not np.array_equal(plain.state(), gpu.state())


@pytest.mark.gpu
def test_turbulence_matches_oracle_dam_break_4k():
    """A 4096-particle dam break (CFL substeps on, so several substeps share
    one step's clock) with curl turbulence, time scale 3 and 5 octaves."""
    from phi_eng_b200 import scenes as S

    sc = S.dam_break_4k()
    cfg = sc.config
    cfg.cfl = 0.4
    cfg.max_substeps = 4
    turb = dict(amplitude=20.0, frequency=2.0, time_scale=3.0, seed=0xC0FFEE, octaves=5, divergence_free=True)
    sims_ = []
    for s in (_GpuTurb(), _OracleTurb(orc.JACOBI)):
        sims.load_scene(s, sc)
        s.config = cfg
        s.set_turbulence(**turb)
        sims_.append(s)
    gpu, ora = sims_
    for k in range(4):
        gpu.step(sc.dt, 10)
        ora.step(sc.dt, 10)
        _compare(gpu, ora, f"step {10 * (k + 1)}")
