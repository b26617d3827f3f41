"""ORACLE — TEST INFRASTRUCTURE ONLY.

ctypes wrapper of oracle/liboracle.so, the C++ restatement of the reference
2D SPH step (crates/dynamics/src/fluid.rs) and 3D step (fluid3.rs). Only tests/, the smoke check and
the CPU-baseline leg of bench.py import this module; the product library
never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from phi_eng_b200._abi import FluidConfig2Ffi, default_config

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

REF_SEQ = 0
JACOBI = 1

_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    lib = C.CDLL(LIB_PATH)
    P, F, D, U32, U8 = C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_uint32), C.POINTER(C.c_uint8)
    I32 = C.POINTER(C.c_int32)
    sig = {
        "orc_new": (P, [C.c_int]),
        "orc_free": (None, [P]),
        "orc_set_config": (None, [P, C.POINTER(FluidConfig2Ffi)]),
        "orc_get_config": (None, [P, C.POINTER(FluidConfig2Ffi)]),
        "orc_set_gravity": (None, [P, C.c_float, C.c_float]),
        "orc_set_turbulence": (None, [P, C.c_int, C.c_float, C.c_float, C.c_float, C.c_uint32, C.c_uint32, C.c_int]),
        "orc_set_wind": (None, [P, C.c_float, C.c_float]),
        "orc_ghosts": (C.c_uint32, [P, C.c_void_p, C.c_uint32]),
        "orc_masses": (C.c_uint32, [P, C.c_void_p, C.c_uint32]),
        "orc3_ghosts": (C.c_uint32, [P, C.c_void_p, C.c_uint32]),
        "orc3_masses": (C.c_uint32, [P, C.c_void_p, C.c_uint32]),
        "orc3_set_turbulence": (None, [P, C.c_int, C.c_float, C.c_float, C.c_float, C.c_uint32, C.c_uint32, C.c_int]),
        "orc_noise2": (None, [C.c_int, C.c_float, C.c_float, C.c_float, C.c_uint32, C.c_uint32, C.POINTER(C.c_float)]),
        "orc_set_cap": (None, [P, C.c_uint32]),
        "orc_set_pow_mode": (None, [P, C.c_int]),
        "orc_add_body": (None, [P, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float,
                                C.c_float, C.c_float, C.c_float, C.c_float]),
        "orc_add_particles": (C.c_uint32, [P, F, U8, C.c_uint32]),
        "orc_step_fluid": (None, [P, C.c_void_p, C.c_uint32, C.c_float, C.c_int]),
        "orc_step_fluid_poly": (None, [P, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_float,
                                       C.c_int]),
        "orc_count": (C.c_uint32, [P]),
        "orc_clear": (None, [P]),
        "orc_set_state": (None, [P, F, C.c_uint32]),
        "orc_set_density_pressure": (None, [P, F, F, C.c_uint32]),
        "orc_get_state": (C.c_uint32, [P, F, C.c_uint32]),
        "orc_get_state64": (C.c_uint32, [P, D, C.c_uint32]),
        "orc_get_density_pressure": (C.c_uint32, [P, F, F, C.c_uint32]),
        "orc_get_density_pressure64": (C.c_uint32, [P, D, D, C.c_uint32]),
        "orc_step": (None, [P, C.c_float, C.c_int]),
        "orc_steps": (C.c_double, [P, C.c_float, C.c_int, C.c_uint32]),
        "orc_substep": (None, [P, C.c_float, C.c_int]),
        "orc_pass_density": (None, [P]),
        "orc_pass_forces": (None, [P]),
        "orc_get_forces": (C.c_uint32, [P, F, C.c_uint32]),
        "orc_get_forces64": (C.c_uint32, [P, D, C.c_uint32]),
        "orc_neighbors": (C.c_uint32, [P, C.c_uint32, U32, C.c_uint32]),
        "orc_all_neighbors": (None, [P, U32, U32, C.c_uint32]),
        "orc_cells": (None, [P, I32, I32]),
        "orc_cfl_substeps": (C.c_uint32, [P, C.c_float]),
        "orc_set_extra_accel": (None, [P, F, C.c_uint32]),
        "orc_features": (C.c_uint32, [P, C.c_float, F, C.c_uint32]),
        "orc_poly6": (C.c_float, [C.c_float, C.c_float]),
        "orc_spiky": (None, [C.c_float, C.c_float, C.c_float, C.c_float, F]),
        "orc_pressure": (C.c_float, [C.c_float, C.c_float, C.c_float, C.c_float]),
        "orc_artificial_pressure": (C.c_float, [C.c_float] * 9),
        "orc_cohesion": (C.c_float, [C.c_float, C.c_float]),
        "orc3_new": (P, [C.c_int]),
        "orc3_free": (None, [P]),
        "orc3_set_config": (None, [P, C.POINTER(FluidConfig2Ffi)]),
        "orc3_set_gravity": (None, [P, C.c_float, C.c_float, C.c_float]),
        "orc3_set_pow_mode": (None, [P, C.c_int]),
        "orc3_set_cap": (None, [P, C.c_uint32]),
        "orc3_add_body": (None, [P, C.c_int] + [C.c_float] * 6),
        "orc3_add_particles": (C.c_uint32, [P, F, U8, C.c_uint32]),
        "orc3_count": (C.c_uint32, [P]),
        "orc3_set_state": (None, [P, F, C.c_uint32]),
        "orc3_get_state": (C.c_uint32, [P, F, C.c_uint32]),
        "orc3_get_density_pressure": (C.c_uint32, [P, F, F, C.c_uint32]),
        "orc3_step": (None, [P, C.c_float, C.c_int]),
        "orc3_steps": (C.c_double, [P, C.c_float, C.c_int, C.c_uint32]),
        "orc3_time": (C.c_float, [P]),
        "orc3_passes": (None, [P, C.c_int]),
        "orc3_get_forces": (C.c_uint32, [P, F, C.c_uint32]),
        "orc3_neighbors": (C.c_uint32, [P, C.c_uint32, U32, C.c_uint32]),
        "orc3_cfl_substeps": (C.c_uint32, [P, C.c_float]),
        "orc3_collide": (C.c_int, [C.c_int] + [C.c_float] * 7 + [F]),
        "orc3_poly6": (C.c_float, [C.c_float, C.c_float]),
        "orc3_spiky": (None, [C.c_float] * 5 + [F]),
        "orc3_step_fluid": (None, [P, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_float,
                                   C.c_int]),
        "orc3_set_wind": (None, [P, C.c_float, C.c_float, C.c_float]),
        "orc3_qrot": (None, [C.c_float] * 4 + [F, F]),
        "orc3_world_inv_inertia": (None, [C.c_float] * 4 + [F, F]),
        "orc3_surface_samples": (C.c_uint32, [C.c_void_p, F, C.c_uint32]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _fp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def lib():
    return _load()


class OracleWorld:
    """A World2-shaped CPU world: static bodies + one SPH fluid.

    mode: REF_SEQ (the reference's in-place integrate) or JACOBI.
    fp64: run the same algorithm in double precision.
    """

    def __init__(self, fp64: bool = False, cap: int = 4096, libm_pow: bool = False):
        """libm_pow: evaluate the Tait power with the platform powf (as the
        reference's f32::powf does) instead of the correctly rounded power."""
        self._l = _load()
        self._h = self._l.orc_new(1 if fp64 else 0)
        self.fp64 = fp64
        self._l.orc_set_cap(self._h, cap)
        self._l.orc_set_pow_mode(self._h, 0 if libm_pow else 1)

    def __del__(self):
        try:
            if self._h:
                self._l.orc_free(self._h)
                self._h = None
        except Exception:
            pass

    # ---- setup ----
    def set_config(self, cfg: FluidConfig2Ffi) -> None:
        self._l.orc_set_config(self._h, C.byref(cfg))

    def get_config(self) -> FluidConfig2Ffi:
        c = FluidConfig2Ffi()
        self._l.orc_get_config(self._h, C.byref(c))
        return c

    def set_gravity(self, gx: float, gy: float) -> None:
        self._l.orc_set_gravity(self._h, gx, gy)

    def masses(self) -> np.ndarray:
        """Particle masses by index."""
        n = self._l.orc_masses(self._h, None, 0)
        out = np.zeros(n, np.float32)
        self._l.orc_masses(self._h, out.ctypes.data, n)
        return out

    def ghosts(self) -> np.ndarray:
        """Boundary ghost positions of the last substep [m][2], generation order."""
        n = self._l.orc_ghosts(self._h, None, 0)
        out = np.zeros((n, 2), np.float32)
        self._l.orc_ghosts(self._h, out.ctypes.data, n)
        return out

    def set_wind(self, wx: float, wy: float) -> None:
        """world.ambient.drag.wind, against which the buoyancy drag acts."""
        self._l.orc_set_wind(self._h, wx, wy)

    def set_turbulence(self, amplitude: float, frequency: float = 1.0, time_scale: float = 1.0, seed: int = 0,
                       octaves: int = 3, divergence_free: bool = False, enabled: bool = True) -> None:
        """world.ambient.turbulence (ambient.rs:108-126), read by the integrate
        at the world clock of each step's start."""
        self._l.orc_set_turbulence(self._h, 1 if enabled else 0, amplitude, frequency, time_scale,
                                   seed & 0xFFFFFFFF, octaves, 1 if divergence_free else 0)

    def set_cap(self, cap: int) -> None:
        self._l.orc_set_cap(self._h, cap)

    def add_box(self, px, py, hx, hy, rot=(1.0, 0.0, 0.0, 1.0)) -> None:
        """Static box; rot = (x_axis.x, x_axis.y, y_axis.x, y_axis.y)."""
        self._l.orc_add_body(self._h, 1, px, py, hx, hy, *rot)

    def add_circle(self, px, py, r, rot=(1.0, 0.0, 0.0, 1.0)) -> None:
        self._l.orc_add_body(self._h, 0, px, py, r, 0.0, *rot)

    def add_particles(self, xy, phases=None) -> int:
        xy = np.ascontiguousarray(xy, dtype=np.float32).reshape(-1, 2)
        n = xy.shape[0]
        ph = None
        if phases is not None:
            ph = np.ascontiguousarray(phases, dtype=np.uint8)
            ph_p = ph.ctypes.data_as(C.POINTER(C.c_uint8))
        else:
            ph_p = None
        return int(self._l.orc_add_particles(self._h, _fp(xy), ph_p, n))

    @property
    def count(self) -> int:
        return int(self._l.orc_count(self._h))

    def set_state(self, xyvv) -> None:
        a = np.ascontiguousarray(xyvv, dtype=np.float32).reshape(-1, 4)
        self._l.orc_set_state(self._h, _fp(a), a.shape[0])

    def set_density_pressure(self, d, p) -> None:
        d = np.ascontiguousarray(d, dtype=np.float32)
        p = np.ascontiguousarray(p, dtype=np.float32)
        self._l.orc_set_density_pressure(self._h, _fp(d), _fp(p), d.shape[0])

    # ---- readback ----
    def state(self) -> np.ndarray:
        n = self.count
        if self.fp64:
            out = np.zeros((n, 4), np.float64)
            self._l.orc_get_state64(self._h, out.ctypes.data_as(C.POINTER(C.c_double)), n)
        else:
            out = np.zeros((n, 4), np.float32)
            self._l.orc_get_state(self._h, _fp(out), n)
        return out

    def density_pressure(self):
        n = self.count
        if self.fp64:
            d = np.zeros(n, np.float64)
            p = np.zeros(n, np.float64)
            D = C.POINTER(C.c_double)
            self._l.orc_get_density_pressure64(self._h, d.ctypes.data_as(D), p.ctypes.data_as(D), n)
        else:
            d = np.zeros(n, np.float32)
            p = np.zeros(n, np.float32)
            self._l.orc_get_density_pressure(self._h, _fp(d), _fp(p), n)
        return d, p

    def forces(self) -> np.ndarray:
        n = self.count
        if self.fp64:
            out = np.zeros((n, 2), np.float64)
            self._l.orc_get_forces64(self._h, out.ctypes.data_as(C.POINTER(C.c_double)), n)
        else:
            out = np.zeros((n, 2), np.float32)
            self._l.orc_get_forces(self._h, _fp(out), n)
        return out

    def neighbors(self, i: int, max_n: int = 256) -> np.ndarray:
        out = np.zeros(max_n, np.uint32)
        k = self._l.orc_neighbors(self._h, i, out.ctypes.data_as(C.POINTER(C.c_uint32)), max_n)
        return out[: min(k, max_n)].copy()

    def all_neighbors(self, max_per: int = 64):
        n = self.count
        counts = np.zeros(n, np.uint32)
        lists = np.zeros(n * max_per, np.uint32)
        U = C.POINTER(C.c_uint32)
        self._l.orc_all_neighbors(self._h, counts.ctypes.data_as(U), lists.ctypes.data_as(U), max_per)
        return counts, lists.reshape(n, max_per)

    def cells(self):
        n = self.count
        cx = np.zeros(n, np.int32)
        cy = np.zeros(n, np.int32)
        I = C.POINTER(C.c_int32)
        self._l.orc_cells(self._h, cx.ctypes.data_as(I), cy.ctypes.data_as(I))
        return cx, cy

    # ---- stepping ----
    def step(self, dt: float, mode: int = REF_SEQ) -> None:
        self._l.orc_step(self._h, dt, mode)

    def steps(self, dt: float, k: int, mode: int = REF_SEQ) -> float:
        """k world steps; returns the wall seconds spent inside C++."""
        return float(self._l.orc_steps(self._h, dt, mode, k))

    def substep(self, dt: float, mode: int = REF_SEQ) -> None:
        self._l.orc_substep(self._h, dt, mode)

    def pass_density(self) -> None:
        self._l.orc_pass_density(self._h)

    def pass_forces(self) -> None:
        self._l.orc_pass_forces(self._h)

    def cfl_substeps(self, dt: float) -> int:
        return int(self._l.orc_cfl_substeps(self._h, dt))

    def step_fluid(self, bodies, dt: float, mode: int = REF_SEQ, poly=None) -> None:
        """FluidState2::step_fluid with `bodies` (a ctypes PhiengBody2 array,
        updated in place) in place of the world's bodies; no clock. poly =
        (xy float32 [m][2], first uint32 [nb], count uint32 [nb]): the local
        vertices of the PHIENG_SHAPE_POLYGON bodies."""
        if poly is None:
            self._l.orc_step_fluid(self._h, C.cast(bodies, C.c_void_p), len(bodies), dt, mode)
            return
        xy, first, count = (np.ascontiguousarray(a) for a in poly)
        self._l.orc_step_fluid_poly(self._h, C.cast(bodies, C.c_void_p), len(bodies), xy.ctypes.data,
                                    first.ctypes.data, count.ctypes.data, dt, mode)

    # ---- learned-closure hooks ----
    def features(self, dt: float) -> np.ndarray:
        """Closure inputs [n][16] at the current state for a substep dt."""
        n = self.count
        out = np.zeros((n, 16), np.float32)
        k = self._l.orc_features(self._h, dt, _fp(out), n)
        assert k == n
        return out

    def set_extra_accel(self, a) -> None:
        """Per-particle acceleration [n][2] added in the next substep's integrate."""
        a = np.ascontiguousarray(a, dtype=np.float32).reshape(-1, 2)
        self._l.orc_set_extra_accel(self._h, _fp(a), a.shape[0])


class OracleWorld3:
    """A World3-shaped CPU world: static sphere / box / capsule bodies + one
    3D SPH fluid (crates/dynamics/src/fluid3.rs). Same modes as OracleWorld."""

    SPHERE, BOX, CAPSULE = 0, 1, 2

    def __init__(self, fp64: bool = False, cap: int = 4096, libm_pow: bool = False):
        self._l = _load()
        self._h = self._l.orc3_new(1 if fp64 else 0)
        self.fp64 = fp64
        self._l.orc3_set_cap(self._h, cap)
        self._l.orc3_set_pow_mode(self._h, 0 if libm_pow else 1)

    def __del__(self):
        try:
            if self._h:
                self._l.orc3_free(self._h)
                self._h = None
        except Exception:
            pass

    def set_config(self, cfg: FluidConfig2Ffi) -> None:
        self._l.orc3_set_config(self._h, C.byref(cfg))

    def masses(self) -> np.ndarray:
        """Particle masses by index."""
        n = self._l.orc3_masses(self._h, None, 0)
        out = np.zeros(n, np.float32)
        self._l.orc3_masses(self._h, out.ctypes.data, n)
        return out

    def ghosts(self) -> np.ndarray:
        """3D boundary ghost positions of the last substep [m][3], generation order."""
        n = self._l.orc3_ghosts(self._h, None, 0)
        out = np.zeros((n, 3), np.float32)
        self._l.orc3_ghosts(self._h, out.ctypes.data, n)
        return out

    def set_turbulence(self, amplitude: float, frequency: float = 1.0, time_scale: float = 1.0, seed: int = 0,
                       octaves: int = 3, divergence_free: bool = False, enabled: bool = True) -> None:
        """world.ambient.turbulence (TurbulenceConfig3), read by the integrate
        at the world clock of each step's start."""
        self._l.orc3_set_turbulence(self._h, 1 if enabled else 0, amplitude, frequency, time_scale,
                                    seed & 0xFFFFFFFF, octaves, 1 if divergence_free else 0)

    def set_gravity(self, gx: float, gy: float, gz: float) -> None:
        self._l.orc3_set_gravity(self._h, gx, gy, gz)

    def add_body(self, shape: int, px, py, pz, a, b=0.0, c=0.0) -> None:
        self._l.orc3_add_body(self._h, shape, px, py, pz, a, b, c)

    def add_particles(self, xyz, phases=None) -> int:
        xyz = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1, 3)
        ph_p = None
        if phases is not None:
            ph = np.ascontiguousarray(phases, dtype=np.uint8)
            ph_p = ph.ctypes.data_as(C.POINTER(C.c_uint8))
        return int(self._l.orc3_add_particles(self._h, _fp(xyz), ph_p, xyz.shape[0]))

    @property
    def count(self) -> int:
        return int(self._l.orc3_count(self._h))

    @property
    def time(self) -> float:
        return float(self._l.orc3_time(self._h))

    def set_state(self, q) -> None:
        a = np.ascontiguousarray(q, dtype=np.float32).reshape(-1, 6)
        self._l.orc3_set_state(self._h, _fp(a), a.shape[0])

    def state(self) -> np.ndarray:
        """[n][6] = x, y, z, vx, vy, vz."""
        out = np.zeros((self.count, 6), np.float32)
        self._l.orc3_get_state(self._h, _fp(out), out.shape[0])
        return out

    def density_pressure(self):
        n = self.count
        d = np.zeros(n, np.float32)
        p = np.zeros(n, np.float32)
        self._l.orc3_get_density_pressure(self._h, _fp(d), _fp(p), n)
        return d, p

    def passes(self, forces: bool = True) -> None:
        """Density (and force) pass on the current state."""
        self._l.orc3_passes(self._h, 1 if forces else 0)

    def forces(self) -> np.ndarray:
        out = np.zeros((self.count, 3), np.float32)
        self._l.orc3_get_forces(self._h, _fp(out), out.shape[0])
        return out

    def neighbors(self, i: int, max_n: int = 512) -> np.ndarray:
        out = np.zeros(max_n, np.uint32)
        k = self._l.orc3_neighbors(self._h, i, out.ctypes.data_as(C.POINTER(C.c_uint32)), max_n)
        return out[: min(k, max_n)].copy()

    def step(self, dt: float, mode: int = REF_SEQ) -> None:
        self._l.orc3_step(self._h, dt, mode)

    def steps(self, dt: float, k: int, mode: int = REF_SEQ) -> float:
        return float(self._l.orc3_steps(self._h, dt, mode, k))

    def cfl_substeps(self, dt: float) -> int:
        return int(self._l.orc3_cfl_substeps(self._h, dt))

    def set_wind(self, x: float, y: float, z: float) -> None:
        """world.ambient.drag.wind, read by the buoyancy drag (fluid3.rs:1196)."""
        self._l.orc3_set_wind(self._h, x, y, z)

    def step_fluid(self, bodies, dt: float, mode: int = REF_SEQ, hulls=None) -> None:
        """FluidState3::step_fluid with `bodies` (a ctypes PhiengBody3 array,
        updated in place) in place of the world's bodies; no clock. hulls =
        (xyz float32 [m][3], first uint32 [nb], count uint32 [nb]): the local
        vertices of the PHIENG_SHAPE3_HULL bodies."""
        if hulls is None:
            self._l.orc3_step_fluid(self._h, C.cast(bodies, C.c_void_p), len(bodies), None, None, None, dt, mode)
            return
        xyz, first, count = (np.ascontiguousarray(a) for a in hulls)
        self._l.orc3_step_fluid(self._h, C.cast(bodies, C.c_void_p), len(bodies), xyz.ctypes.data,
                                first.ctypes.data, count.ctypes.data, dt, mode)


def collide3(shape: int, a: float, b: float, c: float, p, pr: float):
    """Particle at p (body frame, body at the origin) vs one static body:
    (normal xyz, depth) or None when separated."""
    out = np.zeros(4, np.float32)
    hit = _load().orc3_collide(shape, a, b, c, p[0], p[1], p[2], pr, _fp(out))
    return (tuple(float(v) for v in out[:3]), float(out[3])) if hit else None


def qrot3(q, v):
    """v rotated by the unit quaternion q = (x, y, z, w), in the fluid
    phase's f32 evaluation order."""
    vv = np.ascontiguousarray(v, np.float32)
    out = np.zeros(3, np.float32)
    _load().orc3_qrot(q[0], q[1], q[2], q[3], _fp(vv), _fp(out))
    return out


def world_inv_inertia3(q, inv_inertia) -> np.ndarray:
    """(R I^-1) R^T, column-major [9], for R = Mat3::from_quat(q)."""
    ii = np.ascontiguousarray(inv_inertia, np.float32).ravel()
    out = np.zeros(9, np.float32)
    _load().orc3_world_inv_inertia(q[0], q[1], q[2], q[3], _fp(ii), _fp(out))
    return out


def surface_samples3(body) -> np.ndarray:
    """Buoyancy samples of one PhiengBody3: [k][7] = point, outward normal, area."""
    n = _load().orc3_surface_samples(C.addressof(body), None, 0)
    out = np.zeros((n, 7), np.float32)
    _load().orc3_surface_samples(C.addressof(body), _fp(out), n)
    return out


def poly6_3(r2: float, h: float) -> float:
    return float(_load().orc3_poly6(r2, h))


def spiky_grad3(rx: float, ry: float, rz: float, r: float, h: float):
    out = np.zeros(3, np.float32)
    _load().orc3_spiky(rx, ry, rz, r, h, _fp(out))
    return tuple(float(v) for v in out)


# scalar kernels (f32) for the reference's kernel-sanity checks
def poly6(r2: float, h: float) -> float:
    return float(_load().orc_poly6(r2, h))


def spiky_grad(rx: float, ry: float, r: float, h: float):
    out = np.zeros(2, np.float32)
    _load().orc_spiky(rx, ry, r, h, _fp(out))
    return float(out[0]), float(out[1])


def pressure(d: float, rho0: float, k: float, gamma: float) -> float:
    return float(_load().orc_pressure(d, rho0, k, gamma))


def artificial_pressure(dx, dy, vrx, vry, r_sq, h, rho_bar, c, alpha) -> float:
    return float(_load().orc_artificial_pressure(dx, dy, vrx, vry, r_sq, h, rho_bar, c, alpha))


def cohesion(dist: float, h: float) -> float:
    return float(_load().orc_cohesion(dist, h))


__all__ = ["OracleWorld", "OracleWorld3", "REF_SEQ", "JACOBI", "default_config", "build", "lib"]


def noise2(kind: str, x: float, y: float, t: float = 0.0, seed: int = 0, octaves: int = 3):
    """The oracle's f32 restatement of noise.rs: kind "value" (value_noise_2),
    "fbm" (fbm_2) or "curl" (curl_2, a pair)."""
    out = (C.c_float * 2)()
    k = {"value": 0, "fbm": 1, "curl": 2}[kind]
    _load().orc_noise2(k, x, y, t, seed & 0xFFFFFFFF, octaves, out)
    return (out[0], out[1]) if k == 2 else out[0]
