"""Python mirror of the reference's World3 / FluidState3 API over the C ABI.

The reference drives the 3D fluid as

    let mut world = World3::new();
    world.add_body(RigidBody3::static_body(..) with Shape3::Box { half_extents });
    world.fluid.config = FluidConfig3 { .. };
    world.fluid.add_particles(&pts);
    world.step(dt);
    for p in world.fluid.particles.iter() { .. }

(crates/dynamics/src/fluid3.rs, crates/engine/src/ffi.rs:3199-3885). This
module offers the same shape — ``World3()``, ``add_static_body`` with
``Sphere`` / ``Box3`` / ``Capsule``, ``world.fluid.config``,
``world.fluid.add_particles``, ``world.step`` and ``world.fluid.particles`` —
with every call going through libphieng_sph.so; the particle state stays on
the GPU between steps. There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._abi import FluidConfig3Ffi, default_config
from .world import SphError, _fptr


@dataclass
class Sphere:
    """Shape3::Sphere { radius }."""

    radius: float


@dataclass
class Box3:
    """Shape3::Box { half_extents }."""

    hx: float
    hy: float
    hz: float


@dataclass
class Capsule:
    """Shape3::Capsule { radius, half_length } along the body's y axis."""

    radius: float
    half_length: float


def body3(shape, position, rotation=(0.0, 0.0, 0.0, 1.0), density: float | None = None, velocity=(0.0, 0.0, 0.0),
          angular_velocity=(0.0, 0.0, 0.0)) -> "_abi.PhiengBody3":
    """A PhiengBody3 for World3.step_fluid: static when density is None, else
    dynamic with the mass and diagonal inertia of mass_properties_3d
    (body.rs:811-830) for a Sphere or Box3 (inverse inertia 1 / I per axis)."""
    b = _abi.PhiengBody3()
    if isinstance(shape, Sphere):
        b.shape_tag, b.a = _abi.SHAPE3_SPHERE, shape.radius
    elif isinstance(shape, Box3):
        b.shape_tag, b.a, b.b, b.c = _abi.SHAPE3_BOX, shape.hx, shape.hy, shape.hz
    elif isinstance(shape, Capsule):
        b.shape_tag, b.a, b.b = _abi.SHAPE3_CAPSULE, shape.radius, shape.half_length
    else:
        raise TypeError("shape must be Sphere, Box3 or Capsule")
    b.px, b.py, b.pz = (float(v) for v in position)
    b.qx, b.qy, b.qz, b.qw = (float(v) for v in rotation)
    b.vx, b.vy, b.vz = (float(v) for v in velocity)
    b.wx, b.wy, b.wz = (float(v) for v in angular_velocity)
    if density is None:
        b.is_static = 1
        return b
    f = np.float32
    d = f(density)
    if isinstance(shape, Sphere):
        r = f(shape.radius)
        m = ((f(4.0) / f(3.0)) * f(np.pi) * r * r * r) * d
        i = f(0.4) * m * r * r
        diag = (i, i, i)
    elif isinstance(shape, Box3):
        w, h, dd = f(shape.hx) * f(2), f(shape.hy) * f(2), f(shape.hz) * f(2)
        m = (w * h * dd) * d
        diag = (m * (h * h + dd * dd) / f(12), m * (w * w + dd * dd) / f(12), m * (w * w + h * h) / f(12))
    else:
        raise TypeError("dynamic bodies here: Sphere or Box3 (pass inv_mass / inv_inertia yourself for others)")
    b.is_static = 0
    b.inv_mass = f(1) / m
    for k in range(3):
        b.inv_inertia[4 * k] = f(1) / diag[k]
    return b


class FluidState3:
    """world.fluid of a World3: config, particle insertion and read-back."""

    def __init__(self, world: "World3"):
        self._world = world

    @property
    def _lib(self):
        return self._world._lib

    @property
    def _h(self):
        return self._world._h

    @property
    def config(self) -> FluidConfig3Ffi:
        c = FluidConfig3Ffi()
        self._lib.phieng_world3_get_fluid_config(self._h, C.byref(c))
        return c

    @config.setter
    def config(self, cfg: FluidConfig3Ffi) -> None:
        if not self.set_config(cfg):
            raise ValueError("fluid config rejected (fluid3_from_ffi validation)")

    def set_config(self, cfg: FluidConfig3Ffi) -> bool:
        return self._lib.phieng_world3_set_fluid_config(self._h, C.byref(cfg)) == 1

    def add_particles(self, positions) -> int:
        """FluidState3::add_particles: phase 0; returns the number added."""
        p = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 3)
        return int(self._lib.phieng_world3_fluid_add(self._h, _fptr(p), p.shape[0]))

    def add_particles_phase(self, positions, phases) -> int:
        p = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 3)
        ph = np.ascontiguousarray(phases, dtype=np.uint8)
        return int(
            self._lib.phieng_world3_fluid_add_phase(
                self._h, _fptr(p), ph.ctypes.data_as(C.POINTER(C.c_uint8)), p.shape[0]
            )
        )

    def clear(self) -> None:
        self._lib.phieng_world3_fluid_clear(self._h)

    def __len__(self) -> int:
        return int(self._lib.phieng_world3_fluid_count(self._h))

    @property
    def particles(self) -> np.ndarray:
        """[n][6] = x, y, z, vx, vy, vz (phieng_world3_fluid_get)."""
        n = len(self)
        out = np.zeros((n, 6), np.float32)
        k = self._lib.phieng_world3_fluid_get(self._h, _fptr(out), n)
        self._world.check()
        return out[:k]

    def set_state(self, q) -> None:
        a = np.ascontiguousarray(q, dtype=np.float32).reshape(-1, 6)
        if self._lib.phieng_sph3_set_state(self._h, _fptr(a), a.shape[0]) != 1:
            raise ValueError("set_state rejected (count or non-finite values)")

    def density_pressure(self):
        """Per-particle density and pressure of the last density pass."""
        n = len(self)
        d = np.zeros(n, np.float32)
        p = np.zeros(n, np.float32)
        k = self._lib.phieng_sph3_get_density_pressure(self._h, _fptr(d), _fptr(p), n)
        if k != n:
            self._world.check()
        return d, p

    def set_cap(self, cap: int) -> None:
        self._lib.phieng_sph3_set_particle_cap(self._h, cap)


class World3:
    """A 3D world of static bodies and one GPU-resident SPH fluid."""

    def __init__(self):
        self._lib = _abi.load()
        self._h = self._lib.phieng_world3_new()
        if not self._h:
            raise MemoryError("phieng_world3_new returned null")
        self._gravity = (0.0, -9.81, 0.0)
        self.fluid = FluidState3(self)

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.phieng_world3_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def gravity(self):
        return self._gravity

    @gravity.setter
    def gravity(self, g) -> None:
        self._lib.phieng_world3_set_gravity(self._h, float(g[0]), float(g[1]), float(g[2]))
        self._gravity = (float(g[0]), float(g[1]), float(g[2]))

    @property
    def time(self) -> float:
        t = C.c_float()
        self._lib.phieng_world3_get_time(self._h, C.byref(t))
        return float(t.value)

    @property
    def ambient(self) -> "_abi.AmbientConfig3Ffi":
        """The world's AmbientConfig3Ffi (phieng_world3_get_ambient_config)."""
        a = _abi.AmbientConfig3Ffi()
        self._lib.phieng_world3_get_ambient_config(self._h, C.byref(a))
        return a

    def set_turbulence(self, amplitude: float, frequency: float = 1.0, time_scale: float = 1.0, seed: int = 0,
                       octaves: int = 3, divergence_free: bool = False, enabled: bool = True) -> None:
        """world.ambient.turbulence (TurbulenceConfig3, ambient.rs:251-266) through
        phieng_world3_set_ambient_config, the other ambient fields kept."""
        a = self.ambient
        a.turbulence_enabled = 1 if enabled else 0
        a.turbulence_amplitude = amplitude
        a.turbulence_frequency = frequency
        a.turbulence_time_scale = time_scale
        a.turbulence_seed = seed & 0xFFFFFFFF
        a.turbulence_octaves = octaves
        a.turbulence_divergence_free = 1 if divergence_free else 0
        if self._lib.phieng_world3_set_ambient_config(self._h, C.byref(a)) != 1:
            raise ValueError("ambient config rejected")

    def add_static_body(self, position, shape) -> int:
        """A static body through phieng_world3_add_body (identity rotation)."""
        px, py, pz = (float(v) for v in position)
        if isinstance(shape, Sphere):
            args = (_abi.SHAPE3_SPHERE, shape.radius, 0.0, 0.0)
        elif isinstance(shape, Box3):
            args = (_abi.SHAPE3_BOX, shape.hx, shape.hy, shape.hz)
        elif isinstance(shape, Capsule):
            args = (_abi.SHAPE3_CAPSULE, shape.radius, shape.half_length, 0.0)
        else:
            raise TypeError("shape must be Sphere, Box3 or Capsule")
        r = self._lib.phieng_world3_add_body(self._h, px, py, pz, *args, 1.0, 1, 0.5, 0.0)
        if r < 0:
            raise ValueError("invalid static body")
        return int(r)

    def body_count(self) -> int:
        return int(self._lib.phieng_world3_body_count(self._h))

    def step_fluid(self, bodies, dt: float, hulls=None) -> None:
        """FluidState3::step_fluid with the engine's bodies (a ctypes
        PhiengBody3 array, updated in place: velocities and sleep flags), in
        place of the world's static bodies; the clock does not advance.
        hulls = (xyz float32 [m][3], first uint32 [nb], count uint32 [nb]) for
        PHIENG_SHAPE3_HULL bodies."""
        n = len(bodies)
        if hulls is None:
            ok = self._lib.phieng_sph3_step_fluid(self._h, bodies, n, dt)
        else:
            xyz = np.ascontiguousarray(hulls[0], np.float32).reshape(-1, 3)
            first = np.ascontiguousarray(hulls[1], np.uint32)
            count = np.ascontiguousarray(hulls[2], np.uint32)
            U = C.POINTER(C.c_uint32)
            ok = self._lib.phieng_sph3_step_fluid_hull(self._h, bodies, n, _fptr(xyz), first.ctypes.data_as(U),
                                                       count.ctypes.data_as(U), xyz.shape[0], dt)
        if ok != 1:
            self.check()
            raise ValueError("invalid bodies for the fluid phase")

    def step(self, dt: float) -> None:
        self._lib.phieng_world3_step(self._h, dt)
        self.check()

    def step_n(self, dt: float, n: int) -> None:
        if self._lib.phieng_sph3_step_n(self._h, dt, n) != 1:
            self.check()

    def set_stream(self, stream_ptr: int | None) -> None:
        self._lib.phieng_sph3_set_stream(self._h, C.c_void_p(stream_ptr) if stream_ptr else None)

    def sync(self) -> None:
        if self._lib.phieng_sph3_sync(self._h) != 1:
            self.check()

    def status(self) -> _abi.PhiengSphStatus:
        s = _abi.PhiengSphStatus()
        self._lib.phieng_sph3_status(self._h, C.byref(s))
        return s

    def check(self) -> None:
        s = self.status()
        if s.error != _abi.OK:
            msg = self._lib.phieng_sph3_error_string(self._h).decode()
            raise SphError(f"phieng_sph error {s.error}: {msg}")

    def set_profiling(self, on: bool) -> None:
        if self._lib.phieng_sph3_set_profiling(self._h, 1 if on else 0) != 1:
            self.check()

    def phase_times(self):
        """ms of (sort + ranges, density, force + integrate) of the last substep."""
        out = np.zeros(3, np.float32)
        k = self._lib.phieng_sph3_phase_times(self._h, _fptr(out), 3)
        return out[:k].astype(np.float64)

    def save_fluid_block(self, version: int = _abi.SNAPSHOT_SCHEMA) -> bytes:
        """The fluid section of the reference's binary world snapshot
        (snapshot.rs encode_fluid3) for this world's fluid."""
        n = self._lib.phieng_sph3_fluid_block_save(self._h, version, None, 0)
        if n < 0:
            self.check()
            raise ValueError("fluid block save failed (version or world)")
        buf = (C.c_uint8 * n)()
        self._lib.phieng_sph3_fluid_block_save(self._h, version, buf, n)
        return bytes(buf)

    def load_fluid_block(self, data: bytes, version: int = _abi.SNAPSHOT_SCHEMA) -> int:
        """Replace the fluid by a snapshot fluid block (the reference's load
        rules); returns the bytes consumed."""
        buf = (C.c_uint8 * max(len(data), 1)).from_buffer_copy(bytes(data) or b"\0")
        r = self._lib.phieng_sph3_fluid_block_load(self._h, version, buf, len(data))
        if r < 0:
            raise ValueError("malformed fluid block" if r == -2 else "bad arguments")
        return int(r)

    @property
    def precision(self) -> int:
        """_abi.EXACT (default) or _abi.TOLERANCE (phieng_sph3_set_precision)."""
        return int(self._lib.phieng_sph3_get_precision(self._h))

    @precision.setter
    def precision(self, mode: int) -> None:
        if self._lib.phieng_sph3_set_precision(self._h, int(mode)) != 1:
            raise ValueError(f"unknown precision mode {mode}")

    def debug_forces(self):
        """(density, pressure, force [n][3]) of a density + force pass on the
        current state (no integration)."""
        n = len(self.fluid)
        d = np.zeros(n, np.float32)
        p = np.zeros(n, np.float32)
        f = np.zeros((n, 3), np.float32)
        k = self._lib.phieng_sph3_debug_forces(self._h, _fptr(d), _fptr(p), _fptr(f), n)
        if k != n:
            self.check()
        return d, p, f


def dam_break_3d(nx: int, ny: int, nz: int, spacing: float = 0.25, tank=(12.0, 8.0, 6.0)):
    """A 3D dam break: an nx * ny * nz block of particles at `spacing` in the
    corner of a walled tank (floor, four walls) of inner size `tank`.
    Returns (positions [n][3], bodies [(position, shape)])."""
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    pts = np.stack([i, j, k], -1).reshape(-1, 3).astype(np.float32) * np.float32(spacing)
    pts += np.float32(0.5 * spacing)
    lx, ly, lz = tank
    t = 0.5
    bodies = [
        ((lx / 2, -t, lz / 2), Box3(lx / 2 + t, t, lz / 2 + t)),  # floor
        ((-t, ly / 2, lz / 2), Box3(t, ly / 2, lz / 2 + t)),  # x = 0 wall
        ((lx + t, ly / 2, lz / 2), Box3(t, ly / 2, lz / 2 + t)),  # x = lx wall
        ((lx / 2, ly / 2, -t), Box3(lx / 2, ly / 2, t)),  # z = 0 wall
        ((lx / 2, ly / 2, lz + t), Box3(lx / 2, ly / 2, t)),  # z = lz wall
    ]
    return pts, bodies


__all__ = ["World3", "FluidState3", "Sphere", "Box3", "Capsule", "FluidConfig3Ffi", "default_config", "dam_break_3d"]


def main(argv=None) -> None:
    """3D dam break demo: ``python -m phi_eng_b200.world3 --side 64 --steps 100``.

    Builds a side^3 block at 0.25 m spacing in a walled tank 2.5 x 1.5 x 1.5
    times its size, steps it with the default FluidConfig3 at dt = 1/60 and
    prints the front (max x), the peak speed and the time per step."""
    import argparse
    import time

    ap = argparse.ArgumentParser(prog="python -m phi_eng_b200.world3")
    ap.add_argument("--side", type=int, default=32)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--every", type=int, default=0, help="print the front every k steps (0: only at the end)")
    ap.add_argument("--precision", choices=["exact", "tolerance"], default="exact")
    a = ap.parse_args(argv)
    L = a.side * 0.25
    pts, bodies = dam_break_3d(a.side, a.side, a.side, 0.25, tank=(2.5 * L, 1.5 * L, 1.5 * L))
    w = World3()
    w.precision = _abi.TOLERANCE if a.precision == "tolerance" else _abi.EXACT
    w.fluid.set_cap(len(pts))
    for pos, sh in bodies:
        w.add_static_body(pos, sh)
    w.fluid.add_particles(pts)
    t0 = time.perf_counter()
    for k in range(a.steps):
        w.step_n(1.0 / 60.0, 1)
        if a.every and (k + 1) % a.every == 0:
            s = w.fluid.particles
            print(f"step {k + 1:5d}  t={w.time:.3f}s  front={s[:, 0].max():.3f}m", flush=True)
    w.sync()
    el = time.perf_counter() - t0
    s = w.fluid.particles
    speed = float(np.sqrt((s[:, 3:] ** 2).sum(1)).max())
    print(f"{len(pts)} particles, {a.steps} steps: front={s[:, 0].max():.3f}m peak_speed={speed:.3f}m/s "
          f"{1e3 * el / max(a.steps, 1):.4f} ms/step (wall, incl. launch)")


if __name__ == "__main__":
    main()

