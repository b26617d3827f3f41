"""Python mirror of the reference's World2 / FluidState2 API over the C ABI.

The reference drives the fluid as

    let mut world = World2::new();
    world.add_static_body(pos, Shape2::Box { half_extents });
    world.fluid.config = FluidConfig2 { .. };
    world.fluid.add_particles(&pts);
    world.step(dt);
    for p in world.fluid.particles.iter() { .. }

(crates/engine/examples/fluid_dam.rs:12-61). This module offers the same
shape in Python — ``World2()``, ``add_static_body``, ``world.fluid.config``,
``world.fluid.add_particles``, ``world.step`` and ``world.fluid.particles`` —
with every call going through libphieng_sph.so; the particle state stays on
the GPU between steps. There is no CPU fallback: constructing a world loads
the CUDA library or raises.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._abi import FluidConfig2Ffi, default_config


@dataclass
class Box:
    """Shape2::Box { half_extents } (crates/dynamics/src/body.rs)."""

    hx: float
    hy: float


@dataclass
class Circle:
    """Shape2::Circle { radius }."""

    radius: float


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class SphError(RuntimeError):
    pass


class FluidState2:
    """world.fluid: config, particle insertion and read-back."""

    def __init__(self, world: "World2"):
        self._world = world

    @property
    def _lib(self):
        return self._world._lib

    @property
    def _h(self):
        return self._world._h

    # config (ffi.rs:999-1026)
    @property
    def config(self) -> FluidConfig2Ffi:
        c = FluidConfig2Ffi()
        self._lib.phieng_world_get_fluid_config(self._h, C.byref(c))
        return c

    @config.setter
    def config(self, cfg: FluidConfig2Ffi) -> None:
        if self._lib.phieng_world_set_fluid_config(self._h, C.byref(cfg)) != 1:
            raise ValueError("invalid fluid config (rejected by the validation of ffi.rs:773-855)")

    def set_config(self, cfg: FluidConfig2Ffi) -> bool:
        return self._lib.phieng_world_set_fluid_config(self._h, C.byref(cfg)) == 1

    def add_particles(self, positions) -> int:
        """add_particles (fluid.rs:232-236); returns the number added."""
        xy = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 2)
        total = 0
        # the C ABI takes at most 1,000,000 per call (ffi.rs:2493)
        for s in range(0, xy.shape[0], 1_000_000):
            chunk = np.ascontiguousarray(xy[s:s + 1_000_000])
            k = int(self._lib.phieng_world_fluid_add(self._h, _fptr(chunk), chunk.shape[0]))
            total += k
            if k < chunk.shape[0]:
                break
        return total

    def add_particles_phase(self, positions, phases) -> int:
        xy = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 2)
        ph = np.ascontiguousarray(phases, dtype=np.uint8)
        if ph.shape[0] != xy.shape[0]:
            raise ValueError("one phase per particle")
        return int(self._lib.phieng_world_fluid_add_phase(
            self._h, _fptr(xy), ph.ctypes.data_as(C.POINTER(C.c_uint8)), xy.shape[0]))

    def clear(self) -> None:
        self._lib.phieng_world_fluid_clear(self._h)

    def __len__(self) -> int:
        return int(self._lib.phieng_world_fluid_count(self._h))

    def masses(self) -> np.ndarray:
        """Particle masses by id (phieng_sph_fluid_masses)."""
        n = len(self)
        out = np.zeros(n, np.float32)
        self._lib.phieng_sph_fluid_masses(self._h, out.ctypes.data_as(C.POINTER(C.c_float)), n)
        return out

    @property
    def particles(self) -> np.ndarray:
        """(n, 4) float32 [x, y, vx, vy] in insertion order (ffi.rs:2575)."""
        n = len(self)
        out = np.zeros((n, 4), np.float32)
        if n:
            k = self._lib.phieng_world_fluid_get(self._h, _fptr(out), n)
            if k != n:
                self._world.check()
        return out

    def read_into(self, out: np.ndarray) -> int:
        """phieng_world_fluid_get into a caller buffer of (>= n, 4) float32
        (page-locked memory makes the read-back a direct DMA)."""
        if out.dtype != np.float32 or not out.flags.c_contiguous or out.ndim != 2 or out.shape[1] != 4:
            raise ValueError("out must be a C-contiguous (n, 4) float32 array")
        n = min(len(self), out.shape[0])
        k = self._lib.phieng_world_fluid_get(self._h, _fptr(out), n) if n else 0
        if k != n:
            self._world.check()
        return int(k)

    def set_state(self, xyvv) -> None:
        a = np.ascontiguousarray(xyvv, dtype=np.float32).reshape(-1, 4)
        if self._lib.phieng_sph_set_state(self._h, _fptr(a), a.shape[0]) != 1:
            raise ValueError("set_state rejected (non-finite input or too many particles)")

    def density_pressure(self):
        n = len(self)
        d = np.zeros(n, np.float32)
        p = np.zeros(n, np.float32)
        if n:
            self._lib.phieng_sph_get_density_pressure(self._h, _fptr(d), _fptr(p), n)
        return d, p

    def set_cap(self, cap: int) -> None:
        """Lift MAX_PARTICLES_2D (fluid.rs:30) for this fluid."""
        self._lib.phieng_sph_set_particle_cap(self._h, cap)


class World2:
    """A world of static bodies and one GPU-resident SPH fluid."""

    def __init__(self):
        self._lib = _abi.load()
        self._h = self._lib.phieng_world_new()
        if not self._h:
            raise MemoryError("phieng_world_new returned null")
        self._gravity = (0.0, -9.81)
        self.fluid = FluidState2(self)

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.phieng_world_free(self._h)
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

    # ---- world ----
    @property
    def gravity(self):
        return self._gravity

    @gravity.setter
    def gravity(self, g) -> None:
        self._lib.phieng_world_set_gravity(self._h, float(g[0]), float(g[1]))
        self._gravity = (float(g[0]), float(g[1]))

    @property
    def time(self) -> float:
        t = C.c_float()
        self._lib.phieng_world_get_time(self._h, C.byref(t))
        return float(t.value)

    @property
    def ambient(self) -> "_abi.AmbientConfig2Ffi":
        """The world's AmbientConfig2Ffi (phieng_world_get_ambient_config)."""
        a = _abi.AmbientConfig2Ffi()
        self._lib.phieng_world_get_ambient_config(self._h, C.byref(a))
        return a

    def set_turbulence(self, amplitude: float, frequency: float = 1.0, time_scale: float = 1.0, seed: int = 0,
                       octaves: int = 3, divergence_free: bool = False, enabled: bool = True) -> None:
        """world.ambient.turbulence (ambient.rs:108-126) through
        phieng_world_set_ambient_config, the other ambient fields kept."""
        a = self.ambient
        a.turbulence_enabled = 1 if enabled else 0
        a.turbulence_amplitude = amplitude
        a.turbulence_frequency = frequency
        a.turbulence_time_scale = time_scale
        a.turbulence_seed = seed & 0xFFFFFFFF
        a.turbulence_octaves = octaves
        a.turbulence_divergence_free = 1 if divergence_free else 0
        if self._lib.phieng_world_set_ambient_config(self._h, C.byref(a)) != 1:
            raise ValueError("ambient config rejected")

    def add_static_body(self, position, shape) -> int:
        """World2::add_static_body (world.rs:384-392) through phieng_world_add_body."""
        px, py = float(position[0]), float(position[1])
        if isinstance(shape, Box):
            r = self._lib.phieng_world_add_body(self._h, px, py, _abi.SHAPE_BOX, shape.hx, shape.hy, 1.0, 1, 0.4, 0.1)
        elif isinstance(shape, Circle):
            r = self._lib.phieng_world_add_body(self._h, px, py, _abi.SHAPE_CIRCLE, shape.radius, 0.0, 1.0, 1, 0.4, 0.1)
        else:
            raise TypeError("shape must be Box or Circle")
        if r < 0:
            raise ValueError("invalid static body")
        return int(r)

    def body_count(self) -> int:
        return int(self._lib.phieng_world_body_count(self._h))

    def step(self, dt: float) -> None:
        self._lib.phieng_world_step(self._h, dt)
        self.check()

    def reserve(self, n: int) -> None:
        """Allocate the device arrays for n particles ahead of the first step."""
        if self._lib.phieng_sph_reserve(self._h, n) != 1:
            self.check()
            raise SphError("phieng_sph_reserve failed")

    @property
    def precision(self) -> int:
        """_abi.EXACT (default) or _abi.TOLERANCE (phieng_sph_set_precision)."""
        return int(self._lib.phieng_sph_get_precision(self._h))

    @precision.setter
    def precision(self, mode: int) -> None:
        if self._lib.phieng_sph_set_precision(self._h, int(mode)) != 1:
            raise ValueError(f"unknown precision mode {mode}")

    def step_n(self, dt: float, n: int) -> None:
        if self._lib.phieng_sph_step_n(self._h, dt, n) != 1:
            self.check()

    def set_stream(self, stream_ptr: int | None) -> None:
        self._lib.phieng_sph_set_stream(self._h, C.c_void_p(stream_ptr) if stream_ptr else None)

    def sync(self) -> None:
        if self._lib.phieng_sph_sync(self._h) != 1:
            self.check()

    def status(self) -> _abi.PhiengSphStatus:
        s = _abi.PhiengSphStatus()
        self._lib.phieng_sph_status(self._h, C.byref(s))
        return s

    def check(self) -> None:
        s = self.status()
        if s.error != _abi.OK:
            msg = self._lib.phieng_sph_error_string(self._h).decode()
            raise SphError(f"phieng_sph error {s.error}: {msg}")

    def front_metrics(self):
        """(max x, peak speed) over the fluid, reduced on the GPU."""
        out = np.zeros(2, np.float32)
        if self._lib.phieng_sph_front_metrics(self._h, _fptr(out)) != 1:
            self.check()
        return float(out[0]), float(out[1])

    def front_metrics_async(self, raw: np.ndarray) -> None:
        """Enqueue the front metrics' reduction and an 8-byte copy of its raw
        result into raw (a uint32 array of 2, page-locked for the copy to be
        asynchronous) without waiting; decode after the stream has passed it
        (decode_front_metrics)."""
        if raw.dtype != np.uint32 or raw.size < 2 or not raw.flags.c_contiguous:
            raise ValueError("raw must be a contiguous uint32 array of 2")
        if self._lib.phieng_sph_front_metrics_async(self._h, C.c_void_p(raw.ctypes.data)) != 1:
            self.check()

    def decode_front_metrics(self, raw: np.ndarray):
        out = np.zeros(2, np.float32)
        self._lib.phieng_sph_front_metrics_decode(C.c_void_p(raw.ctypes.data), _fptr(out))
        return float(out[0]), float(out[1])

    def set_profiling(self, on: bool) -> None:
        if self._lib.phieng_sph_set_profiling(self._h, 1 if on else 0) != 1:
            self.check()

    def phase_times(self):
        """ms of (sort + ranges, density, force + integrate) of the last substep."""
        out = np.zeros(3, np.float32)
        k = self._lib.phieng_sph_phase_times(self._h, _fptr(out), 3)
        return out[:k].astype(np.float64)

    # ---- device-resident state and the learned closure ----
    def get_state_device(self, dst_ptr: int, max_count: int) -> int:
        """Copy [x, y, vx, vy] of up to max_count particles to device memory."""
        k = self._lib.phieng_sph_get_state_device(self._h, C.c_void_p(dst_ptr), max_count)
        self.check()
        return int(k)

    def set_state_device(self, src_ptr: int, n: int) -> None:
        if self._lib.phieng_sph_set_state_device(self._h, C.c_void_p(src_ptr), n) != 1:
            self.check()
            raise ValueError("set_state_device: count mismatch")

    def load_state_device(self, src_ptr: int, n: int) -> None:
        """Replace every particle by n phase-0 particles from device memory."""
        if self._lib.phieng_sph_load_state_device(self._h, C.c_void_p(src_ptr), n) != 1:
            self.check()
            raise ValueError("load_state_device rejected its arguments")

    def features(self, dt: float, feat_ptr: int) -> None:
        """Closure inputs (n x 16 floats, device) at the current state for a step dt."""
        if self._lib.phieng_sph_features(self._h, dt, C.c_void_p(feat_ptr)) != 1:
            self.check()
            raise ValueError("features failed")

    def set_closure(self, mlp, ratio: int = 4, threshold: float = 0.03,
                    criterion: int = _abi.CLOSURE_JUMP) -> None:
        h = mlp._h if mlp is not None else None
        if self._lib.phieng_sph_set_closure(self._h, h, ratio, threshold, criterion) != 1:
            raise ValueError("set_closure rejected its arguments")
        self._closure = mlp  # keep the network alive while attached

    def closure_step(self, dt_fine: float, coarse_steps: int = 1, stats=None):
        """coarse_steps steps of ratio x dt_fine with the attached closure;
        returns the accumulated PhiengClosureStats."""
        st = stats if stats is not None else _abi.PhiengClosureStats()
        if self._lib.phieng_sph_closure_step(self._h, dt_fine, coarse_steps, C.byref(st)) != 1:
            self.check()
            raise ValueError("closure_step failed (no network attached?)")
        return st

    # ---- diagnostics ----
    def debug_sorted(self):
        n = len(self.fluid)
        ids = np.zeros(n, np.uint32)
        keys = np.zeros(n, np.uint32)
        U = C.POINTER(C.c_uint32)
        self._lib.phieng_sph_debug_sorted(self._h, ids.ctypes.data_as(U), keys.ctypes.data_as(U), n)
        self.check()
        return ids, keys

    def debug_neighbors(self, max_per: int = 64):
        n = len(self.fluid)
        counts = np.zeros(n, np.uint32)
        lists = np.zeros(n * max_per, np.uint32)
        U = C.POINTER(C.c_uint32)
        self._lib.phieng_sph_debug_neighbors(self._h, counts.ctypes.data_as(U), lists.ctypes.data_as(U), max_per, n)
        self.check()
        return counts, lists.reshape(n, max_per)

    def debug_forces(self) -> np.ndarray:
        n = len(self.fluid)
        out = np.zeros((n, 2), np.float32)
        self._lib.phieng_sph_debug_forces(self._h, _fptr(out), n)
        self.check()
        return out

    def save_fluid_block(self, version: int = _abi.SNAPSHOT_SCHEMA) -> bytes:
        """The fluid section of the reference's binary world snapshot
        (snapshot.rs encode_fluid2) for this world's fluid."""
        n = self._lib.phieng_sph_fluid_block_save(self._h, version, None, 0)
        if n < 0:
            self.check()
            raise ValueError("fluid block save failed (version or world)")
        buf = (C.c_uint8 * n)()
        self._lib.phieng_sph_fluid_block_save(self._h, version, buf, n)
        return bytes(buf)

    def load_fluid_block(self, data: bytes, version: int = _abi.SNAPSHOT_SCHEMA) -> int:
        """Replace the fluid by a snapshot fluid block (the reference's load
        rules); returns the bytes consumed."""
        buf = (C.c_uint8 * max(len(data), 1)).from_buffer_copy(bytes(data) or b"\0")
        r = self._lib.phieng_sph_fluid_block_load(self._h, version, buf, len(data))
        if r < 0:
            raise ValueError("malformed fluid block" if r == -2 else "bad arguments")
        return int(r)

    def replan(self) -> None:
        self._lib.phieng_sph_replan(self._h)

    def set_grid(self, log2w: int, log2h: int, cx0: int = 0, cy0: int = 0) -> None:
        """Fix the bucket grid (2^log2w x 2^log2h buckets from cell (cx0, cy0))."""
        if self._lib.phieng_sph_set_grid(self._h, log2w, log2h, cx0, cy0) != 1:
            raise ValueError("invalid bucket grid")


def world_from_scene(scene, cap: int | None = None) -> World2:
    """Build a World2 from a phi_eng_b200.scenes.Scene."""
    w = World2()
    w.gravity = scene.gravity
    for (px, py, hx, hy) in scene.boxes:
        w.add_static_body((px, py), Box(hx, hy))
    for (px, py, r) in scene.circles:
        w.add_static_body((px, py), Circle(r))
    w.fluid.config = scene.config
    w.fluid.set_cap(cap if cap is not None else max(4096, scene.n))
    if scene.phases is not None:
        added = w.fluid.add_particles_phase(scene.xy, scene.phases)
    else:
        added = w.fluid.add_particles(scene.xy)
    if added != scene.n:
        raise RuntimeError(f"added {added} of {scene.n} particles")
    return w


__all__ = ["World2", "FluidState2", "Box", "Circle", "SphError", "world_from_scene", "default_config"]
