"""One scene-building interface over the CPU oracle and the GPU library.

Backends:
  oracle_seq     oracle, the reference's in-place (Gauss-Seidel) integrate
  oracle_jacobi  oracle, Jacobi integrate (what the GPU computes)
  oracle_fp64    oracle, Jacobi integrate in double precision
  gpu            libphieng_sph.so through the C ABI (phi_eng_b200.world)

Bodies added through the GPU's C ABI carry the rotation of
Transform2::from_position_angle(p, 0) (columns (1, 0), (-0, 1)); the oracle
backends use the same matrix so results can be compared bit for bit.
"""
from __future__ import annotations

import numpy as np

from oracle import oracle as orc
from phi_eng_b200._abi import default_config

FFI_ROT = (1.0, 0.0, -0.0, 1.0)


class OracleSim:
    def __init__(self, mode=orc.REF_SEQ, fp64=False, cap=1 << 22, libm_pow=False):
        self.w = orc.OracleWorld(fp64=fp64, cap=cap, libm_pow=libm_pow)
        self.mode = mode

    def add_box(self, px, py, hx, hy):
        self.w.add_box(px, py, hx, hy, FFI_ROT)

    def add_circle(self, px, py, r):
        self.w.add_circle(px, py, r, FFI_ROT)

    def set_gravity(self, gx, gy):
        self.w.set_gravity(gx, gy)

    @property
    def config(self):
        return self.w.get_config()

    @config.setter
    def config(self, c):
        self.w.set_config(c)

    def add_particles(self, xy, phases=None):
        return self.w.add_particles(xy, phases)

    def set_state(self, xyvv):
        self.w.set_state(xyvv)

    def step(self, dt, k=1):
        for _ in range(k):
            self.w.step(dt, self.mode)

    def state(self):
        return self.w.state()

    def density_pressure(self):
        return self.w.density_pressure()

    @property
    def count(self):
        return self.w.count


class GpuSim:
    def __init__(self, cap=1 << 22):
        from phi_eng_b200.world import World2

        self.w = World2()
        self.w.fluid.set_cap(cap)

    def add_box(self, px, py, hx, hy):
        from phi_eng_b200.world import Box

        self.w.add_static_body((px, py), Box(hx, hy))

    def add_circle(self, px, py, r):
        from phi_eng_b200.world import Circle

        self.w.add_static_body((px, py), Circle(r))

    def set_gravity(self, gx, gy):
        self.w.gravity = (gx, gy)

    @property
    def config(self):
        return self.w.fluid.config

    @config.setter
    def config(self, c):
        self.w.fluid.config = c

    def add_particles(self, xy, phases=None):
        if phases is None:
            return self.w.fluid.add_particles(xy)
        return self.w.fluid.add_particles_phase(xy, phases)

    def set_state(self, xyvv):
        self.w.fluid.set_state(xyvv)

    def step(self, dt, k=1):
        if k == 1:
            self.w.step(dt)
        else:
            self.w.step_n(dt, k)

    def state(self):
        return self.w.fluid.particles

    def density_pressure(self):
        return self.w.fluid.density_pressure()

    @property
    def count(self):
        return len(self.w.fluid)


def make(backend: str, **kw):
    if backend == "oracle_seq":
        return OracleSim(orc.REF_SEQ, **kw)
    if backend == "oracle_jacobi":
        return OracleSim(orc.JACOBI, **kw)
    if backend == "oracle_fp64":
        return OracleSim(orc.JACOBI, fp64=True, **kw)
    if backend == "gpu":
        return GpuSim(**kw)
    raise ValueError(backend)


def load_scene(sim, scene):
    sim.set_gravity(*scene.gravity)
    for (px, py, hx, hy) in scene.boxes:
        sim.add_box(px, py, hx, hy)
    for (px, py, r) in scene.circles:
        sim.add_circle(px, py, r)
    sim.config = scene.config
    n = sim.add_particles(scene.xy, scene.phases)
    assert n == scene.n
    return sim


def tank(sim):
    """tank() (crates/dynamics/src/fluid.rs:1151-1170)."""
    sim.add_box(2.0, -1.0, 3.0, 0.5)
    for x in (-1.0, 5.0):
        sim.add_box(x, 2.0, 0.5, 3.5)


def lattice(sim, x0, y0, nx, ny, dx):
    """lattice() (fluid.rs:1173-1182); asserts everything was added."""
    from phi_eng_b200.scenes import lattice as lat

    pts = lat(x0, y0, nx, ny, dx)
    assert sim.add_particles(pts) == pts.shape[0]
    return pts


def default_cfg():
    return default_config()
