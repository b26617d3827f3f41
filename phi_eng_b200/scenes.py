"""Scene builders: the reference's unit-scale tank and the SI dam-break workloads.

Workloads (all synthetic, seeded):
  dam_break_4k   4,096 particles (64 x 64 lattice, spacing 0.01 m) in a 1.0 m wide open-top box
  dam_break_1m   1,048,576 particles (1024 x 1024, spacing 0.001 m) in a 10 x 6 m box
Physical parameters: water (rest density 1 in units of 1000 kg/m^3, particle mass s^2), h = 2 s,
Tait gamma 7 with stiffness 100, XSPH 0.3, max speed 30, particle radius s/2,
gravity (0, -9.81); one world step = one fluid substep at dt = 0.4 h / sqrt(gamma k).
Walls are static boxes 0.1 m thick (floor, left, right, then ceiling for the 1M box).
Lattice particle (ix, iy), index iy * nx + ix, sits at ((ix + 1/2) s + xi_x,
(iy + 1/2) s + xi_y), xi ~ U[-0.01 s, 0.01 s] drawn from SplitMix64 (seed 0x5EED),
two draws per particle in index order.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from ._abi import FluidConfig2Ffi, default_config

MASK64 = (1 << 64) - 1


def splitmix64_stream(seed: int, count: int) -> np.ndarray:
    """`count` outputs of SplitMix64 (Steele, Lea & Flood 2014) from `seed`, as uint64."""
    out = np.empty(count, dtype=np.uint64)
    # vectorised: state_k = seed + (k+1) * golden
    with np.errstate(over="ignore"):
        k = np.arange(1, count + 1, dtype=np.uint64)
        z = np.uint64(seed & MASK64) + k * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    out[:] = z
    return out


def uniform_pm(seed: int, count: int, half_width: float) -> np.ndarray:
    """`count` values uniform in [-half_width, half_width) (53-bit mantissa draws)."""
    u = (splitmix64_stream(seed, count) >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))
    return (2.0 * u - 1.0) * half_width


@dataclass
class Scene:
    """Static walls + particle positions + the fluid config that goes with them."""

    name: str
    boxes: list = field(default_factory=list)  # (px, py, hx, hy), in body order
    circles: list = field(default_factory=list)  # (px, py, r)
    xy: np.ndarray = None  # (n, 2) float32
    phases: np.ndarray | None = None
    config: FluidConfig2Ffi = None
    dt: float = 1.0 / 60.0
    steps: int = 600
    gravity: tuple = (0.0, -9.81)

    @property
    def n(self) -> int:
        return int(self.xy.shape[0])


def si_config(spacing: float, literal_density: bool = False) -> FluidConfig2Ffi:
    """Water at spacing s. Density is expressed in units of 1000 kg/m^3
    (rest density 1, particle mass s^2): the reference's integrate divides
    the pressure sum, which already has units of acceleration, by the density
    once more (fluid.rs:1008), so its pressure term is only correctly scaled
    in the rest-density-1 unit system its defaults use. With the literal
    1000 kg/m^3 (literal_density=True) the pressure acceleration comes out
    1000x too weak and a resting column free-falls into itself."""
    c = default_config()
    rho0 = 1000.0 if literal_density else 1.0
    c.rest_density = rho0
    c.particle_mass = rho0 * spacing * spacing
    c.smoothing_length = 2.0 * spacing
    c.stiffness = 100.0
    c.gamma = 7.0
    c.viscosity = 0.3
    c.artificial_viscosity = 0.0
    c.surface_tension = 0.0
    c.max_velocity = 30.0
    c.particle_radius = 0.5 * spacing
    c.phase_count = 1
    for k in range(4):
        c.phase_rest_density[k] = rho0
        c.phase_mass[k] = c.particle_mass
    return c


def fine_dt(cfg: FluidConfig2Ffi) -> float:
    """The reference's CFL rule (fluid.rs:562-588) with factor 0.4, c0 = sqrt(gamma k)."""
    return float(np.float32(0.4 * cfg.smoothing_length / math.sqrt(cfg.gamma * cfg.stiffness)))


def box_walls(width: float, height: float, t: float = 0.1, ceiling: bool = True) -> list:
    """Floor, left, right (and ceiling) boxes whose inner faces bound [0,W] x [0,H]."""
    walls = [
        (0.5 * width, -0.5 * t, 0.5 * width + t, 0.5 * t),
        (-0.5 * t, 0.5 * height, 0.5 * t, 0.5 * height + t),
        (width + 0.5 * t, 0.5 * height, 0.5 * t, 0.5 * height + t),
    ]
    if ceiling:
        walls.append((0.5 * width, height + 0.5 * t, 0.5 * width + t, 0.5 * t))
    return walls


def jittered_lattice(nx: int, ny: int, spacing: float, seed: int = 0x5EED, jitter: float = 0.01,
                     x0: float = 0.0, y0: float = 0.0) -> np.ndarray:
    n = nx * ny
    xi = uniform_pm(seed, 2 * n, jitter * spacing).reshape(n, 2)
    iy, ix = np.divmod(np.arange(n, dtype=np.int64), nx)
    x = x0 + (ix + 0.5) * spacing + xi[:, 0]
    y = y0 + (iy + 0.5) * spacing + xi[:, 1]
    return np.stack([x, y], axis=1).astype(np.float32)


def dam_break(nx: int, ny: int, spacing: float, width: float, height: float, steps: int,
              name: str, seed: int = 0x5EED, ceiling: bool = True) -> Scene:
    cfg = si_config(spacing)
    return Scene(name=name, boxes=box_walls(width, height, ceiling=ceiling),
                 xy=jittered_lattice(nx, ny, spacing, seed), config=cfg, dt=fine_dt(cfg), steps=steps)


def dam_break_4k() -> Scene:
    """64 x 64 at 0.01 m is a 0.64 m column, taller than the 0.6 m box: with a
    ceiling its top rows would start inside the ceiling box and the
    reference's box-interior branch (always +y, fluid.rs:504-516) would throw
    them out of the tank. The box is therefore open at the top, like the
    reference's own tank() and fluid_dam scenes, with side walls 1.2 m high."""
    return dam_break(64, 64, 0.01, 1.0, 1.2, 1000, "dam_break_4k", ceiling=False)


def dam_break_1m() -> Scene:
    return dam_break(1024, 1024, 0.001, 10.0, 6.0, 200, "dam_break_1m")


def dam_break_scaled(nx: int, ny: int) -> Scene:
    """The 1M workload's construction at another lattice size (for small cases)."""
    return dam_break(nx, ny, 0.001, 10.0, 6.0, 200, f"dam_break_{nx}x{ny}")


# ---- the reference's own unit-scale scenes (crates/dynamics/src/fluid.rs:1151-1182) ----
def tank_boxes() -> list:
    """tank(): floor at (2,-1) half (3,0.5); walls at x = -1 and 5, half (0.5,3.5)."""
    return [(2.0, -1.0, 3.0, 0.5), (-1.0, 2.0, 0.5, 3.5), (5.0, 2.0, 0.5, 3.5)]


def lattice(x0: float, y0: float, nx: int, ny: int, dx: float) -> np.ndarray:
    """lattice(): row-major (iy outer), x0 + ix*dx, y0 + iy*dx, in f32 arithmetic."""
    pts = []
    f = np.float32
    for iy in range(ny):
        for ix in range(nx):
            pts.append((f(x0) + f(ix) * f(dx), f(y0) + f(iy) * f(dx)))
    return np.array(pts, dtype=np.float32)


def reference_tank(nx: int = 8, ny: int = 12) -> Scene:
    """The fluid_dam example / test_fluid_dam_break_contained scene: 8 x 12 at 0.25."""
    return Scene(name=f"tank_{nx}x{ny}", boxes=tank_boxes(), xy=lattice(0.0, 0.0, nx, ny, 0.25),
                 config=default_config(), dt=1.0 / 60.0, steps=600)
