"""ORACLE — TEST INFRASTRUCTURE ONLY.

A second CPU restatement of the reference's 2D SPH step, written from the
reference's C# solver (src/PhiEng.Dynamics/FluidSolver.cs, the managed twin of
crates/dynamics/src/fluid.rs) instead of the Rust source the C++ oracle
(sph_oracle.hpp) follows. The reference's own test
tests/PhiEng.Tests/EquivalenceTests.cs:122-176 asserts that the C# step and
the Rust step agree within 1e-4 in position and 1e-3 in velocity after 60
steps of its scene; tests/test_oracle_pin.py checks this restatement against
the C++ oracle on that scene with that bar, which ties the oracle to a
statement of the algorithm written by the reference's authors.

Scope: the default flag set of that scene (linear or Tait EOS, XSPH, static
boxes and circles, CFL substeps) plus Monaghan artificial viscosity,
cohesion and wall friction; no ghosts, resampling, turbulence or dynamic
bodies. Every operation is an IEEE f32 operation on
numpy float32 scalars in the C# source's evaluation order (System.Numerics
vector ops restated component-wise); slow, for scenes of a few hundred
particles.
"""
from __future__ import annotations

import math

import numpy as np

F = np.float32
EPS = F(1e-6)
EPS_SQ = F(1e-12)
PI = F(math.pi)  # MathF.PI


def poly6(r2, h):
    """FluidSolver.cs:48-57."""
    if r2 >= h * h or r2 < F(0):
        return F(0)
    h2 = h * h
    t = h2 - r2
    return F(4) / (PI * h2 * h2 * h2 * h2) * t * t * t


def spiky_grad(rx, ry, r, h):
    """FluidSolver.cs:60-68: (r_vec / r) * s."""
    if r >= h or r < EPS:
        return F(0), F(0)
    s = F(-30) / (PI * h * h * h * h * h) * (h - r) * (h - r)
    return rx / r * s, ry / r * s


def pressure(density, rest, stiffness, gamma):
    """FluidSolver.cs:75-84 (MathF.Pow as float32 power)."""
    if gamma == F(1):
        return max(F(0), stiffness * (density - rest))
    rho0 = max(rest, EPS)
    return max(F(0), stiffness * rho0 * (F(np.power(density / rho0, gamma, dtype=np.float32)) - F(1)))


def length(x, y):
    return F(np.sqrt(x * x + y * y))


class CsFluid:
    """FluidState2 + FluidIntegration.Substep2 for the scope above."""

    def __init__(self, cfg, bodies, gravity=(0.0, -9.81)):
        self.h_cfg = F(cfg.smoothing_length)
        self.rest = F(cfg.rest_density)
        self.k = F(cfg.stiffness)
        self.gamma = F(cfg.gamma)
        self.visc = F(cfg.viscosity)
        self.av = F(cfg.artificial_viscosity)
        self.friction = F(cfg.wall_friction)
        self.cfl = F(cfg.cfl)
        self.max_substeps = int(cfg.max_substeps)
        self.st = F(cfg.surface_tension)
        self.vmax = F(cfg.max_velocity)
        self.pr = max(F(cfg.particle_radius), F(0))
        self.mass0 = F(cfg.phase_mass[0])
        self.phase_rest0 = F(cfg.phase_rest_density[0])
        # bodies: ("box", px, py, hx, hy) or ("circle", px, py, r), identity rotation
        self.bodies = [tuple(F(v) if not isinstance(v, str) else v for v in b) for b in bodies]
        self.g = (F(gravity[0]), F(gravity[1]))
        self.pos = []
        self.vel = []
        self.mass = []
        self.dens = []
        self.pres = []

    def add_particles(self, xy):
        for x, y in np.asarray(xy, np.float32):
            self.pos.append([F(x), F(y)])
            self.vel.append([F(0), F(0)])
            self.mass.append(self.mass0)
            self.dens.append(F(0))
            self.pres.append(F(0))

    # ---- grid (FluidSolver.cs:111-193)
    def _cell(self, x, y):
        h = self.h_cfg
        return int(math.floor(x / h)), int(math.floor(y / h))

    def _rebuild(self):
        self.grid = {}
        for i, (x, y) in enumerate(self.pos):
            if not (math.isfinite(x) and math.isfinite(y)):
                continue
            self.grid.setdefault(self._cell(x, y), []).append(i)

    def _neighbors(self, i):
        h = self.h_cfg
        px, py = self.pos[i]
        cx, cy = self._cell(px, py)
        out = []
        for oy in (-1, 0, 1):
            for ox in (-1, 0, 1):
                for j in self.grid.get((cx + ox, cy + oy), ()):
                    dx, dy = self.pos[j][0] - px, self.pos[j][1] - py
                    if dx * dx + dy * dy < h * h:
                        out.append(j)
        return out

    # ---- FluidSolver.cs:414-440
    def _density_pressure(self, h):
        n = len(self.pos)
        for i in range(n):
            px, py = self.pos[i]
            rho = F(0)
            for j in self._neighbors(i):
                dx, dy = self.pos[j][0] - px, self.pos[j][1] - py
                rho = rho + self.mass[j] * poly6(dx * dx + dy * dy, h)
            self.dens[i] = min(max(rho, F(0)), F(3) * max(self.rest, EPS))
        for i in range(n):
            self.pres[i] = pressure(self.dens[i], self.phase_rest0, self.k, self.gamma)

    # ---- FluidSolver.cs:283-345 (circle and box branches)
    def _collide(self, px, py, body):
        pr = self.pr
        if body[0] == "circle":
            _, bx, by, r = body
            dx, dy = px - bx, py - by
            dist = length(dx, dy)
            if dist >= r + pr:
                return None
            nx, ny = (dx / dist, dy / dist) if dist > EPS else (F(1), F(0))
            return nx, ny, r + pr - dist
        _, bx, by, hx, hy = body
        lx, ly = px - bx, py - by  # identity rotation
        cxl = min(max(lx, -hx), hx)
        cyl = min(max(ly, -hy), hy)
        ddx, ddy = lx - cxl, ly - cyl
        if ddx * ddx + ddy * ddy > EPS_SQ:
            dist = length(ddx, ddy)
            if dist >= pr:
                return None
            return ddx / dist, ddy / dist, pr - dist
        dxp = hx - F(abs(lx))
        dyp = hy - F(abs(ly))

        def copysign1(v):  # FluidSolver.cs:371-378
            return F(-1) if (v < 0 or (v == 0 and math.copysign(1.0, v) < 0)) else F(1)

        if dxp < dyp:
            return copysign1(lx), F(0), pr + dxp
        return F(0), copysign1(ly), pr + dyp

    # ---- FluidSolver.cs:381-410
    def cfl_substeps(self, dt):
        mx = 1 if self.max_substeps < 1 else self.max_substeps
        if self.cfl <= F(0) or mx <= 1:
            return 1
        h = max(self.h_cfg, EPS)
        rho0 = max(self.rest, EPS)
        k = max(self.k, F(0))
        c0 = F(np.sqrt(k)) if self.gamma == F(1) else F(np.sqrt(self.gamma * k * rho0))
        vmax = F(0)
        for v in self.vel:
            vmax = max(vmax, length(v[0], v[1]))
        speed = c0 + vmax
        if not math.isfinite(speed) or speed <= EPS:
            return 1
        dt_max = self.cfl * h / speed
        if not math.isfinite(dt_max) or dt_max <= F(0):
            return 1
        return max(1, min(int(math.ceil(F(dt) / dt_max)), mx))

    # ---- FluidSolver.cs:27-45: CFL substeps of Substep2
    def step(self, dt):
        if not self.pos or not F(dt) > F(0):
            return
        k = self.cfl_substeps(dt)
        sub = F(dt) / F(k)
        for _ in range(k):
            self.substep(sub)

    # ---- FluidSolver.cs:793-948 + the boundary loop
    def substep(self, dt):
        dt = F(dt)
        h = max(self.h_cfg, EPS)
        n = len(self.pos)
        self._rebuild()
        self._density_pressure(h)
        self.cs = F(np.sqrt(max(self.k, F(0))))
        forces = []
        for i in range(n):
            px, py = self.pos[i]
            rho_i = max(self.dens[i], EPS)
            p_i = self.pres[i]
            fx, fy = F(0), F(0)
            for j in self._neighbors(i):
                if j == i:
                    continue
                rho_j = max(self.dens[j], EPS)
                dx, dy = px - self.pos[j][0], py - self.pos[j][1]
                dist = length(dx, dy)
                gx, gy = spiky_grad(dx, dy, dist, h)
                term = p_i / (rho_i * rho_i) + self.pres[j] / (rho_j * rho_j)
                if self.av > F(0) and dist > EPS:
                    # FluidSolver.cs:89-98, called at :858-862
                    rho_bar = F(0.5) * (rho_i + rho_j)
                    vrx, vry = self.vel[i][0] - self.vel[j][0], self.vel[i][1] - self.vel[j][1]
                    vd = vrx * dx + vry * dy
                    if not vd >= F(0):
                        mu = h * vd / (dist * dist + F(0.01) * h * h)
                        term = term + -self.av * self.cs * mu / max(rho_bar, EPS)
                mt = self.mass[j] * term
                fx = fx - gx * mt
                fy = fy - gy * mt
                if self.st > F(0) and dist > EPS:
                    # FluidSolver.cs:101-108, applied at :864-871
                    coh = F(0) if dist >= h else F(1) - dist / h
                    if coh > F(0):
                        sc = self.st * self.mass[i] * self.mass[j] * coh
                        fx = fx - dx / dist * sc
                        fy = fy - dy / dist * sc
            forces.append((fx, fy))
        for i in range(n):
            nb = self._neighbors(i)  # from the grid of this substep, positions as they are now
            rho_i = max(self.dens[i], EPS)
            ax = self.g[0] + forces[i][0] / rho_i
            ay = self.g[1] + forces[i][1] / rho_i
            vx = self.vel[i][0] + ax * dt
            vy = self.vel[i][1] + ay * dt
            if self.visc > F(0):
                ppx, ppy = self.pos[i]
                v0x, v0y = self.vel[i]
                sx, sy = F(0), F(0)
                for j in nb:
                    if j == i:
                        continue
                    rho_bar = F(0.5) * (rho_i + max(self.dens[j], EPS))
                    ex, ey = self.pos[j][0] - ppx, self.pos[j][1] - ppy
                    w = poly6(ex * ex + ey * ey, h)
                    mr = self.mass[j] / rho_bar
                    sx = sx + (self.vel[j][0] - v0x) * mr * w
                    sy = sy + (self.vel[j][1] - v0y) * mr * w
                vx = vx + sx * self.visc
                vy = vy + sy * self.visc
            speed = length(vx, vy)
            if speed > self.vmax:
                sc = self.vmax / speed
                vx, vy = vx * sc, vy * sc
            if not (math.isfinite(vx) and math.isfinite(vy)):
                vx, vy = F(0), F(0)
            self.vel[i] = [vx, vy]
            x = self.pos[i][0] + vx * dt
            y = self.pos[i][1] + vy * dt
            if math.isfinite(x) and math.isfinite(y):
                self.pos[i] = [x, y]
        for i in range(n):
            for body in self.bodies:
                px, py = self.pos[i]
                hit = self._collide(px, py, body)
                if hit is None or hit[2] <= F(0):
                    continue
                nx, ny, depth = hit
                self.pos[i] = [px + nx * depth, py + ny * depth]
                vn = self.vel[i][0] * nx + self.vel[i][1] * ny
                if vn < F(0):
                    vx, vy = self.vel[i][0] - nx * vn, self.vel[i][1] - ny * vn
                    if self.friction > F(0):
                        # FluidSolver.cs:973-982 against a static body (velocity zero)
                        mu = min(max(self.friction, F(0)), F(1))
                        wn = F(0) * nx + F(0) * ny
                        wtx, wty = F(0) - nx * wn, F(0) - ny * wn
                        vx, vy = vx + (wtx - vx) * mu, vy + (wty - vy) * mu
                    self.vel[i] = [vx, vy]

    def state(self):
        return np.array([[p[0], p[1], v[0], v[1]] for p, v in zip(self.pos, self.vel)], np.float32)
