"""ORACLE — TEST INFRASTRUCTURE ONLY.

A second CPU restatement of the reference's 3D SPH step, written from the
reference's C# solver (src/PhiEng.Dynamics/FluidSolver3.cs, the managed twin
of crates/dynamics/src/fluid3.rs) instead of the Rust source the C++ oracle
(sph_oracle3.hpp) follows. The reference's own test
tests/PhiEng.Tests/EquivalenceTests.cs:177-225 asserts that the C# step and
the Rust step agree within 1e-4 in position per particle after 30 steps of a
3 x 3 x 3 lattice over one static box; tests/test_oracle_pin.py checks this
restatement against the C++ oracle on that scene with that bar, which ties
the 3D oracle to a statement of the algorithm written by the reference's
authors.

Scope: the default flag set (linear or Tait EOS, XSPH, CFL substeps, static
spheres, boxes and capsules at the identity rotation) plus Monaghan artificial viscosity, cohesion
and wall friction; no ghosts, resampling, turbulence or dynamic bodies. System.Numerics operations are
restated component-wise in the C# source's order on numpy float32 scalars:
Vector3.Dot and LengthSquared as (x x' + y y') + z z', Length as the square
root of that, a vector divided by a scalar component by component, and the
identity quaternion's Vector3.Transform as the identity. Slow; for scenes of
a few hundred particles.
"""
from __future__ import annotations

import math

import numpy as np

F = np.float32
EPS = F(1e-6)
EPS_SQ = F(1e-12)
PI = F(math.pi)  # MathF.PI


def dot(a, b):
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


def length(a):
    return F(np.sqrt(dot(a, a)))


def poly6(r2, h):
    """FluidSolver3.cs:41-51: 315 / (64 pi h2 h2 h2 h2 h) * t * t * t."""
    if r2 >= h * h or r2 < F(0):
        return F(0)
    h2 = h * h
    t = h2 - r2
    return F(315) / (F(64) * PI * h2 * h2 * h2 * h2 * h) * t * t * t


def spiky_grad(r_vec, r, h):
    """FluidSolver3.cs:53-62: (r_vec / r) * s, s = -45 / (pi h^6) (h - r) (h - r)."""
    if r >= h or r < EPS:
        return (F(0), F(0), F(0))
    s = F(-45) / (PI * h * h * h * h * h * h) * (h - r) * (h - r)
    return tuple((c / r) * s for c in r_vec)


def pressure(density, rest, stiffness, gamma):
    """FluidSolver3.cs:64-73 (MathF.Pow as numpy's float32 power)."""
    if gamma == F(1):
        return max(F(0), stiffness * (density - rest))
    rho0 = max(rest, EPS)
    return max(F(0), stiffness * rho0 * (F(np.power(F(density / rho0), F(gamma))) - F(1)))


def copysign1(x):
    """FluidSolver3.cs:445-452: -1 for a negative coordinate (the Rust step's
    signum().copysign(1.0) is +1 there)."""
    return F(-1) if (x < F(0) or (x == F(0) and math.copysign(1.0, float(x)) < 0)) else F(1)


def clamp(x, lo, hi):
    """System.Math.Clamp."""
    if x < lo:
        return lo
    if x > hi:
        return hi
    return x


SPHERE, BOX, CAPSULE = 0, 1, 2


class CsFluid3:
    """FluidState3 + FluidIntegration3.StepFluid3 with static identity-rotation
    bodies (shape, (px, py, pz), (a, b, c)) in body order: SPHERE (a =
    radius), BOX (half extents), CAPSULE (a = radius, b = half length along
    y)."""

    def __init__(self, cfg, bodies, gravity=(0.0, -9.81, 0.0), rust_sign=False):
        # rust_sign: a particle inside a box is pushed out along +axis, as the
        # Rust step's signum().copysign(1.0) does (fluid3.rs), instead of the
        # C# Copysign1's -axis for a negative coordinate: the one place where
        # the reference's two statements differ
        self.rust_sign = rust_sign
        self.cfg = cfg
        self.bodies = [(int(sh), tuple(F(v) for v in p), tuple(F(v) for v in e)) for sh, p, e in bodies]
        self.g = tuple(F(v) for v in gravity)
        self.pos, self.vel, self.mass, self.dens, self.pres = [], [], [], [], []
        self.grid = {}

    def add_particles(self, pts):
        # FluidState.cs:238-247: mass = ParticleMass, velocity zero
        for p in pts:
            self.pos.append(tuple(F(v) for v in p))
            self.vel.append((F(0), F(0), F(0)))
            self.mass.append(F(self.cfg.particle_mass))
            self.dens.append(F(0))
            self.pres.append(F(0))

    def state(self):
        return np.array([p + v for p, v in zip(self.pos, self.vel)], np.float32)

    # FluidSolver3.cs:103-153
    def rebuild_grid(self):
        self.grid = {}
        h = F(self.cfg.smoothing_length)
        for i, p in enumerate(self.pos):
            if not all(np.isfinite(c) for c in p):
                continue
            key = tuple(int(math.floor(c / h)) for c in p)
            self.grid.setdefault(key, []).append(i)

    # FluidSolver3.cs:155-184: cells oz, oy, ox; ids in cell order; includes i
    def neighbors(self, i):
        h = F(self.cfg.smoothing_length)
        p = self.pos[i]
        cx, cy, cz = (int(math.floor(c / h)) for c in p)
        out = []
        for oz in (-1, 0, 1):
            for oy in (-1, 0, 1):
                for ox in (-1, 0, 1):
                    for j in self.grid.get((cx + ox, cy + oy, cz + oz), ()):
                        d = tuple(a - b for a, b in zip(self.pos[j], p))
                        if dot(d, d) < h * h:
                            out.append(j)
        return out

    # FluidSolver3.cs:455-486
    def cfl_substeps(self, dt):
        c = self.cfg
        mx = 1 if c.max_substeps < 1 else int(c.max_substeps)
        if F(c.cfl) <= F(0) or mx <= 1:
            return 1
        h = max(F(c.smoothing_length), EPS)
        rho0 = max(F(c.rest_density), EPS)
        k = max(F(c.stiffness), F(0))
        c0 = F(np.sqrt(k)) if F(c.gamma) == F(1) else F(np.sqrt(F(c.gamma) * k * rho0))
        vmax = F(0)
        for v in self.vel:
            vmax = max(vmax, length(v))
        speed = c0 + vmax
        if not np.isfinite(speed) or speed <= EPS:
            return 1
        dt_max = F(c.cfl) * h / speed
        if not np.isfinite(dt_max) or dt_max <= F(0):
            return 1
        n = int(math.ceil(F(dt) / dt_max))
        return max(1, min(n, mx))

    # FluidSolver3.cs:488-518
    def density_pressure(self, h):
        c = self.cfg
        for i in range(len(self.pos)):
            rho = F(0)
            pi = self.pos[i]
            for j in self.neighbors(i):
                d = tuple(a - b for a, b in zip(self.pos[j], pi))
                rho = rho + self.mass[j] * poly6(dot(d, d), h)
            self.dens[i] = clamp(rho, F(0), F(3) * max(F(c.rest_density), EPS))
        for i in range(len(self.pos)):
            self.pres[i] = pressure(self.dens[i], F(c.phase_rest_density[0]), F(c.stiffness), F(c.gamma))

    # CollideParticleBody3 (FluidSolver3.cs:325-443), identity rotation
    def collide(self, p, pr, body):
        shape, bp, ext = body
        if shape == SPHERE:  # :330-342
            delta = tuple(a - c for a, c in zip(p, bp))
            dist = length(delta)
            if dist >= ext[0] + pr:
                return None
            normal = tuple(d / dist for d in delta) if dist > EPS else (F(1), F(0), F(0))
            return normal, ext[0] + pr - dist
        if shape == CAPSULE:  # :386-413
            r, hl = ext[0], ext[1]
            local = tuple(a - c for a, c in zip(p, bp))
            sy = clamp(local[1], -hl, hl)
            diff = (local[0] - F(0), local[1] - sy, local[2] - F(0))
            if dot(diff, diff) > EPS_SQ:
                dist = length(diff)
                if dist >= r + pr:
                    return None
                return tuple(d / dist for d in diff), r + pr - dist
            radial = (local[0], F(0), local[2])
            if dot(radial, radial) > EPS_SQ:
                ln = length(radial)  # NormalizeOrZero
                d = tuple(c / ln for c in radial) if ln > F(0) and np.isfinite(ln) else (F(0), F(0), F(0))
            else:
                d = (F(1), F(0), F(0))
            return d, pr + r - length(diff)
        return self.collide_box(p, pr, bp + ext)

    # BoxShape3 branch (FluidSolver3.cs:343-385)
    def collide_box(self, p, pr, b):
        bp, he = b[:3], b[3:]
        local = tuple(a - c for a, c in zip(p, bp))
        clamped = tuple(clamp(l, -e, e) for l, e in zip(local, he))
        diff = tuple(l - c for l, c in zip(local, clamped))
        if dot(diff, diff) > EPS_SQ:
            dist = length(diff)
            if dist >= pr:
                return None
            return tuple(d / dist for d in diff), pr - dist
        d = [e - abs(l) for e, l in zip(he, local)]
        if d[0] <= d[1] and d[0] <= d[2]:
            ax = 0
        elif d[1] <= d[2]:
            ax = 1
        else:
            ax = 2
        n = [F(0), F(0), F(0)]
        sg = (abs(local[ax]) if np.isnan(local[ax]) else F(1)) if self.rust_sign else copysign1(local[ax])
        n[ax] = F(1) * sg
        return tuple(n), pr + d[ax]

    # FluidSolver3.cs:923-1161
    def substep(self, dt):
        c = self.cfg
        dt = F(dt)
        h = max(F(c.smoothing_length), EPS)
        self.rebuild_grid()
        self.density_pressure(h)
        cs = F(np.sqrt(max(F(c.stiffness), F(0))))
        n = len(self.pos)
        forces = []
        for i in range(n):
            nb = self.neighbors(i)
            pi, rho_i, p_i = self.pos[i], max(self.dens[i], EPS), self.pres[i]
            f = [F(0), F(0), F(0)]
            for j in nb:
                if j == i:
                    continue
                rho_j = max(self.dens[j], EPS)
                delta = tuple(a - b for a, b in zip(pi, self.pos[j]))
                dist = length(delta)
                grad = spiky_grad(delta, dist, h)
                term = p_i / (rho_i * rho_i) + self.pres[j] / (rho_j * rho_j)
                if F(c.artificial_viscosity) > F(0) and dist > EPS:
                    # FluidSolver3.cs:75-85, called at :983-987
                    rho_bar = F(0.5) * (rho_i + rho_j)
                    vrel = tuple(a - b for a, b in zip(self.vel[i], self.vel[j]))
                    vd = dot(vrel, delta)
                    if not vd >= F(0):
                        mu = h * vd / (dist * dist + F(0.01) * h * h)
                        term = term + -F(c.artificial_viscosity) * cs * mu / max(rho_bar, EPS)
                mt = self.mass[j] * term
                f = [fa - g * mt for fa, g in zip(f, grad)]
                if F(c.surface_tension) > F(0) and dist > EPS:
                    # FluidSolver3.cs:87-94, applied at :989-996
                    coh = F(0) if dist >= h else F(1) - dist / h
                    if coh > F(0):
                        sc = F(c.surface_tension) * self.mass[i] * self.mass[j] * coh
                        f = [fa - (d / dist) * sc for fa, d in zip(f, delta)]
            forces.append(f)
        # integrate in place: later particles see the earlier ones' new state
        visc, vmax = F(c.viscosity), F(c.max_velocity)
        for i in range(n):
            nb = self.neighbors(i)
            rho_i = max(self.dens[i], EPS)
            acc = tuple(g + fc / rho_i for g, fc in zip(self.g, forces[i]))
            v = tuple(a + b * dt for a, b in zip(self.vel[i], acc))
            if visc > F(0):
                ppos, vi0 = self.pos[i], self.vel[i]
                smooth = (F(0), F(0), F(0))
                for j in nb:
                    if j == i:
                        continue
                    rho_bar = F(0.5) * (rho_i + max(self.dens[j], EPS))
                    d = tuple(a - b for a, b in zip(self.pos[j], ppos))
                    w = poly6(dot(d, d), h)
                    mr = self.mass[j] / rho_bar
                    smooth = tuple(s + ((vj - v0) * mr) * w for s, vj, v0 in zip(smooth, self.vel[j], vi0))
                v = tuple(a + s * visc for a, s in zip(v, smooth))
            speed = length(v)
            if speed > vmax:
                sc = vmax / speed
                v = tuple(a * sc for a in v)
            if not all(np.isfinite(a) for a in v):
                v = (F(0), F(0), F(0))
            pos = tuple(a + b * dt for a, b in zip(self.pos[i], v))
            if not all(np.isfinite(a) for a in pos):
                pos = self.pos[i]
            self.vel[i], self.pos[i] = v, pos
        # boundary pass, particle by particle, bodies in order (statics take no impulse)
        pr = max(F(c.particle_radius), F(0))
        for i in range(n):
            for b in self.bodies:
                hit = self.collide(self.pos[i], pr, b)
                if hit is None:
                    continue
                normal, depth = hit
                if depth <= F(0):
                    continue
                self.pos[i] = tuple(p + nn * depth for p, nn in zip(self.pos[i], normal))
                v = self.vel[i]
                vn = dot(v, normal)
                if vn < F(0):
                    v = tuple(a - nn * vn for a, nn in zip(v, normal))
                    if F(c.wall_friction) > F(0):
                        mu = clamp(F(c.wall_friction), F(0), F(1))
                        wn = F(0) * normal[0] + F(0) * normal[1] + F(0) * normal[2]
                        wvt = tuple(F(0) - nn * wn for nn in normal)
                        v = tuple(a + (w - a) * mu for a, w in zip(v, wvt))
                    self.vel[i] = v

    def step(self, dt):
        c = self.cfg
        if not c.enabled or not self.pos or not F(dt) > F(0):
            return
        k = self.cfl_substeps(dt)
        sub = F(dt) / F(k)
        for _ in range(k):
            self.substep(sub)
