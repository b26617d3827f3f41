"""Pinning the C++ oracle (a restatement of the reference's Rust fluid step,
fluid.rs) to a second statement of the same algorithm by the reference's
authors: the C# solver (src/PhiEng.Dynamics/FluidSolver.cs), restated in
oracle/fluid_cs.py.

The reference asserts that its C# and Rust steps agree on the scene of
tests/PhiEng.Tests/EquivalenceTests.cs:122-176 (an 8 x 6 lattice at 0.25 in
the three-box tank, default config, 60 steps of 1/60 s) within 1e-4 in
position and 1e-3 in velocity per particle. The C++ oracle in the
reference's own (in-place) order must agree with the C# restatement on that
scene within the same bar; it does so bit for bit where both are IEEE f32 in
the same order, which this test also records.

The 3D oracle (oracle/sph_oracle3.hpp, from fluid3.rs) is pinned the same
way to the C# 3D solver (src/PhiEng.Dynamics/FluidSolver3.cs, restated in
oracle/fluid3_cs.py), on the scene of EquivalenceTests.cs:177-225 (30 steps,
1e-4 in position) and on the reference's five-box test tank.
"""
import numpy as np

import sims
from oracle import fluid_cs
from oracle import oracle as orc

TANK = [("box", 2.0, -1.0, 3.0, 0.5), ("box", -1.0, 2.0, 0.5, 3.5), ("box", 5.0, 2.0, 0.5, 3.5)]


def equivalence_points():
    # EquivalenceTests.cs:133-140: iy outer, ix inner
    return np.array([(ix * 0.25, iy * 0.25) for iy in range(6) for ix in range(8)], np.float32)


def run_both(cfg, steps, pts=None):
    pts = equivalence_points() if pts is None else pts
    cs = fluid_cs.CsFluid(cfg, TANK)
    cs.add_particles(pts)
    o = sims.OracleSim(orc.REF_SEQ)
    sims.tank(o)
    o.config = cfg
    assert o.add_particles(pts) == len(pts)
    for _ in range(steps):
        cs.step(1.0 / 60.0)
        o.step(1.0 / 60.0)
    return cs.state(), o.state()


def test_oracle_matches_csharp_solver_on_the_equivalence_scene():
    cfg = sims.default_cfg()
    a, b = run_both(cfg, 60)
    dp = np.sqrt(((a[:, :2] - b[:, :2]).astype(np.float64) ** 2).sum(1))
    dv = np.sqrt(((a[:, 2:] - b[:, 2:]).astype(np.float64) ** 2).sum(1))
    assert dp.max() < 1e-4 and dv.max() < 1e-3, (dp.max(), dv.max())
    # the two restatements are the same f32 operations in the same order
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_oracle_matches_csharp_solver_tait():
    """The Tait EOS (gamma 7, k 10) on a 12 x 10 lattice at rest spacing for
    40 steps: the two restatements' power functions (the oracle's correctly
    rounded power, numpy's float32 power for MathF.Pow) differ by an ulp now
    and then, and the runs stay within the reference's own bar."""
    cfg = sims.default_cfg()
    cfg.gamma = 7.0
    cfg.stiffness = 10.0
    pts = np.array([(0.125 + ix * 0.25, 0.125 + iy * 0.25) for iy in range(10) for ix in range(12)], np.float32)
    a, b = run_both(cfg, 40, pts)
    dp = np.sqrt(((a[:, :2] - b[:, :2]).astype(np.float64) ** 2).sum(1)).max()
    dv = np.sqrt(((a[:, 2:] - b[:, 2:]).astype(np.float64) ** 2).sum(1)).max()
    assert dp < 1e-4 and dv < 1e-3, (dp, dv)


# ---- 3D: crates/dynamics/src/fluid3.rs against src/PhiEng.Dynamics/FluidSolver3.cs ----

from oracle import fluid3_cs  # noqa: E402
from phi_eng_b200._abi import default_config  # noqa: E402
from test_fluid3 import BOX, TANK as TANK3, lattice, make_oracle  # noqa: E402


def run_both3(cfg, steps, pts, bodies, rust_sign=False):
    cs = fluid3_cs.CsFluid3(cfg, bodies, rust_sign=rust_sign)
    cs.add_particles(pts)
    o = make_oracle(pts, bodies=bodies, cfg=cfg, gravity=(0.0, -9.81, 0.0))
    for _ in range(steps):
        cs.step(1.0 / 60.0)
        o.step(1.0 / 60.0, orc.REF_SEQ)
    a, b = cs.state(), o.state()
    dp = np.sqrt(((a[:, :3] - b[:, :3]).astype(np.float64) ** 2).sum(1)).max()
    dv = np.sqrt(((a[:, 3:] - b[:, 3:]).astype(np.float64) ** 2).sum(1)).max()
    return a, b, dp, dv


def test_oracle3_matches_csharp_solver_on_the_equivalence_scene():
    """EquivalenceTests.cs:177-225: a 3 x 3 x 3 lattice at 0.25 (iz, iy, ix
    loops) over one static box (centre (1, -1, 1), half extents (2, 0.5, 2)),
    default config, 30 steps of 1/60 s; the reference's bar is 1e-4 in
    position. The two restatements agree bit for bit."""
    pts = np.array([(ix * 0.25, iy * 0.25, iz * 0.25) for iz in range(3) for iy in range(3) for ix in range(3)],
                   np.float32)
    a, b, dp, dv = run_both3(default_config(), 30, pts, [(BOX, (1.0, -1.0, 1.0), (2.0, 0.5, 2.0))])
    assert dp < 1e-4, dp
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_oracle3_matches_csharp_solver_tank_cfl_friction():
    """A 6 x 5 x 6 lattice in the reference's five-box test tank, linear EOS
    (k 400: two CFL substeps per step from the start), wall friction, 40
    steps: bit for bit."""
    cfg = default_config()
    cfg.stiffness = 400.0
    cfg.cfl = 0.4
    cfg.max_substeps = 4
    cfg.wall_friction = 0.5
    pts = lattice((0.125, -0.375, 0.125), 6, 5, 6, 0.25)
    cs = fluid3_cs.CsFluid3(cfg, TANK3)
    cs.add_particles(pts)
    assert cs.cfl_substeps(1.0 / 60.0) >= 2
    a, b, dp, dv = run_both3(cfg, 40, pts, TANK3)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (dp, dv)


def test_oracle3_matches_csharp_solver_tait():
    """Tait EOS (gamma 7, k 10) with CFL substeps, 20 steps: the power
    functions differ by an ulp at times (the oracle's correctly rounded power,
    numpy's float32 power for MathF.Pow); the runs stay within the
    reference's bars (1e-4 position, 1e-3 velocity)."""
    cfg = default_config()
    cfg.gamma = 7.0
    cfg.stiffness = 10.0
    cfg.cfl = 0.4
    cfg.max_substeps = 4
    pts = lattice((0.125, -0.375, 0.125), 6, 5, 6, 0.25)
    a, b, dp, dv = run_both3(cfg, 20, pts, TANK3)
    assert dp < 1e-4 and dv < 1e-3, (dp, dv)


def test_oracle_matches_csharp_solver_av_cohesion():
    """Monaghan artificial viscosity (alpha 0.5) and cohesion (surface
    tension 2) on the 2D equivalence scene, 60 steps: bit for bit, and the
    terms change the run."""
    cfg = sims.default_cfg()
    cfg.artificial_viscosity = 0.5
    cfg.surface_tension = 2.0
    a, b = run_both(cfg, 60)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    plain, _ = run_both(sims.default_cfg(), 60)
    assert not np.array_equal(a, plain)


def test_oracle3_matches_csharp_solver_av_cohesion():
    """The same terms (and wall friction) in the 3D tank, 40 steps: bit for
    bit, and the terms change the run."""
    cfg = default_config()
    cfg.artificial_viscosity = 0.5
    cfg.surface_tension = 2.0
    cfg.wall_friction = 0.3
    pts = lattice((0.125, -0.375, 0.125), 6, 5, 6, 0.25)
    a, b, dp, dv = run_both3(cfg, 40, pts, TANK3)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (dp, dv)
    plain, _, _, _ = run_both3(default_config(), 40, pts, TANK3)
    assert not np.array_equal(a, plain)


def test_oracle_matches_csharp_solver_cfl_friction():
    """CFL substeps (k 400: two substeps per 1/60 s step from the start) and
    wall friction on the 2D equivalence scene, 60 steps: bit for bit."""
    cfg = sims.default_cfg()
    cfg.stiffness = 400.0
    cfg.cfl = 0.4
    cfg.max_substeps = 4
    cfg.wall_friction = 0.5
    cs = fluid_cs.CsFluid(cfg, TANK)
    cs.add_particles(equivalence_points())
    assert cs.cfl_substeps(1.0 / 60.0) >= 2
    a, b = run_both(cfg, 60)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_oracle3_matches_csharp_solver_sphere_capsule():
    """A static sphere and an upright capsule in the 3D tank under a falling
    block, 40 steps: bit for bit. At step 30 a fast particle ends a step just
    inside the right wall, where the reference's two statements differ (the
    C# Copysign1 pushes it out along -x, the Rust step along +x); the C#
    restatement takes the Rust sign there (rust_sign), and without it the
    runs part at that particle."""
    from test_fluid3 import CAPSULE, SPHERE

    bodies = TANK3 + [(SPHERE, (1.0, 0.2, 1.0), (0.45, 0.0, 0.0)), (CAPSULE, (3.0, 0.4, 3.0), (0.3, 0.5, 0.0))]
    pts = lattice((0.125, 1.0, 0.125), 6, 4, 6, 0.25)
    pts = np.concatenate([pts, np.array([[3.0, 1.2, 3.0]], np.float32)])
    a, b, dp, dv = run_both3(default_config(), 40, pts, bodies, rust_sign=True)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (dp, dv)
    a, b, dp, dv = run_both3(default_config(), 40, pts, bodies)
    assert not np.array_equal(a, b)


def test_oracle_matches_csharp_solver_circle_obstacle():
    """A static circle in the 2D tank under a falling 10 x 6 block, with wall
    friction, 60 steps: bit for bit."""
    cfg = sims.default_cfg()
    cfg.wall_friction = 0.3
    pts = np.array([(0.125 + ix * 0.25, 1.0 + iy * 0.25) for iy in range(6) for ix in range(10)], np.float32)
    cs = fluid_cs.CsFluid(cfg, TANK + [("circle", 1.2, 0.3, 0.35)])
    cs.add_particles(pts)
    o = sims.OracleSim(orc.REF_SEQ)
    sims.tank(o)
    o.add_circle(1.2, 0.3, 0.35)
    o.config = cfg
    assert o.add_particles(pts) == len(pts)
    touched = False
    for _ in range(60):
        cs.step(1.0 / 60.0)
        o.step(1.0 / 60.0)
        s = cs.state()
        d = np.sqrt((s[:, 0] - 1.2) ** 2 + (s[:, 1] - 0.3) ** 2)
        touched = touched or bool((d < 0.35 + cfg.particle_radius + 1e-3).any())
    a, b = cs.state(), o.state()
    assert touched  # the block reached the circle
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
