"""The reference's behavioural SPH tests (crates/dynamics/src/fluid.rs:1145-2132),
re-run on the CPU oracle (both integrate orders) and on the GPU library.

Each test cites the reference test it restates. Tests that need dynamic
bodies, turbulence, adaptive resolution or boundary ghosts are out of scope
for this library and are not restated here.
"""
import numpy as np
import pytest

import sims
from oracle import oracle as orc

BACKENDS = ["oracle_seq", "oracle_jacobi", pytest.param("gpu", marks=pytest.mark.gpu)]
DT = 1.0 / 60.0


def finite(sim):
    s = sim.state()
    d, _ = sim.density_pressure()
    assert np.isfinite(s).all() and np.isfinite(d).all()


# fluid.rs:1209 test_fluid_kernels_sane
def test_kernels_sane():
    h = 0.5
    peak = orc.poly6(0.0, h)
    assert peak > 0.0
    assert orc.poly6(h * h, h) == 0.0
    assert orc.poly6(h * h * 4.0, h) == 0.0
    assert orc.poly6(h * h * 0.25, h) < peak
    gx, gy = orc.spiky_grad(0.25, 0.0, 0.25, h)
    assert gx < 0.0 and gy == 0.0
    assert orc.spiky_grad(h, 0.0, h, h) == (0.0, 0.0)
    assert orc.spiky_grad(0.0, 0.0, 0.0, h) == (0.0, 0.0)


# fluid.rs:1311 test_fluid_tait_eos_pressure (the one bit-pinned identity)
def test_tait_eos_pressure():
    k, rho0 = 100.0, 1.0
    assert orc.pressure(rho0, rho0, k, 7.0) == 0.0
    assert orc.pressure(0.5, rho0, k, 7.0) == 0.0
    lin = orc.pressure(1.2, rho0, k, 1.0)
    tait = orc.pressure(1.2, rho0, k, 7.0)
    assert lin > 0.0 and tait > lin
    expect = np.float32(k) * (np.float32(1.2) - np.float32(rho0))
    assert np.float32(orc.pressure(1.2, rho0, k, 1.0)).view(np.uint32) == np.float32(expect).view(np.uint32)


# fluid.rs:1333 test_fluid_artificial_pressure_sign
def test_artificial_pressure_sign():
    p_app = orc.artificial_pressure(1.0, 0.0, -2.0, 0.0, 1.0, 0.5, 1.0, 10.0, 1.0)
    p_sep = orc.artificial_pressure(1.0, 0.0, 2.0, 0.0, 1.0, 0.5, 1.0, 10.0, 1.0)
    assert p_app > 0.0
    assert p_sep == 0.0
    assert orc.artificial_pressure(1.0, 0.0, -2.0, 0.0, 1.0, 0.5, 1.0, 10.0, 0.0) == 0.0


# fluid.rs:1353 test_fluid_cohesion_kernel
def test_cohesion_kernel():
    h = 0.5
    assert orc.cohesion(0.1, h) > orc.cohesion(0.4, h)
    assert orc.cohesion(h, h) == 0.0
    assert orc.cohesion(0.9, h) == 0.0


# fluid.rs:1225 test_fluid_dam_break_contained
@pytest.mark.parametrize("backend", BACKENDS)
def test_dam_break_contained(backend):
    sim = sims.make(backend)
    sims.tank(sim)
    sims.lattice(sim, 0.0, 0.0, 8, 12, 0.25)
    peak, max_x = 0.0, 0.0
    for frame in range(600):
        sim.step(DT)
        s = sim.state()
        peak = max(peak, float(np.sqrt((s[:, 2] ** 2 + s[:, 3] ** 2)).max()))
        max_x = max(max_x, float(s[:, 0].max()))
        if frame % 100 == 0:
            finite(sim)
    finite(sim)
    assert max_x > 2.5, max_x
    s = sim.state()
    assert ((s[:, 0] > -1.0) & (s[:, 0] < 5.0) & (s[:, 1] > -0.6)).all()
    assert peak < 30.0
    assert sim.count == 96


# fluid.rs:1292 test_fluid_determinism (bit-identical positions, two runs)
@pytest.mark.parametrize("backend", BACKENDS)
def test_determinism(backend):
    def run():
        sim = sims.make(backend)
        sims.tank(sim)
        sims.lattice(sim, 0.0, 0.0, 6, 8, 0.25)
        for _ in range(120):
            sim.step(DT)
        return sim.state()[:, :2].copy()

    a, b = run(), run()
    assert a.shape == b.shape
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


# fluid.rs:1361 test_fluid_cohesion_attracts
@pytest.mark.parametrize("backend", BACKENDS)
def test_cohesion_attracts(backend):
    sim = sims.make(backend)
    sim.set_gravity(0.0, 0.0)
    assert sim.add_particles(np.array([[0.0, 0.0], [0.4, 0.0]], np.float32)) == 2
    c = sims.default_cfg()
    c.stiffness = 0.0
    c.viscosity = 0.0
    c.surface_tension = 1000.0
    sim.config = c
    sim.step(DT)
    s = sim.state()
    assert s[0, 2] > 0.0 and s[1, 2] < 0.0


# fluid.rs:1385 test_fluid_expansion_tank_stable (Tait + AV + cohesion)
@pytest.mark.parametrize("backend", BACKENDS)
def test_expansion_tank_stable(backend):
    sim = sims.make(backend)
    sims.tank(sim)
    sims.lattice(sim, -0.5, -0.5, 12, 6, 0.25)
    c = sims.default_cfg()
    c.gamma = 7.0
    c.stiffness = 15.0
    c.artificial_viscosity = 1.0
    c.surface_tension = 0.5
    sim.config = c
    peak = 0.0
    for frame in range(400):
        sim.step(DT)
        s = sim.state()
        peak = max(peak, float(np.sqrt(s[:, 2] ** 2 + s[:, 3] ** 2).max()))
        if frame % 100 == 0:
            finite(sim)
    s = sim.state()
    assert ((s[:, 0] > -1.0) & (s[:, 0] < 5.0) & (s[:, 1] > -0.6)).all()
    assert peak < 30.0


# fluid.rs:1421 test_fluid_cfl_substeps
def test_cfl_substeps():
    sim = sims.make("oracle_seq")
    sim.add_particles(np.array([[0.0, 0.0], [0.25, 0.0]], np.float32))
    assert sim.w.cfl_substeps(DT) == 1
    c = sims.default_cfg()
    c.gamma = 7.0
    c.stiffness = 200.0
    c.cfl = 0.4
    c.max_substeps = 8
    sim.config = c
    sim.set_state(np.array([[0.0, 0.0, 20.0, 0.0], [0.25, 0.0, 0.0, 0.0]], np.float32))
    n = sim.w.cfl_substeps(DT)
    assert 2 <= n <= 8
    c.max_substeps = 2
    sim.config = c
    assert sim.w.cfl_substeps(DT) == 2


# fluid.rs:1442 test_fluid_cfl_stabilizes_stiff_tait
@pytest.mark.parametrize("backend", BACKENDS)
def test_cfl_stabilizes_stiff_tait(backend):
    sim = sims.make(backend)
    sims.tank(sim)
    sims.lattice(sim, 0.0, 0.0, 8, 12, 0.25)
    c = sims.default_cfg()
    c.gamma = 7.0
    c.stiffness = 200.0
    c.cfl = 0.4
    c.max_substeps = 8
    sim.config = c
    peak = 0.0
    for _ in range(200):
        sim.step(DT)
        s = sim.state()
        peak = max(peak, float(np.sqrt(s[:, 2] ** 2 + s[:, 3] ** 2).max()))
    finite(sim)
    s = sim.state()
    assert ((s[:, 0] > -1.0) & (s[:, 0] < 5.0) & (s[:, 1] > -0.6)).all()
    assert peak < 30.0


def _hydro_stats(sim):
    """hydrostatic_stats (fluid.rs:1941-1966)."""
    s = sim.state()
    _, p = sim.density_pressure()
    ys = np.sort(s[:, 1])
    n, tenth = ys.shape[0], ys.shape[0] // 10
    bottom = ys[:tenth].mean()
    surface = ys[n - tenth:].mean()
    lo, hi = ys[tenth], ys[n - tenth]
    p_bottom = p[s[:, 1] <= lo].mean()
    p_top = p[s[:, 1] >= hi].mean()
    return p_bottom, p_top, surface - bottom


# fluid.rs:1676 sph_hydrostatic_pressure
@pytest.mark.parametrize("backend", BACKENDS)
def test_hydrostatic_pressure(backend):
    sim = sims.make(backend)
    sims.tank(sim)
    sims.lattice(sim, 0.0, 0.0, 18, 12, 0.25)
    sim.step(DT, 1200)
    finite(sim)
    p_bottom, p_top, height = _hydro_stats(sim)
    expected = 1.0 * 9.81 * height
    assert p_bottom > p_top
    assert 0.3 * expected < p_bottom < 3.0 * expected


# fluid.rs:1970 sph_hydrostatic_tait
@pytest.mark.parametrize("backend", BACKENDS)
def test_hydrostatic_tait(backend):
    sim = sims.make(backend)
    sims.tank(sim)
    c = sims.default_cfg()
    c.gamma = 7.0
    c.stiffness = 15.0
    sim.config = c
    sims.lattice(sim, 0.0, 0.0, 18, 12, 0.25)
    sim.step(DT, 1200)
    finite(sim)
    p_bottom, p_top, height = _hydro_stats(sim)
    expected = 1.0 * 9.81 * height
    assert p_bottom > p_top
    assert 0.5 * expected < p_bottom < 2.0 * expected


def _long_tank(sim):
    sim.add_box(5.0, -0.5, 11.0, 0.5)
    for x in (-1.0, 11.0):
        sim.add_box(x, 5.0, 1.5, 6.0)


# fluid.rs:1734 sph_dam_break_surge_front
@pytest.mark.parametrize("backend", BACKENDS)
def test_surge_front(backend):
    sim = sims.make(backend)
    _long_tank(sim)
    sims.lattice(sim, 0.5, 0.0, 8, 12, 0.25)
    sim.step(DT)
    x0 = sim.state()[:, 0].max()
    sim.step(DT, 159)
    f3 = sim.state()[:, 0].max()
    assert f3 > x0 + 1.0
    finite(sim)
    s = sim.state()
    assert ((s[:, 0] > 0.0) & (s[:, 0] < 9.5) & (s[:, 1] > -1.0)).all()


# fluid.rs:1993 sph_dam_break_obstacle
@pytest.mark.parametrize("backend", BACKENDS)
def test_dam_break_obstacle(backend):
    sim = sims.make(backend)
    _long_tank(sim)
    sim.add_box(4.0, 0.4, 0.6, 0.9)
    sims.lattice(sim, 0.5, 0.0, 8, 12, 0.25)
    sim.step(DT, 400)
    finite(sim)
    s = sim.state()
    assert (s[:, 0] > 6.0).sum() > 5
    d = s[:, :2] - np.array([4.0, 0.4], np.float32)
    inside = (np.abs(d[:, 0]) < 0.6 - 0.05) & (np.abs(d[:, 1]) < 0.9 - 0.05)
    assert not inside.any()


# fluid.rs:1775 sph_droplet_cohesion
@pytest.mark.parametrize("backend", BACKENDS)
def test_droplet_cohesion(backend):
    sim = sims.make(backend)
    sim.set_gravity(0.0, 0.0)
    c = sims.default_cfg()
    c.surface_tension = 8.0
    c.viscosity = 0.1
    c.max_velocity = 10.0
    sim.config = c
    pts = []
    for iy in range(-6, 7):
        for ix in range(-6, 7):
            x, y = np.float32(ix) * np.float32(0.25), np.float32(iy) * np.float32(0.25)
            if x * x + y * y <= np.float32(1.25) * np.float32(1.25):
                pts.append((x, y))
    sim.add_particles(np.array(pts, np.float32))
    r0 = np.sqrt((sim.state()[:, :2] ** 2).sum(1)).max()
    sim.step(DT, 600)
    finite(sim)
    r1 = np.sqrt((sim.state()[:, :2] ** 2).sum(1)).max()
    assert r1 < 2.0 * r0


# fluid.rs:1812 sph_free_blob_energy_bounded
@pytest.mark.parametrize("backend", BACKENDS)
def test_free_blob_energy_bounded(backend):
    sim = sims.make(backend)
    sim.set_gravity(0.0, 0.0)
    c = sims.default_cfg()
    c.viscosity = 0.0
    c.drag = 0.0
    c.max_velocity = 100.0
    sim.config = c
    pts = sims.lattice(sim, -1.0, -1.0, 8, 8, 0.25)
    st = np.zeros((pts.shape[0], 4), np.float32)
    st[:, :2] = pts
    st[:, 2] = 1.0
    sim.set_state(st)
    m = c.particle_mass

    def ke():
        s = sim.state()
        return m * (0.5 * (s[:, 2] ** 2 + s[:, 3] ** 2)).sum()

    e0 = ke()
    sim.step(DT, 600)
    finite(sim)
    e1 = ke()
    assert 0.0 < e1 < 2.0 * e0


def _channel(sim, mu):
    sim.set_gravity(4.0, 0.0)
    c = sims.default_cfg()
    c.max_velocity = 100.0
    c.wall_friction = mu
    return c


# fluid.rs:1846 sph_poiseuille_profile. The reference asserts the curved
# profile on the single frame 600; the band means flip back and forth between
# frames even in the reference's own integrate order (at frame 300 the centre
# band is slower than the bottom one), so that snapshot is a property of one
# chaotic trajectory. The reference order keeps the exact snapshot check; the
# Jacobi backends check the same profile averaged over frames 300-600.
@pytest.mark.parametrize("backend", BACKENDS)
def test_poiseuille_profile(backend):
    sim = sims.make(backend)
    c = _channel(sim, 1.0)
    c.artificial_viscosity = 0.5
    sim.config = c
    sim.add_box(0.0, 0.0, 4.0, 0.5)
    sim.add_box(0.0, 3.0, 4.0, 0.5)
    sims.lattice(sim, -3.0, 0.5, 24, 9, 0.25)

    def bands(s):
        out = []
        for lo, hi in ((0.5, 1.1), (1.1, 1.9), (1.9, 2.5)):
            m = (s[:, 1] >= lo) & (s[:, 1] < hi)
            out.append(s[m, 2].mean() if m.any() else 0.0)
        return np.array(out, np.float64)

    if backend == "oracle_seq":
        sim.step(DT, 600)
        bottom, middle, top = bands(sim.state())
    else:
        sim.step(DT, 300)
        acc = np.zeros(3)
        for _ in range(30):
            sim.step(DT, 10)
            acc += bands(sim.state())
        bottom, middle, top = acc / 30
    finite(sim)
    assert middle > bottom and middle > top


# fluid.rs:1903 sph_wall_friction_slows_flow
@pytest.mark.parametrize("backend", BACKENDS)
def test_wall_friction_slows_flow(backend):
    def run(mu):
        sim = sims.make(backend)
        sim.config = _channel(sim, mu)
        sim.add_box(0.0, 0.0, 4.0, 0.5)
        sim.add_box(0.0, 3.0, 4.0, 0.5)
        sims.lattice(sim, -3.0, 0.5, 24, 9, 0.25)
        sim.step(DT, 600)
        return sim.state()[:, 2].mean()

    assert run(1.0) < run(0.0)


# fluid.rs:2048 sph_sloshing_settles
@pytest.mark.parametrize("backend", BACKENDS)
def test_sloshing_settles(backend):
    sim = sims.make(backend)
    sims.tank(sim)
    pts = sims.lattice(sim, -0.5, -0.5, 12, 6, 0.25)
    st = np.zeros((pts.shape[0], 4), np.float32)
    st[:, :2] = pts
    st[:, 2] = 2.0
    sim.set_state(st)

    def peak():
        s = sim.state()
        return np.sqrt(s[:, 2] ** 2 + s[:, 3] ** 2).max()

    k0 = peak()
    sim.step(DT, 300)
    k1 = peak()
    sim.step(DT, 300)
    k2 = peak()
    finite(sim)
    assert k1 < k0 and k2 < k1


# fluid.rs:2080 sph_two_phase_heavy_sinks (per-particle mass and rest density)
@pytest.mark.parametrize("backend", BACKENDS)
def test_two_phase_heavy_sinks(backend):
    sim = sims.make(backend)
    sims.tank(sim)
    c = sims.default_cfg()
    c.phase_count = 2
    for k, v in enumerate([2.0, 1.0, 1.0, 1.0]):
        c.phase_rest_density[k] = v
    for k, v in enumerate([0.125, 0.0625, 0.0625, 0.0625]):
        c.phase_mass[k] = v
    sim.config = c
    f = np.float32
    light = np.array([(f(ix) * f(0.25), f(iy) * f(0.25)) for iy in range(8) for ix in range(18)], np.float32)
    heavy = np.array([(f(ix) * f(0.25), f(iy) * f(0.25)) for iy in range(8, 12) for ix in range(6, 12)], np.float32)
    sim.add_particles(light, np.ones(light.shape[0], np.uint8))
    sim.add_particles(heavy, np.zeros(heavy.shape[0], np.uint8))
    nl = light.shape[0]
    y0 = sim.state()[nl:, 1].mean()
    sim.step(DT, 600)
    finite(sim)
    y1 = sim.state()[nl:, 1].mean()
    assert y1 < y0
