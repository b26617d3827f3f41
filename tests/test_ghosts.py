"""Boundary ghost particles (FluidConfig2.boundary_particles, fluid.rs:617-818):
static bodies sampled at h / 2, their density and pressure from the fluid
each substep, their pressure on the fluid after the fluid pairs.

CPU: the reference's ghost tests on the oracle (present and deterministic,
fluid.rs:1572-1599; contained, fluid.rs:1602-1627). GPU: the generated set
equals the oracle's, it is generated once for a static scene and persists
(fluid.rs:1630-1662), and trajectories are bit-exact against the oracle's
Jacobi integrate, with Tait / AV / obstacles and through the fluid phase with
polygon bodies.
"""
import ctypes as C

import numpy as np
import pytest

import sims
from oracle import oracle as orc
from phi_eng_b200 import _abi


def ghost_scene(sim, nx=6, ny=8, cfg=None, circle=False):
    sims.tank(sim)
    if circle:
        sim.add_circle(2.5, 0.4, 0.35)
    c = cfg if cfg is not None else sims.default_cfg()
    c.boundary_particles = 1
    sim.config = c
    sims.lattice(sim, 0.0, 0.0, nx, ny, 0.25)
    return sim


def sorted_rows(a):
    a = np.ascontiguousarray(a, np.float32)
    return a[np.lexsort((a[:, 1], a[:, 0]))]


# ---------------------------------------------------------------- oracle (CPU)
def test_oracle_ghosts_present_and_deterministic():
    a = ghost_scene(sims.OracleSim(orc.REF_SEQ))
    b = ghost_scene(sims.OracleSim(orc.REF_SEQ))
    a.step(1 / 60)
    b.step(1 / 60)
    ga, gb = a.w.ghosts(), b.w.ghosts()
    assert len(ga) > 0
    assert np.array_equal(ga.view(np.uint32), gb.view(np.uint32))


def test_oracle_ghosts_contained():
    s = ghost_scene(sims.OracleSim(orc.REF_SEQ), 8, 12)
    peak = 0.0
    for _ in range(300):
        s.step(1 / 60)
        st = s.state()
        peak = max(peak, float(np.sqrt((st[:, 2:] ** 2).sum(1)).max()))
    st = s.state()
    assert np.isfinite(st).all()
    assert (st[:, 0] > -1.0).all() and (st[:, 0] < 5.0).all() and (st[:, 1] > -0.6).all()
    assert peak < 30.0


def test_ghosts_change_the_flow():
    on = ghost_scene(sims.OracleSim(orc.JACOBI))
    off = sims.OracleSim(orc.JACOBI)
    sims.tank(off)
    off.config = sims.default_cfg()
    sims.lattice(off, 0.0, 0.0, 6, 8, 0.25)
    # the reference samples a box on its left and bottom sides, up from its
    # top-left corner and right from its bottom-right one (fluid.rs:686-691):
    # the fluid meets ghosts at the right wall's inner face, after ~1 s
    on.step(1 / 60, 120)
    off.step(1 / 60, 120)
    assert not np.array_equal(on.state(), off.state())


# ---------------------------------------------------------------- GPU
def gpu_ghosts(sim):
    lib, h = sim.w._lib, sim.w._h
    regens = C.c_uint64()
    n = lib.phieng_sph_ghosts(h, None, 0, C.byref(regens))
    xy = np.zeros((n, 2), np.float32)
    lib.phieng_sph_ghosts(h, xy.ctypes.data_as(C.POINTER(C.c_float)), n, None)
    return xy, regens.value


@pytest.mark.gpu
def test_gpu_ghosts_equal_oracle_and_persist():
    g = ghost_scene(sims.GpuSim(), circle=True)
    o = ghost_scene(sims.OracleSim(orc.JACOBI), circle=True)
    g.step(1 / 60, 10)
    o.step(1 / 60, 10)
    xy, regens = gpu_ghosts(g)
    assert regens == 1  # a static scene generates its ghosts once
    ref = o.w.ghosts()
    assert len(xy) == len(ref) > 0
    assert np.array_equal(sorted_rows(xy).view(np.uint32), sorted_rows(ref).view(np.uint32))
    g.step(1 / 60, 10)
    xy2, regens = gpu_ghosts(g)
    assert regens == 1 and np.array_equal(xy2.view(np.uint32), xy.view(np.uint32))
    # a change of h regenerates them
    c = g.config
    c.smoothing_length = 0.45
    g.config = c
    g.step(1 / 60)
    assert gpu_ghosts(g)[1] == 2


def _parity(cfg, steps, circle=False, nx=6, ny=8, every=20):
    g = ghost_scene(sims.GpuSim(), nx, ny, cfg=cfg, circle=circle)
    o = ghost_scene(sims.OracleSim(orc.JACOBI), nx, ny, cfg=cfg, circle=circle)
    for k in range(0, steps, every):
        g.step(1 / 60, every)
        o.step(1 / 60, every)
        a, b = g.state(), o.state()
        bad = np.nonzero(a.view(np.uint32) != b.view(np.uint32))[0]
        assert bad.size == 0, f"step {k + every}: {bad.size} words differ, first particle {bad[0] // 4}"


@pytest.mark.gpu
def test_ghosts_bit_exact_reference_tank():
    _parity(sims.default_cfg(), 200)


@pytest.mark.gpu
def test_ghosts_bit_exact_tait_av_obstacle():
    c = sims.default_cfg()
    c.gamma = 7.0
    c.stiffness = 40.0
    c.artificial_viscosity = 0.1
    c.cfl = 0.4
    c.max_substeps = 4
    _parity(c, 150, circle=True, nx=8, ny=12, every=25)


@pytest.mark.gpu
def test_ghosts_bit_exact_fluid_phase_with_polygons():
    """Ghosts of the fluid phase's own static bodies, a polygon among them
    (its local vertices sampled edge by edge, fluid.rs:714-738)."""
    from test_dynamic_bodies import RAMP, TANK, coupled_parity, floating_bodies, poly_arrays, polygon_body

    c = _abi.default_config()
    c.boundary_particles = 1
    ramp, vr = polygon_body(1.2, 0.3, RAMP, angle=0.2)
    bodies = floating_bodies()
    bodies.insert(3, ramp)
    poly = poly_arrays([None, None, None, vr] + [None] * (len(bodies) - 4))
    coupled_parity(c, bodies, 60, poly=poly)
