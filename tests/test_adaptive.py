"""Adaptive resolution (FluidConfig2.adaptive_resolution, FluidState2::resample,
fluid.rs:826-893): after the first density pass, over-dense close pairs
merge (index order, mass and momentum conserved) and under-dense particles
split into two half-mass children (up to MAX_PARTICLES_2D), then the
substep's sort and density run again on the new set.

CPU: the reference's resample tests on the oracle (mass conserved over 200
steps, count within the cap, contained, fluid.rs:1518-1548; a lone particle
splits, fluid.rs:1551-1568). GPU: trajectories, counts and masses bit-exact
against the oracle's Jacobi integrate, merges and splits both occurring.
"""
import numpy as np
import pytest

import sims
from oracle import oracle as orc


def calm_tank(sim, cfg=None, nx=12, ny=6):
    sims.tank(sim)
    c = cfg if cfg is not None else sims.default_cfg()
    c.adaptive_resolution = 1
    sim.config = c
    sims.lattice(sim, -0.5, -0.5, nx, ny, 0.25)
    return sim


def masses(sim):
    if isinstance(sim, sims.OracleSim):
        return sim.w.masses()
    return sim.w.fluid.masses()


def test_oracle_adaptive_conserves_mass_and_stays_contained():
    s = calm_tank(sims.OracleSim(orc.REF_SEQ))
    m0 = float(masses(s).sum())
    for _ in range(200):
        s.step(1 / 60)
    st = s.state()
    assert np.isfinite(st).all()
    assert abs(float(masses(s).sum()) - m0) < 1e-3
    assert len(st) <= 4096
    assert (st[:, 0] > -1.0).all() and (st[:, 0] < 5.0).all() and (st[:, 1] > -0.6).all()


def test_oracle_lone_particle_splits():
    """An isolated particle is under-dense (its density is its own kernel
    weight): the first substep splits it into two half-mass children."""
    s = sims.OracleSim(orc.JACOBI)
    c = sims.default_cfg()
    c.adaptive_resolution = 1
    s.config = c
    s.add_particles(np.array([[0.0, 3.0]], np.float32))
    m0 = float(masses(s).sum())
    s.step(1 / 60)
    assert s.count == 2
    assert abs(float(masses(s).sum()) - m0) < 1e-6


def _dense_cfg():
    # a compressed column: the lower rows exceed merge_density_ratio * rest
    c = sims.default_cfg()
    c.merge_density_ratio = 1.15
    c.split_density_ratio = 0.55
    return c


@pytest.mark.gpu
@pytest.mark.parametrize("cfg_name", ["default", "dense"])
def test_adaptive_bit_exact(cfg_name):
    cfg = sims.default_cfg() if cfg_name == "default" else _dense_cfg()
    g = calm_tank(sims.GpuSim(), cfg, 14, 10)
    o = calm_tank(sims.OracleSim(orc.JACOBI), cfg, 14, 10)
    n0 = o.count
    counts = set()
    for k in range(8):
        g.step(1 / 60, 15)
        o.step(1 / 60, 15)
        assert g.count == o.count, f"step {15 * (k + 1)}: counts {g.count} vs {o.count}"
        counts.add(o.count)
        a, b = g.state(), o.state()
        bad = np.nonzero(a.view(np.uint32) != b.view(np.uint32))[0]
        assert bad.size == 0, f"step {15 * (k + 1)}: {bad.size} words differ, first particle {bad[0] // 4}"
        assert np.array_equal(masses(g).view(np.uint32), masses(o).view(np.uint32))
    assert counts != {n0}  # the resampling changed the particle count


def _sparse_points(n, spacing, x0=0.0, y0=0.5):
    """n isolated particles on a row-major grid `spacing` apart (> h, so each
    one's density is its own kernel weight: under split_density_ratio)."""
    nx = int(np.ceil(np.sqrt(n)))
    i = np.arange(n)
    return np.stack([x0 + (i % nx) * spacing, y0 + (i // nx) * spacing], axis=1).astype(np.float32)


def test_oracle_split_output_exceeds_the_add_cap():
    """More than MAX_PARTICLES_2D / 2 under-dense particles: the first 2048
    split (the output reaches 4096), the rest are kept, so one pass leaves
    n + 2048 particles, beyond the 4096 cap of add_particles (the reference's
    output is a Vec with no cap of its own, fluid.rs:873-889)."""
    s = sims.OracleSim(orc.JACOBI)
    c = sims.default_cfg()
    c.adaptive_resolution = 1
    s.config = c
    s.set_gravity(0.0, 0.0)
    assert s.add_particles(_sparse_points(3000, 2.0)) == 3000
    s.step(1 / 60)
    assert s.count == 3000 + 2048


@pytest.mark.gpu
def test_adaptive_split_beyond_cap_bit_exact():
    """The same pass on the GPU: the world's buffers hold the n + 2048 output
    (no write past them), and counts, states and masses equal the oracle's
    over further steps in which the grown set resamples again."""
    c = sims.default_cfg()
    c.adaptive_resolution = 1
    pts = _sparse_points(3000, 2.0)
    g, o = sims.GpuSim(), sims.OracleSim(orc.JACOBI)
    for s in (g, o):
        s.set_gravity(0.0, -9.81)
        s.config = c
        assert s.add_particles(pts) == 3000
    for k in range(4):
        g.step(1 / 60)
        o.step(1 / 60)
        assert g.count == o.count, f"step {k + 1}: counts {g.count} vs {o.count}"
        a, b = g.state(), o.state()
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), f"step {k + 1}: states differ"
        assert np.array_equal(masses(g).view(np.uint32), masses(o).view(np.uint32))
    assert o.count > 5000
    assert g.w.status().error == 0
