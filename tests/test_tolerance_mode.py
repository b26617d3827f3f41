"""Tolerance mode (phieng_sph_set_precision(world, PHIENG_SPH_TOLERANCE)).

The plain force pass reassociates its sums (fused multiply-adds, one
approximate reciprocal square root and one approximate reciprocal per
neighbour pair); the density pass, neighbour sets, sort order and visit
order stay the exact mode's. Bars, all through the C ABI:
  * from identical state: density and pressure bit-exact (and so within the
    stated 1e-5), force within 1e-4 of its RMS against the oracle (the
    reference's f32 arithmetic); pressure also through check_pressure, the
    bar a reassociated density would have to meet (its Tait EOS amplifies
    density rounding near rest density);
  * the same state recomputed in FP64 by the oracle states both paths'
    error: the tolerance path's error stays within a small multiple of the
    exact f32 path's;
  * runs are bit-reproducible, and staging the neighbour rows in shared
    memory (a launch shape) changes no bit;
  * trajectories stay close to the exact mode's.
"""
import ctypes as C

import numpy as np
import pytest

import sims
from oracle import oracle as orc
from phi_eng_b200 import _abi, scenes
from phi_eng_b200.autotune import apply as apply_tuning


def rel_rms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    rms = np.sqrt((b ** 2).mean())
    return float(np.sqrt(((a - b) ** 2).mean()) / max(rms, 1e-30))


def test_precision_mode_abi():
    """Valid modes are taken, unknown ones refused with the world unchanged
    (no GPU needed: the device is set up on the first step)."""
    from phi_eng_b200.world import World2

    w = World2()
    assert w.precision == _abi.EXACT
    w.precision = _abi.TOLERANCE
    assert w.precision == _abi.TOLERANCE
    with pytest.raises(ValueError):
        w.precision = 7
    assert w.precision == _abi.TOLERANCE
    lib = w._lib
    assert lib.phieng_sph_set_precision(None, 0) == 0
    assert lib.phieng_sph_get_precision(None) == _abi.EXACT
    t = _abi.PhiengSphTuning(128, 128, 2.0, 8)  # stage bits beyond 2 are refused
    assert lib.phieng_sph_set_tuning(w._h, C.byref(t)) == 0
    t = _abi.PhiengSphTuning(128, 128, 2.0, 4)  # bit 2: the force pass's lane balancing
    assert lib.phieng_sph_set_tuning(w._h, C.byref(t)) == 1
    w.close()


def check_pressure(cfg, d_gpu, p_gpu, d_o, p_o):
    """Pressure is the EOS of the density (fluid.rs:290-297). Near rest
    density the Tait EOS is ill-conditioned, p ~ k gamma (rho / rho0 - 1), so
    the density's reassociation rounding (within 1e-5 of its RMS) is
    amplified by ~ 1 / |rho / rho0 - 1| in the pressure. The bar: the GPU's
    pressure is the EOS of the GPU's density within 5e-6 of the pressure
    RMS, and its difference to the oracle's pressure is the density
    difference carried through dp / drho (to first order) within 1e-5."""
    g, k = float(cfg.gamma), float(cfg.stiffness)
    r0 = max(float(cfg.phase_rest_density[0]), 1e-6)
    d = d_gpu.astype(np.float64)
    eos = np.maximum(k * r0 * ((d / r0) ** g - 1.0), 0.0) if g != 1.0 else np.maximum(k * (d - r0), 0.0)
    rms = np.sqrt(np.mean(p_o.astype(np.float64) ** 2))
    assert np.sqrt(np.mean((p_gpu - eos) ** 2)) <= 5e-6 * rms
    dpdr = np.where(eos > 0, k * g * (d / r0) ** (g - 1.0) if g != 1.0 else k, 0.0)
    lin = p_o.astype(np.float64) + dpdr * (d - d_o.astype(np.float64))
    assert np.sqrt(np.mean((p_gpu - lin) ** 2)) <= 1e-5 * rms


SCENES = {
    "tank_8x12": (scenes.reference_tank, 30),
    "dam_break_4k": (scenes.dam_break_4k, 200),
    "dam_break_128x128": (lambda: scenes.dam_break_scaled(128, 128), 100),
}


def _gpu(sc, tolerance=True, stage=3):
    g = sims.load_scene(sims.make("gpu"), sc)
    if tolerance:
        g.w.precision = _abi.TOLERANCE
    apply_tuning(g.w, dict(density_block=128, force_block=128, buckets_per_particle=2.0, stage=stage))
    return g


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(SCENES))
@pytest.mark.parametrize("stage", [0, 3, 4])
def test_identical_state_within_tolerance(name, stage):
    make, steps = SCENES[name]
    sc = make()
    g = _gpu(sc, stage=stage)
    g.step(sc.dt, steps)
    st = g.state()
    f_gpu = g.w.debug_forces()
    d_gpu, p_gpu = g.density_pressure()
    o = sims.load_scene(sims.OracleSim(orc.JACOBI), sc)
    o.set_state(st)
    o.w.pass_density()
    d_o, p_o = o.density_pressure()
    o.w.pass_forces()
    f_o = o.w.forces()
    assert rel_rms(d_gpu, d_o) <= 1e-5
    assert rel_rms(f_gpu, f_o) <= 1e-4
    check_pressure(sc.config, d_gpu, p_gpu, d_o, p_o)
    # the density pass is the exact one, staged in shared memory or not
    assert np.array_equal(d_gpu, d_o) and np.array_equal(p_gpu, p_o)


@pytest.mark.gpu
def test_fp64_error_of_both_paths():
    """One step's density and force recomputed in FP64 on the oracle from the
    same state: the error of the exact f32 path and of the tolerance path."""
    sc = scenes.dam_break_4k()
    g = _gpu(sc)
    g.step(sc.dt, 200)
    st = g.state()
    f_tol = g.w.debug_forces()
    d_tol, _ = g.density_pressure()
    g.w.precision = _abi.EXACT
    f_ex = g.w.debug_forces()
    d_ex, _ = g.density_pressure()
    o = sims.load_scene(sims.OracleSim(orc.JACOBI, fp64=True), sc)
    o.set_state(st)
    o.w.pass_density()
    d64, _ = o.density_pressure()
    o.w.pass_forces()
    f64 = o.w.forces()
    e_ex_d, e_tol_d = rel_rms(d_ex, d64), rel_rms(d_tol, d64)
    e_ex_f, e_tol_f = rel_rms(f_ex, f64), rel_rms(f_tol, f64)
    print(f"vs FP64: density exact {e_ex_d:.2e} tolerance {e_tol_d:.2e}; force exact {e_ex_f:.2e} "
          f"tolerance {e_tol_f:.2e}")
    assert e_ex_d <= 1e-5 and e_tol_d <= 1e-5
    assert e_ex_f <= 1e-4 and e_tol_f <= 1e-4
    assert e_tol_d <= 10 * e_ex_d + 1e-7
    assert e_tol_f <= 10 * e_ex_f + 1e-6


@pytest.mark.gpu
def test_bit_reproducible_and_staging_invariant():
    sc = scenes.dam_break_4k()
    runs = []
    for stage in (3, 3, 0, 1, 2, 4, 5, 6):
        g = _gpu(sc, stage=stage)
        g.step(sc.dt, 150)
        runs.append(g.state())
        g.w.close()
    for r in runs[1:]:
        assert np.array_equal(r.view(np.uint32), runs[0].view(np.uint32))


@pytest.mark.gpu
def test_trajectory_close_to_exact_mode():
    """200 steps of the 4k dam break: positions stay within a small fraction
    of the spacing of the exact run's, the front and the kinetic energy
    agree closely."""
    sc = scenes.dam_break_4k()
    a = _gpu(sc, tolerance=False)
    b = _gpu(sc)
    a.step(sc.dt, 200)
    b.step(sc.dt, 200)
    sa, sb = a.state(), b.state()
    spacing = 0.01
    assert np.abs(sa[:, :2] - sb[:, :2]).max() < 0.05 * spacing
    ke = lambda s: float((s[:, 2] ** 2 + s[:, 3] ** 2).sum())  # noqa: E731
    assert abs(ke(sa) - ke(sb)) <= 1e-3 * ke(sa)
    assert abs(sa[:, 0].max() - sb[:, 0].max()) < 0.01 * spacing


@pytest.mark.gpu
def test_full_size_step_within_tolerance():
    """The 1,048,576-particle dam break: after 5 steps, density and force
    from identical state within the tolerances, on the oracle's Jacobi pass."""
    sc = scenes.dam_break_1m()
    g = _gpu(sc)
    g.step(sc.dt, 5)
    st = g.state()
    f_gpu = g.w.debug_forces()
    d_gpu, p_gpu = g.density_pressure()
    o = sims.load_scene(sims.OracleSim(orc.JACOBI), sc)
    o.set_state(st)
    o.w.pass_density()
    d_o, p_o = o.density_pressure()
    o.w.pass_forces()
    f_o = o.w.forces()
    assert rel_rms(d_gpu, d_o) <= 1e-5
    assert rel_rms(f_gpu, f_o) <= 1e-4
    check_pressure(sc.config, d_gpu, p_gpu, d_o, p_o)


@pytest.mark.gpu
def test_batch_scenes_equal_each_world_alone():
    """A batch in tolerance mode: every scene bit for bit equal to its world
    stepped alone in tolerance mode (the reassociated arithmetic is per
    particle; block and staging windows may span scenes without effect)."""
    from phi_eng_b200 import batch
    from phi_eng_b200.world import world_from_scene

    scs = batch.batched_scenes(12, n_min=256, n_max=4096)
    dt = scs[0].dt
    b = batch.Batch.from_scenes(scs)
    b.world.precision = _abi.TOLERANCE
    b.step(dt, 40)
    for k, sc in enumerate(scs):
        w = world_from_scene(sc)
        w.precision = _abi.TOLERANCE
        w.step_n(dt, 40)
        assert np.array_equal(b.scene_particles(k).view(np.uint32), w.fluid.particles.view(np.uint32)), k
        w.close()
    b.close()
