"""GPU vs oracle parity, through the C ABI (libphieng_sph.so).

Bars:
  * bucket keys, sort order, cell membership, neighbour lists: exact;
  * density and force from identical state: bit-exact against the oracle
    (the reference's density and force passes read only pre-step state, so
    both orders agree); checked against the stated tolerances as well
    (density 1e-5, force 1e-4 relative to RMS);
  * a whole substep and a trajectory: bit-exact against the oracle's Jacobi
    integrate. Against the reference's in-place order the integrate differs
    by design (a parallel update reads pre-update neighbours); that
    difference is bounded separately.
Floating-point values are compared with ``==`` (so -0.0 == +0.0).
"""
import numpy as np
import pytest

import sims
from oracle import oracle as orc
from phi_eng_b200 import scenes

pytestmark = pytest.mark.gpu


def rel_rms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    rms = np.sqrt((b ** 2).mean())
    return float(np.sqrt(((a - b) ** 2).mean()) / max(rms, 1e-30))


def pair(scene, mode=orc.JACOBI, fp64=False):
    g = sims.load_scene(sims.make("gpu"), scene)
    o = sims.load_scene(sims.OracleSim(mode, fp64=fp64), scene)
    return g, o


def expected_keys(world, xy, h):
    st = world.status()
    W, H = 1 << st.grid_log2_w, 1 << st.grid_log2_h
    q = np.floor(xy.astype(np.float32) / np.float32(h))
    cx = q[:, 0].astype(np.int64)
    cy = q[:, 1].astype(np.int64)
    bx = (cx - st.grid_cx0) & (W - 1)
    by = (cy - st.grid_cy0) & (H - 1)
    return (by * W + bx).astype(np.uint32)


SMALL_SCENES = {
    "tank_8x12": scenes.reference_tank,
    "dam_break_4k": scenes.dam_break_4k,
    "dam_break_128x128": lambda: scenes.dam_break_scaled(128, 128),
}


@pytest.mark.parametrize("name", list(SMALL_SCENES))
def test_sorted_order_and_membership(name):
    sc = SMALL_SCENES[name]()
    g, o = pair(sc)
    ids, keys = g.w.debug_sorted()
    exp = expected_keys(g.w, sc.xy, sc.config.smoothing_length)
    order = np.lexsort((np.arange(sc.n), exp))
    assert np.array_equal(ids, order)
    assert np.array_equal(keys, exp[ids])
    # each bucket holds exactly the oracle's cell list (ascending ids)
    cx, cy = o.w.cells()
    cells = {}
    for i in range(sc.n):
        cells.setdefault((int(cx[i]), int(cy[i])), []).append(i)
    bounds = np.flatnonzero(np.diff(keys.astype(np.int64))) + 1
    groups = np.split(ids, bounds)
    got = sorted(tuple(gr.tolist()) for gr in groups)
    want = sorted(tuple(v) for v in cells.values())
    assert got == want


@pytest.mark.parametrize("name", list(SMALL_SCENES))
def test_neighbor_lists_exact(name):
    sc = SMALL_SCENES[name]()
    g, o = pair(sc)
    gc, gl = g.w.debug_neighbors(64)
    oc, ol = o.w.all_neighbors(64)
    assert np.array_equal(gc, oc)
    assert gc.max() <= 64
    for i in range(sc.n):
        k = int(oc[i])
        assert np.array_equal(gl[i, :k], ol[i, :k]), i


def _advance_identical(sc, steps):
    """Run the GPU `steps` steps, then load that state into a fresh oracle."""
    g = sims.load_scene(sims.make("gpu"), sc)
    g.step(sc.dt, steps)
    st = g.state()
    o = sims.load_scene(sims.OracleSim(orc.JACOBI), sc)
    o.set_state(st)
    return g, o, st


@pytest.mark.parametrize("name,steps", [("tank_8x12", 30), ("dam_break_4k", 200), ("dam_break_128x128", 100)])
def test_density_force_identical_state(name, steps):
    sc = SMALL_SCENES[name]()
    g, o, _ = _advance_identical(sc, steps)
    f_gpu = g.w.debug_forces()
    d_gpu, p_gpu = g.density_pressure()
    o.w.pass_density()
    d_o, p_o = o.density_pressure()
    o.w.pass_forces()
    f_o = o.w.forces()
    assert rel_rms(d_gpu, d_o) <= 1e-5  # the stated tolerances
    assert rel_rms(p_gpu, p_o) <= 1e-5
    assert rel_rms(f_gpu, f_o) <= 1e-4
    assert np.array_equal(d_gpu, d_o)  # and bit-exact
    assert np.array_equal(p_gpu, p_o)
    assert np.array_equal(f_gpu, f_o)


def test_pressure_vs_platform_powf():
    """The reference evaluates the Tait power with the platform powf
    (fluid.rs:295); glibc's is one ulp off the correctly rounded power on
    ~0.07% of inputs. Against an oracle that calls powf the GPU stays within
    the stated tolerances."""
    sc = scenes.dam_break_4k()
    g = sims.load_scene(sims.make("gpu"), sc)
    g.step(sc.dt, 200)
    st = g.state()
    f_gpu = g.w.debug_forces()
    d_gpu, p_gpu = g.density_pressure()
    o = sims.load_scene(sims.OracleSim(orc.JACOBI, libm_pow=True), sc)
    o.set_state(st)
    o.w.pass_density()
    d_o, p_o = o.density_pressure()
    o.w.pass_forces()
    f_o = o.w.forces()
    assert np.array_equal(d_gpu, d_o)
    assert rel_rms(p_gpu, p_o) <= 1e-5
    assert (p_gpu != p_o).mean() <= 2e-3
    assert rel_rms(f_gpu, f_o) <= 1e-4


@pytest.mark.parametrize("name", list(SMALL_SCENES))
def test_one_substep_bit_exact_jacobi(name):
    sc = SMALL_SCENES[name]()
    g, o = pair(sc)
    g.step(sc.dt)
    o.step(sc.dt)
    assert np.array_equal(g.state(), o.state())
    dg, pg = g.density_pressure()
    do, po = o.density_pressure()
    assert np.array_equal(dg, do)


def test_trajectory_bit_exact_jacobi_4k():
    sc = scenes.dam_break_4k()
    g, o = pair(sc)
    for k in range(4):
        g.step(sc.dt, 50)
        o.step(sc.dt, 50)
        assert np.array_equal(g.state(), o.state()), f"after {(k + 1) * 50} steps"


def test_trajectory_bit_exact_jacobi_reference_tank():
    sc = scenes.reference_tank()
    g, o = pair(sc)
    for k in range(6):
        g.step(sc.dt, 100)
        o.step(sc.dt, 100)
        assert np.array_equal(g.state(), o.state()), f"after {(k + 1) * 100} steps"


def test_vs_reference_order_one_step():
    """One substep from identical state against the reference's in-place
    sweep: the GPU equals the oracle's Jacobi order bit for bit, and the
    in-place order moves no particle by more than the step's largest
    displacement."""
    sc = scenes.dam_break_4k()
    g, o = pair(sc, mode=orc.REF_SEQ)
    g.step(sc.dt)
    o.step(sc.dt)
    oj = sims.load_scene(sims.OracleSim(orc.JACOBI), sc)
    oj.step(sc.dt)
    gs, os_, js = g.state(), o.state(), oj.state()
    assert np.array_equal(gs, js)
    disp = np.abs(os_[:, :2].astype(np.float64) - sc.xy).max()
    assert np.abs(gs[:, :2].astype(np.float64) - os_[:, :2]).max() <= disp


def test_vs_reference_order_trajectory():
    """The dam break on the GPU (Jacobi reads) against the reference's
    in-place order: the front (max x, the reference's collapse reach,
    fluid_dam.rs:50) agrees within 3% over the 600 steps before it reaches
    the far wall, and the kinetic energy within 25%."""
    sc = scenes.dam_break_4k()
    g, o = pair(sc, mode=orc.REF_SEQ)
    m = sc.config.particle_mass
    for k in range(6):
        g.step(sc.dt, 100)
        o.step(sc.dt, 100)
        gs, os_ = g.state().astype(np.float64), o.state().astype(np.float64)
        front_g, front_o = gs[:, 0].max(), os_[:, 0].max()
        assert abs(front_g - front_o) <= 0.03 * front_o, (k, front_g, front_o)
        ke_g = 0.5 * m * (gs[:, 2:] ** 2).sum()
        ke_o = 0.5 * m * (os_[:, 2:] ** 2).sum()
        assert abs(ke_g - ke_o) <= 0.25 * ke_o, (k, ke_g, ke_o)


def test_fp64_error_statement():
    """f32 error of the GPU path (== the oracle's f32 path) against the FP64
    recompute of one step from the same state."""
    sc = scenes.dam_break_4k()
    g, o, st = _advance_identical(sc, 200)
    f_gpu = g.w.debug_forces()
    d_gpu, _ = g.density_pressure()
    o64 = sims.load_scene(sims.OracleSim(orc.JACOBI, fp64=True), sc)
    o64.set_state(st)
    o64.w.pass_density()
    d64, _ = o64.density_pressure()
    o64.w.pass_forces()
    f64 = o64.w.forces()
    e_d = rel_rms(d_gpu, d64)
    e_f = rel_rms(f_gpu, f64)
    print(f"f32 vs fp64: density rel-RMS {e_d:.2e}, force rel-RMS {e_f:.2e}")
    assert e_d < 1e-6
    assert e_f < 1e-4


def test_run_to_run_bit_identical():
    sc = scenes.dam_break_4k()
    outs = []
    for _ in range(2):
        g = sims.load_scene(sims.make("gpu"), sc)
        g.step(sc.dt, 300)
        outs.append(g.state())
    assert np.array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32))


# ---- optional branches (AV, cohesion, wall friction, CFL, phases) ----
def _unit_scene(cfg_mut, grav=(0.0, -9.81), nx=12, ny=10):
    sc = scenes.reference_tank(nx, ny)
    c = sc.config
    cfg_mut(c)
    sc.config = c
    sc.gravity = grav
    return sc


@pytest.mark.parametrize("label", ["av_cohesion_tait", "friction", "cfl", "no_visc"])
def test_optional_branches_bit_exact(label):
    def mut(c):
        if label == "av_cohesion_tait":
            c.gamma = 7.0
            c.stiffness = 15.0
            c.artificial_viscosity = 1.0
            c.surface_tension = 0.5
        elif label == "friction":
            c.wall_friction = 0.7
        elif label == "cfl":
            c.gamma = 7.0
            c.stiffness = 200.0
            c.cfl = 0.4
            c.max_substeps = 8
        elif label == "no_visc":
            c.viscosity = 0.0

    sc = _unit_scene(mut)
    g, o = pair(sc)
    for _ in range(3):
        g.step(sc.dt, 40)
        o.step(sc.dt, 40)
        assert np.array_equal(g.state(), o.state())


def test_two_phase_bit_exact():
    sc = scenes.reference_tank(18, 8)
    c = sc.config
    c.phase_count = 2
    for k, v in enumerate([2.0, 1.0, 1.0, 1.0]):
        c.phase_rest_density[k] = v
    for k, v in enumerate([0.125, 0.0625, 0.0625, 0.0625]):
        c.phase_mass[k] = v
    sc.config = c
    sc.phases = (np.arange(sc.n) % 3 == 0).astype(np.uint8)
    g, o = pair(sc)
    g.step(sc.dt, 100)
    o.step(sc.dt, 100)
    assert np.array_equal(g.state(), o.state())


def test_circle_walls_bit_exact():
    sc = scenes.reference_tank()
    sc.circles = [(1.0, 1.5, 0.4), (3.0, 0.5, 0.3)]
    g, o = pair(sc)
    g.step(sc.dt, 200)
    o.step(sc.dt, 200)
    assert np.array_equal(g.state(), o.state())


# ---- full size ----
def test_full_size_1m_one_step_bit_exact():
    """The 1,048,576-particle workload: one step from the initial lattice is
    bit-exact against the oracle's Jacobi order (density, pressure, state)."""
    sc = scenes.dam_break_1m()
    g, o = pair(sc)
    g.step(sc.dt)
    o.step(sc.dt)
    assert np.array_equal(g.state(), o.state())
    dg, pg = g.density_pressure()
    do, po = o.density_pressure()
    assert np.array_equal(dg, do) and np.array_equal(pg, po)


def test_full_size_1m_properties():
    """20 steps at full size: finite, contained, particle count kept, keys
    sorted, run-to-run bit-identical."""
    sc = scenes.dam_break_1m()
    runs = []
    for _ in range(2):
        g = sims.load_scene(sims.make("gpu"), sc)
        g.step(sc.dt, 20)
        runs.append(g.state())
        ids, keys = g.w.debug_sorted()
        assert (np.diff(keys.astype(np.int64)) >= 0).all()
        assert np.array_equal(np.sort(ids), np.arange(sc.n))
    s = runs[0]
    assert np.isfinite(s).all() and s.shape[0] == sc.n
    assert (s[:, 0] >= 0).all() and (s[:, 0] <= 10.0).all() and (s[:, 1] >= 0).all()
    assert np.array_equal(runs[0].view(np.uint32), runs[1].view(np.uint32))


# ---- edge cases ----
def test_aliased_buckets_and_wrap_seams():
    """Two clusters far apart force a bucket grid smaller than the particle
    span, so distinct cells share buckets and rows cross the wrap seam;
    neighbour lists and the step stay exact."""
    a = scenes.jittered_lattice(40, 30, 0.01, seed=1)
    b = scenes.jittered_lattice(40, 30, 0.01, seed=2, x0=37.3, y0=-11.7)
    sc = scenes.Scene(name="clusters", boxes=[], xy=np.concatenate([a, b]), config=scenes.si_config(0.01),
                      dt=scenes.fine_dt(scenes.si_config(0.01)))
    g, o = pair(sc)
    st = g.w.status()
    gc, gl = g.w.debug_neighbors(64)
    st = g.w.status()
    span_cells = (37.3 + 0.4) / 0.02
    assert (1 << st.grid_log2_w) < span_cells  # the grid really aliases
    oc, ol = o.w.all_neighbors(64)
    assert np.array_equal(gc, oc)
    for i in range(sc.n):
        assert np.array_equal(gl[i, :oc[i]], ol[i, :oc[i]])
    g.step(sc.dt, 30)
    o.step(sc.dt, 30)
    assert np.array_equal(g.state(), o.state())


def test_negative_coordinates_and_coincident_particles():
    xy = scenes.jittered_lattice(20, 20, 0.01, x0=-0.37, y0=-0.21)
    xy = np.concatenate([xy, xy[:5], xy[:5]])  # exact duplicates: r = 0 pairs
    sc = scenes.Scene(name="coincident", boxes=[(-0.1, -0.3, 0.5, 0.05)], xy=xy, config=scenes.si_config(0.01),
                      dt=scenes.fine_dt(scenes.si_config(0.01)))
    g, o = pair(sc)
    g.step(sc.dt, 20)
    o.step(sc.dt, 20)
    assert np.array_equal(g.state(), o.state())


def test_single_particle_free_fall():
    sc = scenes.Scene(name="one", boxes=[], xy=np.array([[0.3, 0.7]], np.float32), config=scenes.si_config(0.01),
                      dt=1e-3)
    g, o = pair(sc)
    g.step(sc.dt, 10)
    o.step(sc.dt, 10)
    assert np.array_equal(g.state(), o.state())
    assert g.state()[0, 3] < 0


def test_step_guards_and_clock():
    from phi_eng_b200.world import World2

    w = World2()
    w.step(0.05)  # empty world: clock advances, nothing else
    assert abs(w.time - 0.05) < 1e-7
    w.fluid.add_particles(np.array([[0.0, 0.0]], np.float32))
    w.step(10.0)  # clamped to 1/15 s (ffi.rs:80)
    assert abs(w.time - (0.05 + 1.0 / 15.0)) < 1e-6
    assert w.status().substeps == 1
    c = w.fluid.config
    c.enabled = 0
    w.fluid.config = c
    before = w.fluid.particles.copy()
    w.step(0.01)  # disabled fluid: no substep (fluid.rs:550)
    assert w.status().substeps == 1
    assert np.array_equal(before, w.fluid.particles)


def test_unsupported_feature_fails_cleanly():
    """The fluid phase with the engine's bodies (phieng_sph_step_fluid) does
    not take adaptive resolution (the world step does): it reports
    PHIENG_SPH_E_UNSUPPORTED and leaves the particles unchanged."""
    from phi_eng_b200._abi import PhiengBody2
    from phi_eng_b200.world import World2

    w = World2()
    w.fluid.add_particles(np.array([[0.0, 0.0], [0.1, 0.0]], np.float32))
    c = w.fluid.config
    c.adaptive_resolution = 1
    w.fluid.config = c
    before = w.fluid.particles.copy()
    assert w._lib.phieng_sph_step_fluid(w._h, (PhiengBody2 * 1)(), 0, 0.01) == 0
    assert w.status().error == 3  # PHIENG_SPH_E_UNSUPPORTED
    assert np.array_equal(before, w.fluid.particles)


def test_add_and_clear_between_steps():
    sc = scenes.dam_break_4k()
    g, o = pair(sc)
    g.step(sc.dt, 10)
    o.step(sc.dt, 10)
    extra = scenes.jittered_lattice(8, 8, 0.01, seed=9, x0=0.8, y0=0.3)
    assert g.add_particles(extra) == 64 and o.add_particles(extra) == 64
    g.step(sc.dt, 10)
    o.step(sc.dt, 10)
    assert np.array_equal(g.state(), o.state())
    g.w.fluid.clear()
    assert g.count == 0
    g.step(sc.dt)
    assert g.count == 0


@pytest.mark.parametrize("log2", [(2, 2), (3, 4), (5, 3)])
def test_forced_tiny_grid_exact(log2):
    """A bucket grid far smaller than the fluid: every bucket aliases many
    cells and a large share of particles sit on the wrap seam (the K6
    fallback walk). Neighbour lists, the sort and a trajectory stay exact."""
    sc = scenes.dam_break_4k()
    g, o = pair(sc)
    g.w.set_grid(log2[0], log2[1], -3, 5)
    ids, keys = g.w.debug_sorted()
    exp = expected_keys(g.w, sc.xy, sc.config.smoothing_length)
    assert np.array_equal(ids, np.lexsort((np.arange(sc.n), exp)))
    gc, gl = g.w.debug_neighbors(64)
    oc, ol = o.w.all_neighbors(64)
    assert np.array_equal(gc, oc)
    for i in range(0, sc.n, 7):
        assert np.array_equal(gl[i, :oc[i]], ol[i, :oc[i]])
    g.step(sc.dt, 40)
    o.step(sc.dt, 40)
    assert np.array_equal(g.state(), o.state())


def test_front_metrics_async_equal_sync():
    """phieng_sph_front_metrics_async: the metric of every step copied into
    its own page-locked slot without waiting equals the synchronous read of
    the same state."""
    import torch

    sc = scenes.dam_break_4k()
    a = sims.load_scene(sims.make("gpu"), sc).w
    b = sims.load_scene(sims.make("gpu"), sc).w
    ring = torch.zeros((6, 2), dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    want = []
    for k in range(6):
        a.step(sc.dt)
        a.front_metrics_async(ring[k])
        b.step(sc.dt)
        want.append(b.front_metrics())
    a.sync()
    got = [a.decode_front_metrics(ring[k]) for k in range(6)]
    assert got == want
