"""Two-way coupling of the 3D fluid with rigid bodies: FluidState3::step_fluid
with the engine's bodies (crates/dynamics/src/fluid3.rs:591-607, 990-1213)
through phieng_sph3_step_fluid / phieng_sph3_step_fluid_hull.

The rigid side of World3::step (gravity, contacts, integration) belongs to
the host engine; a small host loop stands in for it here (kick, fluid phase,
drift with a quaternion update), identical for the oracle and the GPU. CPU
tests check the oracle's rotation arithmetic, buoyancy samples, a
hand-computed reaction and the reference's own floating-box test
(fluid3.rs:1349-1396); GPU tests check the CUDA path bit for bit against the
oracle (Jacobi order): particle state and every body's velocity, angular
velocity and sleep flag after each step, with rotated boxes, capsules,
spheres and hulls, with and without wall friction, through CFL substeps,
wind and turbulence.
"""
import ctypes as C
import math

import numpy as np
import pytest

from oracle import oracle as orc
from oracle.oracle import JACOBI, REF_SEQ
from phi_eng_b200 import _abi
from phi_eng_b200._abi import PhiengBody3, default_config
from test_fluid3 import TANK, assert_bit_equal, bits, has_gpu, lattice, make_gpu, make_oracle

f32 = np.float32
G = f32(-9.81)
DT = 1 / 60


def quat(axis, angle):
    a = np.asarray(axis, np.float64)
    a = a / np.linalg.norm(a)
    s = math.sin(angle / 2)
    return tuple(float(f32(v)) for v in (a[0] * s, a[1] * s, a[2] * s, math.cos(angle / 2)))


def static3(shape, pos, ext, rot=(0.0, 0.0, 0.0, 1.0)):
    b = PhiengBody3()
    b.shape_tag = shape
    b.a, b.b, b.c = ext
    b.px, b.py, b.pz = pos
    b.qx, b.qy, b.qz, b.qw = rot
    b.is_static = 1
    return b


def dynamic3(shape, pos, ext, inv_mass, inv_inertia, rot=(0.0, 0.0, 0.0, 1.0)):
    b = static3(shape, pos, ext, rot)
    b.is_static = 0
    b.inv_mass = inv_mass
    for k in range(3):
        b.inv_inertia[4 * k] = inv_inertia[k]
    return b


def dynamic_box3(pos, he, density, rot=(0.0, 0.0, 0.0, 1.0)):
    """mass_properties_3d for Shape3::Box (body.rs:819-828), inverse 1 / I per axis."""
    w, h, d = (f32(v) * f32(2) for v in he)
    m = (w * h * d) * f32(density)
    diag = (m * (h * h + d * d) / f32(12), m * (w * w + d * d) / f32(12), m * (w * w + h * h) / f32(12))
    return dynamic3(_abi.SHAPE3_BOX, pos, he, f32(1) / m, [f32(1) / x for x in diag], rot)


def dynamic_sphere3(pos, r, density):
    r = f32(r)
    m = ((f32(4.0) / f32(3.0)) * f32(math.pi) * r * r * r) * f32(density)
    i = f32(0.4) * m * r * r
    return dynamic3(_abi.SHAPE3_SPHERE, pos, (r, 0.0, 0.0), f32(1) / m, [f32(1) / i] * 3)


def tank_bodies():
    return [static3(shape, pos, ext) for shape, pos, ext in TANK]


def body_list(bodies):
    arr = (PhiengBody3 * len(bodies))()
    for k, b in enumerate(bodies):
        arr[k] = b
    return arr


def copy_bodies(arr):
    out = (PhiengBody3 * len(arr))()
    C.memmove(out, arr, C.sizeof(out))
    return out


def body_bits(arr):
    return np.array([[b.vx, b.vy, b.vz, b.wx, b.wy, b.wz, b.px, b.py, b.pz, b.qx, b.qy, b.qz, b.qw] for b in arr],
                    np.float32).view(np.uint32)


def kick(arr, dt):
    for b in arr:
        if not b.is_static:
            b.vy = f32(b.vy) + G * f32(dt)


def drift(arr, dt):
    """Position by velocity; rotation q + (dt / 2) (w, 0) q, renormalised (f32)."""
    h = f32(0.5) * f32(dt)
    for b in arr:
        if b.is_static:
            continue
        b.px = f32(b.px) + f32(b.vx) * f32(dt)
        b.py = f32(b.py) + f32(b.vy) * f32(dt)
        b.pz = f32(b.pz) + f32(b.vz) * f32(dt)
        wx, wy, wz = f32(b.wx), f32(b.wy), f32(b.wz)
        x, y, z, w = f32(b.qx), f32(b.qy), f32(b.qz), f32(b.qw)
        dx = wx * w + (wy * z - wz * y)
        dy = wy * w + (wz * x - wx * z)
        dz = wz * w + (wx * y - wy * x)
        dw = -(wx * x + wy * y + wz * z)
        x, y, z, w = x + h * dx, y + h * dy, z + h * dz, w + h * dw
        n = f32(np.sqrt(f32(x * x + y * y + z * z + w * w)))
        b.qx, b.qy, b.qz, b.qw = x / n, y / n, z / n, w / n


# ---- CPU: the oracle's pieces -------------------------------------------------

def test_qrot_rotates():
    v = np.array([0.3, -1.2, 2.5], np.float32)
    assert (orc.qrot3((0.0, 0.0, 0.0, 1.0), v) == v).all()  # identity: unchanged
    q = quat((0, 0, 1), math.pi / 2)
    np.testing.assert_allclose(orc.qrot3(q, [1, 0, 0]), [0, 1, 0], atol=1e-6)
    rng = np.random.default_rng(1)
    for _ in range(20):
        q = quat(rng.standard_normal(3), float(rng.uniform(-3, 3)))
        u = orc.qrot3(q, v)
        assert abs(np.linalg.norm(u) - np.linalg.norm(v)) < 1e-5
        back = orc.qrot3((-q[0], -q[1], -q[2], q[3]), u)  # the conjugate undoes it
        np.testing.assert_allclose(back, v, atol=1e-5)


def test_world_inv_inertia_rotates_the_tensor():
    ii = np.diag([1.0, 2.0, 3.0]).astype(np.float32).T.ravel()
    assert (orc.world_inv_inertia3((0.0, 0.0, 0.0, 1.0), ii) == ii).all()
    q = quat((0, 0, 1), math.pi / 2)  # swaps x and y
    np.testing.assert_allclose(orc.world_inv_inertia3(q, ii).reshape(3, 3).T, np.diag([2.0, 1.0, 3.0]), atol=1e-6)
    q = quat((1, 2, 3), 0.7)
    r = np.array([orc.qrot3(q, e) for e in np.eye(3)]).T  # columns: the rotated axes
    np.testing.assert_allclose(orc.world_inv_inertia3(q, ii).reshape(3, 3).T, r @ np.diag([1, 2, 3]) @ r.T,
                               atol=1e-5)


def test_surface_samples_cover_the_surface():
    """fluid3.rs:371-467: counts, total area, unit normals; box points all at
    each face's -he coordinate, as the reference writes them."""
    q = quat((1, 1, 0), 0.4)
    s = orc.surface_samples3(static3(_abi.SHAPE3_SPHERE, (1.0, 2.0, 3.0), (0.5, 0, 0), q))
    assert s.shape == (14, 7)
    np.testing.assert_allclose(s[:, 6].sum(), 4 * math.pi * 0.25, rtol=1e-6)
    np.testing.assert_allclose(np.linalg.norm(s[:, :3] - [1, 2, 3], axis=1), 0.5, rtol=1e-5)
    np.testing.assert_allclose(np.linalg.norm(s[:, 3:6], axis=1), 1.0, rtol=1e-5)
    b = orc.surface_samples3(static3(_abi.SHAPE3_BOX, (0.0, 0.0, 0.0), (0.3, 0.2, 0.1)))
    assert b.shape == (24, 7)
    np.testing.assert_allclose(b[:, 6].sum(), 8 * (0.06 + 0.02 + 0.03), rtol=1e-6)
    assert (b[:8, 1] == f32(-0.2)).all() and (b[8:16, 0] == f32(-0.3)).all() and (b[16:, 2] == f32(-0.1)).all()
    c = orc.surface_samples3(static3(_abi.SHAPE3_CAPSULE, (0.0, 0.0, 0.0), (0.2, 0.5, 0.0)))
    assert c.shape == (18, 7)
    np.testing.assert_allclose(c[:, 6].sum(), 4 * math.pi * 0.2 * 0.5 + 4 * math.pi * 0.04, rtol=1e-6)
    hull = static3(_abi.SHAPE3_HULL, (0.0, 0.0, 0.0), (0.0, 0.0, 0.0))
    assert orc.surface_samples3(hull).shape == (0, 7)  # impulse-coupled only


def one_particle_world(vx):
    cfg = default_config()
    o = orc.OracleWorld3()
    o.set_config(cfg)
    o.set_gravity(0.0, 0.0, 0.0)
    o.add_particles(np.array([[1.02, 0.0, 0.0]], np.float32))
    o.set_state(np.array([[1.02, 0.0, 0.0, vx, 0.0, 0.0]], np.float32))
    return o, cfg


def test_oracle_reaction_hand_computed():
    """One particle driven into a dynamic unit sphere: the push-out, the
    removed approach velocity and the impulse n (vn m) on the body
    (fluid3.rs:1156-1166, body.rs:1349-1361; no torque: the contact point lies
    on the line through the centre)."""
    o, cfg = one_particle_world(-2.0)
    arr = body_list([dynamic_sphere3((0.0, 0.0, 0.0), 1.0, 1.0)])
    o.step_fluid(arr, f32(DT), REF_SEQ)
    x = f32(1.02) + f32(-2.0) * f32(DT)  # no neighbours, no gravity: v unchanged by the integrate
    pr = f32(cfg.particle_radius)
    assert x < f32(1.0) + pr
    vn = f32(-2.0)
    m = f32(cfg.particle_mass)
    assert arr[0].vx == f32(f32(vn * m) * f32(arr[0].inv_mass))
    assert arr[0].vy == 0.0 and arr[0].vz == 0.0 and (arr[0].wx, arr[0].wy, arr[0].wz) == (0.0, 0.0, 0.0)
    s = o.state()[0]
    assert s[0] == f32(f32(1.0) + pr) and s[3] == 0.0  # pushed to the surface, approach removed
    # moving away: contact without reaction
    o, cfg = one_particle_world(+2.0)
    o.set_state(np.array([[0.95, 0.0, 0.0, 2.0, 0.0, 0.0]], np.float32))
    arr = body_list([dynamic_sphere3((0.0, 0.0, 0.0), 1.0, 1.0)])
    o.step_fluid(arr, f32(DT), REF_SEQ)
    assert arr[0].vx == 0.0


def test_oracle_box_floats():
    """fluid3.rs:1349-1396 on the oracle: still water in a pool inside the
    tank, then a half-density box set just above the surface stays afloat."""
    pool = [(_abi.SHAPE3_BOX, p, e) for p, e in [
        ((0.375, 1.0, 1.5), (0.125, 2.0, 1.25)), ((2.625, 1.0, 1.5), (0.125, 2.0, 1.25)),
        ((1.5, 1.0, 0.375), (1.0, 2.0, 0.125)), ((1.5, 1.0, 2.625), (1.0, 2.0, 0.125))]]
    o = make_oracle(lattice((0.75, -0.5, 0.75), 6, 8, 6, 0.25), bodies=TANK + pool)
    for _ in range(200):
        o.step(DT, REF_SEQ)
    arr = body_list([static3(*b) for b in TANK + pool] + [dynamic_box3((1.5, 1.4, 1.5), (0.3, 0.3, 0.3), 0.5)])
    for frame in range(400):
        kick(arr, DT)
        o.step_fluid(arr, f32(DT), REF_SEQ)
        drift(arr, DT)
        if frame % 100 == 0:
            assert np.isfinite(o.state()).all()
    y = arr[-1].py
    assert 0.0 < y < 2.0, y
    assert np.isfinite(o.state()).all()


def test_step_fluid3_arguments():
    lib = _abi.load()
    w = lib.phieng_world3_new()
    arr = body_list(tank_bodies())
    assert lib.phieng_sph3_step_fluid(None, arr, len(arr), f32(DT)) == 0
    assert lib.phieng_sph3_step_fluid(w, None, 1, f32(DT)) == 0
    bad = copy_bodies(arr)
    bad[0].shape_tag = 7
    assert lib.phieng_sph3_step_fluid(w, bad, len(bad), f32(DT)) == 0
    bad = copy_bodies(arr)
    bad[1].qw = 0.9  # not a unit quaternion
    assert lib.phieng_sph3_step_fluid(w, bad, len(bad), f32(DT)) == 0
    bad = copy_bodies(arr)
    bad[2].inv_inertia[4] = float("nan")
    assert lib.phieng_sph3_step_fluid(w, bad, len(bad), f32(DT)) == 0
    hull = body_list([static3(_abi.SHAPE3_HULL, (0.0, 0.0, 0.0), (0.0, 0.0, 0.0))])
    assert lib.phieng_sph3_step_fluid(w, hull, 1, f32(DT)) == 0  # hulls only through the hull entry
    xyz = np.zeros((4, 3), np.float32)
    U = C.POINTER(C.c_uint32)
    first, count = np.array([2], np.uint32), np.array([3], np.uint32)  # past the 4 vertices
    F = C.POINTER(C.c_float)
    assert lib.phieng_sph3_step_fluid_hull(w, hull, 1, xyz.ctypes.data_as(F), first.ctypes.data_as(U),
                                           count.ctypes.data_as(U), 4, f32(DT)) == 0
    xyz[1, 0] = float("inf")
    first[0] = 0
    assert lib.phieng_sph3_step_fluid_hull(w, hull, 1, xyz.ctypes.data_as(F), first.ctypes.data_as(U),
                                           count.ctypes.data_as(U), 4, f32(DT)) == 0
    # no particles: the reference's early return, nothing touched
    assert lib.phieng_sph3_step_fluid(w, arr, len(arr), f32(DT)) == 1
    lib.phieng_world3_free(w)


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_step_fluid3_without_device_fails_loudly():
    lib = _abi.load()
    w = lib.phieng_world3_new()
    p = lattice((0.0, 0.0, 0.0), 3, 3, 3, 0.25)
    assert lib.phieng_world3_fluid_add(w, p.ctypes.data_as(C.POINTER(C.c_float)), len(p)) == len(p)
    arr = body_list(tank_bodies())
    assert lib.phieng_sph3_step_fluid(w, arr, len(arr), f32(DT)) == 0
    st = _abi.PhiengSphStatus()
    lib.phieng_sph3_status(w, C.byref(st))
    assert st.error == _abi.E_NO_DEVICE
    lib.phieng_world3_free(w)


# ---- GPU parity -----------------------------------------------------------------

def set_gpu_ambient(w, wind=(0.0, 0.0, 0.0), turb=None):
    a = _abi.AmbientConfig3Ffi()
    assert w._lib.phieng_world3_get_ambient_config(w._h, C.byref(a)) == 1
    a.wind_x, a.wind_y, a.wind_z = wind
    if turb:
        a.turbulence_enabled = 1
        a.turbulence_amplitude = turb["amplitude"]
        a.turbulence_frequency = turb.get("frequency", 1.0)
        a.turbulence_seed = turb.get("seed", 0)
        a.turbulence_divergence_free = 1 if turb.get("divergence_free") else 0
    assert w._lib.phieng_world3_set_ambient_config(w._h, C.byref(a)) == 1


def coupled_parity3(cfg, bodies, frames, settle=40, pts=None, wind=None, turb=None, hulls=None):
    pts = lattice((0.0, -0.4, 0.0), 12, 6, 12, 0.25) if pts is None else pts
    o = make_oracle(pts, cfg=cfg)
    w = make_gpu(pts, cfg=cfg)
    if wind or turb:
        set_gpu_ambient(w, wind or (0.0, 0.0, 0.0), turb)
        o.set_wind(*(wind or (0.0, 0.0, 0.0)))
        if turb:
            o.set_turbulence(**turb)
    for _ in range(settle):
        o.step(DT, JACOBI)
        w.step(DT)
    assert_bit_equal(o.state(), w.fluid.particles, "settled state")
    a = body_list(bodies)
    b = copy_bodies(a)
    for f in range(frames):
        kick(a, DT)
        kick(b, DT)
        o.step_fluid(a, f32(DT), JACOBI, hulls)
        w.step_fluid(b, f32(DT), hulls)
        drift(a, DT)
        drift(b, DT)
        # a body that blows up turns NaN on both sides with different NaN
        # bits; say so instead of reporting a bit difference
        assert np.isfinite(body_bits(a).view(np.float32)).all(), f"oracle bodies non-finite at frame {f}"
        assert (body_bits(a) == body_bits(b)).all(), f"bodies differ at frame {f}"
        assert [x.is_sleeping for x in a] == [x.is_sleeping for x in b]
        if f % 10 == 9 or f == frames - 1:
            assert_bit_equal(o.state(), w.fluid.particles, f"frame {f}")
    w.close()
    return a


def floating_bodies3():
    caps = dynamic3(_abi.SHAPE3_CAPSULE, (3.2, 1.3, 1.0), (0.18, 0.3, 0.0), 4.0, (9.0, 14.0, 9.0),
                    quat((1, 0, 0.5), 1.1))
    return tank_bodies() + [
        dynamic_box3((1.2, 1.25, 2.2), (0.35, 0.2, 0.3), 0.5, quat((1, 2, 0.5), 0.4)),
        dynamic_sphere3((2.6, 1.2, 2.8), 0.3, 0.6),
        caps,
        static3(_abi.SHAPE3_BOX, (0.8, 0.0, 0.8), (0.5, 0.15, 0.4), quat((0, 0, 1), 0.5)),  # a tilted ramp
    ]


@pytest.mark.gpu
def test_step_fluid3_statics_equal_world_step():
    """The tank as the call's static bodies (identity rotation) steps the
    fluid exactly as the world's own statics do."""
    pts = lattice((0.0, -0.4, 0.0), 12, 6, 12, 0.25)
    w1, w2 = make_gpu(pts), make_gpu(pts, bodies=[])
    arr = body_list(tank_bodies())
    for _ in range(60):
        w1.step(DT)
        w2.step_fluid(arr, f32(DT))
    assert_bit_equal(w1.fluid.particles, w2.fluid.particles, "statics through the fluid phase")
    w1.close()
    w2.close()


@pytest.mark.gpu
def test_step_fluid3_bit_exact_frictionless():
    # drag 1 instead of the default 4: the buoyancy pass applies the
    # quadratic drag explicitly, sample after sample, and the light box
    # (inverse inertia ~275) spins up without bound under drag 4 (the
    # oracle's box goes to inf at frame 35, as the reference's would)
    c = default_config()
    c.drag = 1.0
    a = coupled_parity3(c, floating_bodies3(), 80)
    assert any(abs(b.wx) + abs(b.wy) + abs(b.wz) > 0 for b in a[5:8])  # the coupling produced torque
    assert any(b.vy != 0 for b in a[5:8])


@pytest.mark.gpu
def test_step_fluid3_bit_exact_friction_and_substeps():
    c = default_config()
    c.wall_friction = 0.5
    c.gamma = 7.0
    c.stiffness = 40.0
    c.cfl = 0.4
    c.max_substeps = 4
    c.drag = 2.0
    bodies = floating_bodies3()
    bodies[-1].vx = 0.3  # a moving static: its velocity enters the no-slip term
    coupled_parity3(c, bodies, 60)


@pytest.mark.gpu
def test_step_fluid3_bit_exact_wind_and_turbulence():
    c = default_config()
    c.drag = 2.0
    coupled_parity3(c, floating_bodies3(), 50, wind=(3.0, -0.5, 1.0),
                    turb=dict(amplitude=3.0, frequency=0.7, seed=11, divergence_free=True))


@pytest.mark.gpu
def test_step_fluid3_bit_exact_hulls():
    """A static rotated hull and a dynamic one (nearest-vertex spheres,
    fluid3.rs:568-585) among the walls, with friction."""
    c = default_config()
    c.wall_friction = 0.3
    rng = np.random.default_rng(7)
    cube = np.array([(x, y, z) for x in (-0.3, 0.3) for y in (-0.3, 0.3) for z in (-0.3, 0.3)], np.float32)
    blob = (rng.standard_normal((40, 3)) * 0.25).astype(np.float32)
    hs = static3(_abi.SHAPE3_HULL, (1.0, 0.2, 1.0), (0, 0, 0), quat((1, 1, 1), 0.6))
    hd = dynamic3(_abi.SHAPE3_HULL, (3.0, 1.3, 3.0), (0, 0, 0), 2.0, (6.0, 6.0, 6.0), quat((0, 1, 0), 0.3))
    bodies = tank_bodies() + [hs, hd]
    xyz = np.concatenate([cube, blob])
    first = np.array([0] * 5 + [0, len(cube)], np.uint32)
    count = np.array([0] * 5 + [len(cube), len(blob)], np.uint32)
    a = coupled_parity3(c, bodies, 60, hulls=(xyz, first, count))
    assert abs(a[6].vx) + abs(a[6].vy) + abs(a[6].vz) > 0  # the dynamic hull took impulses


@pytest.mark.gpu
def test_gpu_box_floats():
    """fluid3.rs:1349-1396 through the GPU fluid phase."""
    pool = [(_abi.SHAPE3_BOX, p, e) for p, e in [
        ((0.375, 1.0, 1.5), (0.125, 2.0, 1.25)), ((2.625, 1.0, 1.5), (0.125, 2.0, 1.25)),
        ((1.5, 1.0, 0.375), (1.0, 2.0, 0.125)), ((1.5, 1.0, 2.625), (1.0, 2.0, 0.125))]]
    w = make_gpu(lattice((0.75, -0.5, 0.75), 6, 8, 6, 0.25), bodies=TANK + pool)
    for _ in range(200):
        w.step(DT)
    arr = body_list([static3(*b) for b in TANK + pool] + [dynamic_box3((1.5, 1.4, 1.5), (0.3, 0.3, 0.3), 0.5)])
    for _ in range(400):
        kick(arr, DT)
        w.step_fluid(arr, f32(DT))
        drift(arr, DT)
    assert 0.0 < arr[-1].py < 2.0
    assert np.isfinite(w.fluid.particles).all()
    w.close()
