"""Two-way coupling with rigid bodies: FluidState2::step_fluid with the engine's
bodies (crates/dynamics/src/fluid.rs:541-557, :1056-1135) through
phieng_sph_step_fluid.

The rigid side of World2::step (gravity kick, contacts, integration) belongs
to the host engine; here a small host loop stands in for it (kick, fluid
phase, drift), identical for the oracle and the GPU. CPU tests run the
oracle against the reference's own floating-box test (fluid.rs:1258-1289)
and hand-computed reactions; GPU tests check the CUDA path bit for bit
against the oracle (Jacobi order): particle state and every body's velocity
after each step, with and without wall friction, through CFL substeps.
"""
import ctypes as C
import math

import numpy as np
import pytest

from oracle.oracle import JACOBI, REF_SEQ, OracleWorld
from phi_eng_b200 import _abi
from phi_eng_b200._abi import PhiengBody2, default_config

F = C.POINTER(C.c_float)
f32 = np.float32


def fp(a):
    return a.ctypes.data_as(F)


def has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


# the reference's 2D test tank (fluid.rs:1150-1170): floor top at y = -0.5,
# inner walls at x = -0.5 and 4.5
TANK = [((2.0, -1.0), (3.0, 0.5)), ((-1.0, 2.0), (0.5, 3.5)), ((5.0, 2.0), (0.5, 3.5))]


def static_box(px, py, hx, hy):
    b = PhiengBody2()
    b.shape_tag = _abi.SHAPE_BOX
    b.a, b.b, b.px, b.py = hx, hy, px, py
    b.xax, b.xay, b.yax, b.yay = 1.0, 0.0, -0.0, 1.0
    b.is_static = 1
    return b


def dynamic_box(px, py, hx, hy, density, angle=0.0):
    """RigidBody2 with Shape2::Box at `density` (body.rs:612-654, :791-797)."""
    b = static_box(px, py, hx, hy)
    b.is_static = 0
    set_angle(b, angle)
    w, h = f32(hx) * f32(2), f32(hy) * f32(2)
    m = (w * h) * f32(density)
    inertia = m * (w * w + h * h) / f32(12)
    b.inv_mass = f32(1) / max(m, f32(1e-6))
    b.inv_inertia = f32(1) / max(inertia, f32(1e-6))
    return b


def dynamic_circle(px, py, r, density):
    b = PhiengBody2()
    b.shape_tag = _abi.SHAPE_CIRCLE
    b.a, b.px, b.py = r, px, py
    b.xax, b.xay, b.yax, b.yay = 1.0, 0.0, -0.0, 1.0
    m = (f32(math.pi) * f32(r) * f32(r)) * f32(density)
    inertia = f32(0.5) * m * f32(r) * f32(r)
    b.inv_mass = f32(1) / m
    b.inv_inertia = f32(1) / inertia
    return b


def set_angle(b, angle):
    c, s = f32(math.cos(angle)), f32(math.sin(angle))
    b.xax, b.xay, b.yax, b.yay = c, s, -s, c


def body_list(bodies):
    arr = (PhiengBody2 * len(bodies))()
    for k, b in enumerate(bodies):
        arr[k] = b
    return arr


def kick(arr, dt, g=-9.81):
    for b in arr:
        if not b.is_static:
            b.vy = f32(b.vy) + f32(g) * f32(dt)


def drift(arr, dt, angles):
    for k, b in enumerate(arr):
        if not b.is_static:
            b.px = f32(b.px) + f32(b.vx) * f32(dt)
            b.py = f32(b.py) + f32(b.vy) * f32(dt)
            angles[k] = f32(angles[k]) + f32(b.w) * f32(dt)
            if b.shape_tag in (_abi.SHAPE_BOX, _abi.SHAPE_POLYGON):
                set_angle(b, float(angles[k]))


def lattice(x0, y0, nx, ny, dx):
    return np.array([(x0 + ix * dx, y0 + iy * dx) for iy in range(ny) for ix in range(nx)], np.float32)


def oracle_world(pts, cfg=None):
    o = OracleWorld()
    if cfg is not None:
        o.set_config(cfg)
    for (px, py), (hx, hy) in TANK:
        o.add_box(px, py, hx, hy)
    o.add_particles(pts)
    return o


def run_oracle(o, arr, frames, dt=1 / 60, mode=REF_SEQ, poly=None):
    angles = [0.0] * len(arr)
    for _ in range(frames):
        kick(arr, dt)
        o.step_fluid(arr, dt, mode, poly)
        drift(arr, dt, angles)


def polygon_body(px, py, verts, dynamic=False, inv_mass=2.0, inv_inertia=6.0, angle=0.0):
    """A Shape2::Polygon body; returns (body, local vertices)."""
    b = PhiengBody2()
    b.shape_tag = _abi.SHAPE_POLYGON
    b.px, b.py = px, py
    set_angle(b, angle)
    b.is_static = 0 if dynamic else 1
    if dynamic:
        b.inv_mass, b.inv_inertia = inv_mass, inv_inertia
    return b, np.asarray(verts, np.float32)


def poly_arrays(entries):
    """(xy, first, count) for phieng_sph_step_fluid_poly from per-body vertex
    arrays (None for non-polygons)."""
    xy, first, count = [], [], []
    for v in entries:
        first.append(sum(len(a) for a in xy))
        count.append(0 if v is None else len(v))
        if v is not None:
            xy.append(v)
    flat = np.concatenate(xy).astype(np.float32) if xy else np.zeros((0, 2), np.float32)
    return np.ascontiguousarray(flat), np.asarray(first, np.uint32), np.asarray(count, np.uint32)


def point_in_poly(x, y, v):
    inside = False
    j = len(v) - 1
    for i in range(len(v)):
        if (v[i][1] > y) != (v[j][1] > y) and x < (v[j][0] - v[i][0]) * (y - v[i][1]) / (v[j][1] - v[i][1]) + v[i][0]:
            inside = not inside
        j = i
    return inside


RAMP = [(-1.0, -0.4), (1.0, -0.4), (-1.0, 0.6)]          # triangle, counter-clockwise
ELL = [(0.0, 0.0), (0.8, 0.0), (0.8, 0.2), (0.2, 0.2), (0.2, 0.7), (0.0, 0.7)]  # concave L
PENTAGON = [(0.25 * math.cos(2 * math.pi * k / 5), 0.25 * math.sin(2 * math.pi * k / 5)) for k in range(5)]


# ---- oracle (CPU) -----------------------------------------------------------

def test_oracle_box_floats():
    """fluid.rs:1258-1289 on the oracle with the host loop above: a
    half-density box set just above still water stays afloat."""
    o = oracle_world(lattice(-0.5, -0.5, 12, 6, 0.25))
    o.steps(1 / 60, 300)
    arr = body_list([static_box(*p, *e) for p, e in TANK] + [dynamic_box(2.0, 1.6, 0.3, 0.3, 0.5)])
    ys = []
    for _ in range(6):
        run_oracle(o, arr, 100)
        ys.append(float(arr[3].py))
        assert np.isfinite(o.state()).all()
    assert all(0.0 < y < 2.0 for y in ys), ys
    assert abs(arr[3].vy) < 1.0


def test_oracle_heavy_box_sinks_light_box_floats():
    """Archimedes: with the same start the denser box ends lower."""
    ends = {}
    for density in (0.3, 3.0):
        o = oracle_world(lattice(-0.5, -0.5, 12, 6, 0.25))
        o.steps(1 / 60, 200)
        arr = body_list([static_box(*p, *e) for p, e in TANK] + [dynamic_box(2.0, 1.2, 0.3, 0.3, density)])
        run_oracle(o, arr, 200)
        ends[density] = float(arr[3].py)
    assert ends[3.0] < ends[0.3] - 0.2, ends


def test_oracle_wind_drifts_floating_body():
    """fluid.rs:1467-1494 on the oracle: a box floating in the settled tank
    drifts downwind under ambient.drag.wind = (3, 0)."""
    o = oracle_world(lattice(-0.5, -0.5, 12, 6, 0.25))
    for _ in range(200):
        o.step(1 / 60, REF_SEQ)
    o.set_wind(3.0, 0.0)
    arr = body_list([static_box(*p, *e) for p, e in TANK] + [dynamic_box(2.0, 1.6, 0.3, 0.3, 0.5)])
    x0 = arr[3].px
    run_oracle(o, arr, 400)
    assert arr[3].px > x0 + 0.05, (x0, arr[3].px)


def test_oracle_polygon_ramp_holds_and_deflects_fluid():
    """A static triangular ramp in the tank (fluid.rs:518-530): fluid poured
    on it ends outside the triangle and runs down its slope."""
    o = OracleWorld()
    for (px, py), (hx, hy) in TANK:
        o.add_box(px, py, hx, hy)
    o.add_particles(lattice(-0.2, 1.0, 8, 4, 0.2))
    ramp, v = polygon_body(1.0, 0.2, RAMP)
    arr = body_list([static_box(*p, *e) for p, e in TANK] + [ramp])
    poly = poly_arrays([None, None, None, v])
    run_oracle(o, arr, 240, poly=poly)
    s = o.state()
    world = [(x + 1.0, y + 0.2) for x, y in RAMP]
    assert np.isfinite(s).all()
    assert sum(point_in_poly(x, y, world) for x, y in s[:, :2]) == 0
    assert s[:, 0].mean() > 0.9  # ran down the slope towards +x


def test_oracle_polygon_body_takes_impulses():
    """A dynamic pentagon hit by falling fluid picks up velocity and spin
    from the boundary impulses (polygons get no buoyancy, fluid.rs:415-418)."""
    o = oracle_world(lattice(1.5, 1.2, 6, 3, 0.2))
    pent, v = polygon_body(2.0, 0.6, PENTAGON, dynamic=True)
    arr = body_list([static_box(*p, *e) for p, e in TANK] + [pent])
    poly = poly_arrays([None, None, None, v])
    vy0 = []
    for _ in range(40):
        o.step_fluid(arr, 1 / 60, REF_SEQ, poly)  # no kick: only the fluid moves the body
        vy0.append(arr[3].vy)
    assert min(vy0) < 0.0 and arr[3].is_sleeping == 0


def test_oracle_reaction_hand_computed():
    """One particle moving into a resting dynamic circle, no gravity: the
    body receives n * (vn * m) (apply_impulse, body.rs:675-687)."""
    c = default_config()
    c.viscosity = 0.0
    o = OracleWorld()
    o.set_config(c)
    o.set_gravity(0.0, 0.0)
    o.add_particles(np.array([[1.0, 0.0]], np.float32))
    o.set_state(np.array([[1.0, 0.0, -2.0, 0.0]], np.float32))
    arr = body_list([dynamic_circle(0.0, 0.0, 1.0, 1.0)])
    dt = f32(1 / 60)
    o.step_fluid(arr, float(dt))
    # the particle moved to x = 1 - 2 dt, penetrates by r + pr - dist and
    # is pushed out along +x; vn = -2, impulse = (vn * m, 0)
    m = f32(0.0625)
    inv_m = f32(1) / (f32(math.pi) * f32(1) * f32(1) * f32(1))
    assert arr[0].vx == f32(f32(0) + (f32(1) * (f32(-2) * m)) * inv_m)
    assert arr[0].vy == 0.0 and arr[0].w == 0.0 and arr[0].is_sleeping == 0
    s = o.state()
    assert s[0, 2] == 0.0  # approach velocity removed


def test_step_fluid_arguments(lib=None):
    lib = _abi.load()
    w = lib.phieng_world_new()
    arr = body_list([dynamic_circle(0.0, 0.0, 1.0, 1.0)])
    assert lib.phieng_sph_step_fluid(None, arr, 1, 0.01) == 0
    assert lib.phieng_sph_step_fluid(w, None, 1, 0.01) == 0
    assert lib.phieng_sph_step_fluid(w, arr, 1, 0.01) == 1  # no particles: nothing to do
    bad = body_list([dynamic_circle(0.0, 0.0, 1.0, 1.0)])
    bad[0].shape_tag = 7
    assert lib.phieng_sph_step_fluid(w, bad, 1, 0.01) == 0
    bad = body_list([dynamic_circle(0.0, 0.0, 1.0, 1.0)])
    bad[0].vx = float("nan")
    assert lib.phieng_sph_step_fluid(w, bad, 1, 0.01) == 0
    # polygons: only through phieng_sph_step_fluid_poly, with a valid vertex range
    pb, v = polygon_body(0.0, 0.0, RAMP)
    arr = body_list([pb])
    xy, first, count = poly_arrays([v])
    U = C.POINTER(C.c_uint32)

    def call(xy_, first_, count_, nverts):
        return lib.phieng_sph_step_fluid_poly(w, arr, 1, None if xy_ is None else fp(xy_),
                                             None if first_ is None else first_.ctypes.data_as(U),
                                             None if count_ is None else count_.ctypes.data_as(U), nverts, 0.01)

    assert lib.phieng_sph_step_fluid(w, arr, 1, 0.01) == 0
    assert call(xy, first, count, 3) == 1
    assert call(None, first, count, 3) == 0
    assert call(xy, first, count, 2) == 0  # range past the vertex count
    assert call(xy, first, np.asarray([2], np.uint32), 3) == 0  # fewer than 3 vertices
    xy_bad = xy.copy()
    xy_bad[1, 0] = np.inf
    assert call(xy_bad, first, count, 3) == 0
    lib.phieng_world_free(w)


# ---- GPU parity ---------------------------------------------------------------

def gpu_world(pts, cfg=None):
    lib = _abi.load()
    w = lib.phieng_world_new()
    if cfg is not None:
        assert lib.phieng_world_set_fluid_config(w, C.byref(cfg)) == 1
    for (px, py), (hx, hy) in TANK:
        assert lib.phieng_world_add_body(w, px, py, _abi.SHAPE_BOX, hx, hy, 1.0, 1, 0.5, 0.0) >= 0
    p = np.ascontiguousarray(pts, np.float32)
    assert lib.phieng_world_fluid_add(w, fp(p.ravel()), len(p)) == len(p)
    return lib, w


def gpu_state(lib, w):
    n = lib.phieng_world_fluid_count(w)
    out = np.zeros((n, 4), np.float32)
    assert lib.phieng_world_fluid_get(w, fp(out), n) == n
    return out


def copy_bodies(arr):
    out = (PhiengBody2 * len(arr))()
    C.memmove(out, arr, C.sizeof(out))
    return out


def body_bits(arr):
    return np.array([[b.vx, b.vy, b.w, b.px, b.py] for b in arr], np.float32).view(np.uint32)


def set_gpu_ambient(lib, w, wind=(0.0, 0.0), turb=None):
    a = _abi.default_ambient()
    a.wind_x, a.wind_y = wind
    if turb:
        a.turbulence_enabled = 1
        a.turbulence_amplitude = turb["amplitude"]
        a.turbulence_frequency = turb.get("frequency", 1.0)
        a.turbulence_seed = turb.get("seed", 0)
        a.turbulence_divergence_free = 1 if turb.get("divergence_free") else 0
    assert lib.phieng_world_set_ambient_config(w, C.byref(a)) == 1


def coupled_parity(cfg, bodies, frames, settle=60, pts=None, wind=None, turb=None, poly=None):
    pts = lattice(-0.5, -0.5, 16, 8, 0.25) if pts is None else pts
    o = oracle_world(pts, cfg)
    lib, w = gpu_world(pts, cfg)
    if wind or turb:
        set_gpu_ambient(lib, w, wind or (0.0, 0.0), turb)
        o.set_wind(*(wind or (0.0, 0.0)))
        if turb:
            o.set_turbulence(**turb)
    for _ in range(settle):
        o.step(1 / 60, JACOBI)
        lib.phieng_world_step(w, 1 / 60)
    a = body_list(bodies)
    b = copy_bodies(a)
    angles_a, angles_b = [0.0] * len(a), [0.0] * len(b)
    dt = 1 / 60
    for f in range(frames):
        kick(a, dt)
        kick(b, dt)
        o.step_fluid(a, dt, JACOBI, poly)
        if poly is None:
            assert lib.phieng_sph_step_fluid(w, b, len(b), dt) == 1
        else:
            xy, first, count = poly
            U = C.POINTER(C.c_uint32)
            assert lib.phieng_sph_step_fluid_poly(w, b, len(b), fp(xy), first.ctypes.data_as(U),
                                                  count.ctypes.data_as(U), len(xy), dt) == 1
        drift(a, dt, angles_a)
        drift(b, dt, angles_b)
        assert (body_bits(a) == body_bits(b)).all(), f"bodies differ at frame {f}"
        assert [x.is_sleeping for x in a] == [x.is_sleeping for x in b]
        if f % 10 == 9 or f == frames - 1:
            s_ref, s = o.state(), gpu_state(lib, w)
            bad = np.nonzero(s_ref.view(np.uint32) != s.view(np.uint32))[0]
            assert bad.size == 0, f"frame {f}: {bad.size} particles differ, first {bad[0]}"
    lib.phieng_world_free(w)
    return a


def floating_bodies():
    return [static_box(*p, *e) for p, e in TANK] + [
        dynamic_box(1.2, 1.4, 0.3, 0.2, 0.5, angle=0.3),
        dynamic_circle(3.0, 1.5, 0.25, 0.6),
    ]


@pytest.mark.gpu
def test_step_fluid_bit_exact_frictionless():
    a = coupled_parity(default_config(), floating_bodies(), 120)
    assert any(abs(b.w) > 0 for b in a[3:])  # the coupling produced torque


@pytest.mark.gpu
def test_step_fluid_bit_exact_friction_and_substeps():
    c = default_config()
    c.wall_friction = 0.5
    c.gamma = 7.0
    c.stiffness = 40.0
    c.cfl = 0.4
    c.max_substeps = 4
    c.drag = 2.0
    coupled_parity(c, floating_bodies(), 100)


@pytest.mark.gpu
def test_step_fluid_bit_exact_wind_and_turbulence():
    """The world's ambient config in the fluid phase: the wind in the
    buoyancy drag (fluid.rs:1121-1124) and curl turbulence at the world clock,
    bodies and particles bit for bit against the oracle."""
    c = default_config()
    c.drag = 2.0
    coupled_parity(c, floating_bodies(), 90, wind=(3.0, -0.5),
                   turb=dict(amplitude=3.0, frequency=0.7, seed=11, divergence_free=True))


@pytest.mark.gpu
def test_step_fluid_bit_exact_polygons():
    """A static triangular ramp, a static concave L and a dynamic rotating
    pentagon among the walls, with friction: bodies and particles bit for bit
    against the oracle."""
    c = default_config()
    c.wall_friction = 0.3
    ramp, vr = polygon_body(1.2, 0.3, RAMP, angle=0.2)
    ell, ve = polygon_body(2.8, -0.45, ELL)
    pent, vp = polygon_body(3.6, 1.2, PENTAGON, dynamic=True, angle=0.4)
    bodies = [static_box(*p, *e) for p, e in TANK] + [ramp, ell, pent, dynamic_circle(0.6, 1.8, 0.2, 0.5)]
    poly = poly_arrays([None, None, None, vr, ve, vp, None])
    a = coupled_parity(c, bodies, 100, pts=lattice(-0.4, 0.8, 16, 10, 0.2), poly=poly)
    assert abs(a[5].vx) + abs(a[5].vy) > 0  # the pentagon took impulses


@pytest.mark.gpu
def test_gpu_box_floats():
    """fluid.rs:1258-1289 through the GPU fluid phase."""
    lib, w = gpu_world(lattice(-0.5, -0.5, 12, 6, 0.25))
    for _ in range(300):
        lib.phieng_world_step(w, 1 / 60)
    arr = body_list([static_box(*p, *e) for p, e in TANK] + [dynamic_box(2.0, 1.6, 0.3, 0.3, 0.5)])
    angles = [0.0] * len(arr)
    for _ in range(600):
        kick(arr, 1 / 60)
        assert lib.phieng_sph_step_fluid(w, arr, len(arr), 1 / 60) == 1
        drift(arr, 1 / 60, angles)
    assert 0.0 < arr[3].py < 2.0
    assert np.isfinite(gpu_state(lib, w)).all()
    lib.phieng_world_free(w)


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_step_fluid_without_device_fails_loudly():
    lib, w = gpu_world(lattice(0.0, 0.0, 3, 3, 0.25))
    arr = body_list(floating_bodies())
    assert lib.phieng_sph_step_fluid(w, arr, len(arr), 1 / 60) == 0
    st = _abi.PhiengSphStatus()
    lib.phieng_sph_status(w, C.byref(st))
    assert st.error == _abi.E_NO_DEVICE
    lib.phieng_world_free(w)
