"""Launch tuning: validation (CPU) and result invariance + the tuner (GPU).

The knobs (threads per block of the density and force passes, bucket budget
per particle) must not change any result: the trajectory under every tuning
equals the default one bit for bit, and equals the oracle's.
"""
import ctypes as C

import numpy as np
import pytest

import sims
from oracle import oracle as orc
from phi_eng_b200 import _abi, autotune, scenes
from phi_eng_b200.world import world_from_scene


def test_tuning_validation_and_roundtrip():
    w = world_from_scene(scenes.dam_break_4k())
    lib = w._lib
    assert autotune.current(w) == autotune.DEFAULT
    for bad in [(96, 256, 2.0), (256, 512, 2.0), (256, 256, 0.0), (256, 256, 64.0), (256, 256, float("nan"))]:
        t = _abi.PhiengSphTuning(bad[0], bad[1], bad[2], 0)
        assert lib.phieng_sph_set_tuning(w._h, C.byref(t)) == 0
    assert autotune.current(w) == autotune.DEFAULT
    autotune.apply(w, dict(density_block=128, force_block=64, buckets_per_particle=0.5, stage=1))
    assert autotune.current(w) == dict(density_block=128, force_block=64, buckets_per_particle=0.5, stage=1)
    assert lib.phieng_sph_set_tuning(None, None) == 0
    w.close()


@pytest.mark.gpu
@pytest.mark.parametrize("tuning", [dict(density_block=128, force_block=64, buckets_per_particle=0.5),
                                    dict(density_block=64, force_block=128, buckets_per_particle=4.0),
                                    dict(density_block=256, force_block=256, buckets_per_particle=0.125)])
def test_results_do_not_depend_on_tuning(tuning):
    sc = scenes.dam_break_4k()
    w = world_from_scene(sc)
    autotune.apply(w, tuning)
    w.step_n(sc.dt, 40)
    o = sims.load_scene(sims.OracleSim(orc.JACOBI), sc)
    o.step(sc.dt, 40)
    np.testing.assert_array_equal(w.fluid.particles, o.state())
    w.close()


@pytest.mark.gpu
def test_autotune_applies_the_fastest_and_keeps_the_state():
    sc = scenes.dam_break_4k()
    w = world_from_scene(sc)
    w.step_n(sc.dt, 5)
    before = w.fluid.particles.copy()
    r = autotune.autotune(w, sc.dt, steps=4,
                          candidates=dict(density_block=(128, 256), force_block=(256,), buckets_per_particle=(1.0, 2.0)))
    assert len(r["table"]) == 4 and r["ms"] == min(t["ms"] for t in r["table"])
    assert autotune.current(w) == r["tuning"]
    np.testing.assert_array_equal(w.fluid.particles, before)
    ref = world_from_scene(sc)
    ref.step_n(sc.dt, 5)
    w.step_n(sc.dt, 10)
    ref.step_n(sc.dt, 10)
    np.testing.assert_array_equal(w.fluid.particles, ref.fluid.particles)
