"""Golden fixtures (tests/golden, made by tests/golden/make_golden.py).

CPU: the oracle and the scene generators reproduce the committed vectors bit
for bit. GPU: the CUDA step reproduces the Jacobi-integrate vectors bit for
bit (the GPU integrate is the Jacobi form of fluid.rs:1003-1050).
"""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

import sims
from oracle import oracle as orc
from phi_eng_b200 import scenes

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load():
    dam = np.load(os.path.join(GOLD, "dam_break_4k.npz"))
    tank = np.load(os.path.join(GOLD, "tank_8x12.npz"))
    with open(os.path.join(GOLD, "golden.json")) as f:
        meta = json.load(f)
    return dam, tank, meta


def _run(sim, scene, marks):
    sims.load_scene(sim, scene)
    out, done = {}, 0
    for m in sorted(marks):
        sim.step(scene.dt, m - done)
        done = m
        out[m] = np.array(sim.state(), dtype=np.float32)
    return out


def _sha(a):
    import hashlib

    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float32).tobytes()).hexdigest()


def test_generators_match_golden():
    dam, _, meta = _load()
    sc = scenes.dam_break_4k()
    np.testing.assert_array_equal(np.asarray(sc.xy, np.float32), dam["dam_initial"])
    assert sc.dt == meta["dam_break_4k"]["dt"]
    assert scenes.reference_tank().n == meta["tank_8x12"]["n"]


@pytest.mark.parametrize("name,mode", [("seq", orc.REF_SEQ), ("jacobi", orc.JACOBI)])
def test_oracle_matches_golden(name, mode):
    dam, tank, meta = _load()
    st = _run(sims.OracleSim(mode), scenes.dam_break_4k(), (1, 10, 100))
    for m in (1, 10):
        np.testing.assert_array_equal(st[m], dam[f"dam_{name}_{m}"])
    assert _sha(st[100]) == meta["dam_break_4k"]["sha256"][f"{name}_100"]
    st = _run(sims.OracleSim(mode), scenes.reference_tank(), (1, 10, 60))
    for m in (1, 10, 60):
        np.testing.assert_array_equal(st[m], tank[f"tank_{name}_{m}"])


def test_integrate_orders_differ():
    """The two integrate orders are distinct fixtures (the in-place sweep reads
    already-advected neighbours), so a mode mix-up cannot pass silently."""
    dam, _, _ = _load()
    assert not np.array_equal(dam["dam_seq_10"], dam["dam_jacobi_10"])


@pytest.mark.gpu
def test_gpu_matches_golden_jacobi():
    dam, tank, meta = _load()
    st = _run(sims.GpuSim(), scenes.dam_break_4k(), (1, 10, 100))
    for m in (1, 10):
        np.testing.assert_array_equal(st[m], dam[f"dam_jacobi_{m}"])
    assert _sha(st[100]) == meta["dam_break_4k"]["sha256"]["jacobi_100"]
    st = _run(sims.GpuSim(), scenes.reference_tank(), (1, 10, 60))
    for m in (1, 10, 60):
        np.testing.assert_array_equal(st[m], tank[f"tank_jacobi_{m}"])
