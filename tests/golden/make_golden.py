"""Regenerate the golden fixtures in this folder from the CPU oracle.

    python tests/golden/make_golden.py

The reference ships no numeric vectors for its SPH step (its tests are
behavioural), so these fixtures are the oracle's own outputs, pinned so a
change to the oracle or to the GPU path shows up as a diff:

  dam_break_4k.npz   64 x 64 block, spacing 0.01 m, jitter +-1% from
                     SplitMix64(0x5EED), rho0 = 1 units, h = 0.02, Tait gamma 7,
                     k = 100, open-top 1.0 m box; dt = 0.4 h / sqrt(gamma k).
                     Full f32 states after 1 and 10 steps and SHA-256 of the
                     state after 100 steps, for the in-place (Gauss-Seidel)
                     integrate and the Jacobi integrate.
  tank_8x12.npz      the reference's test tank (crates/dynamics/src/fluid.rs:
                     1151-1182): 8 x 12 at 0.25 m, default FluidConfig2,
                     dt = 1/60; full states after 1, 10 and 60 steps.

Each array is [x, y, vx, vy] f32 per particle in insertion order.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.dirname(HERE)):
    if p not in sys.path:
        sys.path.insert(0, p)

from oracle import oracle as orc  # noqa: E402
from phi_eng_b200 import scenes  # noqa: E402
import sims  # noqa: E402

MODES = {"seq": orc.REF_SEQ, "jacobi": orc.JACOBI}
DAM_FULL = (1, 10)
DAM_HASH = (100,)
TANK_FULL = (1, 10, 60)


def sha(state: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(state, dtype=np.float32).tobytes()).hexdigest()


def run(scene, mode, marks):
    sim = sims.load_scene(sims.OracleSim(mode), scene)
    out, done = {}, 0
    for m in sorted(marks):
        sim.step(scene.dt, m - done)
        done = m
        out[m] = np.array(sim.state(), dtype=np.float32)
    return out


def generate():
    dam = scenes.dam_break_4k()
    tank = scenes.reference_tank()
    arrays, meta = {}, {"dam_break_4k": {"dt": dam.dt, "n": dam.n, "sha256": {}},
                        "tank_8x12": {"dt": tank.dt, "n": tank.n}}
    arrays["dam_initial"] = np.array(dam.xy, dtype=np.float32)
    for name, mode in MODES.items():
        st = run(dam, mode, DAM_FULL + DAM_HASH)
        for m in DAM_FULL:
            arrays[f"dam_{name}_{m}"] = st[m]
        for m in DAM_HASH:
            meta["dam_break_4k"]["sha256"][f"{name}_{m}"] = sha(st[m])
    tank_arrays = {}
    for name, mode in MODES.items():
        st = run(tank, mode, TANK_FULL)
        for m in TANK_FULL:
            tank_arrays[f"tank_{name}_{m}"] = st[m]
    return arrays, tank_arrays, meta


def main():
    orc.build()
    arrays, tank_arrays, meta = generate()
    np.savez_compressed(os.path.join(HERE, "dam_break_4k.npz"), **arrays)
    np.savez_compressed(os.path.join(HERE, "tank_8x12.npz"), **tank_arrays)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
        f.write("\n")


if __name__ == "__main__":
    main()
