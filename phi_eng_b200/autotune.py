"""Launch-shape autotuner for the SPH step (threads per block of the density
and force passes, bucket-grid budget per particle).

None of the knobs changes results: the neighbour visit order and every sum
are fixed by the cell grid, whatever the bucket grid or block size (the
parity tests run under several of them). The tuner times each candidate on
the caller's own world (or batch) from the same saved device state, with CUDA
events on the world's stream, and keeps the fastest. Choices are cached in a
JSON file keyed by GPU name and workload signature:

  - the file named by $PHIENG_SPH_TUNING_CACHE, else
    ~/.cache/phieng_sph/tuning.json (written by `autotune(..., save=True)`);
  - phi_eng_b200/tuning_b200.json ships the choices measured on B200 for the
    benchmark workloads and is read when the user cache has no entry.
"""
from __future__ import annotations

import ctypes as C
import itertools
import json
import os

import numpy as np

from . import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
SHIPPED = os.path.join(HERE, "tuning_b200.json")
DEFAULT = dict(density_block=256, force_block=256, buckets_per_particle=2.0, stage=0)
CANDIDATES = dict(density_block=(128, 256), force_block=(64, 128, 256), buckets_per_particle=(0.5, 1.0, 2.0, 4.0),
                  stage=(0,))
# tolerance-mode worlds also try the passes without shared-memory staging
CANDIDATES_TOLERANCE = dict(CANDIDATES, stage=(0, 1, 2, 3, 4, 5))


def cache_path() -> str:
    p = os.environ.get("PHIENG_SPH_TUNING_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "phieng_sph", "tuning.json")


def gpu_name() -> str:
    import torch

    return torch.cuda.get_device_name(0) if torch.cuda.is_available() else "cpu"


def signature(world) -> str:
    """Workload signature: particle count (to 2 significant digits), scenes,
    smoothing length, bucket-grid shape of the default plan."""
    st = world.status()
    n = int(st.particles)
    n2 = int(float(f"{n:.2g}")) if n else 0
    scenes = int(world._lib.phieng_sph_batch_scenes(world._h)) or 1
    h = float(world.fluid.config.smoothing_length) if scenes == 1 else 0.0
    mode = "|tol" if int(world._lib.phieng_sph_get_precision(world._h)) == _abi.TOLERANCE else ""
    return f"n{n2}|s{scenes}|h{h:.3g}{mode}"


def _load(path: str) -> dict:
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def lookup(world, gpu: str | None = None):
    """The cached tuning for this world's workload on this GPU, or None."""
    key = f"{gpu or gpu_name()}|{signature(world)}"
    for path in (cache_path(), SHIPPED):
        t = _load(path).get(key)
        if t:
            return dict(t["tuning"])
    return None


def apply(world, tuning: dict) -> None:
    t = _abi.PhiengSphTuning(int(tuning["density_block"]), int(tuning["force_block"]),
                             float(tuning["buckets_per_particle"]), int(tuning.get("stage", 0)))
    if world._lib.phieng_sph_set_tuning(world._h, C.byref(t)) != 1:
        raise ValueError(f"invalid tuning {tuning}")


def current(world) -> dict:
    t = _abi.PhiengSphTuning()
    world._lib.phieng_sph_get_tuning(world._h, C.byref(t))
    return dict(density_block=int(t.density_block), force_block=int(t.force_block),
                buckets_per_particle=float(t.buckets_per_particle), stage=int(t.stage))


def time_steps(world, dt: float, steps: int, warmup: int = 2) -> float:
    """Mean ms per step on the world's stream (CUDA events)."""
    import torch

    s = torch.cuda.Stream()
    world.set_stream(s.cuda_stream)
    world.step_n(dt, warmup)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    world.step_n(dt, steps)
    e1.record(s)
    e1.synchronize()
    world.set_stream(None)
    return e0.elapsed_time(e1) / steps


def autotune(world, dt: float, steps: int = 20, candidates: dict | None = None, save: bool = False,
             log=None) -> dict:
    """Time every candidate from the world's current state (restored between
    candidates) and leave the fastest applied. Returns {tuning, ms, table}."""
    import torch

    tol = int(world._lib.phieng_sph_get_precision(world._h)) == _abi.TOLERANCE
    cand = candidates or (CANDIDATES_TOLERANCE if tol else CANDIDATES)
    n = int(world.status().particles)
    saved = torch.empty((max(n, 1), 4), dtype=torch.float32, device="cuda")
    world.get_state_device(saved.data_ptr(), n)
    world.sync()
    table = []
    for db, fb, bpp, stg in itertools.product(cand["density_block"], cand["force_block"],
                                              cand["buckets_per_particle"], cand.get("stage", (0,))):
        t = dict(density_block=db, force_block=fb, buckets_per_particle=bpp, stage=stg)
        apply(world, t)
        world.set_state_device(saved.data_ptr(), n)
        ms = time_steps(world, dt, steps)
        table.append((ms, t))
        if log:
            log(f"{t}: {ms:.4f} ms/step")
    world.set_state_device(saved.data_ptr(), n)
    ms, best = min(table, key=lambda r: r[0])
    apply(world, best)
    world.sync()
    if save:
        path = cache_path()
        os.makedirs(os.path.dirname(path), exist_ok=True)
        d = _load(path)
        d[f"{gpu_name()}|{signature(world)}"] = dict(tuning=best, ms_per_step=ms)
        with open(path, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
    return dict(tuning=best, ms=ms, table=[dict(ms=m, **t) for m, t in table],
                default_ms=next((m for m, t in table if t == DEFAULT), None))


def _main(argv=None) -> None:
    """python -m phi_eng_b200.autotune [--workload NAME] [--out PATH] [--precision MODE]: tune the
    benchmark workloads and write their entries (GPU name + signature) to a
    JSON table."""
    import argparse

    from . import scenes as S
    from .batch import Batch, batched_scenes
    from .world import world_from_scene

    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", action="append", choices=["dam_break_1m", "dam_break_4k", "batch_512"])
    ap.add_argument("--out", default=None, help="JSON table to update (default: the user cache)")
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--precision", choices=["exact", "tolerance"], default="exact",
                    help="tune the worlds in this arithmetic mode (phieng_sph_set_precision)")
    a = ap.parse_args(argv)
    mode = _abi.TOLERANCE if a.precision == "tolerance" else _abi.EXACT
    out = {}
    for name in a.workload or ["dam_break_1m", "dam_break_4k", "batch_512"]:
        if name == "batch_512":
            scs = batched_scenes(512)
            b = Batch.from_scenes(scs)
            w, dt, keep = b.world, scs[0].dt, b
        else:
            sc = S.dam_break_1m() if name == "dam_break_1m" else S.dam_break_4k()
            w, dt, keep = world_from_scene(sc), sc.dt, None
        w.precision = mode
        w.step_n(dt, 3)
        r = autotune(w, dt, steps=a.steps)
        key = f"{gpu_name()}|{signature(w)}"
        out[key] = dict(tuning=r["tuning"], ms_per_step=r["ms"], default_ms_per_step=r["default_ms"], workload=name)
        print(json.dumps(dict(workload=name, key=key, **r)), flush=True)
        if keep is not None:
            keep.close()
        else:
            w.close()
    path = a.out or cache_path()
    d = _load(path)
    d.update(out)
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    _main()
