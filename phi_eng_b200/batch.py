"""Batches of independent SPH scenes advanced together on one GPU.

The batched workload: 512 dam-break scenes whose particle counts are
log-uniform in [1,024, 32,768], block aspect ratios uniform in [0.5, 2],
gravity tilted uniformly within +-15 degrees, each in its own walled box
2.5x its block's width and 1.5x its height, with the 4k workload's
parameters (spacing 0.01 m). Scene k's block is the first N_k points of an
nx x ny lattice, nx = round(sqrt(N_k * a)), ny = ceil(N_k / nx), jittered by
+-1% of the spacing from SplitMix64 seeded 0x5EED + k; the scene draws come
from SplitMix64 seeded 0xBA7C, three per scene (size, aspect, tilt).

A batch is a World2 holding copies of the scenes' worlds (phieng_sph_batch_new):
one phieng_world_step advances every scene by one substep, and each scene's
result equals stepping its world alone.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _abi, scenes
from .world import World2, world_from_scene


def batched_scenes(count: int = 512, seed: int = 0xBA7C, n_min: int = 1024, n_max: int = 32768,
                   spacing: float = 0.01) -> list:
    u = (scenes.splitmix64_stream(seed, 3 * count) >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))
    u = u.reshape(count, 3)
    out = []
    cfg = scenes.si_config(spacing)
    dt = scenes.fine_dt(cfg)
    for k in range(count):
        n_k = int(round(math.exp(math.log(n_min) + u[k, 0] * (math.log(n_max) - math.log(n_min)))))
        a = 0.5 + 1.5 * u[k, 1]
        theta = math.radians(-15.0 + 30.0 * u[k, 2])
        nx = max(1, int(round(math.sqrt(n_k * a))))
        ny = int(math.ceil(n_k / nx))
        xy = scenes.jittered_lattice(nx, ny, spacing, seed=0x5EED + k)[:n_k]
        width, height = 2.5 * nx * spacing, 1.5 * ny * spacing
        g = (9.81 * math.sin(theta), -9.81 * math.cos(theta))
        out.append(scenes.Scene(name=f"batch_{k}", boxes=scenes.box_walls(width, height), xy=xy,
                                config=cfg, dt=dt, steps=500, gravity=g))
    return out


def partition_lpt(sizes, nparts: int) -> list:
    """Longest-processing-time split of scene indices into nparts groups
    balanced by particle count (largest scene first, to the lightest group).
    Deterministic: ties go to the lowest group index."""
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i))
    loads = [0] * nparts
    groups = [[] for _ in range(nparts)]
    for i in order:
        g = min(range(nparts), key=lambda j: (loads[j], j))
        groups[g].append(i)
        loads[g] += int(sizes[i])
    return [sorted(gr) for gr in groups]


class _BatchView(World2):
    """World2 entry points (step, read-back, status, streams) on a batch handle
    owned by a Batch; closing the view does not free the handle."""

    def __init__(self, lib, handle):
        from .world import FluidState2

        self._lib = lib
        self._h = handle
        self._gravity = (0.0, 0.0)
        self.fluid = FluidState2(self)

    def close(self) -> None:
        self._h = None


class Batch:
    """A GPU batch built from worlds (kept alive by the caller)."""

    def __init__(self, worlds):
        self._lib = _abi.load()
        self.worlds = list(worlds)
        arr = (C.c_void_p * len(self.worlds))(*[w._h for w in self.worlds])
        self._h = self._lib.phieng_sph_batch_new(arr, len(self.worlds))
        if not self._h:
            raise ValueError("phieng_sph_batch_new rejected the worlds")
        self._arr = arr
        self.world = _BatchView(self._lib, self._h)

    @classmethod
    def from_scenes(cls, scs):
        worlds = [world_from_scene(sc) for sc in scs]
        return cls(worlds)

    @property
    def scenes(self) -> int:
        return int(self._lib.phieng_sph_batch_scenes(self._h))

    def scene_range(self, k: int):
        f, c = C.c_uint32(), C.c_uint32()
        if self._lib.phieng_sph_batch_scene_range(self._h, k, C.byref(f), C.byref(c)) != 1:
            raise IndexError(k)
        return int(f.value), int(c.value)

    def step(self, dt: float, n: int = 1) -> None:
        self.world.step_n(dt, n)

    def particles(self) -> np.ndarray:
        return self.world.fluid.particles

    def scene_particles(self, k: int) -> np.ndarray:
        f, c = self.scene_range(k)
        return self.particles()[f:f + c]

    def store(self) -> None:
        if self._lib.phieng_sph_batch_store(self._h, self._arr, len(self.worlds)) != 1:
            raise RuntimeError("phieng_sph_batch_store failed")

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.phieng_world_free(self._h)
            self._h = None
            self.world._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gpu_stepper(scs, steps: int, dt: float | None = None) -> list:
    """Advance scenes together on this process's GPU; returns each scene's
    final [x, y, vx, vy] state."""
    if not scs:
        return []
    b = Batch.from_scenes(scs)
    b.step(scs[0].dt if dt is None else dt, steps)
    out = [b.scene_particles(k).copy() for k in range(len(scs))]
    b.close()
    return out


def run_sharded(scs, steps: int, rank: int = 0, world_size: int = 1, stepper=gpu_stepper) -> dict:
    """Deal the scenes over the ranks (partition_lpt by particle count), let
    every rank advance its share with `stepper`, and return every scene's
    final state on every rank (torch.distributed all_gather_object when
    world_size > 1). Scenes are independent, so no data crosses ranks during
    the steps; the gather is the only collective."""
    parts = partition_lpt([sc.n for sc in scs], world_size)
    mine = parts[rank]
    states = stepper([scs[i] for i in mine], steps)
    local = {i: st for i, st in zip(mine, states)}
    if world_size == 1:
        return local
    import torch.distributed as dist

    gathered = [None] * world_size
    dist.all_gather_object(gathered, local)
    out = {}
    for part in gathered:
        out.update(part)
    return out
