"""Batches of independent scenes: the workload generator, the per-rank split
and (on a GPU) bit-exact agreement of every scene with stepping it alone.
The two-rank sharded run is exercised with gloo on the CPU, each rank
stepping its scenes with the oracle."""
import math
import os

import numpy as np
import pytest

import sims
from oracle import oracle as orc
from phi_eng_b200 import batch, scenes


def test_batched_workload_shape():
    scs = batch.batched_scenes(512)
    assert len(scs) == 512
    n = np.array([sc.n for sc in scs])
    assert n.min() >= 1024 and n.max() <= 32768
    # log-uniform: mean of log N near the middle of [ln 1024, ln 32768]
    assert abs(np.log(n).mean() - 0.5 * (math.log(1024) + math.log(32768))) < 0.15
    tilt = np.degrees(np.arctan2([sc.gravity[0] for sc in scs], [-sc.gravity[1] for sc in scs]))
    assert np.abs(tilt).max() <= 15.0 + 1e-9
    for sc in scs[:20]:
        xs, ys = sc.xy[:, 0], sc.xy[:, 1]
        width = sc.boxes[2][0] - sc.boxes[2][2]  # inner face of the right wall
        assert xs.max() < width and ys.min() > 0.0
    assert batch.batched_scenes(4)[2].xy.tobytes() == batch.batched_scenes(4)[2].xy.tobytes()


def test_partition_lpt_balanced_and_complete():
    sizes = [sc.n for sc in batch.batched_scenes(512)]
    for parts in (1, 2, 3, 8):
        groups = batch.partition_lpt(sizes, parts)
        flat = sorted(i for g in groups for i in g)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[i] for i in g) for g in groups]
        assert max(loads) - min(loads) <= max(sizes)


def oracle_stepper(scs, steps):
    out = []
    for sc in scs:
        o = sims.load_scene(sims.OracleSim(orc.JACOBI), sc)
        o.step(sc.dt, steps)
        out.append(o.state())
    return out


def _rank_main(rank, world_size, port, result_path):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world_size)
    scs = batch.batched_scenes(6, n_min=64, n_max=256)
    res = batch.run_sharded(scs, 5, rank, world_size, stepper=oracle_stepper)
    if rank == 0:
        np.savez(result_path, **{str(k): v for k, v in res.items()})
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_run_two_ranks_gloo(tmp_path):
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    path = str(tmp_path / "res.npz")
    mp.spawn(_rank_main, args=(2, port, path), nprocs=2, join=True)
    got = np.load(path)
    scs = batch.batched_scenes(6, n_min=64, n_max=256)
    want = oracle_stepper(scs, 5)
    assert sorted(int(k) for k in got.files) == list(range(6))
    for k in range(6):
        assert np.array_equal(got[str(k)], want[k])


def _mixed_scenes():
    out = []
    base = scenes.reference_tank(8, 6)
    out.append(base)
    a = scenes.reference_tank(10, 5)
    c = a.config
    c.gamma = 7.0
    c.stiffness = 15.0
    c.artificial_viscosity = 1.0
    c.surface_tension = 0.5
    a.config = c
    a.gravity = (1.5, -9.0)
    out.append(a)
    b = scenes.reference_tank(6, 9)
    b.circles = [(1.0, 1.2, 0.3)]
    c = b.config
    c.wall_friction = 0.5
    b.config = c
    out.append(b)
    t = scenes.reference_tank(12, 4)
    c = t.config
    c.phase_count = 2
    for k, v in enumerate([2.0, 1.0, 1.0, 1.0]):
        c.phase_rest_density[k] = v
    for k, v in enumerate([0.125, 0.0625, 0.0625, 0.0625]):
        c.phase_mass[k] = v
    t.config = c
    t.phases = (np.arange(t.n) % 2).astype(np.uint8)
    out.append(t)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["generated", "mixed"])
def test_batch_equals_each_world_alone(which):
    from phi_eng_b200.world import world_from_scene

    scs = batch.batched_scenes(12, n_min=256, n_max=4096) if which == "generated" else _mixed_scenes()
    dt = scs[0].dt
    b = batch.Batch.from_scenes(scs)
    b.step(dt, 40)
    for k, sc in enumerate(scs):
        w = world_from_scene(sc)
        w.step_n(dt, 40)
        assert np.array_equal(b.scene_particles(k), w.fluid.particles), k
        w.close()
    b.store()
    for k in range(len(scs)):
        assert np.array_equal(b.worlds[k].fluid.particles, b.scene_particles(k))
    b.close()


@pytest.mark.gpu
def test_batch_matches_oracle_on_generated_scenes():
    scs = batch.batched_scenes(4, n_min=512, n_max=2048)
    got = batch.gpu_stepper(scs, 25)
    want = oracle_stepper(scs, 25)
    for k in range(len(scs)):
        assert np.array_equal(got[k], want[k])


@pytest.mark.gpu
def test_batch_rejects_bad_input():
    from phi_eng_b200.world import World2

    w = World2()
    w.fluid.add_particles(np.zeros((4, 2), np.float32) + np.arange(4, dtype=np.float32)[:, None])
    c = w.fluid.config
    c.cfl = 0.4
    c.max_substeps = 4
    w.fluid.config = c
    with pytest.raises(ValueError):
        batch.Batch([w])


def workload_slice():
    """32 scenes of the 512-scene workload generator itself: its 8 largest
    (32,768-particle end of the log-uniform range) and 24 spread over the rest
    by index."""
    scs = batch.batched_scenes(512)
    by_size = sorted(range(len(scs)), key=lambda i: (-scs[i].n, i))
    largest = by_size[:8]
    rest = [i for i in range(0, 512, 21) if i not in largest][:24]
    idx = sorted(largest + rest)
    return [scs[i] for i in idx]


def test_workload_slice_covers_the_range():
    scs = workload_slice()
    n = [sc.n for sc in scs]
    assert len(scs) == 32
    assert max(n) >= 32000 and min(n) < 2048


@pytest.mark.gpu
def test_batch_workload_slice_matches_oracle():
    """The slice advanced together in one batch for 20 steps: every scene bit
    for bit equal to the oracle's Jacobi step of that scene alone."""
    scs = workload_slice()
    got = batch.gpu_stepper(scs, 20)
    want = oracle_stepper(scs, 20)
    for k in range(len(scs)):
        assert np.array_equal(got[k].view(np.uint32), want[k].view(np.uint32)), (k, scs[k].n)
