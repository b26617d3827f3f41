"""Slab decomposition of one scene over ranks (phi_eng_b200/slab.py).

CPU: gloo ranks (2 and 3) each step their slab plus a 2-cell halo on an
oracle engine defined here (Jacobi order, the order the GPU computes) and
exchange halos and migrating particles with their neighbours; the gathered
state equals the single-domain oracle run bit for bit, with and without CFL
substeps.
GPU: one rank on the library (no peers) equals the plain world, and two gloo
ranks that both drive the library's engine (the product default) on the one
GPU, exchanging host tensors, equal the single-domain GPU world bit for bit.
Each rank's kernels run on their own; no kernel waits on another rank.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import sims
from oracle import oracle as orc
from phi_eng_b200 import scenes


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _scene(cfl: bool):
    sc = scenes.dam_break_4k()
    if cfl:
        cfg = sc.config
        cfg.cfl = 0.4
        cfg.max_substeps = 4
        sc.config = cfg
        sc.dt = 2.5 * sc.dt
    return sc


class OracleEngine:
    """Test engine: the oracle in Jacobi order (what the GPU computes)."""

    def __init__(self, scene):
        self.scene = scene

    def step(self, state, dt: float):
        import torch

        from phi_eng_b200.slab import _no_cfl

        sc = self.scene
        o = orc.OracleWorld(cap=max(state.shape[0], 1))
        o.set_gravity(*sc.gravity)
        for (px, py, hx, hy) in sc.boxes:
            o.add_box(px, py, hx, hy, (1.0, 0.0, -0.0, 1.0))
        for (px, py, r) in sc.circles:
            o.add_circle(px, py, r, (1.0, 0.0, -0.0, 1.0))
        o.set_config(_no_cfl(sc.config))
        st = state.numpy()
        if st.shape[0]:
            o.add_particles(np.ascontiguousarray(st[:, :2]))
            o.set_state(st)
            o.step(dt, orc.JACOBI)
        return torch.from_numpy(o.state().reshape(-1, 4).copy())


def _worker(rank, size, port, steps, cfl, out, gpu=False, halo_cap=None):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=size)
    from phi_eng_b200.slab import DeviceSlabRun, SlabRun

    sc = _scene(cfl)
    if gpu == "device":
        run = DeviceSlabRun(sc, rank, size, halo_cap=halo_cap)
    else:
        run = SlabRun(sc, rank, size, engine=None if gpu else OracleEngine(sc))  # None: the library's GpuEngine
    for _ in range(steps):
        run.step(sc.dt)
    if gpu == "device" and halo_cap is not None:
        try:
            run.owned()
            ok = 1
        except RuntimeError:
            ok = 0
        np.save(out + f".ok{rank}.npy", np.array([ok]))
        run.close()
        dist.barrier()
        dist.destroy_process_group()
        return
    full = run.gather()
    if gpu == "device":
        run.close()
    elif gpu:
        run.engine.close()
    if rank == 0:
        np.save(out, full)
    moved = np.array([run.comm_bytes], np.int64)
    np.save(out + f".bytes{rank}.npy", moved)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("size,cfl", [(2, False), (3, False), (2, True)])
def test_slab_ranks_equal_single_domain(tmp_path, size, cfl):
    steps = 60
    out = str(tmp_path / "state.npy")
    mp.start_processes(_worker, args=(size, _free_port(), steps, cfl, out), nprocs=size, start_method="spawn")
    got = np.load(out)
    sc = _scene(cfl)
    o = sims.load_scene(sims.OracleSim(orc.JACOBI), sc)
    o.step(sc.dt, steps)
    np.testing.assert_array_equal(got, o.state())
    for r in range(size):
        assert np.load(out + f".bytes{r}.npy")[0] > 0  # halos crossed every edge


def test_slab_edges_split_evenly():
    from phi_eng_b200.slab import cell_column, slab_edges

    import torch

    sc = scenes.dam_break_4k()
    h = float(sc.config.smoothing_length)
    e = slab_edges(sc.xy, h, 4)
    cx = cell_column(torch.from_numpy(sc.xy[:, 0].copy()), h).numpy()
    counts = [int(((cx >= e[r]) & (cx < e[r + 1])).sum()) for r in range(4)]
    assert sum(counts) == sc.n and max(counts) - min(counts) <= 2 * 64 + 64
    assert all(e[r + 1] - e[r] >= 2 for r in range(1, 3))


@pytest.mark.gpu
def test_slab_gpu_single_rank_equals_world():
    import torch

    from phi_eng_b200.slab import GpuEngine, SlabRun
    from phi_eng_b200.world import world_from_scene

    sc = scenes.dam_break_4k()
    eng = GpuEngine(sc, cap=sc.n)
    run = SlabRun(sc, 0, 1, engine=eng, device="cuda")
    for _ in range(30):
        run.step(sc.dt)
    w = world_from_scene(sc)
    w.step_n(sc.dt, 30)
    np.testing.assert_array_equal(run.gather(), w.fluid.particles)
    torch.cuda.synchronize()
    eng.close()
    w.close()


@pytest.mark.gpu
@pytest.mark.parametrize("cfl", [False, True])
def test_slab_two_ranks_on_gpu_engine_equal_world(tmp_path, cfl):
    """Two gloo ranks, each stepping its slab + halo on the library's GPU
    engine (the default engine), exchange host tensors; 50 steps of the 4k
    dam break gathered equal a single-domain GPU world bit for bit."""
    from phi_eng_b200.world import world_from_scene

    steps, size = 50, 2
    out = str(tmp_path / "state.npy")
    mp.start_processes(_worker, args=(size, _free_port(), steps, cfl, out, True), nprocs=size, start_method="spawn")
    got = np.load(out)
    sc = _scene(cfl)
    w = world_from_scene(sc)
    for _ in range(steps):
        w.step(sc.dt)
    ref = w.fluid.particles
    w.close()
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    for r in range(size):
        assert np.load(out + f".bytes{r}.npy")[0] > 0


@pytest.mark.gpu
@pytest.mark.parametrize("cfl", [False, True])
def test_device_slab_two_ranks_equal_world(tmp_path, cfl):
    """Two gloo ranks on persistent rank worlds with the device-side exchange
    (pack / unpack kernels, fixed-size buffers with in-band counts, order
    tags, halo and migrants in place): 50 steps of the 4k dam break gathered
    equal the single-domain GPU world bit for bit."""
    from phi_eng_b200.world import world_from_scene

    steps, size = 50, 2
    out = str(tmp_path / "state.npy")
    mp.start_processes(_worker, args=(size, _free_port(), steps, cfl, out, "device"), nprocs=size,
                       start_method="spawn")
    got = np.load(out)
    sc = _scene(cfl)
    w = world_from_scene(sc)
    for _ in range(steps):
        w.step(sc.dt)
    ref = w.fluid.particles
    w.close()
    assert got.shape == ref.shape
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    for r in range(size):
        assert np.load(out + f".bytes{r}.npy")[0] > 0


@pytest.mark.gpu
def test_device_slab_single_rank_equals_world():
    from phi_eng_b200.slab import DeviceSlabRun
    from phi_eng_b200.world import world_from_scene

    sc = _scene(False)
    run = DeviceSlabRun(sc, 0, 1)
    w = world_from_scene(sc)
    for _ in range(30):
        run.step(sc.dt)
        w.step(sc.dt)
    got = run.gather()
    run.close()
    ref = w.fluid.particles
    w.close()
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


@pytest.mark.gpu
def test_device_slab_reports_overflow(tmp_path):
    """A halo buffer too small for the edge is reported (the pack kernel
    drops what does not fit and flags it), not written past its end."""
    steps, size = 2, 2
    out = str(tmp_path / "state.npy")
    mp.start_processes(_worker, args=(size, _free_port(), steps, False, out, "device", 8), nprocs=size,
                       start_method="spawn")
    assert [int(np.load(out + f".ok{r}.npy")[0]) for r in range(size)] == [0, 0]


@pytest.mark.gpu
@pytest.mark.parametrize("size,cfl", [(2, False), (3, True)])
def test_local_slab_group_equals_world(size, cfl):
    """All ranks in one process on the one GPU, buffers moved by device
    copies: the same bit-identical result as the process-group ranks."""
    from phi_eng_b200.slab import LocalSlabGroup
    from phi_eng_b200.world import world_from_scene

    sc = _scene(cfl)
    g = LocalSlabGroup(sc, size)
    w = world_from_scene(sc)
    for _ in range(40):
        g.step(sc.dt)
        w.step(sc.dt)
    got = g.gather()
    assert g.copied > 0
    g.close()
    ref = w.fluid.particles
    w.close()
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


@pytest.mark.gpu
def test_local_slab_group_migrants_cross_the_edge():
    """An edge four columns behind the initial dam front: the collapsing
    column pushes particles across it into the right rank, and the gathered
    state still equals the single-domain world bit for bit."""
    import torch

    from phi_eng_b200.slab import LocalSlabGroup, cell_column
    from phi_eng_b200.world import world_from_scene

    sc = _scene(False)
    h = float(sc.config.smoothing_length)
    cx = cell_column(torch.from_numpy(np.ascontiguousarray(sc.xy[:, 0])), h)
    edge = int(cx.max()) - 4
    g = LocalSlabGroup(sc, 2, edges=[-(1 << 40), edge, 1 << 40])
    w = world_from_scene(sc)
    before = [set(r.owned()[1].tolist()) for r in g.ranks]
    for _ in range(80):  # on the oracle, 43 particles have crossed by step 60
        g.step(sc.dt)
        w.step(sc.dt)
    after = [set(r.owned()[1].tolist()) for r in g.ranks]
    got = g.gather()
    g.close()
    ref = w.fluid.particles
    w.close()
    assert len(after[1] - before[1]) > 0  # particles moved into the right rank
    assert sum(len(a) for a in after) == sc.n
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


@pytest.mark.gpu
def test_local_slab_group_reports_a_full_owned_region():
    """An owned region with no spare slot (the right rank's own_cap is its
    initial count): the migrants that arrive there find no free slot, which
    is reported (the unpack drops them), not written past the region."""
    import torch

    from phi_eng_b200.slab import LocalSlabGroup, cell_column

    sc = _scene(False)
    h = float(sc.config.smoothing_length)
    cx = cell_column(torch.from_numpy(np.ascontiguousarray(sc.xy[:, 0])), h)
    edge = int(cx.max()) - 4
    n_right = int((cx >= edge).sum())
    # the right rank starts full (own_cap = its initial count; the left one's region is its own count)
    g = LocalSlabGroup(sc, 2, edges=[-(1 << 40), edge, 1 << 40], own_cap=n_right)
    for _ in range(80):
        g.step(sc.dt)
    with pytest.raises(RuntimeError):
        g.ranks[1].owned()
    g.close()


@pytest.mark.gpu
def test_local_slab_group_tolerance_mode_equals_world():
    """In the tolerance mode too, the rank worlds visit every owned
    particle's neighbours in the single domain's order, so the gathered
    state equals a single-domain tolerance-mode world bit for bit."""
    from phi_eng_b200 import _abi
    from phi_eng_b200.slab import LocalSlabGroup
    from phi_eng_b200.world import world_from_scene

    sc = _scene(False)
    g = LocalSlabGroup(sc, 3, precision=_abi.TOLERANCE)
    w = world_from_scene(sc)
    w.precision = _abi.TOLERANCE
    for _ in range(40):
        g.step(sc.dt)
        w.step(sc.dt)
    got = g.gather()
    g.close()
    ref = w.fluid.particles
    w.close()
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
