"""Slab decomposition of one scene over ranks (phi_eng_b200/slab.py).

CPU: gloo ranks (2 and 3) each step their slab plus a 2-cell halo on an
oracle engine defined here (Jacobi order, the order the GPU computes) and
exchange halos and migrating particles with their neighbours; the gathered
state equals the single-domain oracle run bit for bit, with and without CFL
substeps. Both the engine-based protocol (SlabRun: halo, step, migrants)
and the device ranks' one-exchange protocol (restated here as
OneExchangeRank) are checked this way.
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
    # inner slabs span two halo bands: a migrant from the far side never lands in the near band
    assert all(e[r + 1] - e[r] >= 4 for r in range(1, 3))
    # many ranks on a narrow block: the edges still keep that width, and the outer slabs absorb the rest
    e8 = slab_edges(sc.xy, h, 8)
    assert all(e8[r + 1] - e8[r] >= 4 for r in range(1, 7))
    assert e8 == sorted(e8)


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


class OneExchangeRank:
    """The protocol of the device slab ranks (phi_eng_b200/slab.py
    DeviceSlabRun, sph_slab.cu) restated on the CPU with the oracle engine:
    once before the first step each rank sends each neighbour the particles
    within HALO_CELLS columns of their shared edge; then every substep it
    steps owned ∪ halo in ascending global id and keeps the owned results,
    packs for each side the particles that left the slab towards it
    (migrants) and the stayers within HALO_CELLS columns of that edge (halo),
    exchanges once, adds the received migrants to its own particles, and
    takes as each side's halo the received halo rows plus its own migrants to
    that side."""

    def __init__(self, sc, rank, size, edges=None):
        import torch

        from phi_eng_b200.slab import HALO_CELLS, cell_column, slab_edges

        self.sc, self.rank, self.size = sc, rank, size
        self.h = float(sc.config.smoothing_length)
        self.band = HALO_CELLS
        self.cell = lambda x: cell_column(torch.from_numpy(np.ascontiguousarray(x, np.float32)), self.h).numpy()
        edges = edges or slab_edges(sc.xy, self.h, size)
        self.lo, self.hi = edges[rank], edges[rank + 1]
        cx = self.cell(sc.xy[:, 0])
        mine = np.nonzero((cx >= self.lo) & (cx < self.hi))[0]
        self.ids = mine.astype(np.int64)
        self.st = np.zeros((mine.shape[0], 4), np.float32)
        self.st[:, :2] = sc.xy[mine]
        self.has = (rank > 0, rank < size - 1)
        self.halo = [(np.zeros((0, 4), np.float32), np.zeros(0, np.int64)) for _ in range(2)]
        self.engine = OracleEngine(sc)
        self.primed = False
        self.migrated = 0

    def _exchange(self, out):
        import torch
        import torch.distributed as dist

        got = [None, None]
        peers = [(k, self.rank + (1 if k else -1)) for k in (0, 1) if self.has[k]]
        cnt = {k: torch.zeros(1, dtype=torch.int64) for k, _ in peers}
        ops = []
        for k, p in peers:
            ops += [dist.P2POp(dist.isend, torch.tensor([out[k].shape[0]], dtype=torch.int64), p),
                    dist.P2POp(dist.irecv, cnt[k], p)]
        if ops:
            for q in dist.batch_isend_irecv(ops):
                q.wait()
        ops, buf = [], {}
        for k, p in peers:
            buf[k] = torch.zeros((int(cnt[k].item()), 6), dtype=torch.float64)
            if out[k].shape[0]:
                ops.append(dist.P2POp(dist.isend, torch.from_numpy(out[k]), p))
            if buf[k].shape[0]:
                ops.append(dist.P2POp(dist.irecv, buf[k], p))
        if ops:
            for q in dist.batch_isend_irecv(ops):
                q.wait()
        for k, _ in peers:
            got[k] = buf[k].numpy()
        return got

    @staticmethod
    def _rows(st, ids, migrant):
        r = np.zeros((st.shape[0], 6), np.float64)  # float64 carries the f32 state and the id exactly
        r[:, :4] = st
        r[:, 4] = ids
        r[:, 5] = 1.0 if migrant else 0.0
        return r

    def _pack(self, migrants):
        cx = self.cell(self.st[:, 0])
        gl = self.has[0] & (cx < self.lo) if migrants else np.zeros(cx.shape, bool)
        gr = self.has[1] & ~gl & (cx >= self.hi) if migrants else np.zeros(cx.shape, bool)
        stay = ~(gl | gr)
        hl = stay & self.has[0] & (cx < self.lo + self.band)
        hr = stay & self.has[1] & (cx >= self.hi - self.band)
        out = []
        for go, hb in ((gl, hl), (gr, hr)):
            out.append(np.concatenate([self._rows(self.st[go], self.ids[go], True),
                                       self._rows(self.st[hb], self.ids[hb], False)]))
        mig = [(self.st[gl], self.ids[gl]), (self.st[gr], self.ids[gr])]
        self.st, self.ids = self.st[stay], self.ids[stay]
        return out, mig

    def _unpack(self, got, mig):
        for k in (0, 1):
            if not self.has[k]:
                continue
            r = got[k]
            m = r[:, 5] > 0
            self.migrated += int(m.sum())
            self.st = np.concatenate([self.st, r[m, :4].astype(np.float32)])
            self.ids = np.concatenate([self.ids, r[m, 4].astype(np.int64)])
            hs = np.concatenate([r[~m, :4].astype(np.float32), mig[k][0]])
            hi = np.concatenate([r[~m, 4].astype(np.int64), mig[k][1]])
            self.halo[k] = (hs, hi)

    def _substep(self, dt):
        import torch

        st = np.concatenate([self.st, self.halo[0][0], self.halo[1][0]])
        ids = np.concatenate([self.ids, self.halo[0][1], self.halo[1][1]])
        order = np.argsort(ids, kind="stable")
        new = self.engine.step(torch.from_numpy(np.ascontiguousarray(st[order])), dt).numpy()
        back = np.empty_like(new)
        back[order] = new
        self.st = back[: self.ids.shape[0]].copy()
        out, mig = self._pack(True)
        self._unpack(self._exchange(out), mig)

    def step(self, dt):
        import torch
        import torch.distributed as dist

        from phi_eng_b200.slab import cfl_count

        if not self.primed:
            out, mig = self._pack(False)
            self._unpack(self._exchange(out), mig)
            self.primed = True
        cfg = self.sc.config
        n_sub = 1
        if float(cfg.cfl) > 0 and int(cfg.max_substeps) > 1:
            v = np.sqrt(self.st[:, 2].astype(np.float32) ** 2 + self.st[:, 3].astype(np.float32) ** 2)
            t = torch.tensor([float(np.nan_to_num(v, nan=0.0).max()) if v.size else 0.0], dtype=torch.float32)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            n_sub = cfl_count(cfg, dt, float(t.item()))
        sub = float(np.float32(dt) / np.float32(n_sub))
        for _ in range(n_sub):
            self._substep(sub)

    def gather(self):
        import torch.distributed as dist

        parts = [None] * self.size
        dist.all_gather_object(parts, (self.ids, self.st))
        out = np.zeros((sum(p[0].shape[0] for p in parts), 4), np.float32)
        for i, s in parts:
            out[i] = s
        return out


def _front_edges(sc):
    """Two slabs split four columns behind the dam front: the collapsing
    column pushes particles across the edge."""
    import torch

    from phi_eng_b200.slab import cell_column

    cx = cell_column(torch.from_numpy(np.ascontiguousarray(sc.xy[:, 0])), float(sc.config.smoothing_length))
    return [-(1 << 40), int(cx.max()) - 4, 1 << 40]


def _one_exchange_worker(rank, size, port, steps, cfl, out, front=False):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=size)
    sc = _scene(cfl)
    r = OneExchangeRank(sc, rank, size, edges=_front_edges(sc) if front else None)
    for _ in range(steps):
        r.step(sc.dt)
    full = r.gather()
    if rank == 0:
        np.save(out, full)
    np.save(out + f".mig{rank}.npy", np.array([r.migrated], np.int64))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("size,cfl,front", [(2, False, False), (3, False, False), (2, True, False),
                                             (2, False, True)])
def test_one_exchange_protocol_equals_single_domain(tmp_path, size, cfl, front):
    """The device ranks' one-exchange protocol, on gloo ranks with the
    oracle as each rank's engine: 80 steps gathered equal the single-domain
    oracle run bit for bit; particles changed rank in every case but the
    two-rank split at the column's middle."""
    steps = 80
    out = str(tmp_path / "state.npy")
    mp.start_processes(_one_exchange_worker, args=(size, _free_port(), steps, cfl, out, front), nprocs=size,
                       start_method="spawn")
    got = np.load(out)
    sc = _scene(cfl)
    o = sims.load_scene(sims.OracleSim(orc.JACOBI), sc)
    o.step(sc.dt, steps)
    np.testing.assert_array_equal(got, o.state())
    migrated = sum(int(np.load(out + f".mig{r}.npy")[0]) for r in range(size))
    assert migrated > 0 or (size == 2 and not cfl and not front)
