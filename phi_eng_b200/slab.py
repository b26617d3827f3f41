"""One SPH scene split over ranks in x slabs, with halo exchange.

Rank r owns the particles whose cell column cx = floor(x / h) lies in
[edges[r], edges[r+1]). Every substep:

  1. halo: each rank sends its neighbours the particles in the two cell
     columns next to the shared edge (2h: the neighbours of a particle reach
     one cell, and their densities need one more);
  2. the rank steps its owned particles together with the received halo, in
     ascending global id, on its engine (one substep, no CFL splitting);
  3. it keeps the owned particles' new states (those are exactly the
     single-domain results: every neighbour, and every neighbour's density,
     is present, and the in-cell visit order is ascending global id) and
     drops the halo's;
  4. migration: owned particles whose new cell column left the slab go to
     the adjacent rank (a particle moves less than one cell per substep).

With CFL substeps enabled the substep count comes from the global maximum
speed (one all-reduce), as the single-domain step computes it. Results are
bit-identical to the single-domain step.

Communication is neighbour point-to-point (torch.distributed isend / irecv:
NCCL over NVLink for CUDA tensors, gloo for CPU tensors): first the counts,
then one float32 payload per direction, [x, y, vx, vy, id bits].
"""
from __future__ import annotations

import numpy as np

HALO_CELLS = 2


def cell_column(x, h: float):
    """floor(x / h) in f32 arithmetic, saturated to i32 (NaN -> 0), as the
    kernels and the reference compute it (fluid.rs:350-356)."""
    import torch

    q = torch.floor(x.to(torch.float32) / torch.tensor(np.float32(h), device=x.device))
    q = torch.nan_to_num(q, nan=0.0, posinf=2147483647.0, neginf=-2147483648.0)
    return q.clamp(-2147483648.0, 2147483647.0).to(torch.int64)


def slab_edges(xy: np.ndarray, h: float, size: int) -> list:
    """Cell-column edges that split the particles into `size` slabs of equal
    count (each inner slab at least two halo bands, 2 * HALO_CELLS columns,
    wide)."""
    import torch

    cx = cell_column(torch.from_numpy(np.ascontiguousarray(xy[:, 0])), h).numpy()
    cols = np.sort(cx)
    edges = [-(1 << 40)]
    for r in range(1, size):
        e = int(cols[min(len(cols) - 1, (len(cols) * r) // size)])
        e = max(e, edges[-1] + 2 * HALO_CELLS if r > 1 else e)
        edges.append(e)
    edges.append(1 << 40)
    return edges


def cfl_count(cfg, dt: float, vmax: float) -> int:
    """cfl_substeps (fluid.rs:562-588) from a global maximum speed, in the
    f32 arithmetic of the single-domain step."""
    f = np.float32
    mx = max(int(cfg.max_substeps), 1)
    if not (f(cfg.cfl) > 0) or mx <= 1:
        return 1
    h = max(f(cfg.smoothing_length), f(1e-6))
    rho0 = max(f(cfg.rest_density), f(1e-6))
    k = max(f(cfg.stiffness), f(0))
    c0 = np.sqrt(k) if f(cfg.gamma) == f(1) else np.sqrt(f(cfg.gamma) * k * rho0)
    speed = f(c0) + f(vmax)
    if not np.isfinite(speed) or speed <= f(1e-6):
        return 1
    dt_max = f(cfg.cfl) * h / speed
    if not np.isfinite(dt_max) or dt_max <= 0:
        return 1
    q = np.ceil(f(dt) / dt_max)
    if q != q:
        return 1
    return int(max(1, min(float(q), mx)))


class GpuEngine:
    """The rank's engine: one library world whose particle set is replaced
    from device memory each substep. `state` may live on the host (gloo
    exchange) or on the GPU (NCCL exchange); the result comes back on the
    same device."""

    def __init__(self, scene, cap: int):
        from .world import world_from_scene

        self.world = world_from_scene(_empty_scene(scene))
        self.world.fluid.config = _no_cfl(scene.config)
        self.world.fluid.set_cap(cap)

    def close(self) -> None:
        self.world.close()

    def step(self, state, dt: float):
        import torch

        from .closure import torch_stream_handle

        home = state.device
        dev = state if state.is_cuda else state.to("cuda")
        n = dev.shape[0]
        w = self.world
        w.set_stream(torch_stream_handle())  # ordered after the torch ops that built `state`
        w.load_state_device(dev.data_ptr(), n)
        w.step(dt)
        out = torch.empty_like(dev)
        if n:
            w.get_state_device(out.data_ptr(), n)
        w.sync()
        return out if home == out.device else out.to(home)


class DeviceSlabRun:
    """This rank's part of one scene on a persistent rank world with the
    exchange on the device (phieng_sph_slab_*): the world holds the owned
    slots and two halo regions at a fixed capacity (unused slots are NaN
    particles, which no neighbour walk visits, so the step's CUDA graph never
    changes), buckets are ordered by global id (order tags), and each
    substep packs, exchanges whole fixed-size buffers, unpacks, steps, then
    does the same for the migrants. With NCCL the buffers move on the
    world's stream and a substep never waits on the host; with CFL substeps
    one all-reduced maximum speed is read per step. gloo moves host copies of
    the same buffers (tests on one GPU)."""

    def __init__(self, scene, rank: int, size: int, edges=None, own_cap: int | None = None,
                 halo_cap: int | None = None, precision: int | None = None):
        import torch

        from . import _abi
        from .closure import torch_stream_handle
        from .world import world_from_scene

        self.scene = scene
        self.rank, self.size = rank, size
        self.h = float(scene.config.smoothing_length)
        self.edges = edges or slab_edges(scene.xy, self.h, size)
        self.lo, self.hi = self.edges[rank], self.edges[rank + 1]
        xy = torch.from_numpy(np.ascontiguousarray(scene.xy, dtype=np.float32))
        cx = cell_column(xy[:, 0], self.h)
        ids = torch.nonzero((cx >= self.lo) & (cx < self.hi)).squeeze(1)
        n0 = int(ids.shape[0])
        if halo_cap is None:
            # twice the fullest halo band at the start (the HALO_CELLS columns on either side of an inner
            # edge), plus a margin; an exchange that overflows is reported, never written past the end
            band = 0
            for e in self.edges[1:-1]:
                band = max(band, int(((cx >= e - HALO_CELLS) & (cx < e)).sum()),
                           int(((cx >= e) & (cx < e + HALO_CELLS)).sum()))
            halo_cap = 2 * band + 1024
        halo_cap = max(1, min(int(halo_cap), max(scene.n, 1)))
        if own_cap is None:
            own_cap = min(max(scene.n, 1), n0 + n0 // 8 + 2 * halo_cap)
        own_cap = max(int(own_cap), n0)
        self.own_cap, self.halo_cap = own_cap, halo_cap
        cap = own_cap + 4 * halo_cap
        st = torch.zeros((cap, 4), dtype=torch.float32)
        st[:, :2] = float("nan")
        st[:n0, :2] = xy[ids]
        tags = torch.full((cap,), -1, dtype=torch.int32)  # PHIENG_SPH_SLAB_FREE
        tags[:n0] = ids.to(torch.int32)
        self.world = world_from_scene(_empty_scene(scene))
        self.world.fluid.config = _no_cfl(scene.config)
        self.world.fluid.set_cap(cap)
        if precision is not None:
            self.world.precision = precision  # the owned results equal a single-domain world's in either mode
        self.world.set_stream(torch_stream_handle())
        self._lib = _abi.load()
        st_d, tags_d = st.cuda(), tags.cuda()
        self.world.load_state_device(st_d.data_ptr(), cap)
        if self._lib.phieng_sph_set_order(self.world._h, tags_d.data_ptr(), cap) != 1:
            self.world.check()
            raise RuntimeError("phieng_sph_set_order")
        nbytes = 16 + 20 * halo_cap
        self.send = [torch.zeros(nbytes, dtype=torch.uint8, device="cuda") for _ in range(2)]
        self.recv = [torch.zeros(nbytes, dtype=torch.uint8, device="cuda") for _ in range(2)]
        self.left = rank - 1 if rank > 0 else None
        self.right = rank + 1 if rank < size - 1 else None
        nb = (1 if self.left is not None else 0) | (2 if self.right is not None else 0)
        i32 = lambda v: int(max(-(1 << 31), min((1 << 31) - 1, v)))
        ok = self._lib.phieng_sph_slab_setup(self.world._h, i32(self.lo), i32(self.hi), nb, own_cap, halo_cap,
                                             self.send[0].data_ptr(), self.send[1].data_ptr(),
                                             self.recv[0].data_ptr(), self.recv[1].data_ptr())
        if ok != 1:
            self.world.check()
            raise RuntimeError("phieng_sph_slab_setup")
        torch.cuda.current_stream().synchronize()  # st_d / tags_d were read on the stream
        self.backend = None
        if size > 1:
            import torch.distributed as dist

            if dist.is_available() and dist.is_initialized():
                self.backend = dist.get_backend()
        self.vmax = torch.zeros(1, dtype=torch.float32, device="cuda")
        self.comm_bytes = 0
        self.substeps = 0
        self.primed = False

    def close(self) -> None:
        self.world.close()

    def _exchange(self):
        if self.size == 1:
            return
        import torch
        import torch.distributed as dist

        peers = [(k, p) for k, p in ((0, self.left), (1, self.right)) if p is not None]
        if self.backend == "nccl":
            ops = []
            for k, p in peers:
                ops += [dist.P2POp(dist.isend, self.send[k], p), dist.P2POp(dist.irecv, self.recv[k], p)]
            for q in dist.batch_isend_irecv(ops):
                q.wait()
        else:
            hs = {k: self.send[k].cpu() for k, _ in peers}
            hr = {k: torch.empty_like(hs[k]) for k, _ in peers}
            ops = []
            for k, p in peers:
                ops += [dist.P2POp(dist.isend, hs[k], p), dist.P2POp(dist.irecv, hr[k], p)]
            for q in dist.batch_isend_irecv(ops):
                q.wait()
            for k, _ in peers:
                self.recv[k].copy_(hr[k])
        self.comm_bytes += sum(self.send[k].numel() for k, _ in peers)

    def _call(self, name: str, *args) -> None:
        if getattr(self._lib, name)(self.world._h, *args) != 1:
            self.world.check()
            raise RuntimeError(name)

    def pack(self, phase: int) -> None:
        self._call("phieng_sph_slab_pack", phase)

    def unpack(self, phase: int) -> None:
        self._call("phieng_sph_slab_unpack", phase)

    def local_vmax(self):
        """Max |v| over the owned particles (device tensor of one float)."""
        self._call("phieng_sph_slab_vmax", self.vmax.data_ptr())
        return self.vmax

    def prime(self) -> None:
        """The first halo (before the first step)."""
        self.pack(0)
        self._exchange()
        self.unpack(0)
        self.primed = True

    def _substep(self, dt: float) -> None:
        self.substeps += 1
        self.world.step(dt)
        self.pack(1)
        self._exchange()
        self.unpack(1)

    def step(self, dt: float) -> None:
        """One world step of dt (CFL substeps from the global maximum speed)."""
        if not self.primed:
            self.prime()
        cfg = self.scene.config
        n_sub = 1
        if float(cfg.cfl) > 0 and int(cfg.max_substeps) > 1:
            v = self.local_vmax()
            if self.size > 1:
                import torch.distributed as dist

                if self.backend == "nccl":
                    dist.all_reduce(v, op=dist.ReduceOp.MAX)
                else:
                    v = v.cpu()
                    dist.all_reduce(v, op=dist.ReduceOp.MAX)
            n_sub = cfl_count(cfg, dt, float(v.item()))
        sub = float(np.float32(dt) / np.float32(n_sub))
        for _ in range(n_sub):
            self._substep(sub)

    def owned(self):
        """(state [k][4], global ids [k]) of this rank's particles (host)."""
        st = np.zeros((self.own_cap, 4), np.float32)
        tg = np.zeros(self.own_cap, np.uint32)
        k = self._lib.phieng_sph_slab_owned(self.world._h, st.ctypes.data, tg.ctypes.data, self.own_cap)
        if self._lib.phieng_sph_slab_status(self.world._h) != 1:
            raise RuntimeError("a slab exchange overflowed its buffers or the owned slots")
        return st[:k], tg[:k].astype(np.int64)

    def gather(self):
        """Every particle's state in global id order (all ranks)."""
        st, ids = self.owned()
        if self.size == 1:
            out = np.zeros((ids.shape[0], 4), np.float32)
            out[ids] = st
            return out
        import torch.distributed as dist

        parts = [None] * self.size
        dist.all_gather_object(parts, (ids, st))
        n = sum(p[0].shape[0] for p in parts)
        out = np.zeros((n, 4), np.float32)
        for i, s in parts:
            out[i] = s
        return out


class LocalSlabGroup:
    """All ranks of a slab decomposition in one process on one GPU: the host
    runs each phase on every rank world in turn and moves the exchange
    buffers with device-to-device copies (no kernel waits on another rank).
    Bit-identical to the single-domain step, like the ranks of a real run;
    used to test the decomposition without a process group and to measure
    what the device-side exchange adds per substep."""

    def __init__(self, scene, size: int, halo_cap: int | None = None, edges=None, own_cap: int | None = None,
                 precision: int | None = None):
        edges = edges or slab_edges(scene.xy, float(scene.config.smoothing_length), size)
        self.scene = scene
        self.ranks = [DeviceSlabRun(scene, r, size, edges=edges, halo_cap=halo_cap, own_cap=own_cap,
                                    precision=precision) for r in range(size)]
        self.copied = 0

    def close(self) -> None:
        for r in self.ranks:
            r.close()

    def _exchange(self) -> None:
        rk = self.ranks
        for i, r in enumerate(rk):
            if r.left is not None:
                r.recv[0].copy_(rk[i - 1].send[1])
                self.copied += r.recv[0].numel()
            if r.right is not None:
                r.recv[1].copy_(rk[i + 1].send[0])
                self.copied += r.recv[1].numel()

    def _phase(self, phase: int) -> None:
        for r in self.ranks:
            r.pack(phase)
        self._exchange()
        for r in self.ranks:
            r.unpack(phase)

    def _substep(self, dt: float) -> None:
        for r in self.ranks:
            r.world.step(dt)
        self._phase(1)

    def step(self, dt: float) -> None:
        import torch

        if not self.ranks[0].primed:
            self._phase(0)
            for r in self.ranks:
                r.primed = True
        cfg = self.scene.config
        n_sub = 1
        if float(cfg.cfl) > 0 and int(cfg.max_substeps) > 1:
            v = torch.stack([r.local_vmax().clone() for r in self.ranks]).max()
            n_sub = cfl_count(cfg, dt, float(v.item()))
        sub = float(np.float32(dt) / np.float32(n_sub))
        for _ in range(n_sub):
            self._substep(sub)

    def gather(self):
        parts = [r.owned() for r in self.ranks]
        n = sum(p[1].shape[0] for p in parts)
        out = np.zeros((n, 4), np.float32)
        for st, ids in parts:
            out[ids] = st
        return out


def _empty_scene(scene):
    import copy

    s = copy.copy(scene)
    s.xy = np.zeros((0, 2), np.float32)
    s.phases = None
    return s


def _no_cfl(cfg):
    from ._abi import FluidConfig2Ffi
    import ctypes as C

    c = FluidConfig2Ffi()
    C.memmove(C.byref(c), C.byref(cfg), C.sizeof(cfg))
    c.cfl = 0.0
    c.max_substeps = 1
    return c


def _pack(state, ids):
    import torch

    return torch.cat([state, ids.to(torch.int32).view(torch.float32).unsqueeze(1)], 1)


def _unpack(buf):
    import torch

    return buf[:, :4].contiguous(), buf[:, 4].contiguous().view(torch.int32).to(torch.int64)


class SlabRun:
    """This rank's part of one scene (owned particles, their global ids)."""

    def __init__(self, scene, rank: int, size: int, engine=None, device: str = "cpu", edges=None):
        import torch

        self.scene = scene
        self.rank, self.size = rank, size
        self.device = device
        self.h = float(scene.config.smoothing_length)
        self.edges = edges or slab_edges(scene.xy, self.h, size)
        self.lo, self.hi = self.edges[rank], self.edges[rank + 1]
        xy = torch.from_numpy(np.ascontiguousarray(scene.xy, dtype=np.float32))
        cx = cell_column(xy[:, 0], self.h)
        mine = (cx >= self.lo) & (cx < self.hi)
        ids = torch.nonzero(mine).squeeze(1)
        st = torch.zeros((ids.shape[0], 4), dtype=torch.float32)
        st[:, :2] = xy[ids]
        self.ids = ids.to(device)
        self.state = st.to(device)
        self.engine = engine if engine is not None else GpuEngine(scene, cap=max(scene.n, 1))
        self.comm_bytes = 0

    # ---- neighbour exchange ----
    def _exchange(self, to_left, to_right):
        """Send packed rows to the neighbours, receive theirs (variable sizes)."""
        import torch
        import torch.distributed as dist

        left = self.rank - 1 if self.rank > 0 else None
        right = self.rank + 1 if self.rank < self.size - 1 else None
        dev = self.device
        cnt = {}
        ops = []
        for peer, buf in ((left, to_left), (right, to_right)):
            if peer is None:
                continue
            s = torch.tensor([buf.shape[0]], dtype=torch.int64, device=dev)
            r = torch.zeros(1, dtype=torch.int64, device=dev)
            cnt[peer] = r
            ops += [dist.P2POp(dist.isend, s, peer), dist.P2POp(dist.irecv, r, peer)]
        if ops:
            for q in dist.batch_isend_irecv(ops):
                q.wait()
        got = {}
        ops = []
        for peer, buf in ((left, to_left), (right, to_right)):
            if peer is None:
                continue
            k = int(cnt[peer].item())
            got[peer] = torch.empty((k, 5), dtype=torch.float32, device=dev)
            if buf.shape[0]:
                ops.append(dist.P2POp(dist.isend, buf.contiguous(), peer))
                self.comm_bytes += buf.numel() * 4
            if k:
                ops.append(dist.P2POp(dist.irecv, got[peer], peer))
        if ops:
            for q in dist.batch_isend_irecv(ops):
                q.wait()
        empty = torch.empty((0, 5), dtype=torch.float32, device=dev)
        return got.get(left, empty), got.get(right, empty)

    def _substep(self, dt: float):
        import torch

        cx = cell_column(self.state[:, 0], self.h)
        packed = _pack(self.state, self.ids)
        to_l = packed[cx < self.lo + HALO_CELLS] if self.size > 1 else packed[:0]
        to_r = packed[cx >= self.hi - HALO_CELLS] if self.size > 1 else packed[:0]
        from_l, from_r = self._exchange(to_l, to_r) if self.size > 1 else (packed[:0], packed[:0])
        hl_s, hl_i = _unpack(from_l)
        hr_s, hr_i = _unpack(from_r)
        ids = torch.cat([self.ids, hl_i, hr_i])
        st = torch.cat([self.state, hl_s, hr_s])
        order = torch.argsort(ids)
        new = self.engine.step(st[order].contiguous(), dt).to(self.device)
        owned = order < self.ids.shape[0]  # rows that came from this rank's own particles
        self.ids = ids[order][owned]
        self.state = new[owned]
        # migration
        if self.size > 1:
            cx = cell_column(self.state[:, 0], self.h)
            go_l, go_r = cx < self.lo, cx >= self.hi
            if self.rank == 0:
                go_l = torch.zeros_like(go_l)
            if self.rank == self.size - 1:
                go_r = torch.zeros_like(go_r)
            packed = _pack(self.state, self.ids)
            in_l, in_r = self._exchange(packed[go_l], packed[go_r])
            keep = ~(go_l | go_r)
            a_s, a_i = _unpack(in_l)
            b_s, b_i = _unpack(in_r)
            ids = torch.cat([self.ids[keep], a_i, b_i])
            st = torch.cat([self.state[keep], a_s, b_s])
            order = torch.argsort(ids)
            self.ids, self.state = ids[order], st[order].contiguous()

    def step(self, dt: float):
        """One world step of dt (CFL substeps from the global max speed)."""
        import torch

        cfg = self.scene.config
        n_sub = 1
        if float(cfg.cfl) > 0 and int(cfg.max_substeps) > 1:
            v = torch.sqrt(self.state[:, 2] ** 2 + self.state[:, 3] ** 2)
            v = torch.nan_to_num(v, nan=0.0)
            vmax = v.max() if v.numel() else torch.zeros((), device=self.device)
            vmax = vmax.reshape(1).to(torch.float32)
            if self.size > 1:
                import torch.distributed as dist

                dist.all_reduce(vmax, op=dist.ReduceOp.MAX)
            n_sub = cfl_count(cfg, dt, float(vmax.item()))
        sub = float(np.float32(dt) / np.float32(n_sub))
        for _ in range(n_sub):
            self._substep(sub)

    def gather(self):
        """Every particle's state in global id order (all ranks)."""
        import torch

        if self.size == 1:
            return self.state.cpu().numpy()
        import torch.distributed as dist

        parts = [None] * self.size
        dist.all_gather_object(parts, (self.ids.cpu().numpy(), self.state.cpu().numpy()))
        n = sum(p[0].shape[0] for p in parts)
        out = np.zeros((n, 4), np.float32)
        for ids, st in parts:
            out[ids] = st
        return out


def bench_local(workload: str = "dam_break_1m", ranks: int = 2, steps: int = 20, warmup: int = 3,
                precision: str = "tolerance") -> dict:
    """Device time per step of the single-domain world and of `ranks` rank
    worlds run one after another on this GPU (LocalSlabGroup), split into the
    rank worlds' steps and the exchange (pack, buffer copies, unpack); CUDA
    events on the current stream, L2 not flushed."""
    import torch

    from . import scenes
    from .closure import torch_stream_handle
    from .world import world_from_scene

    from . import _abi

    mode = _abi.TOLERANCE if precision == "tolerance" else _abi.EXACT
    sc = {"dam_break_1m": scenes.dam_break_1m, "dam_break_4k": scenes.dam_break_4k}[workload]()
    w = world_from_scene(sc)
    w.precision = mode
    w.set_stream(torch_stream_handle())
    for _ in range(warmup):
        w.step(sc.dt)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        w.step(sc.dt)
    e1.record()
    e1.synchronize()
    single = e0.elapsed_time(e1) / steps
    w.close()

    g = LocalSlabGroup(sc, ranks, precision=mode)
    for _ in range(warmup):
        g.step(sc.dt)
    torch.cuda.synchronize()

    def n_substeps():
        if float(sc.config.cfl) > 0 and int(sc.config.max_substeps) > 1:
            v = torch.stack([r.local_vmax().clone() for r in g.ranks]).max()
            return cfl_count(sc.config, sc.dt, float(v.item()))
        return 1

    # LocalSlabGroup.step with CUDA events around the rank worlds' steps and the exchange
    marks = []
    substeps = 0
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(steps):
        n_sub = n_substeps()
        sub = float(np.float32(sc.dt) / np.float32(n_sub))
        for _ in range(n_sub):
            substeps += 1
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            ev[0].record()
            for r in g.ranks:
                r.world.step(sub)
            ev[1].record()
            g._phase(1)
            ev[2].record()
            marks.append(ev)
    t1.record()
    t1.synchronize()
    total = t0.elapsed_time(t1) / steps
    world = sum(e[0].elapsed_time(e[1]) for e in marks)
    exch = sum(e[1].elapsed_time(e[2]) for e in marks)
    # the same exchange captured once in a CUDA graph (all ranks' packs, the buffer copies, all
    # unpacks): its device time without the host's per-call launch latency
    cap_stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    for r in g.ranks:  # outside the capture: switching streams synchronises the old one
        r.world.set_stream(cap_stream.cuda_stream)
    gr = torch.cuda.CUDAGraph()
    with torch.cuda.graph(gr, stream=cap_stream):
        g._phase(1)
    for r in g.ranks:
        r.world.set_stream(torch_stream_handle())
    torch.cuda.synchronize()
    gexch = 0.0
    gsub = 0
    for _ in range(steps):
        n_sub = n_substeps()
        sub = float(np.float32(sc.dt) / np.float32(n_sub))
        for _ in range(n_sub):
            gsub += 1
            for r in g.ranks:
                r.world.step(sub)
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record()
            gr.replay()
            a1.record()
            a1.synchronize()
            gexch += a0.elapsed_time(a1)
    rows = int(sum(r.own_cap for r in g.ranks))
    halo = [r.halo_cap for r in g.ranks]
    status = all(r._lib.phieng_sph_slab_status(r.world._h) == 1 for r in g.ranks)
    gathered = g.gather()
    g.close()
    # the graph-replayed substeps continue the same trajectory: still the single domain's, bit for bit
    w = world_from_scene(sc)
    w.precision = mode
    for _ in range(warmup + 2 * steps):
        w.step(sc.dt)
    same = bool(np.array_equal(gathered.view(np.uint32), w.fluid.particles.view(np.uint32)))
    w.close()
    return {"workload": workload, "precision": precision, "particles": sc.n, "ranks": ranks, "steps": steps,
            "substeps": substeps,
            "single_ms_per_step": single, "ranks_ms_per_step": total,
            "rank_worlds_ms_per_step": world / steps, "exchange_ms_per_step": exch / steps,
            "exchange_us_per_substep": 1000.0 * exch / substeps,
            "exchange_graph_us_per_substep": 1000.0 * gexch / gsub,
            "owned_slots": rows, "halo_cap": halo, "buffer_bytes": 16 + 20 * halo[0], "clean": status,
            "bit_identical_to_single_domain": same}


def main(argv=None) -> None:
    import argparse
    import json

    ap = argparse.ArgumentParser(description="slab decomposition on one GPU: rank worlds run in turn")
    ap.add_argument("cmd", choices=["bench"])
    ap.add_argument("--workload", default="dam_break_1m")
    ap.add_argument("--ranks", type=int, default=2)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--precision", choices=["tolerance", "exact"], default="tolerance")
    a = ap.parse_args(argv)
    print(json.dumps(bench_local(a.workload, a.ranks, a.steps, a.warmup, a.precision)), flush=True)


if __name__ == "__main__":
    main()
