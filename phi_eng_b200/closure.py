"""Learned closure for coarse SPH steps (no counterpart in the reference).

A per-particle network (16 -> 64 -> 64 -> 2, SiLU, BF16 weights on the tensor
cores, FP32 accumulate; phi_eng_b200/csrc/sph_mlp.cu) reads 16 neighbour
aggregate features (sph_device.cuh: feat_pair / wall_feature / feat_finish)
and predicts the displacement correction, in units of the smoothing length h,
that makes one substep of ratio * dt track ratio plain substeps of dt. The
plain step is both the teacher and the fallback: training pairs come from the
plain GPU step only, and a coarse step whose density check exceeds the
threshold is undone and replaced by plain substeps (phieng_sph_closure_step).

Device memory is held in torch tensors (allocation only); every computation
runs in the library's kernels.
"""
from __future__ import annotations

import ctypes as C
import os
import time

import numpy as np

from . import _abi
from .world import World2, world_from_scene

NPARAMS = _abi.MLP_PARAMS
NNORM = _abi.MLP_NORM
NFEAT = _abi.MLP_FEATURES


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("the closure needs a CUDA device")
    return torch


def _fp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class Mlp:
    """The closure network on the current CUDA device."""

    def __init__(self, seed: int = 0x5EED):
        self._lib = _abi.load()
        self._h = self._lib.phieng_mlp_new(seed)
        if not self._h:
            raise MemoryError("phieng_mlp_new")
        self.check()

    def check(self) -> None:
        e = self._lib.phieng_mlp_status(self._h)
        if e != _abi.OK:
            raise RuntimeError(f"closure network error {e}")

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.phieng_mlp_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- parameters ----
    def get(self):
        p = np.zeros(NPARAMS, np.float32)
        nrm = np.zeros(NNORM, np.float32)
        if self._lib.phieng_mlp_get_params(self._h, _fp(p), _fp(nrm)) != 1:
            self.check()
        return p, nrm

    def set(self, params, norm) -> None:
        p = np.ascontiguousarray(params, np.float32)
        nrm = np.ascontiguousarray(norm, np.float32)
        assert p.size == NPARAMS and nrm.size == NNORM
        if self._lib.phieng_mlp_set_params(self._h, _fp(p), _fp(nrm)) != 1:
            self.check()

    @property
    def steps(self) -> int:
        return int(self._lib.phieng_mlp_step_count(self._h))

    def save(self, path: str, **meta) -> None:
        p, nrm = self.get()
        np.savez(path, params=p, norm=nrm, **meta)

    @classmethod
    def load(cls, path: str) -> "Mlp":
        z = np.load(path)
        m = cls()
        m.set(z["params"], z["norm"])
        return m

    # ---- compute (device tensors, on torch's current stream) ----
    def _on_current_stream(self):
        torch = _torch()
        self._lib.phieng_mlp_set_stream(self._h, C.c_void_p(torch.cuda.current_stream().cuda_stream))
        return torch

    def forward(self, x):
        torch = self._on_current_stream()
        x = x.contiguous()
        y = torch.empty((x.shape[0], 2), dtype=torch.float32, device=x.device)
        if self._lib.phieng_mlp_forward(self._h, x.data_ptr(), x.shape[0], y.data_ptr()) != 1:
            self.check()
        return y

    def grad(self, x, t, batch: int, seed: int, it: int):
        self._on_current_stream()
        g = np.zeros(NPARAMS, np.float32)
        loss = np.zeros(1, np.float32)
        if self._lib.phieng_mlp_grad(self._h, x.data_ptr(), t.data_ptr(), x.shape[0], batch, seed, it, _fp(g),
                                     _fp(loss)) != 1:
            self.check()
            raise ValueError("phieng_mlp_grad rejected its arguments")
        return float(loss[0]), g

    def train(self, x, t, batch: int = 65536, iters: int = 20000, lr: float = 1e-3, seed: int = 0xC105E):
        self._on_current_stream()
        hist = np.zeros(iters, np.float32)
        if self._lib.phieng_mlp_train(self._h, x.data_ptr(), t.data_ptr(), x.shape[0], batch, iters, lr, seed,
                                      _fp(hist)) != 1:
            self.check()
            raise ValueError("phieng_mlp_train rejected its arguments")
        return hist


def sample_indices(npairs: int, batch: int, seed: int, it: int):
    torch = _torch()
    out = torch.empty(batch, dtype=torch.int32, device="cuda")
    lib = _abi.load()
    if lib.phieng_mlp_sample_indices(npairs, batch, seed, it, out.data_ptr(), None) != 1:
        raise ValueError("sample_indices")
    torch.cuda.synchronize()
    return out.cpu().numpy().view(np.uint32).astype(np.int64)


# ---------------------------------------------------------------- training data
def generate_pairs(scs, ratio: int = 4, samples: int = 40, every: int = 50, first: int = 50):
    """(features, targets) on the device from the plain GPU step.

    The scenes advance together as one batch with the plain fine step dt
    (the scenes' own). At `samples` instants (after `first` steps, then every
    `every` steps) the state S is saved and
      features  = closure inputs at S for a coarse step ratio * dt
      coarse    = one plain substep of ratio * dt from S
      fine      = ratio plain substeps of dt from S (the trajectory continues here)
      target    = (x_fine - x_coarse) / h   per particle
    """
    from .batch import Batch

    torch = _torch()
    lib = _abi.load()
    dt = scs[0].dt
    h = float(scs[0].config.smoothing_length)
    assert all(s.dt == dt and float(s.config.smoothing_length) == h for s in scs)
    b = Batch.from_scenes(scs)
    w = b.world
    n = sum(s.n for s in scs)
    S = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    Cs = torch.empty_like(S)
    F = torch.empty_like(S)
    X = torch.empty((samples * n, NFEAT), dtype=torch.float32, device="cuda")
    T = torch.empty((samples * n, 2), dtype=torch.float32, device="cuda")
    ws = torch.cuda.current_stream().cuda_stream
    w.set_stream(ws)
    b.step(dt, first)
    for k in range(samples):
        if k:
            b.step(dt, every)
        w.get_state_device(S.data_ptr(), n)
        w.features(ratio * dt, X[k * n:(k + 1) * n].data_ptr())
        b.step(ratio * dt, 1)
        w.get_state_device(Cs.data_ptr(), n)
        w.set_state_device(S.data_ptr(), n)
        b.step(dt, ratio)
        w.get_state_device(F.data_ptr(), n)
        if lib.phieng_mlp_targets(F.data_ptr(), Cs.data_ptr(), n, 1.0 / h, T[k * n:(k + 1) * n].data_ptr(),
                                  C.c_void_p(ws)) != 1:
            raise RuntimeError("phieng_mlp_targets")
    w.sync()
    w.set_stream(None)
    b.close()
    return X, T


def normalisation(X, T, sample: int = 1 << 20, seed: int = 7) -> np.ndarray:
    """mu / isd of the features and out_scale of the targets (per-component
    standard deviations) from a seeded subsample of the pairs."""
    torch = _torch()
    g = torch.Generator(device="cpu").manual_seed(seed)
    idx = torch.randint(0, X.shape[0], (min(sample, X.shape[0]),), generator=g).to(X.device)
    xs = X[idx].double().cpu().numpy()
    ts = T[idx].double().cpu().numpy()
    mu = xs.mean(0)
    sd = xs.std(0)
    isd = np.where(sd > 1e-12, 1.0 / np.maximum(sd, 1e-12), 1.0)
    osc = np.maximum(ts.std(0), 1e-12)
    return np.concatenate([mu, isd, osc]).astype(np.float32)


def train_closure(scs=None, ratio: int = 4, samples: int = 40, every: int = 50, batch: int = 65536,
                  iters: int = 20000, lr: float = 1e-3, seed: int = 0x5EED, log=print):
    """Generate pairs on the batched scenes (the 256-scene slice of the batched
    workload by default) and train a network; returns (mlp, info)."""
    from .batch import batched_scenes

    torch = _torch()
    scs = scs if scs is not None else batched_scenes(256)
    t0 = time.perf_counter()
    X, T = generate_pairs(scs, ratio=ratio, samples=samples, every=every)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    mlp = Mlp(seed)
    p, _ = mlp.get()
    nrm = normalisation(X, T)
    mlp.set(p, nrm)
    hist = mlp.train(X, T, batch=batch, iters=iters, lr=lr, seed=seed ^ 0xA5A5)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    info = dict(pairs=int(X.shape[0]), scenes=len(scs), gen_s=t1 - t0, train_s=t2 - t1,
                loss_first=float(hist[:100].mean()), loss_last=float(hist[-100:].mean()), iters=iters,
                batch=batch, lr=lr, ratio=ratio)
    if log:
        log(f"closure training: {info}")
    del X, T
    return mlp, info


# ---------------------------------------------------------------- evaluation
def fluid_metrics(w: World2, mass: float, rho0: float):
    """Dam front (max x), kinetic energy sum(m |v|^2 / 2) and density
    deviation statistics of the current state (density recomputed for it)."""
    st = w.fluid.particles
    w.debug_forces()  # refreshes density / pressure for the current state
    dens, _ = w.fluid.density_pressure()
    rel = dens.astype(np.float64) / rho0 - 1.0
    v2 = st[:, 2].astype(np.float64) ** 2 + st[:, 3].astype(np.float64) ** 2
    return dict(front=float(np.max(st[:, 0])), ke=float(0.5 * mass * v2.sum()),
                dev_mean=float(np.abs(rel).mean()), comp_max=float(max(rel.max(), 0.0)))


def evaluate(scene, mlp: Mlp, coarse_steps: int = 50, ratio: int = 4, threshold: float = 0.03,
             criterion: int = _abi.CLOSURE_JUMP, record_every: int = 1, timing_reps: int = 1):
    """Closure (coarse_steps x ratio*dt) against the plain run (coarse_steps x
    ratio plain steps of dt) from the same initial state.

    Errors are taken at every `record_every`-th coarse step: dam-front
    position (relative to the plain front, and relative to the plain front's
    travel), kinetic energy, mean |rho/rho0 - 1| and the largest compression.
    Speed: simulated seconds per wall second of each run, timed on the device
    with CUDA events over the whole run (metric reads excluded; the closure's
    per-step density check and its host read are included)."""
    torch = _torch()
    dt = scene.dt
    mass = float(scene.config.particle_mass)
    rho0 = float(scene.config.rest_density)
    # ---- trajectories with metrics
    plain = world_from_scene(scene)
    clo = world_from_scene(scene)
    clo.set_closure(mlp, ratio, threshold, criterion)
    rows = []
    stats = _abi.PhiengClosureStats()
    for k in range(1, coarse_steps + 1):
        plain.step_n(dt, ratio)
        clo.closure_step(dt, 1, stats)
        if k % record_every == 0 or k == coarse_steps:
            rows.append((k, fluid_metrics(plain, mass, rho0), fluid_metrics(clo, mass, rho0)))
    x0 = float(np.max(scene.xy[:, 0]))
    err = dict(front_rel=0.0, front_travel_rel=0.0, ke_rel=0.0, density_dev_abs=0.0, comp_max_abs=0.0)
    for k, p, c in rows:
        err["front_rel"] = max(err["front_rel"], abs(c["front"] - p["front"]) / abs(p["front"]))
        travel = abs(p["front"] - x0)
        if travel > 0:
            err["front_travel_rel"] = max(err["front_travel_rel"], abs(c["front"] - p["front"]) / travel)
        if p["ke"] > 0:
            err["ke_rel"] = max(err["ke_rel"], abs(c["ke"] - p["ke"]) / p["ke"])
        err["density_dev_abs"] = max(err["density_dev_abs"], abs(c["dev_mean"] - p["dev_mean"]))
        err["comp_max_abs"] = max(err["comp_max_abs"], abs(c["comp_max"] - p["comp_max"]))
    plain.close()
    clo.close()

    # ---- timing (fresh worlds, no metric reads)
    def timed(run):
        best = None
        for _ in range(timing_reps):
            w = world_from_scene(scene)
            s = torch.cuda.Stream()
            w.set_stream(s.cuda_stream)
            if run is not None:
                w.set_closure(mlp, ratio, threshold, criterion)
            w.step_n(dt, 1)  # upload, plan, first graphs outside the timing
            w.sync()
            st = _abi.PhiengClosureStats()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(s):
                e0.record(s)
                if run is None:
                    w.step_n(dt, coarse_steps * ratio)
                else:
                    w.closure_step(dt, coarse_steps, st)
                e1.record(s)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            best = (ms, st) if best is None or ms < best[0] else best
            w.close()
        return best

    t_plain, _ = timed(None)
    t_clo, st = timed("closure")
    sim = coarse_steps * ratio * dt
    out = dict(
        particles=scene.n, coarse_steps=coarse_steps, ratio=ratio, dt_fine=dt, threshold=threshold,
        criterion="jump" if criterion == _abi.CLOSURE_JUMP else "compression",
        plain_ms=t_plain, closure_ms=t_clo,
        plain_sim_s_per_wall_s=sim / (t_plain / 1000.0), closure_sim_s_per_wall_s=sim / (t_clo / 1000.0),
        speedup=t_plain / t_clo, accepted=int(stats.accepted), fallbacks=int(stats.fallbacks),
        max_check=float(stats.max_check), timed_fallbacks=int(st.fallbacks), **err,
        final_plain=rows[-1][1], final_closure=rows[-1][2])
    return out


# ---------------------------------------------------------------- command line
WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "closure_mlp.npz")


def _main(argv=None) -> None:
    """python -m phi_eng_b200.closure train [--out PATH] [--iters N] ...
    python -m phi_eng_b200.closure eval [--weights PATH] [--workload NAME] ..."""
    import argparse
    import json

    from . import scenes as S

    ap = argparse.ArgumentParser(prog="python -m phi_eng_b200.closure")
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--out", default=WEIGHTS)
    t.add_argument("--scenes", type=int, default=256)
    t.add_argument("--samples", type=int, default=40)
    t.add_argument("--every", type=int, default=50)
    t.add_argument("--iters", type=int, default=20000)
    t.add_argument("--batch", type=int, default=65536)
    t.add_argument("--lr", type=float, default=1e-3)
    t.add_argument("--seed", type=lambda s: int(s, 0), default=0x5EED)
    e = sub.add_parser("eval")
    e.add_argument("--weights", default=WEIGHTS)
    e.add_argument("--workload", default="dam_break_1m", choices=["dam_break_1m", "dam_break_4k"])
    e.add_argument("--coarse-steps", type=int, default=50)
    e.add_argument("--threshold", type=float, default=0.03)
    e.add_argument("--criterion", choices=["jump", "compression"], default="jump")
    e.add_argument("--zero", action="store_true", help="evaluate a zero network (no correction)")
    a = ap.parse_args(argv)
    if a.cmd == "train":
        from .batch import batched_scenes

        mlp, info = train_closure(batched_scenes(a.scenes), samples=a.samples, every=a.every, batch=a.batch,
                                  iters=a.iters, lr=a.lr, seed=a.seed, log=None)
        os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
        mlp.save(a.out, **{k: np.asarray(v) for k, v in info.items()})
        print(json.dumps(dict(trained=a.out, **info)))
        return
    sc = S.dam_break_1m() if a.workload == "dam_break_1m" else S.dam_break_4k()
    mlp = Mlp() if a.zero else Mlp.load(a.weights)
    crit = _abi.CLOSURE_JUMP if a.criterion == "jump" else _abi.CLOSURE_COMPRESSION
    r = evaluate(sc, mlp, coarse_steps=a.coarse_steps, threshold=a.threshold, criterion=crit)
    print(json.dumps(dict(workload=a.workload, weights=None if a.zero else a.weights, **r)))


if __name__ == "__main__":
    _main()
