#!/usr/bin/env python
"""SPH dam-break throughput on B200: particle-updates/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload dam_break_1m|dam_break_4k|batch_512]
                    [--precision tolerance|exact] [--no-cpu-baseline]

One step = one fluid substep of the whole scene (sort, ranges, density,
force + integrate + walls). Default workload: 1,048,576 particles (1024 x
1024 lattice, 1 mm spacing) in a 10 x 6 m box, dt = 0.4 h / sqrt(gamma k),
in the tolerance mode (phieng_sph_set_precision: reassociated density and
force sums within the stated tolerances); the exact mode (the reference's
f32 arithmetic bit for bit) is timed beside it, and so are steps 150..200 of
the workload and the 512-scene batched workload.
Inputs are resident in HBM when timing starts; L2 is flushed (256 MiB write)
between timed steps, outside the timed events. Under torchrun each rank runs
its own replica of the scene (the single-scene step has no exchange), so
scaling is weak and `value` sums all ranks' particle-updates over the max
rank time.

--impl reference times the reference's CPU step on the host: the reference
is Rust (no toolchain here), so its algorithm runs as the C++ restatement
in oracle/ in the reference's own in-place order, single-threaded like the
reference's fluid step.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from phi_eng_b200 import scenes  # noqa: E402

METRIC = "particle-updates/s"
HBM_FALLBACK = 6650.0

# Algorithmic bytes per particle-update of the reference's step (payload
# bytes only, each array read or written once, neighbour re-reads not
# counted): K1 hash 16 (read pos 8, write key + id 8); K2 radix sort of
# (key, id) with 3 digit passes 16 * 3 + 4 = 52; K3 cell ranges 4 + 8 c
# (c = occupied cells per particle, 0.25 at rest density) = 6; K4 reorder 32
# (read pos + vel 16, write them sorted 16); K5 density 16 (read pos 8,
# write density + pressure 8); K6 force + integrate 40 (read pos, vel,
# density, pressure 24, write pos + vel 16). Whole step 162.
ALG_BYTES = dict(hash=16, sort=52, ranges=6, reorder=32, density=16, force=40)
STEP_ALG_BYTES = sum(ALG_BYTES.values())
# the bench's phases: the library's sort phase holds K2-K4, its force pass
# also writes the next keys (K1, counted nowhere else)
PHASE_ALG_BYTES = dict(sort_ranges=ALG_BYTES["sort"] + ALG_BYTES["ranges"] + ALG_BYTES["reorder"],
                       density=ALG_BYTES["density"], force_integrate=ALG_BYTES["force"] + ALG_BYTES["hash"])

# What this implementation moves per particle (each of its arrays read or
# written once; B/N = buckets per particle):
#   sort:    scan: read counts twice, write start + cursor, clear counts
#            (20 B per bucket); place: read id 4 + key 4, write (key, id) 8;
#            fixup: read (key, id) 8 + start 8, write (key, id) 8,
#            gather state 16 -> write pos 8 + vel 8                = 72 + 20 B/N
#   density: read pos 8 + key 4; write (density, q) 8 + pressure 4,
#            three 32-bit neighbour-row masks 12                    = 36
#   force:   read pos 8, vel 8, (density, q) 8, key 4, id 4, masks 12;
#            write state 16 + next key 4                             = 64
DENSITY_BYTES = 36
FORCE_BYTES = 64
# DRAM bytes (read + write) of one launch of the named kernel on the named
# workload and precision mode, from an ncu capture (profiles/).
PROFILED_TRAFFIC = {("dam_break_1m", "exact", "force_integrate"): 48.333312e6 + 1.921792e6,
                    ("dam_break_1m", "tolerance", "force_integrate"): 48.337664e6 + 1.710592e6}
PROFILED_TRAFFIC_3D = {"force_integrate": 85.545216e6 + 14.838528e6}  # 100^3 3D dam break
KERNELS_PER_STEP = 5  # single-pass scan, place, fixup, density, force


def sort_bytes(buckets_per_particle: float) -> float:
    return 72 + 20 * buckets_per_particle


def hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK, "fallback"


class ClockSampler:
    """SM clock and clock-event (throttle) reasons, polled through NVML every
    ~2 ms on a background thread while the timed steps run (read-only)."""

    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, cuda_index: int):
        self.cuda_index = cuda_index
        self.samples = []
        self._stop = None
        self._thread = None
        self.error = None

    def _handle(self):
        import pynvml
        import torch

        pynvml.nvmlInit()
        try:
            uuid = str(torch.cuda.get_device_properties(self.cuda_index).uuid)
            return pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return pynvml.nvmlDeviceGetHandleByIndex(self.cuda_index)

    def start(self):
        import threading

        try:
            import pynvml

            h = self._handle()
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
        except Exception as e:  # no NVML: report that instead of numbers
            self.error = f"nvml unavailable: {e}"
            return
        self._stop = threading.Event()

        def run():
            while not self._stop.is_set():
                try:
                    sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                    rs = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.samples.append((sm, rs))
                except Exception:
                    pass
                self._stop.wait(0.002)

        self._thread = threading.Thread(target=run, daemon=True)
        self._thread.start()

    def stop(self):
        if self._thread is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [self.error or "not sampled"], "samples": 0}
        self._stop.set()
        self._thread.join()
        sm = [x[0] for x in self.samples]
        reasons = set()
        for _, r in self.samples:
            for bit, name in self.REASONS.items():
                if r & bit:
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvml"}


WORKLOADS = ("dam_break_1m", "dam_break_4k", "batch_512")


def make_scene(name: str):
    return {"dam_break_1m": scenes.dam_break_1m, "dam_break_4k": scenes.dam_break_4k}[name]()


def workload_scenes(name: str) -> list:
    if name == "batch_512":
        from phi_eng_b200 import batch

        return batch.batched_scenes(512)
    return [make_scene(name)]


def workload_desc(name: str, scs) -> str:
    sc = scs[0]
    n = sum(s.n for s in scs)
    if len(scs) > 1:
        return (f"{name}: {len(scs)} independent dam-break scenes, {n} particles in total "
                f"({min(s.n for s in scs)}..{max(s.n for s in scs)} per scene), one CUDA graph per step, "
                f"h={sc.config.smoothing_length:g} m, Tait gamma={sc.config.gamma:g}, dt={sc.dt:.4e} s")
    return (f"{sc.name}: {sc.n} particles, SPH dam break, h={sc.config.smoothing_length:g} m, "
            f"Tait gamma={sc.config.gamma:g} k={sc.config.stiffness:g}, XSPH {sc.config.viscosity:g}, "
            f"dt={sc.dt:.4e} s, {len(sc.boxes)} static box walls")


class Job:
    """The workload on this GPU: one world, or a batch of scene worlds."""

    def __init__(self, scs):
        from phi_eng_b200.batch import Batch
        from phi_eng_b200.world import world_from_scene

        self.scs = scs
        self.n = sum(sc.n for sc in scs)
        self.dt = scs[0].dt
        if len(scs) == 1:
            self.batch = None
            self.world = world_from_scene(scs[0])
        else:
            self.batch = Batch.from_scenes(scs)
            self.world = self.batch.world

    def close(self):
        if self.batch is not None:
            self.batch.close()
            for w in self.batch.worlds:
                w.close()
        else:
            self.world.close()


def oracle_world(sc):
    from oracle import oracle as orc

    o = orc.OracleWorld(cap=max(sc.n, 4096), libm_pow=True)
    o.set_gravity(*sc.gravity)
    for (px, py, hx, hy) in sc.boxes:
        o.add_box(px, py, hx, hy, (1.0, 0.0, -0.0, 1.0))
    for (px, py, r) in sc.circles:
        o.add_circle(px, py, r, (1.0, 0.0, -0.0, 1.0))
    o.set_config(sc.config)
    o.add_particles(sc.xy, sc.phases)
    return o


def cpu_baseline(scs, budget_s: float = 15.0, max_steps: int = 20):
    """The reference algorithm on one host core (oracle, in-place order), on
    the first scene(s) of the workload for a bounded number of steps."""
    from oracle import oracle as orc

    t = 0.0
    updates = 0
    used = 0
    steps_done = 0
    for sc in scs:
        o = oracle_world(sc)
        dt = o.steps(sc.dt, 1, orc.REF_SEQ)
        steps = 1
        left = budget_s / max(len(scs), 1) if len(scs) > 1 else budget_s
        more = int(min(max_steps - 1, max(0, left / max(dt, 1e-9) - 1)))
        if more > 0:
            dt += o.steps(sc.dt, more, orc.REF_SEQ)
            steps += more
        t += dt
        updates += sc.n * steps
        used += 1
        steps_done = steps
        if t > budget_s:
            break
    what = (f"first {steps_done} steps of {scs[0].name} ({scs[0].n} particles)" if used == 1 else
            f"{used} of {len(scs)} scenes, about {steps_done} steps each")
    return {"value": updates / t, "unit": METRIC, "cores": 1, "kind": "port",
            "sample": f"{what}, reference (in-place) order, C++ restatement of fluid.rs, 1 thread, {t:.1f} s"}


def run_reference(args, rank: int):
    if rank != 0:
        return
    scs = workload_scenes(args.workload)
    if len(scs) > 1:
        line = cpu_baseline(scs, budget_s=120.0, max_steps=max(args.steps, 1))
        out = {"impl": "reference", "metric": METRIC, "value": line["value"], "unit": METRIC, "n_gpus": args.gpus,
               "steps": args.steps, "warmup": 0, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f32", "data": "synthetic",
               "config": {"workload": workload_desc(args.workload, scs), "particles": sum(x.n for x in scs)},
               "cpu_baseline": line,
               "e2e": {"value": line["value"], "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(out), flush=True)
        return
    sc = scs[0]
    from oracle import oracle as orc

    o = oracle_world(sc)
    t1 = o.steps(sc.dt, 1, orc.REF_SEQ)  # one step to size the run
    budget = 150.0
    warm = max(0, min(args.warmup - 1, int(budget * 0.1 / max(t1, 1e-9))))
    if warm:
        o.steps(sc.dt, warm, orc.REF_SEQ)
    k = max(1, min(args.steps, int(budget / max(t1, 1e-9))))
    t = o.steps(sc.dt, k, orc.REF_SEQ)
    v = sc.n * k / t
    sample = (f"{k} timed steps (of {args.steps} requested; capped to ~{budget:.0f} s) after {warm + 1} warm-up "
              f"steps of {sc.name}, reference (in-place) order, C++ restatement of fluid.rs (the Rust reference "
              f"cannot be built here), 1 thread: the reference fluid step is single-threaded")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": args.gpus,
            "steps": k, "warmup": warm + 1, "ms_per_step": 1000.0 * t / k, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload_desc(args.workload, scs), "particles": sc.n},
            "cpu_baseline": {"value": v, "unit": METRIC, "cores": 1, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def apply_tuning(world, mode: str, dt: float) -> dict:
    """Launch tuning for the timed world: "auto" = the cached / shipped
    choice for this GPU and workload, else the defaults; "tune" = run the
    autotuner now (outside the timed region); "default" = the defaults."""
    from phi_eng_b200 import autotune as at

    if mode == "tune":
        world.step_n(dt, 2)
        r = at.autotune(world, dt, steps=10)
        return dict(r["tuning"], source="autotuned in this run")
    if mode == "auto":
        t = at.lookup(world)
        if t:
            at.apply(world, t)
            return dict(t, source="tuning table")
    return dict(at.DEFAULT, source="defaults")


def closure_line(sc, precision: int) -> dict:
    """The learned closure against the plain fine run on this workload, with
    the shipped weights: 50 coarse steps of 4 dt against 200 fine steps
    (speed and accuracy), under the per-particle jump criterion and under the
    literal rule (max relative density deviation above 3%), and a longer
    horizon of 300 coarse steps (jump criterion) over which the plain dam
    front travels further. Errors are maxima over the recorded instants:
    front error relative to the plain front's travel x_f(t) - x_f(0)
    (x_f = max x, as fluid_dam prints it; also over the instants at which the
    plain front has moved at least h, and at the last instant), kinetic
    energy relative to the plain run's, and the difference in mean
    |rho/rho0 - 1|."""
    from phi_eng_b200 import _abi
    from phi_eng_b200 import closure as cl

    if not os.path.exists(cl.WEIGHTS):
        return {"unavailable": "no trained weights"}
    mlp = cl.Mlp.load(cl.WEIGHTS)

    def run(steps, crit, every):
        r = cl.evaluate(sc, mlp, coarse_steps=steps, threshold=0.03, criterion=crit, record_every=every,
                        precision=precision)
        fp, fc = r["final_plain"], r["final_closure"]
        return {"ratio": r["speedup"], "learned": r["closure_sim_s_per_wall_s"],
                "plain": r["plain_sim_s_per_wall_s"], "accepted": r["accepted"], "fallbacks": r["fallbacks"],
                "front_travel_err": r["front_travel_rel"], "front_travel_err_moved": r["front_travel_rel_moved"],
                "front_travel_err_final": r["front_travel_rel_final"], "front_err_abs_x": r["front_rel"],
                "ke_err": r["ke_rel"], "density_err": r["density_dev_abs"],
                "final": {"plain": {"front": fp["front"], "ke": fp["ke"], "dev_mean": fp["dev_mean"]},
                          "closure": {"front": fc["front"], "ke": fc["ke"], "dev_mean": fc["dev_mean"]}},
                "front_travel_plain": fp["front"] - float(np.max(sc.xy[:, 0])), "coarse_steps": steps}

    out = {"metric": "simulated s per wall s", "dt_ratio": 4, "threshold": 0.03,
           "precision": f"tolerance (fast pair arithmetic, network on {mlp.closure_engine})"
           if precision == _abi.TOLERANCE else "exact (network on mma.sync)"}
    jump = run(50, _abi.CLOSURE_JUMP, 10)
    out.update(jump, criterion="jump (largest per-particle density increase over the coarse step)")
    out["literal_rule"] = dict(run(50, _abi.CLOSURE_COMPRESSION, 10),
                               criterion="max relative density deviation (rho/rho0 - 1) > 3%")
    out["long_horizon"] = dict(run(300, _abi.CLOSURE_JUMP, 50), criterion="jump")
    return out


# 3D (fluid3.rs) chain, bytes per particle of each phase:
#   sort:    place 16 (read key + previous slot id, write key, id); fixup 64
#            + 8 (read key, id, start pair; write key, id; gather pos 16 +
#            vel 16 -> write 32)                                  = 104 + 20 B/N
#   density: read pos 16 + key 4; write (density, q) 8 + pressure 4 + nine
#            32-bit row masks 36                                     = 68
#   force:   read pos 16, vel 16, (density, q) 8, key 4, id 4, masks 36;
#            write pos 16 + vel 16 + next key 4                       = 120
DENSITY3_BYTES = 68
FORCE3_BYTES = 120


def fluid3d_line(steps: int, warmup: int, side: int = 100) -> dict:
    """The 3D step (phieng_world3_*) on a side^3-particle dam break: a block at
    the reference's lattice spacing 0.25 m in a walled tank 2.5 x 1.5 x 1.5
    times its size, the reference's default FluidConfig3 and world step
    dt = 1/60 (its tests' step). Device-timed like the main line (L2 flushed
    between timed steps), with the oracle's in-place CPU step on the
    reference's particle cap (4096) beside it."""
    import torch

    from phi_eng_b200 import _abi
    from phi_eng_b200.world3 import World3, dam_break_3d

    L = side * 0.25
    pts, bodies = dam_break_3d(side, side, side, 0.25, tank=(2.5 * L, 1.5 * L, 1.5 * L))
    n = len(pts)
    w = World3()
    w.fluid.set_cap(n)
    for pos, sh in bodies:
        w.add_static_body(pos, sh)
    assert w.fluid.add_particles(pts) == n
    stream = torch.cuda.Stream()
    w.set_stream(stream.cuda_stream)
    dt = 1.0 / 60.0
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    for _ in range(max(warmup, 3)):
        w.step(dt)
    s0 = w.fluid.particles  # both modes are timed from this state

    def timed():
        w.fluid.set_state(s0)
        for _ in range(3):
            w.step(dt)
        w.set_profiling(True)
        w.step(dt)
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        phases = []
        for k in range(steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            ev[k][0].record(stream)
            w.step(dt)
            ev[k][1].record(stream)
            phases.append(w.phase_times())
        torch.cuda.synchronize()
        w.set_profiling(False)
        return sum(a.elapsed_time(b) for a, b in ev) / steps, np.array(phases).mean(axis=0)

    # the exact mode, then the tolerance mode (the line's value), each from s0
    ms_exact, ph_exact = timed()
    w.precision = _abi.TOLERANCE
    ms, ph = timed()
    buckets = w.status().grid_buckets
    names = ["sort_ranges", "density", "force_integrate"]
    bytes_pp = [104 + 20 * buckets / n, DENSITY3_BYTES, FORCE3_BYTES]
    top = int(np.argmax(ph))
    peak, _ = hbm_peak()
    achieved = bytes_pp[top] * n / (ph[top] / 1000.0) / 1e9
    s = w.fluid.particles
    w.close()
    # the reference's algorithm on the CPU at its particle cap
    from oracle.oracle import REF_SEQ, OracleWorld3

    cpts, cbodies = dam_break_3d(16, 16, 16, 0.25, tank=(10.0, 6.0, 6.0))
    o = OracleWorld3()
    for pos, sh in cbodies:
        o.add_body(1, *pos, sh.hx, sh.hy, sh.hz)
    o.add_particles(cpts)
    o.steps(dt, 2, REF_SEQ)
    k = 20
    secs = o.steps(dt, k, REF_SEQ)
    return {"metric": METRIC, "value": n / (ms / 1000.0), "ms_per_step": ms, "particles": n,
            "workload": f"3D dam break, {side}^3 particles at 0.25 m in a {2.5 * L:g} x {1.5 * L:g} x {1.5 * L:g} m "
                        "tank (floor + 4 walls), FluidConfig3 defaults, dt = 1/60",
            "precision": "tolerance",
            "phases_ms": {nm: float(v) for nm, v in zip(names, ph)}, "buckets": int(buckets),
            "exact_mode": {"value": n / (ms_exact / 1000.0), "ms_per_step": ms_exact,
                           "phases_ms": {nm: float(v) for nm, v in zip(names, ph_exact)}},
            "roofline": {"bound": "hbm", "kernel": names[top], "bytes_per_particle": bytes_pp[top],
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": PROFILED_TRAFFIC_3D.get(names[top]) if side == 100 else None,
                         "traffic_source": "ncu capture of the exact-mode force pass (the tolerance-mode pass "
                                           "reads and writes the same arrays)"},
            "finite": bool(np.isfinite(s).all()),
            "cpu_baseline": {"value": 4096 * k / secs, "unit": METRIC, "cores": 1, "kind": "port",
                             "sample": f"{k} in-place steps of a 4096-particle 3D dam break (the reference's cap)"}}


# kernels per substep of a slab rank: halo pack + unpack, the world's five
# (scan, placement, fixup, density, force), migrant pack + unpack + settle
SLAB_KERNELS_PER_SUBSTEP = 10


def run_slab(args, rank: int, world: int, local_rank: int) -> None:
    """The single scene split in x slabs over the ranks, each a persistent
    rank world with the device-side exchange (pack / unpack kernels, whole
    fixed-size buffers over NCCL point-to-point on the world's stream,
    phi_eng_b200/slab.py DeviceSlabRun); strong scaling. The timed region is
    bracketed by barriers and CUDA events on the default stream; the max over
    ranks is reported."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    from phi_eng_b200.slab import DeviceSlabRun

    torch.cuda.set_device(local_rank)
    dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    from phi_eng_b200 import _abi

    sc = workload_scenes(args.workload)[0]
    run = DeviceSlabRun(sc, rank, world,
                        precision=_abi.TOLERANCE if args.precision == "tolerance" else _abi.EXACT)
    for _ in range(args.warmup):
        run.step(sc.dt)
    torch.cuda.synchronize()
    dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sub0 = run.substeps
    e0.record()
    for _ in range(args.steps):
        run.step(sc.dt)
    e1.record()
    torch.cuda.synchronize()
    t = torch.tensor([e0.elapsed_time(e1)], device="cuda", dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    if rank == 0:
        value = sc.n * args.steps / (total_ms / 1000.0)
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": workload_desc(args.workload, [sc]), "particles": sc.n,
                           "parallelism": f"slab{world}", "l2": "not flushed (inputs move between ranks)"},
                "gpu_launches": SLAB_KERNELS_PER_SUBSTEP * (run.substeps - sub0)}
        print(json.dumps(line), flush=True)
    try:
        run.owned()  # raises if an exchange overflowed
        ok = True
    except RuntimeError:
        ok = False
    run.close()
    dist.barrier()
    dist.destroy_process_group()
    if not ok:
        raise RuntimeError("slab exchange")


def timed_steps(w, dt: float, steps: int, stream, flush, phases: bool = True):
    """Device time of `steps` world steps on `stream` (CUDA events around each
    step, L2 flushed before each one outside the events); returns
    (ms per step list, per-phase ms array of shape (steps, 3) or None)."""
    import torch

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    ph = []
    for k in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        ev[k][0].record(stream)
        w.step(dt)
        ev[k][1].record(stream)
        if phases:
            ph.append(w.phase_times())
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in ev], (np.array(ph) if phases else None)


def roofline_of(phase_ms, n: int, workload: str, precision: str, buckets: int) -> dict:
    """Roofline of the dominant phase's kernel at its algorithmic bytes per
    particle (ALG_BYTES; the force pass is held to the reference's K6 bytes,
    40, although it also writes the next keys), with this implementation's
    own bytes and the profiled DRAM traffic beside it."""
    names = ["sort_ranges", "density", "force_integrate"]
    alg = [PHASE_ALG_BYTES["sort_ranges"], ALG_BYTES["density"], ALG_BYTES["force"]]
    impl = [sort_bytes(buckets / n), DENSITY_BYTES, FORCE_BYTES]
    top = int(np.argmax(phase_ms))
    peak, peak_kind = hbm_peak()
    achieved = alg[top] * n / (phase_ms[top] / 1000.0) / 1e9
    traffic = PROFILED_TRAFFIC.get((workload, precision, names[top]))
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "kernel": names[top], "bytes_per_particle": alg[top],
            "implementation_bytes_per_particle": impl[top],
            "traffic_over_algorithmic": (traffic / (alg[top] * n)) if traffic else None,
            "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
            else "fallback 6650 GB/s"}


def whole_step_of(ms_per_step: float, n: int) -> dict:
    peak, _ = hbm_peak()
    gbs = STEP_ALG_BYTES * n / (ms_per_step / 1000.0) / 1e9
    return {"bytes_per_particle": STEP_ALG_BYTES, "achieved_gbs": gbs, "frac": gbs / peak,
            "bytes": "K1 hash 16 + K2 sort (3 digit passes) 52 + K3 ranges 6 + K4 reorder 32 + K5 density 16 + "
                     "K6 force 40"}


def batch_line(steps: int, warmup: int, tuning_mode: str, cpu: bool, precision: int) -> dict:
    """The batched workload (512 independent scenes, one CUDA graph of the
    step's kernels for all of them per step), device-timed like the main
    line, with the oracle's in-place CPU step on a sample of its scenes."""
    import torch

    from phi_eng_b200 import _abi

    scs = workload_scenes("batch_512")
    job = Job(scs)
    n = job.n
    w = job.world
    w.precision = precision
    tuning = apply_tuning(w, tuning_mode, job.dt)
    stream = torch.cuda.Stream()
    w.set_stream(stream.cuda_stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    for _ in range(max(warmup, 3)):
        w.step(job.dt)
    w.set_profiling(True)
    w.step(job.dt)
    buckets = w.status().grid_buckets
    torch.cuda.synchronize()
    step_ms, ph = timed_steps(w, job.dt, steps, stream, flush)
    ms = sum(step_ms) / steps
    ph_mean = ph.mean(axis=0)
    job.close()
    out = {"metric": METRIC, "value": n / (ms / 1000.0), "ms_per_step": ms, "particles": n,
           "scenes": len(scs), "workload": workload_desc("batch_512", scs), "buckets": int(buckets),
           "tuning": tuning, "precision": "tolerance" if precision == _abi.TOLERANCE else "exact",
           "phases_ms": {k: float(v) for k, v in zip(["sort_ranges", "density", "force_integrate"], ph_mean)},
           "roofline": roofline_of(ph_mean, n, "batch_512",
                                   "tolerance" if precision == _abi.TOLERANCE else "exact", buckets), "whole_step": whole_step_of(ms, n),
           "step_ms_min_max": [float(min(step_ms)), float(max(step_ms))]}
    if cpu:
        sample = [scs[i] for i in range(0, len(scs), 64)]  # 8 scenes spread over the size range
        out["cpu_baseline"] = cpu_baseline(sample, budget_s=15.0, max_steps=10)
    return out


def run_ours(args, rank: int, world: int, local_rank: int):
    import torch

    from phi_eng_b200 import _abi

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist  # noqa: F811
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120))

    scs = workload_scenes(args.workload)
    single = len(scs) == 1
    mode = _abi.TOLERANCE if args.precision == "tolerance" else _abi.EXACT
    job = Job(scs)
    n_total, dt = job.n, job.dt
    w = job.world
    w.precision = mode
    tuning = apply_tuning(w, args.tuning, dt)
    stream = torch.cuda.Stream()
    w.set_stream(stream.cuda_stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    for _ in range(args.warmup):
        w.step(dt)
    w.set_profiling(True)
    w.step(dt)  # capture the profiled graph outside the timed region
    st = w.status()
    buckets = st.grid_buckets
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()

    sampler = ClockSampler(local_rank) if rank == 0 else None
    if sampler:
        sampler.start()
    step_ms, ph = timed_steps(w, dt, args.steps, stream, flush)
    clocks = sampler.stop() if sampler else None
    total_ms = sum(step_ms)
    if dist:
        t = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = n_total * args.steps * world / (total_ms / 1000.0)
    ph_mean = ph.mean(axis=0)
    names = ["sort_ranges", "density", "force_integrate"]
    precision = "tolerance" if mode == _abi.TOLERANCE else "exact"
    roofline = roofline_of(ph_mean, n_total, args.workload, precision, buckets)
    whole = whole_step_of(total_ms / args.steps, n_total)

    # the exact mode (the reference's f32 arithmetic bit for bit) on the same
    # world, from where the timed steps left it
    exact = None
    if single and mode == _abi.TOLERANCE and not args.no_exact:
        w.precision = _abi.EXACT
        for _ in range(3):
            w.step(dt)
        e_ms, e_ph = timed_steps(w, dt, args.steps, stream, flush)
        e_mean = e_ph.mean(axis=0)
        em = sum(e_ms) / args.steps
        exact = {"value": n_total / (em / 1000.0), "ms_per_step": em,
                 "phases_ms": {k: float(v) for k, v in zip(names, e_mean)},
                 "roofline": roofline_of(e_mean, n_total, args.workload, "exact", buckets),
                 "whole_step": whole_step_of(em, n_total)}
        w.precision = mode

    # later in the flow: steps 150..200 of the 200-step workload
    late = None
    if single and args.workload == "dam_break_1m" and not args.no_late:
        w.set_profiling(False)
        done = args.warmup + 1 + args.steps + (args.steps + 3 if exact else 0)
        if done < 150:
            w.step_n(dt, 150 - done)
        w.set_profiling(True)
        w.step(dt)
        l_ms, l_ph = timed_steps(w, dt, 50, stream, flush)
        lm = sum(l_ms) / 50
        late = {"steps": f"{max(done, 150) + 1}..{max(done, 150) + 50}", "ms_per_step": lm,
                "value": n_total / (lm / 1000.0),
                "phases_ms": {k: float(v) for k, v in zip(names, l_ph.mean(axis=0))},
                "front_x": w.front_metrics()[0]}

    # end to end through the C ABI from host buffers: the worlds are built and
    # filled from host arrays outside the timed region; timed: the first
    # step's upload of the particles, K x (phieng_world_step +
    # phieng_sph_front_metrics, an 8-byte read-back), and the final read-back
    # of every particle's state (phieng_world_fluid_get)
    job.close()
    job2 = Job(scs)
    from phi_eng_b200 import autotune as at

    job2.world.precision = mode
    at.apply(job2.world, tuning)
    if job2.batch is None:
        job2.world.reserve(n_total)  # device arrays allocated before the clock starts
    # the read-back lands in page-locked host memory, as the inputs do (the
    # library keeps its host mirror page-locked)
    final = torch.empty((n_total, 4), dtype=torch.float32, pin_memory=True).numpy()
    # every step's metric lands in its own page-locked slot (an 8-byte copy
    # per step, enqueued behind the step; no host wait between steps)
    ring = torch.zeros((args.steps, 2), dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for k in range(args.steps):
        job2.world.step(dt)
        job2.world.front_metrics_async(ring[k])
    job2.world.fluid.read_into(final)
    fronts = [job2.world.decode_front_metrics(ring[k])[0] for k in range(args.steps)]
    e2e_s = time.perf_counter() - t0
    if not all(math.isfinite(f) for f in fronts):
        raise RuntimeError("non-finite front metric")
    job2.close()
    e2e = {"value": n_total * args.steps * world / e2e_s, "unit": METRIC,
           "h2d_bytes_per_step": int(n_total * 16 / args.steps),
           "d2h_bytes_per_step": int(8 + final.nbytes / args.steps),
           "timed": "(device arrays reserved beforehand) first-step upload of the page-locked host particle "
                    "arrays, grid plan and graph capture + K x (phieng_world_step + "
                    "phieng_sph_front_metrics_async: the step's metric reduced and copied, 8 bytes, into its "
                    "own page-locked slot without a host wait) + phieng_world_fluid_get into page-locked memory "
                    "+ decoding the K metrics, wall clock"}
    if dist:
        t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e["value"] = n_total * args.steps * world / float(t.item())

    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base = cpu_baseline(scs)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": workload_desc(args.workload, scs), "particles": n_total, "parallelism":
                           ("replicas" if world > 1 else "single"),
                           "l2": "flushed between timed steps (256 MiB write, outside the timed events)",
                           "buckets": int(buckets), "tuning": tuning, "precision": precision},
                "roofline": roofline, "whole_step": whole,
                "phases_ms": {n: float(v) for n, v in zip(names, ph_mean)},
                "cpu_baseline": base, "e2e": e2e, "gpu_launches": KERNELS_PER_STEP * args.steps,
                "clocks": clocks}
        if exact:
            line["exact_mode"] = exact
        if late:
            line["late_flow"] = late
        if args.batch and world == 1 and args.workload != "batch_512":
            line["batch"] = batch_line(args.steps, args.warmup, args.tuning, not args.no_cpu_baseline, mode)
        if args.closure and single and world == 1:
            line["closure"] = closure_line(scs[0], mode)
        if args.fluid3d and world == 1:
            line["fluid3d"] = fluid3d_line(args.steps, args.warmup)
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="dam_break_1m", choices=list(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tuning", choices=["auto", "default", "tune"], default="auto")
    ap.add_argument("--parallel", choices=["replicas", "slab"], default="replicas",
                    help="N > 1: independent replicas (weak scaling) or the scene split in x slabs (strong)")
    ap.add_argument("--no-closure", dest="closure", action="store_false",
                    help="skip the learned-closure comparison line")
    ap.add_argument("--no-fluid3d", dest="fluid3d", action="store_false",
                    help="skip the 3D step line")
    ap.add_argument("--no-batch", dest="batch", action="store_false",
                    help="skip the batched-scenes line (512 scenes)")
    ap.add_argument("--precision", choices=["tolerance", "exact"], default="tolerance",
                    help="arithmetic of the plain passes (phieng_sph_set_precision); the other mode is "
                         "timed beside it unless --no-exact")
    ap.add_argument("--no-exact", action="store_true", help="skip the exact-mode comparison")
    ap.add_argument("--no-late", action="store_true", help="skip the late-flow timing (steps 150..200)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.parallel == "slab" and world > 1:
        run_slab(args, rank, world, local_rank)
        return
    run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
