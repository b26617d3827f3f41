#!/usr/bin/env python
"""SPH dam-break throughput on B200: particle-updates/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload dam_break_1m|dam_break_4k] [--no-cpu-baseline]

One step = one fluid substep of the whole scene (sort, ranges, density,
force + integrate + walls). Default workload: 1,048,576 particles (1024 x
1024 lattice, 1 mm spacing) in a 10 x 6 m box, dt = 0.4 h / sqrt(gamma k).
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

# Algorithmic bytes per particle of each phase (every array read or written
# once; neighbour re-reads not counted). B/N = buckets per particle.
#   sort:    scan: read counts twice, write start + cursor, clear counts
#            (20 B per bucket); place: read id 4 + key 4, write (key, id) 8;
#            fixup: read (key, id) 8 + start 8, write (key, id) 8,
#            gather state 16 -> write pos 8 + vel 8                = 72 + 20 B/N
#   density: read pos 8 + key 4, write (density, q) 8 + pressure 4   = 24
#   force:   read pos 8, vel 8, (density, q) 8, key 4, id 4;
#            write state 16 + next key 4                             = 52
DENSITY_BYTES = 24
FORCE_BYTES = 52
KERNELS_PER_STEP = 6  # scan reduce, scan down, place, fixup, density, force


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
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_scene(name: str):
    return {"dam_break_1m": scenes.dam_break_1m, "dam_break_4k": scenes.dam_break_4k}[name]()


def workload_desc(sc) -> str:
    return (f"{sc.name}: {sc.n} particles, SPH dam break, h={sc.config.smoothing_length:g} m, "
            f"Tait gamma={sc.config.gamma:g} k={sc.config.stiffness:g}, XSPH {sc.config.viscosity:g}, "
            f"dt={sc.dt:.4e} s, {len(sc.boxes)} static box walls")


def cpu_baseline(sc, budget_s: float = 15.0, max_steps: int = 20):
    """The reference algorithm on one host core (oracle, in-place order)."""
    from oracle import oracle as orc

    o = orc.OracleWorld(cap=sc.n, libm_pow=True)
    o.set_gravity(*sc.gravity)
    for (px, py, hx, hy) in sc.boxes:
        o.add_box(px, py, hx, hy, (1.0, 0.0, -0.0, 1.0))
    o.set_config(sc.config)
    o.add_particles(sc.xy)
    t = o.steps(sc.dt, 1, orc.REF_SEQ)
    steps = 1
    more = int(min(max_steps - 1, max(0, budget_s / max(t, 1e-9) - 1)))
    if more > 0:
        t += o.steps(sc.dt, more, orc.REF_SEQ)
        steps += more
    return {"value": sc.n * steps / t, "unit": METRIC, "cores": 1, "kind": "port",
            "sample": f"first {steps} steps of {sc.name} ({sc.n} particles), reference (in-place) order, "
                      f"C++ restatement of fluid.rs, 1 thread, {t:.1f} s"}


def run_reference(args, rank: int):
    if rank != 0:
        return
    sc = make_scene(args.workload)
    from oracle import oracle as orc

    o = orc.OracleWorld(cap=sc.n, libm_pow=True)
    o.set_gravity(*sc.gravity)
    for (px, py, hx, hy) in sc.boxes:
        o.add_box(px, py, hx, hy, (1.0, 0.0, -0.0, 1.0))
    o.set_config(sc.config)
    o.add_particles(sc.xy)
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
            "config": {"workload": workload_desc(sc), "particles": sc.n},
            "cpu_baseline": {"value": v, "unit": METRIC, "cores": 1, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, rank: int, world: int, local_rank: int):
    import torch

    from phi_eng_b200.world import world_from_scene

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist  # noqa: F811
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120))

    sc = make_scene(args.workload)
    stream = torch.cuda.Stream()
    w = world_from_scene(sc)
    w.set_stream(stream.cuda_stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    for _ in range(args.warmup):
        w.step(sc.dt)
    w.set_profiling(True)
    w.step(sc.dt)  # capture the profiled graph outside the timed region
    st = w.status()
    buckets = (1 << st.grid_log2_w) * (1 << st.grid_log2_h)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()

    sampler = ClockSampler(local_rank) if rank == 0 else None
    if sampler:
        sampler.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    phases = []
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        ev[k][0].record(stream)
        w.step(sc.dt)
        ev[k][1].record(stream)
        phases.append(w.phase_times())
    torch.cuda.synchronize()
    clocks = sampler.stop() if sampler else None
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = sum(step_ms)
    if dist:
        t = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = sc.n * args.steps * world / (total_ms / 1000.0)

    ph = np.array(phases)
    ph_mean = ph.mean(axis=0)
    names = ["sort_ranges", "density", "force_integrate"]
    bytes_pp = [sort_bytes(buckets / sc.n), DENSITY_BYTES, FORCE_BYTES]
    top = int(np.argmax(ph_mean))
    peak, peak_kind = hbm_peak()
    achieved = bytes_pp[top] * sc.n / (ph_mean[top] / 1000.0) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": None, "kernel": names[top], "bytes_per_particle": bytes_pp[top],
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                else "fallback 6650 GB/s"}
    step_bytes = sum(bytes_pp) * sc.n
    whole = {"bytes_per_particle": sum(bytes_pp),
             "achieved_gbs": step_bytes / (total_ms / args.steps / 1000.0) / 1e9}

    # end to end through the C ABI from host buffers: world creation, upload,
    # K steps each followed by the (max x, peak speed) read-back, final state read
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    w2 = world_from_scene(sc)
    for _ in range(args.steps):
        w2.step(sc.dt)
        w2.front_metrics()
    final = w2.fluid.particles
    e2e_s = time.perf_counter() - t0
    w2.close()
    e2e = {"value": sc.n * args.steps * world / e2e_s, "unit": METRIC,
           "h2d_bytes_per_step": int(sc.n * 8 / args.steps),
           "d2h_bytes_per_step": int(8 + final.nbytes / args.steps),
           "timed": "phieng_world_new + fluid_add from host arrays + K x (phieng_world_step + "
                    "phieng_sph_front_metrics) + phieng_world_fluid_get, wall clock"}
    if dist:
        t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e["value"] = sc.n * args.steps * world / float(t.item())

    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base = cpu_baseline(sc)

    if rank == 0:
        kernels_per_step = KERNELS_PER_STEP
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": workload_desc(sc), "particles": sc.n, "parallelism":
                           ("replicas" if world > 1 else "single"),
                           "l2": "flushed between timed steps (256 MiB write, outside the timed events)",
                           "grid": f"{1 << st.grid_log2_w}x{1 << st.grid_log2_h} buckets"},
                "roofline": roofline, "whole_step": whole,
                "phases_ms": {n: float(v) for n, v in zip(names, ph_mean)},
                "cpu_baseline": base, "e2e": e2e, "gpu_launches": kernels_per_step * args.steps,
                "clocks": clocks}
        print(json.dumps(line), flush=True)
    w.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="dam_break_1m", choices=["dam_break_1m", "dam_break_4k"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
