#!/usr/bin/env python
"""Throughput of the lattice-Boltzmann tick on B200 (MLUPS).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--storage f32|f16|bf16]

Workload (default): D3Q19 TRT (magic parameter 3/16), 128^3 periodic box,
tau = 0.7, rho0 = 1, uniform Guo body force 1e-6 along x, one coupled squirmer
of radius 8 at the box centre, B1 = 5e-4, beta = +5, seeded unit orientation;
populations stored as shifted FP32.  One "step" is one tick (collision +
streaming + bounce-back + Ladd coupling + particle update) of the whole box.
Multi-GPU: replicas only (one independent model per GPU, no exchange).

Prints one JSON line (rank 0).  `value` is device-timed (CUDA events on the
library's stream) with the populations resident in HBM; `e2e` goes through
the C ABI from host buffers; `roofline` is the bulk stream-collide kernel
against the measured copy bandwidth; `cpu_baseline` is the FP64 CPU oracle
(a restatement of the reference's tick) on this host's cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "lbmengine.jl_b200")
sys.path.insert(0, PKG)

METRIC = "MLUPS/% HBM roofline: mixed-precision & batched vs plain FP32, 1 B200, err≤1e-3"
BYTES = {"f32": 4, "f16": 2, "bf16": 2, "f64": 8}
FALLBACK_HBM_GBS = 6650.0


def unit_vector(seed, dims):
    import numpy as np
    v = np.random.default_rng(seed).standard_normal(dims)
    return list(v / np.sqrt((v * v).sum()))


def workload(side=128, storage="f32", device=-1):
    """The 128^3 D3Q19 TRT squirmer workload (coordinates centred on the origin)."""
    h = side // 2
    model = dict(dims=3, velocities="D3Q19", collisionModel="trt", kineticParameter=3 / 16,
                 latticeParameter=1.0, relaxationTimeRatio=0.7, xlims=(-float(h), float(side - h - 1)),
                 forceDensity=[1e-6, 0.0, 0.0], storage=storage, device=device)
    radius = 8 if side >= 32 else max(2, side // 4)
    squirmer = dict(radius=radius, position=[0.0, 0.0, 0.0], swimmingSpeed=5e-4 / 1.5, beta=5.0,
                    swimmingDirection=unit_vector(2024, 3), coupleForces=True, coupleTorques=True)
    return model, squirmer


def workload_name(side, storage):
    return (f"D3Q19 TRT(3/16) {side}^3 periodic, tau=0.7, Guo F=1e-6 x, 1 squirmer r=8 B1=5e-4 beta=+5, "
            f"{storage} shifted storage")


def measured_peak():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def bulk_traffic(storage, cells):
    """DRAM bytes per bulk launch from the ncu capture summarised in profiles/bulk_traffic.txt."""
    path = os.path.join(REPO, "profiles", "bulk_traffic.txt")
    try:
        for line in open(path):
            parts = line.split()
            if len(parts) == 2 and parts[0] == storage and not line.startswith("#"):
                return round(float(parts[1]) * cells)
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.file = None

    def __enter__(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", str(self.gpu)], stdout=self.file,
                                         stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if self.file is None:
            return out
        self.file.flush()
        try:
            lines = open(self.file.name).read().strip().splitlines()
            os.unlink(self.file.name)
        except Exception:
            return out
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if sm:
            loaded = [s for s in sm if s > 0.5 * max(sm)] or sm
            out.update(sm_mhz=statistics.median(loaded), sm_max_mhz=max(mx), samples=len(sm))
        out["reasons"] = sorted(reasons)
        return out


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
    return world, rank, local, dist


def reduce_max(dist, x):
    if dist is None:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


def oracle_mlups(side, ticks, warm, threads=None):
    """FP64 CPU oracle on a side^3 box of the workload: (MLUPS, seconds, threads)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle  # CPU baseline leg only
    from lbmengine import config
    oracle.build()
    if threads:
        oracle.set_threads(threads)
    mkw, skw = workload(side)
    res = config.resolve_model(**mkw)
    m = oracle.OracleModel(res)
    m.add_particle(config.resolve_squirmer(3, **skw))
    m.step(warm)
    t0 = time.perf_counter()
    m.step(ticks)
    dt = time.perf_counter() - t0
    return side ** 3 * ticks / dt / 1e6, dt, oracle.max_threads()


def oracle_side_for(ticks_total, budget_s):
    """Largest box (multiple of 8, 16..128) whose ticks fit the time budget."""
    rate, _, _ = oracle_mlups(24, 2, 1)
    cells = rate * 1e6 * budget_s / max(1, ticks_total)
    side = int(cells ** (1 / 3)) // 8 * 8
    return max(16, min(128, side))


def run_reference(args):
    world, rank, _, _ = dist_setup_env_only()
    if rank != 0:
        return 0
    side = oracle_side_for(args.steps + args.warmup, budget_s=150.0)
    mlups, dt, threads = oracle_mlups(side, args.steps, args.warmup)
    line = {
        "metric": METRIC, "impl": "reference", "value": round(mlups, 4), "unit": "MLUPS", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / max(1, args.steps),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload_name(128, "f64"), "parallelism": "replicas"},
        "cpu_baseline": {"value": round(mlups, 4), "unit": "MLUPS", "cores": threads, "kind": "port",
                         "sample": f"{side}^3 box of the workload (same physics, one squirmer), {args.steps} ticks "
                                   f"after {args.warmup} warm-up ticks; FP64 C++ restatement of the reference's "
                                   f"GPU-module tick (Julia reference not runnable here)"},
        "e2e": {"value": round(mlups, 4), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def dist_setup_env_only():
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")), None)


def run_ours(args):
    import numpy as np
    from lbmengine import _capi, config, model as lbm_model
    world, rank, local, dist = dist_setup()
    side = args.side
    storage = args.storage
    mkw, skw = workload(side, storage, device=local)
    res = config.resolve_model(**mkw)
    m = lbm_model.LBMmodel(res)
    lbm_model._add(m, config.resolve_squirmer(3, **skw))
    cells = side ** 3
    q = 19
    lib = m._lib

    m.step(max(3, args.warmup))
    barrier(dist)
    lib.lbm_set_profiling(m.handle, 1)
    with ClockSampler(local) as clk:
        m.step(args.steps)
    prof = _capi.LbmProfile()
    m._check(lib.lbm_get_profile(m.handle, prof))
    lib.lbm_set_profiling(m.handle, 0)
    total_ms = reduce_max(dist, prof.total_ms)
    barrier(dist)
    value = cells * args.steps * world / (total_ms / 1e3) / 1e6

    # roofline of the dominant (bulk) kernel: its mean launch duration from CUDA
    # events around back-to-back launches on the library's stream, right after
    # the timed region and on the same model (state saved and restored)
    kern = {}
    for name, kid in (("bulk", 0), ("fixup", 1), ("particles", 2)):
        ms = __import__("ctypes").c_double(0.0)
        rc = lib.lbm_time_kernel(m.handle, kid, 200 if kid == 0 else 50, __import__("ctypes").byref(ms))
        kern[name] = ms.value if rc == 0 else None
    bpp = BYTES[storage]
    bulk_bytes = prof.bulk_cells * 2 * q * bpp
    achieved = bulk_bytes / (kern["bulk"] / 1e3) / 1e9 if kern["bulk"] else None
    peak, peak_kind = measured_peak()
    traffic = bulk_traffic(storage, prof.bulk_cells)
    roofline = {"bound": "hbm", "achieved": round(achieved, 1) if achieved else None, "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4) if achieved else None, "traffic": traffic,
                "peak_source": f"{peak_kind} copy bandwidth (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                else "fallback 6.65 TB/s",
                "kernel": f"k_bulk_v4<D3Q19,{storage},TRT>", "bytes_per_launch": bulk_bytes,
                "algorithmic_bytes_per_cell": 2 * q * bpp, "kernel_ms": kern,
                "fixup_entries": prof.fixup_entries,
                "timing": "value: CUDA events around the timed lbm_step call (graph replays); kernel_ms: mean of "
                          "back-to-back launches of each kernel alone, events on the same stream"}
    launches = int(prof.launches)
    tick_ms = total_ms / max(1, args.steps)

    # end to end through the C ABI from host buffers
    e2e_steps = max(1, min(args.steps, args.e2e_steps))
    barrier(dist)
    t0 = time.perf_counter()
    mkw2 = dict(mkw)
    rho0 = np.ones((side,) * 3, dtype=np.float64)
    u0 = np.zeros((side,) * 3 + (3,), dtype=np.float64)
    mkw2.update(massDensity=rho0, fluidVelocity=u0)
    m2 = lbm_model.LBMmodel(config.resolve_model(**mkw2))
    lbm_model._add(m2, config.resolve_squirmer(3, **skw))
    state_bytes = 0
    for _ in range(e2e_steps):
        m2.step(1)
        st = m2.particle_states()
        state_bytes += len(st) * __import__("ctypes").sizeof(_capi.LbmParticleState)
    rho_out = m2.massDensity
    u_out = m2.fluidVelocity
    e2e_s = time.perf_counter() - t0
    e2e_s = reduce_max(dist, e2e_s)
    m2.close()
    h2d = (rho0.nbytes + u0.nbytes) / e2e_steps
    d2h = (state_bytes + rho_out.nbytes + u_out.nbytes) / e2e_steps
    e2e = {"value": round(cells * e2e_steps * world / e2e_s / 1e6, 2), "unit": "MLUPS",
           "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
           "steps": e2e_steps,
           "path": "lbm_create(host rho,u) + lbm_add_particle + per tick lbm_step(1) + lbm_get_particles, "
                   "then lbm_get_fields; host wall clock"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ticks = args.cpu_ticks
        mlups, dt, threads = oracle_mlups(side, ticks, 1)
        cpu = {"value": round(mlups, 4), "unit": "MLUPS", "cores": threads, "kind": "port",
               "sample": f"{ticks} ticks (after 1 warm-up tick) of the full {side}^3 workload, FP64 C++ restatement "
                         f"of the reference's GPU-module tick, OpenMP over cells ({dt:.1f} s)"}
    clocks = clk.summary()
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": round(tick_ms, 6), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if storage == "f64" else "f32",
            "data": "synthetic",
            "config": {"workload": workload_name(side, storage), "cells": cells, "storage": storage,
                       "parallelism": "replicas" if world > 1 else "single",
                       "l2": f"inputs larger than L2: populations 2 x {cells * q * bpp / 1e6:.0f} MB"},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
            "clocks": {"sm_mhz": clocks["sm_mhz"], "sm_max_mhz": clocks["sm_max_mhz"], "reasons": clocks["reasons"],
                       "samples": clocks["samples"]},
        }
        print(json.dumps(line), flush=True)
    m.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--warmup", type=int, default=200)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--storage", choices=["f32", "f16", "bf16", "f64"], default="f32")
    ap.add_argument("--side", type=int, default=128)
    ap.add_argument("--e2e-steps", type=int, default=2000)
    ap.add_argument("--cpu-ticks", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args(argv)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
