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


# The body force accelerates the whole periodic box (u_x = 1e-6 t), so the
# squirmer of the 128^3 workload is carried x ~ 5e-7 t^2 and reaches the x
# boundary near tick 10,550.  There the reference's particle geometry is not
# periodic: the torque arm and the slip velocity use the unwrapped X - R
# (src/gpu/fluids.jl:206-208, src/gpu/particles.jl getNodeVelocity), so a link
# across the boundary gets an arm of about one box length and the coupling
# diverges in every storage format, FP64 included (near tick 11,000).  The
# default timed run (200 warm-up + 10,000 ticks) ends before the crossing.
VALID_TICKS_128 = 10_500


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


def workload_name(side, storage=None):
    name = f"D3Q19 TRT(3/16) {side}^3 periodic, tau=0.7, Guo F=1e-6 x, 1 squirmer r=8 B1=5e-4 beta=+5"
    return name if storage is None else f"{name}, {storage} shifted storage"


def bench_config(side, world):
    """The `config` object of the JSON line; both arms print the same one."""
    return {"workload": workload_name(side), "cells": side ** 3,
            "ticks_valid": f"the squirmer crosses the periodic x boundary near tick {VALID_TICKS_128} (128^3), "
                           "after which the reference's unwrapped torque arm makes the coupling diverge",
            "parallelism": "replicas" if world > 1 else "single",
            "l2": f"inputs larger than L2: D3Q19 populations 2 x {side ** 3 * 19 * 4 / 1e6:.0f} MB (FP32), no "
                  "flush; each tick walks its tiles in the order opposite to the previous tick's and so reads "
                  "part of its populations (about 45 % at 128^3 FP32) from what the previous tick left in L2"}


def measured_peak():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def bulk_traffic(storage, cells):
    """DRAM bytes per bulk launch, replayed from an earlier ncu capture of the same kernel
    (bytes per cell, profiles/bulk_traffic.txt) scaled to `cells`: not measured by this run."""
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


ORACLE_SEMANTICS = ("FP64 C++ restatement of the reference's tick (fluid step of src/gpu/fluids.jl:132-226 "
                    "with the GPU module's particle update, the path this library replaces; the CPU module's "
                    "particle rules are a switch of the same code), OpenMP over cells; the reference itself is "
                    "Julia and cannot run here")


def oracle_mlups(side, ticks, warm, threads=None, budget_s=None):
    """FP64 CPU oracle on a side^3 box of the workload: (MLUPS, seconds, threads,
    ticks timed).  With budget_s, at most the ticks that fit the budget are
    timed (measured from the first warm-up tick), at least one."""
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
    t0 = time.perf_counter()
    m.step(max(1, warm))
    per_tick = (time.perf_counter() - t0) / max(1, warm)
    if budget_s is not None:
        ticks = max(1, min(ticks, int(budget_s / max(per_tick, 1e-9))))
    t0 = time.perf_counter()
    m.step(ticks)
    dt = time.perf_counter() - t0
    return side ** 3 * ticks / dt / 1e6, dt, oracle.max_threads(), ticks


def oracle_side_for(ticks_total, budget_s):
    """Largest box (multiple of 8, 16..128) whose ticks fit the time budget."""
    rate, _, _, _ = oracle_mlups(24, 2, 1)
    cells = rate * 1e6 * budget_s / max(1, ticks_total)
    side = int(cells ** (1 / 3)) // 8 * 8
    return max(16, min(128, side))


def run_reference(args):
    world, rank, _, _ = dist_setup_env_only()
    if rank != 0:
        return 0
    side = args.side
    # each timed tick is the full workload; at most ~60 s of CPU ticks are timed
    warm = max(1, min(args.warmup, 3))
    mlups, dt, threads, timed = oracle_mlups(side, args.steps, warm, budget_s=60.0)
    line = {
        "metric": METRIC, "impl": "reference", "value": round(mlups, 4), "unit": "MLUPS", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / max(1, timed),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": bench_config(side, world),
        "cpu_baseline": {"value": round(mlups, 4), "unit": "MLUPS", "cores": threads, "kind": "port",
                         "sample": f"the full {side}^3 workload, {timed} of the {args.steps} ticks (at most ~60 s) "
                                   f"after {warm} warm-up ticks on this host's cores; {ORACLE_SEMANTICS}"},
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

    if side == 128 and max(3, args.warmup) + args.steps > VALID_TICKS_128:
        print(f"bench: {max(3, args.warmup) + args.steps} ticks run past the periodic-boundary crossing near tick "
              f"{VALID_TICKS_128}, where the reference's coupling diverges; expect LBM_ERR_NUMERIC", file=sys.stderr)
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
                "frac_of_nominal_8000": round(achieved / 8000.0, 4) if achieved else None,
                "peak_source": f"{peak_kind} copy bandwidth (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                else "fallback 6.65 TB/s",
                "traffic_source": "replayed from an earlier ncu capture of consecutive live launches without cache "
                                  "flushing (profiles/bulk_traffic.txt), not this run: each pass reads about 45 % "
                                  "(FP32) of its populations from L2, so DRAM traffic is below the algorithmic bytes",
                "kernel": f"k_bulk_v4<D3Q19,{storage},TRT,64>", "bytes_per_launch": bulk_bytes,
                "algorithmic_bytes_per_cell": 2 * q * bpp, "kernel_ms": kern,
                "fixup_entries": prof.fixup_entries,
                "timing": "value: CUDA events around the timed lbm_step call (graph replays); kernel_ms: mean of "
                          "back-to-back launches of each kernel alone, events on the same stream"}
    launches = int(prof.launches)
    tick_ms = total_ms / max(1, args.steps)

    # end to end through the public API from host buffers: the initial fields
    # from pinned, column-major host arrays (a Julia array's layout), every
    # tick's particle state read back (the device trajectory ring, read in
    # blocks), the final fields into pinned host arrays; host wall clock
    import torch
    from lbmengine import output as lbm_output
    e2e_steps = max(1, min(args.steps, args.e2e_steps))

    def pinned(shape):
        t = torch.empty(int(np.prod(shape)), dtype=torch.float64, pin_memory=True)
        return t, t.numpy().reshape(shape, order="F")

    keep = [pinned((side,) * 3), pinned((side,) * 3 + (3,)), pinned((side,) * 3), pinned((side,) * 3 + (3,))]
    rho0, u0, rho_out, u_out = (k[1] for k in keep)
    rho0[...] = 1.0
    u0[...] = 0.0
    ring = lbm_output.RING_TICKS
    rows = np.empty(ring * 9, dtype=np.float64)
    got = __import__("ctypes").c_int64()
    # one untimed pass of the same calls (2 ticks): the process's first use of
    # each of them (kernel modules, pinned transfers) is not the steady state
    mw = lbm_model.LBMmodel(config.resolve_model(**dict(mkw, massDensity=rho0, fluidVelocity=u0)))
    lbm_model._add(mw, config.resolve_squirmer(3, **skw))
    mw._check(lib.lbm_record_trajectories(mw.handle, ring))
    mw.step(2)
    mw._check(lib.lbm_read_trajectories(mw.handle, rows.ctypes.data_as(_capi._dp), 2, __import__("ctypes").byref(got)))
    mw.read_fields(rho_out, u_out)
    mw.close()
    barrier(dist)
    t0 = time.perf_counter()
    m2 = lbm_model.LBMmodel(config.resolve_model(**dict(mkw, massDensity=rho0, fluidVelocity=u0)))
    lbm_model._add(m2, config.resolve_squirmer(3, **skw))
    m2._check(lib.lbm_record_trajectories(m2.handle, ring))
    done = rows_read = 0
    while done < e2e_steps:
        seg = min(ring, e2e_steps - done)
        m2.step(seg)
        m2._check(lib.lbm_read_trajectories(m2.handle, rows.ctypes.data_as(_capi._dp), seg, __import__("ctypes").byref(got)))
        rows_read += got.value
        done += seg
    m2.read_fields(rho_out, u_out)
    e2e_s = time.perf_counter() - t0
    e2e_s = reduce_max(dist, e2e_s)
    m2.close()
    h2d = (rho0.nbytes + u0.nbytes) / e2e_steps
    d2h = (rows_read * 9 * 8 + rho_out.nbytes + u_out.nbytes) / e2e_steps
    e2e = {"value": round(cells * e2e_steps * world / e2e_s / 1e6, 2), "unit": "MLUPS",
           "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
           "steps": e2e_steps, "ticks_with_particle_state_read": int(rows_read),
           "path": "modelInit with pinned column-major host rho/u (lbm_create) + addSquirmer + LBMpropagate in "
                   f"blocks of up to {ring} ticks, each block's per-tick particle states read from the device "
                   "trajectory ring (lbm_read_trajectories), then massDensity/fluidVelocity into pinned host "
                   "arrays (lbm_get_fields); host wall clock, including any graph builds (a model's first call "
                   "of up to 32 ticks launches its ticks directly, later calls build the graphs they need), after "
                   "one untimed 2-tick pass of the same calls (whose freed device blocks the library keeps for "
                   "reuse, as for any model built after another in a process)"}
    del keep

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ticks = args.cpu_ticks
        mlups, dt, threads, _ = oracle_mlups(side, ticks, 1)
        cpu = {"value": round(mlups, 4), "unit": "MLUPS", "cores": threads, "kind": "port",
               "sample": f"{ticks} ticks (after 1 warm-up tick) of the full {side}^3 workload ({dt:.1f} s); "
                         f"{ORACLE_SEMANTICS}"}
    clocks = clk.summary()
    forms = run_forms(args, local) if rank == 0 and world == 1 else None
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": round(tick_ms, 6), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if storage == "f64" else "f32",
            "data": "synthetic",
            "config": bench_config(side, world), "storage": storage,
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
            "clocks": {"sm_mhz": clocks["sm_mhz"], "sm_max_mhz": clocks["sm_max_mhz"], "reasons": clocks["reasons"],
                       "samples": clocks["samples"]},
            "forms": forms,
        }
        if forms:
            line["forms_summary"] = forms_summary(forms)  # last key: survives a tail of the output
        print(json.dumps(line), flush=True)
    m.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------
# The three forms beside the plain FP32 path: shifted FP16/BF16 storage,
# batches of replicas, and adjoint gradients.  Each entry states its config
# and what its numbers were measured against.
# ---------------------------------------------------------------------------
def _ms_per_tick(m, n):
    from lbmengine import _capi
    lib = m._lib
    lib.lbm_set_profiling(m.handle, 1)
    m.step(n)
    p = _capi.LbmProfile()
    m._check(lib.lbm_get_profile(m.handle, p))
    lib.lbm_set_profiling(m.handle, 0)
    return p.total_ms / n


def _rel_l2(a, b):
    import numpy as np
    return float(np.sqrt(np.sum((np.asarray(a) - np.asarray(b)) ** 2) / max(np.sum(np.asarray(b) ** 2), 1e-300)))


def form_precision_c2(device):
    """C2 workload per storage format: MLUPS over 5000 ticks (squirmer inside the
    box throughout), and the error after 500 ticks against FP64 storage."""
    from lbmengine import config, model as M
    out = {"config": workload_name(128, "<storage>") + "; throughput over ticks 200..5200, error after 500 ticks",
           "reference_for_error": "FP64 storage on the GPU (equal to the FP64 CPU oracle to 1e-10 in the parity tests)"}
    fields = {}
    for st in ("f32", "f16", "bf16", "f64"):
        mkw, skw = workload(128, st, device=device)
        m = M.LBMmodel(config.resolve_model(**mkw))
        M._add(m, config.resolve_squirmer(3, **skw))
        m.step(500)
        fields[st] = (m.massDensity, m.fluidVelocity, list(m.particle_states()[0].position[:3]))
        if st != "f64":
            ms = _ms_per_tick(m, 5000)
            out[st] = {"mlups": round(128 ** 3 / ms / 1e3, 1), "ms_per_tick": round(ms, 5)}
        m.close()
    import numpy as np
    for st in ("f32", "f16", "bf16"):
        rho, u, R = fields[st]
        out[st].update(u_rel_l2=_rel_l2(u, fields["f64"][1]), rho_rel_l2=_rel_l2(rho, fields["f64"][0]),
                       position_abs_err=float(np.max(np.abs(np.array(R) - np.array(fields["f64"][2])))))
    for st in ("f16", "bf16"):
        out[f"{st}_vs_f32"] = round(out[st]["mlups"] / out["f32"]["mlups"], 3)
    return out


def c3_particles(seed=3):
    """64 non-overlapping squirmers of radius 6 in a 192^3 box: centres uniform in
    [r+1, 190-r]^3 (0-based nodes) by rejection with centre distance >= 2r+2."""
    import numpy as np
    rng = np.random.default_rng(seed)
    r, side, centres = 6, 192, []
    while len(centres) < 64:
        c = rng.uniform(r + 1, side - 2 - r, 3)
        if all(np.linalg.norm(c - q) >= 2 * r + 2 for q in centres):
            centres.append(c)
    parts = []
    for c in centres:
        e = rng.standard_normal(3)
        parts.append(dict(radius=float(r), position=list(c - side // 2), swimmingSpeed=5e-4 / 1.5,
                          beta=float(rng.uniform(-5, 5)), swimmingDirection=list(e / np.linalg.norm(e)),
                          coupleForces=True, coupleTorques=True))
    return parts


def form_precision_c3(device, ticks=3000, density=3.0):
    """C3 geometry: 192^3 D3Q19 TRT (tau 0.6, magic 1/4), 64 squirmers r=6.
    With the reference's default particle density (1, as the configuration
    leaves it) the explicit Ladd coupling diverges within a few hundred ticks
    even in FP64 (reported as `as_specified`); the storage formats are compared
    on particles of density `density`, over `ticks` ticks (before squirmers,
    which do not interact, swim into one another)."""
    import numpy as np
    from lbmengine import config, model as M
    model = dict(dims=3, velocities="D3Q19", collisionModel="trt", kineticParameter=0.25, latticeParameter=1.0,
                 relaxationTimeRatio=0.6, xlims=(-96.0, 95.0), device=device)
    parts = c3_particles()
    res = {}
    out = {"config": f"D3Q19 TRT 192^3 periodic, tau=0.6, magic parameter 1/4, 64 squirmers r=6 (seeded, gap >= 2), "
                     f"B1=5e-4, beta~U[-5,5], particle density {density}; {ticks} ticks; error against FP64 storage "
                     f"on the GPU"}
    m = M.LBMmodel(config.resolve_model(**dict(model, storage="f64")))
    for p in parts:
        M._add(m, config.resolve_squirmer(3, **p))
    from lbmengine._capi import LbmError
    diverged = None
    for _ in range(20):
        try:
            m.step(100)  # the density sentinel raises once the run has diverged
        except LbmError:
            diverged = m.tick
            break
        if not np.isfinite(m.fluidVelocity).all():
            diverged = m.tick
            break
    m.close()
    out["as_specified"] = {"particle_density": 1.0, "fp64_nonfinite_by_tick": diverged, "checked_ticks": 2000}
    for st in ("f64", "f16", "bf16", "f32"):
        m = M.LBMmodel(config.resolve_model(**dict(model, storage=st)))
        for p in parts:
            M._add(m, config.resolve_squirmer(3, **dict(p, massDensity=density)))
        ms = _ms_per_tick(m, ticks)
        R = np.array([ps.position[:3] for ps in m.particle_states()])
        res[st] = (m.massDensity, m.fluidVelocity, R)
        out[st] = {"mlups": round(192 ** 3 / ms / 1e3, 1), "ms_per_tick": round(ms, 5)}
        m.close()
    for st in ("f16", "bf16", "f32"):
        rho, u, R = res[st]
        d = np.linalg.norm(R - res["f64"][2], axis=1)
        out[st].update(u_rel_l2=_rel_l2(u, res["f64"][1]), rho_rel_l2=_rel_l2(rho, res["f64"][0]),
                       position_err_max=float(d.max()), position_err_mean=float(d.mean()))
    return out


def c4_replicas(n=512, seed=4):
    """C4: D2Q9 TRT squirmer replicas: side in {64,96,128,192,256}, radius in
    6..12, beta~U[-5,5], tau~U[0.55,1], B1=1e-3, seeded centre and orientation."""
    import numpy as np
    rng = np.random.default_rng(seed)
    specs = []
    for _ in range(n):
        side = int(rng.choice([64, 96, 128, 192, 256]))
        r = int(rng.integers(6, 13))
        beta, tau, ang = float(rng.uniform(-5, 5)), float(rng.uniform(0.55, 1.0)), float(rng.uniform(0, 2 * np.pi))
        h = side // 2
        pos = [float(rng.uniform(r + 1, side - 2 - r)) - h for _ in range(2)]
        specs.append((dict(dims=2, latticeParameter=1.0, relaxationTimeRatio=tau, collisionModel="trt",
                           xlims=(-float(h), float(side - h - 1))),
                      [("squirmer", dict(radius=float(r), position=pos, swimmingSpeed=1e-3 / 1.5, beta=beta,
                                         swimmingDirection=[float(np.cos(ang)), float(np.sin(ang))],
                                         coupleForces=True, coupleTorques=True))]))
    return specs


def form_batch(device, ticks=2000, sampled=8):
    import numpy as np
    from lbmengine import LBMbatch, config, model as M
    specs = c4_replicas()
    for mkw, _ in specs:
        mkw["device"] = device
    b = LBMbatch(specs)
    chosen, cands = b.autotune(ticks=32)
    b.set_profiling(1)
    b.step(ticks)
    ms = b.profile().total_ms / ticks
    nonfinite = [i for i, r in enumerate(b.replicas) if not np.isfinite(r.fluidVelocity).all()]
    out = {"config": f"512 D2Q9 TRT squirmer replicas (side in {{64..256}}, r 6..12, beta~U[-5,5], tau~U[0.55,1], "
                     f"B1=1e-3), {ticks} ticks, FP32", "cells": b.cells,
           "mlups": round(b.cells / ms / 1e3, 1), "ms_per_tick": round(ms, 5),
           "tuning": vars(chosen), "candidates": len(cands),
           "hbm_frac_of_measured": round(b.cells * 72 / (ms / 1e3) / 1e9 / measured_peak()[0], 4),
           "replicas_nonfinite_at_end": len(nonfinite),
           "replicas_diverged": sum(1 for st in b.status() if st != 0),
           "note": "replicas with low tau and a large radius diverge under the reference's explicit Ladd coupling at "
                   "particle density 1 (the FP64 oracle diverges on them too); they cost the same per tick"}
    # the same replicas one at a time (each model's own graph-replayed tick)
    tot = 0.0
    for mkw, parts in specs:
        m = M.LBMmodel(config.resolve_model(**mkw))
        for _, pkw in parts:
            M._add(m, config.resolve_squirmer(2, **pkw))
        m.step(16)
        tot += _ms_per_tick(m, 32)
        m.close()
    out["one_at_a_time_mlups"] = round(b.cells / tot / 1e3, 1)
    out["batch_vs_one_at_a_time"] = round(tot / ms, 2)
    # per-replica error against the FP64 CPU oracle on sampled replicas
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle  # the checker
    oracle.build()
    idx = sorted(np.random.default_rng(8).choice(len(specs), sampled, replace=False).tolist())
    errs = []
    for i in idx:
        mkw, parts = specs[i]
        orc = oracle.OracleModel(config.resolve_model(**mkw))
        orc.add_particle(config.resolve_squirmer(2, **parts[0][1]))
        orc.step(ticks)
        rho_o, u_o = orc.fields()
        rep = b.replicas[i]
        R_o = np.array(orc.particles()[0].position[:2])
        errs.append({"replica": i, "side": rep._shape[0], "gpu_finite": bool(np.isfinite(rep.fluidVelocity).all()),
                     "oracle_finite": bool(np.isfinite(u_o).all()),
                     "u_rel_l2": _rel_l2(rep.fluidVelocity.reshape(-1, 2, order="F").T, u_o),
                     "rho_rel_l2": _rel_l2(rep.massDensity.ravel(order="F"), rho_o),
                     "position_abs_err": float(np.max(np.abs(np.array(rep.particle_states()[0].position[:2]) - R_o)))})
        orc.close()
    out["oracle_check"] = errs
    b.close()
    return out


def c5_case(side=96, storage="f32"):
    h = side // 2
    model = dict(dims=3, velocities="D3Q19", collisionModel="trt", kineticParameter=3 / 16, latticeParameter=1.0,
                 relaxationTimeRatio=0.7, xlims=(-float(h), float(side - h - 1)), forceDensity=[1e-6, 0.0, 0.0],
                 storage=storage)
    squirmer = dict(radius=8.0, position=[0.0, 0.0, 0.0], swimmingSpeed=5e-4 / 1.5, beta=-2.0,
                    swimmingDirection=unit_vector(2024, 3), coupleForces=True, coupleTorques=True)
    return model, squirmer


def form_gradients(device, ticks=3000, window=(1000, 3000), dual_side=32, dual_ticks=600, dual_window=(200, 600)):
    import numpy as np
    from lbmengine.adjoint import build_swimmer, swimming_speed_gradient
    out = {"config": f"D3Q19 TRT 96^3, one squirmer r=8, B1=5e-4, beta=-2, tau=0.7 (magic 3/16), F=(1e-6,0,0); "
                     f"observable: velocity along the initial orientation averaged over ticks {window[0]}..{window[1]}; "
                     f"at most 32 stored states"}
    for st in ("f32", "f64"):
        mkw, skw = c5_case(96, st)
        mkw["device"] = device
        m = build_swimmer(mkw, skw)
        g = swimming_speed_gradient(m, ticks, window, snapshots=32)
        m.close()
        out[st] = {"value": g.value, "grad": g.grad, "ms": round(g.ms, 1), "forward_ticks": g.forward_ticks,
                   "snapshots_used": g.snapshots_used}
    # central differences of FP64 forward runs
    mkw, skw = c5_case(96, "f64")
    mkw["device"] = device
    B1 = 1.5 * skw["swimmingSpeed"]
    theta = np.array([B1, skw["beta"] * B1, 0.7, 1e-6, 0.0, 0.0])

    def observable(th):
        m = build_swimmer(mkw, skw, th)
        e0 = np.array(skw["swimmingDirection"])
        J = 0.0
        track = []
        for t in range(1, ticks + 1):
            m.step(1)
            st = m.particle_states()[0]
            track.append(np.array(st.position[:3]))
            if window[0] <= t <= window[1]:
                J += float(np.dot(st.velocity[:3], e0)) / (window[1] - window[0] + 1)
        m.close()
        return J, track

    axis = np.arange(96, dtype=np.float64) - 48.0  # node coordinates of the 96^3 box

    def flips(tp, tm, r=8.0):
        """Nodes inside one run's sphere and outside the other's (the getSphere test
        (x-R1)^2+(y-R2)^2+(z-R3)^2 < r^2 in FP64), summed over the ticks."""
        total, ticks_with = 0, 0
        for a, b in zip(tp, tm):
            lo = np.floor(np.minimum(a, b) - r - 1).astype(int) + 48
            hi = np.ceil(np.maximum(a, b) + r + 1).astype(int) + 48
            x, y, z = (axis[max(0, lo[k]):min(96, hi[k] + 1)] for k in range(3))
            X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
            ina = ((X - a[0]) * (X - a[0]) + (Y - a[1]) * (Y - a[1])) + (Z - a[2]) * (Z - a[2]) < r * r
            inb = ((X - b[0]) * (X - b[0]) + (Y - b[1]) * (Y - b[1])) + (Z - b[2]) * (Z - b[2]) < r * r
            n = int(np.count_nonzero(ina != inb))
            total += n
            ticks_with += n > 0
        return {"node_flips": total, "ticks_with_flips": ticks_with}

    fd = {}
    for rel in (1e-4, 1e-6, 1e-8):
        fd[str(rel)] = {}
        for k, nm in enumerate(("B1", "B2", "tau", "Fx")):
            h = rel * abs(theta[k])
            tp, tm = theta.copy(), theta.copy()
            tp[k] += h
            tm[k] -= h
            (Jp, trp), (Jm, trm) = observable(tp), observable(tm)
            d = (Jp - Jm) / (2 * h)
            fd[str(rel)][nm] = {"fd": d, "rel_err_f64_adjoint": abs(out["f64"]["grad"][nm] - d) / abs(d),
                                "rel_err_f32_adjoint": abs(out["f32"]["grad"][nm] - d) / abs(d),
                                **flips(trp, trm)}
    out["central_differences"] = fd
    # the drag of the same squirmer held in place: no node ever changes sides,
    # so central differences at the configured step h = 1e-4 hold
    from lbmengine.adjoint import drag_gradient
    skw_held = dict(skw, coupleForces=False, coupleTorques=False)
    m = build_swimmer(mkw, skw_held)
    gd = drag_gradient(m, ticks, window, snapshots=32)
    m.close()

    def drag(th):
        m = build_swimmer(mkw, skw_held, th)
        m.record_force(1)
        e0 = np.array(skw["swimmingDirection"])
        J = 0.0
        for t in range(1, ticks + 1):
            m.step(1)
            if window[0] <= t <= window[1]:
                J += float(np.dot(m.particle_states()[0].last_force[:3], e0)) / (window[1] - window[0] + 1)
        m.close()
        return J

    dfd = {}
    for k, nm in enumerate(("B1", "B2", "tau", "Fx")):
        h = 1e-4 * abs(theta[k])
        tp, tm = theta.copy(), theta.copy()
        tp[k] += h
        tm[k] -= h
        d = (drag(tp) - drag(tm)) / (2 * h)
        dfd[nm] = {"fd": d, "adjoint": gd.grad[nm], "rel_err": abs(gd.grad[nm] - d) / abs(d)}
    out["drag"] = {"observable": "momentum-exchange force on the held squirmer along its orientation, averaged "
                                 f"over ticks {window[0]}..{window[1]} (FP64 storage)",
                   "value": gd.value, "ms": round(gd.ms, 1), "central_differences_h1e-4": dfd,
                   "fd_rel_err_max": max(v["rel_err"] for v in dfd.values())}
    # forward-mode dual numbers through the CPU oracle on the same setup at dual_side^3
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle  # the checker
    from lbmengine import config
    oracle.build()
    # (the bench runs the dual check over dual_ticks; the same check over the
    # full 3000-tick schedule takes minutes of CPU time)
    ticks, window = dual_ticks, dual_window
    mkw, skw = c5_case(dual_side, "f64")
    res = config.resolve_model(**mkw)
    t0 = time.perf_counter()
    dual = oracle.DualOracle(res)
    p = config.resolve_squirmer(3, **skw)
    dual.add_particle(p)
    e0 = np.array(p.swimming_direction[:3])
    dJ = np.zeros(len(oracle.DIRECTIONS))
    for t in range(1, ticks + 1):
        dual.step(1)
        if window[0] <= t <= window[1]:
            _, der = dual.particle(1)
            dJ += (e0 @ der["velocity"][:3]) / (window[1] - window[0] + 1)
    dual.close()
    dual_s = time.perf_counter() - t0
    m = build_swimmer(dict(mkw, device=device), skw)
    g = swimming_speed_gradient(m, ticks, window, snapshots=32)
    m.close()
    out["dual_check"] = {"side": dual_side, "ticks": ticks, "window": list(window), "cpu_seconds": round(dual_s, 1),
                         "rel_err": {nm: abs(g.grad[nm] - v) / abs(v) for nm, v in zip(oracle.DIRECTIONS, dJ)
                                     if abs(v) > 0}}
    return out


def _oracle_errors(res, gpu, orc):
    """Errors of a GPU model against an oracle model: rel. L2 of rho and u, the
    largest position error (lattice units), the force error relative to the
    oracle's largest component."""
    import numpy as np
    rho_o, u_o = orc.fields()
    d = res.dims
    rho_g = gpu.massDensity.ravel(order="F")
    u_g = gpu.fluidVelocity.reshape(-1, d, order="F").T
    a, b = gpu.particle_states()[0], orc.particles()[0]
    fo = np.array(b.last_force[:d])
    return {"rho_rel_l2": _rel_l2(rho_g, rho_o), "u_rel_l2": _rel_l2(u_g, u_o),
            "position_abs_err": float(np.max(np.abs(np.array(a.position[:d]) - np.array(b.position[:d])))),
            "force_rel_err": float(np.max(np.abs(np.array(a.last_force[:d]) - fo)) / max(1e-30, np.max(np.abs(fo))))}


def form_parity(device, c2_ticks=500, c1_ticks=5000):
    """The plain-method workloads against the FP64 CPU oracle at full size:
    the 128^3 D3Q19 TRT squirmer box for beta in {-5, 0, +5} over c2_ticks
    ticks (FP32, FP16, BF16 storage against one oracle run per beta), and the
    256 x 128 D2Q9 BGK squirmer over c1_ticks ticks (centred coordinates; as
    specified, with the squirmer 4x too light by the reference's origin-centred
    mass, both the oracle and the GPU diverge, and the tick of the GPU's
    divergence report is given)."""
    import numpy as np
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle  # the checker
    from lbmengine import _capi, config, model as M
    oracle.build()
    out = {"c2": {"config": workload_name(128) + f" with beta in (-5, 0, +5); {c2_ticks} ticks; oracle FP64"}}
    for beta in (-5.0, 0.0, 5.0):
        mkw, skw = workload(128, "f64", device=device)
        skw = dict(skw, beta=beta)
        t0 = time.perf_counter()
        orc = oracle.OracleModel(config.resolve_model(**mkw))
        orc.add_particle(config.resolve_squirmer(3, **skw))
        orc.step(c2_ticks)
        ent = {"oracle_s": round(time.perf_counter() - t0, 1)}
        for st in ("f32", "f16", "bf16"):
            mkw2, _ = workload(128, st, device=device)
            res = config.resolve_model(**mkw2)
            g = M.LBMmodel(res)
            M._add(g, config.resolve_squirmer(3, **skw))
            g.step(c2_ticks)
            ent[st] = _oracle_errors(res, g, orc)
            g.close()
        orc.close()
        out["c2"][f"beta={beta:+g}"] = ent
    # C1
    out["c1"] = {"config": f"D2Q9 BGK 256x128, tau=0.8, squirmer r=10 B1=1e-3 beta=+3, angle 0; {c1_ticks} ticks"}
    for centred in (True, False):
        lims = dict(xlims=(-128.0, 127.0), ylims=(-64.0, 63.0)) if centred else dict(xlims=(0.0, 255.0),
                                                                                  ylims=(0.0, 127.0))
        pos = [-64.0, 0.0] if centred else [64.0, 64.0]
        prm = config.resolve_squirmer(2, radius=10, position=pos, swimmingDirection=[1.0, 0.0],
                                      swimmingSpeed=1e-3 / 1.5, beta=3.0, coupleForces=True, coupleTorques=True)
        key = "centred" if centred else "as_specified"
        ent = {}
        for st in ("f64", "f32"):
            res = config.resolve_model(dims=2, latticeParameter=1.0, relaxationTimeRatio=0.8, collisionModel="bgk",
                                       storage=st, device=device, **lims)
            orc = oracle.OracleModel(res)
            orc.add_particle(prm)
            g = M.LBMmodel(res)
            M._add(g, prm)
            if centred:
                orc.step(c1_ticks)
                g.step(c1_ticks)
                ent[st] = _oracle_errors(res, g, orc)
            else:
                orc.step(1000)
                g.step(1000)
                ent[st] = {"at_tick_1000": _oracle_errors(res, g, orc)}
                reported = None
                while g.tick < c1_ticks:
                    try:
                        g.step(250)
                    except _capi.LbmError as exc:
                        reported = (g.tick, exc.code)
                        break
                orc.step(c1_ticks - 1000)
                ent[st]["gpu_divergence_reported_at_tick"] = reported[0] if reported else None
                ent[st]["oracle_finite_at_end"] = bool(np.isfinite(orc.fields()[1]).all())
            g.close()
            orc.close()
        out["c1"][key] = ent
    return out


def _r(x, n=3):
    return None if x is None else float(f"{x:.{n}g}")


def forms_summary(forms):
    """One compact entry per form (throughput ratios and the largest errors)."""
    out = {}
    f = forms.get("precision_c2", {})
    if "f32" in f:
        out["precision_c2"] = {"mlups": {k: f[k]["mlups"] for k in ("f32", "f16", "bf16")},
                               "f16_vs_f32": f.get("f16_vs_f32"), "bf16_vs_f32": f.get("bf16_vs_f32"),
                               "u_err_vs_f64": {k: _r(f[k]["u_rel_l2"]) for k in ("f32", "f16", "bf16")}}
    f = forms.get("precision_c3", {})
    if "f32" in f:
        out["precision_c3"] = {"mlups": {k: f[k]["mlups"] for k in ("f32", "f16", "bf16")},
                               "f16_vs_f32": round(f["f16"]["mlups"] / f["f32"]["mlups"], 3),
                               "u_err_vs_f64": {k: _r(f[k]["u_rel_l2"]) for k in ("f32", "f16", "bf16")}}
    f = forms.get("batching_c4", {})
    if "mlups" in f:
        chk = [e for e in f.get("oracle_check", []) if e["oracle_finite"]]
        out["batching_c4"] = {"mlups": f["mlups"], "hbm_frac": f["hbm_frac_of_measured"],
                              "vs_one_at_a_time": f["batch_vs_one_at_a_time"],
                              "diverged_replicas": f.get("replicas_diverged"),
                              "oracle_u_err_max": _r(max((e["u_rel_l2"] for e in chk), default=None))}
    f = forms.get("gradients_c5", {})
    if "f32" in f:
        cd = f.get("central_differences", {})
        out["gradients_c5"] = {"s": round(f["f32"]["ms"] / 1e3, 1),
                               "dual_rel_err_max": _r(max(f["dual_check"]["rel_err"].values())),
                               # per step h and parameter: [FD vs adjoint rel. error, nodes that
                               # changed sides between the +h and -h runs]
                               "fd_err_and_flips": {h: {k: [_r(v["rel_err_f64_adjoint"], 2), v.get("node_flips")]
                                                        for k, v in cd[h].items()} for h in cd},
                               "fd_rel_err_max_flip_free": _r(max((v["rel_err_f64_adjoint"] for h in cd
                                                                   for v in cd[h].values()
                                                                   if v.get("node_flips") == 0), default=None))}
        if "drag" in f:
            out["gradients_c5"]["drag_fd_rel_err_max"] = f["drag"].get("fd_rel_err_max")
    f = forms.get("parity", {})
    if "c2" in f:
        out["parity_c2_500"] = {b: {st: {"u": _r(v[st]["u_rel_l2"], 2), "rho": _r(v[st]["rho_rel_l2"], 2),
                                         "pos": _r(v[st]["position_abs_err"], 2)} for st in ("f32", "f16", "bf16")}
                                for b, v in f["c2"].items() if b.startswith("beta")}
        c1 = f["c1"]
        out["parity_c1_5000"] = {"centred": {st: {"u": _r(c1["centred"][st]["u_rel_l2"], 2),
                                                  "pos": _r(c1["centred"][st]["position_abs_err"], 2)}
                                             for st in ("f64", "f32")},
                                 "as_specified_diverges_at": c1["as_specified"]["f64"]["gpu_divergence_reported_at_tick"]}
    for k, v in forms.items():
        if "error" in v:
            out[k] = {"error": v["error"][:200]}
        if k in out:
            out[k]["wall_s"] = v.get("wall_s")
    return out


def run_forms(args, device):
    forms = {}
    for name, fn in (("precision_c2", lambda: form_precision_c2(device)),
                     ("precision_c3", lambda: form_precision_c3(device)),
                     ("batching_c4", lambda: form_batch(device)),
                     ("gradients_c5", lambda: form_gradients(device)),
                     ("parity", lambda: form_parity(device))):
        if name in args.skip_forms:
            continue
        t0 = time.perf_counter()
        try:
            forms[name] = fn()
        except Exception as exc:  # reported, not hidden: the form's entry carries the error
            forms[name] = {"error": f"{type(exc).__name__}: {exc}"}
        forms[name]["wall_s"] = round(time.perf_counter() - t0, 1)
    return forms


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10000)
    ap.add_argument("--warmup", type=int, default=200)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--storage", choices=["f32", "f16", "bf16", "f64"], default="f32")
    ap.add_argument("--side", type=int, default=128)
    ap.add_argument("--e2e-steps", type=int, default=2000)
    ap.add_argument("--cpu-ticks", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--skip-forms", default="",
                    help="comma-separated forms to skip: precision_c2, precision_c3, batching_c4, gradients_c5, parity "
                         "(all: skip every form)")
    args = ap.parse_args(argv)
    args.skip_forms = {"precision_c2", "precision_c3", "batching_c4", "gradients_c5", "parity"} \
        if args.skip_forms == "all" else set(filter(None, args.skip_forms.split(",")))
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
