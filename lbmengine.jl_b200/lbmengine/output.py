"""The :saveData output of LBMengine.jl: trajectory and field CSV files.

Restates writeTrajectories / writeParticleTrajectory (src/gpu/aux.jl:271-356)
and the checkpoint logic of LBMpropagate! (src/gpu/fluids.jl:243-259):
``output.lbm/fluidTrj_<tick>.csv`` at ``ticksSaved`` checkpoints and one row
per particle and tick in ``output.lbm/particlesTrj.csv``.  The particle
states of every tick are recorded on the device (lbm_record_trajectories) and
read back in blocks, so stepping stays graph-replayed; the large field files
are formatted and written by the library on a host thread
(lbm_write_fluid_csv) while stepping goes on.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import shutil
from fractions import Fraction

import numpy as np

from . import _capi as capi

OUTPUT_DIR = "output.lbm"
RING_TICKS = 1024  # ticks of particle states the device ring holds between reads


def julia_float(x: float) -> str:
    """Julia's print(::Float64), as CSV.jl writes numbers: shortest round-trip
    digits, plain notation for 1e-4 <= |x| < 1e6 ("1.0", "0.0001"), else
    "d.ddde<exp>" ("1.0e-5", "1.234567e6")."""
    x = float(x)
    if math.isnan(x):
        return "NaN"
    if math.isinf(x):
        return "Inf" if x > 0 else "-Inf"
    if x == 0.0:
        return "-0.0" if math.copysign(1.0, x) < 0 else "0.0"
    r = repr(abs(x))
    if "e" in r:
        mant, e = r.split("e")
        e10 = int(e)
    else:
        mant, e10 = r, None
    digits = mant.replace(".", "")
    if e10 is None:  # plain repr: find the decimal exponent of the leading digit
        ip, _, fp = mant.partition(".")
        if ip != "0":
            e10 = len(ip) - 1
            digits = (ip + fp).rstrip("0") or "0"
        else:
            z = len(fp) - len(fp.lstrip("0"))
            e10 = -(z + 1)
            digits = fp.lstrip("0")
    else:
        digits = digits.rstrip("0") or "0"
    digits = digits.lstrip("0") or "0"
    sign = "-" if x < 0 else ""
    if e10 < -4 or e10 >= 6:
        return f"{sign}{digits[0]}.{digits[1:] or '0'}e{e10}"
    if e10 < 0:
        return f"{sign}0.{'0' * (-e10 - 1)}{digits}"
    ip = e10 + 1
    if len(digits) <= ip:
        return f"{sign}{digits}{'0' * (ip - len(digits))}.0"
    return f"{sign}{digits[:ip]}.{digits[ip:]}"


def julia_round(x: Fraction) -> int:
    """round(x) of Julia (RoundNearest: ties to even) on an exact rational."""
    f = math.floor(x)
    r = x - f
    if r > Fraction(1, 2) or (r == Fraction(1, 2) and f % 2 == 1):
        return f + 1
    return f


def checkpoints(tick0: int, dt: float, ticks: int, ticks_saved: int):
    """Ticks after which LBMpropagate! writes the fluid (src/gpu/fluids.jl:243-247):
    round.(range(tick, stop = tick + floor(simulationTime / dt), length = ticksSaved))."""
    fdt = Fraction(dt)
    sim_time = fdt * ticks  # time[end] of range(dt, length = ticks, step = dt)
    total = math.floor(sim_time / fdt)
    if ticks_saved == 1:
        return {tick0}
    step = Fraction(total, ticks_saved - 1)
    return {julia_round(tick0 + i * step) for i in range(ticks_saved)}


def prepare_directory():
    """modelInit(saveData = true): rm("output.lbm"; recursive) then mkdir (src/gpu/initMethods.jl:671-675)."""
    shutil.rmtree(OUTPUT_DIR, ignore_errors=True)
    os.makedirs(OUTPUT_DIR)


def write_fluid(model) -> None:
    """writeTrajectories(model): output.lbm/fluidTrj_<tick>.csv, written by the library's host thread."""
    path = os.path.join(OUTPUT_DIR, f"fluidTrj_{model.tick}.csv")
    model._check(model._lib.lbm_write_fluid_csv(model.handle, path.encode()))


def _particle_header(dims):
    if dims == 2:
        return ["tick", "time", "particleId", "position_x", "position_y", "velocity_x", "velocity_y",
                "angularVelocity"]
    return ["tick", "time", "particleId", "position_x", "position_y", "position_z", "velocity_x", "velocity_y",
            "velocity_z", "angularVelocity_x", "angularVelocity_y", "angularVelocity_z"]


def append_particle_rows(dims, rows) -> None:
    """Append rows (tick, time, id, R, v, w) to output.lbm/particlesTrj.csv
    (the header first when the file does not exist yet, as CSV.write does)."""
    path = os.path.join(OUTPUT_DIR, "particlesTrj.csv")
    new = not os.path.isfile(path)
    nw = 1 if dims == 2 else 3
    with open(path, "a") as f:
        if new:
            f.write(",".join(_particle_header(dims)) + "\n")
        for tick, time, pid, R, v, w in rows:
            vals = [str(int(tick)), julia_float(time), str(int(pid))]
            vals += [julia_float(x) for x in R[:dims]] + [julia_float(x) for x in v[:dims]]
            vals += [julia_float(x) for x in w[:nw]]
            f.write(",".join(vals) + "\n")


def write_particle(model, state) -> None:
    """writeParticleTrajectory(particle, model) for one particle state (at its addition)."""
    append_particle_rows(model._dims, [(model.tick, model.time, state.id, list(state.position),
                                        list(state.velocity), list(state.angular_velocity))])


def propagate(model, ticks: int, ticks_saved) -> None:
    """LBMpropagate! with :saveData: step `ticks` ticks, writing the fluid at the
    checkpoints and every particle's state after every tick."""
    lib, h = model._lib, model.handle
    dims = model._dims
    t0 = model.tick
    cps = checkpoints(t0, model.spaceTime.timeStep, ticks, 100 if ticks_saved is None else int(ticks_saved))
    nparts = len(model.particle_states())
    if nparts:
        model._check(lib.lbm_record_trajectories(h, RING_TICKS))
    dt = model.spaceTime.timeStep
    done = 0
    time = model.time
    try:
        while done < ticks:
            nxt = min([c - t0 for c in cps if c - t0 > done] + [ticks])
            seg = min(nxt - done, RING_TICKS)
            model.step(seg)
            tick_start = t0 + done
            done += seg
            if nparts:
                buf = np.zeros(seg * nparts * 9)
                got = C.c_int64()
                model._check(lib.lbm_read_trajectories(h, buf.ctypes.data_as(capi._dp), seg, C.byref(got)))
                buf = buf.reshape(seg, nparts, 9)
                rows = []
                for t in range(seg):
                    time = time + dt  # model.time += dt in every tick!
                    for p in range(nparts):
                        r = buf[t, p]
                        rows.append((tick_start + t + 1, time, p + 1, r[0:3], r[3:6], r[6:9]))
                append_particle_rows(dims, rows)
            if model.tick in cps:
                write_fluid(model)
    finally:
        if nparts:
            lib.lbm_record_trajectories(h, 0)
        model._check(lib.lbm_output_flush(h))
