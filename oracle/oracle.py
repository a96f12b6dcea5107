"""ctypes driver of the FP64 CPU oracle (TEST INFRASTRUCTURE ONLY).

Loaded only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg,
always as the checker or the timed CPU baseline, never as a product path.
The oracle restates LBMengine.jl's GPU-module time step in FP64, and with
lbm_config.particle_rules == LBM_RULES_CPU_MODULE the CPU module's particle
update; parity is unpinned by the reference itself (it ships no tests or
golden vectors and its Julia toolchain is not available to run it).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
PKG = os.path.join(REPO, "lbmengine.jl_b200")
if PKG not in sys.path:
    sys.path.insert(0, PKG)

from lbmengine import _capi as capi  # noqa: E402  (struct layouts of include/lbm_b200.h)

LIB_PATH = os.path.join(HERE, "_build", "liblbm_oracle.so")

_lib = None


def build(quiet: bool = True) -> str:
    """Compile the oracle with its Makefile (g++, OpenMP, no FP contraction)."""
    out = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)
    return LIB_PATH


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    lib = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    dp = C.POINTER(C.c_double)
    lib.orc_last_error.restype = C.c_char_p
    lib.orc_set_threads.argtypes = [C.c_int]
    lib.orc_max_threads.restype = C.c_int
    lib.orc_create.argtypes = [C.POINTER(capi.LbmConfig), C.POINTER(vp)]
    lib.orc_add_particle.argtypes = [vp, C.POINTER(capi.LbmParticleParams), C.POINTER(C.c_int32)]
    lib.orc_step.argtypes = [vp, C.c_int64]
    lib.orc_get_fields.argtypes = [vp, dp, dp]
    lib.orc_get_distributions.argtypes = [vp, dp]
    lib.orc_set_distributions.argtypes = [vp, dp]
    lib.orc_get_particles.argtypes = [vp, C.POINTER(capi.LbmParticleState), C.c_int32, C.POINTER(C.c_int32)]
    lib.orc_get_mask.argtypes = [vp, C.c_int32, C.POINTER(C.c_uint8)]
    lib.orc_set_particle.argtypes = [vp, C.c_int32, C.POINTER(capi.LbmParticleState)]
    lib.orc_record_force.argtypes = [vp, C.c_int32, C.c_int32]
    lib.orc_get_stress.argtypes = [vp, dp]
    lib.orc_set_interactions.argtypes = [vp, C.POINTER(capi.LbmInteraction), C.c_int32]
    lib.ord_record_force.argtypes = [vp, C.c_int32, C.c_int32]
    lib.ord_particle_force.argtypes = [vp, C.c_int32, dp, dp]
    lib.orc_get_links.argtypes = [vp, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int8), C.c_int64,
                                  C.POINTER(C.c_int64)]
    lib.orc_get_info.argtypes = [vp, C.POINTER(capi.LbmInfo)]
    lib.orc_velocity_set.argtypes = [C.c_int32, C.POINTER(C.c_int8), dp, C.POINTER(C.c_int32)]
    lib.orc_destroy.argtypes = [vp]
    lib.ord_directions.restype = C.c_int
    lib.ord_create.argtypes = [C.POINTER(capi.LbmConfig), dp, dp, dp, C.POINTER(vp)]
    lib.ord_add_particle.argtypes = [vp, C.POINTER(capi.LbmParticleParams), dp, dp, C.POINTER(C.c_int32)]
    lib.ord_step.argtypes = [vp, C.c_int64]
    lib.ord_particle.argtypes = [vp, C.c_int32, dp, dp]
    lib.ord_get_fields.argtypes = [vp, dp, dp]
    lib.ord_destroy.argtypes = [vp]
    _lib = lib
    return lib


def _check(code):
    if code != 0:
        raise capi.LbmError(code, load().orc_last_error().decode())


def velocity_set(q: int):
    lib = load()
    c = np.zeros((q, 3), dtype=np.int8)
    w = np.zeros(q, dtype=np.float64)
    opp = np.zeros(q, dtype=np.int32)
    _check(lib.orc_velocity_set(q, c.ctypes.data_as(C.POINTER(C.c_int8)), w.ctypes.data_as(C.POINTER(C.c_double)),
                                opp.ctypes.data_as(C.POINTER(C.c_int32))))
    return c, w, opp


def set_threads(n: int) -> None:
    load().orc_set_threads(int(n))


def max_threads() -> int:
    return int(load().orc_max_threads())


class OracleModel:
    """One FP64 CPU model built from a resolved config (lbmengine.config.resolve_model)."""

    def __init__(self, resolved):
        self.lib = load()
        self.res = resolved
        self.h = C.c_void_p()
        _check(self.lib.orc_create(C.byref(resolved.cfg), C.byref(self.h)))
        info = self.info()
        self.q = info.q
        self.dims = info.dims
        self.shape = tuple(info.n[a] for a in range(self.dims))
        self.cells = info.cells

    def info(self):
        inf = capi.LbmInfo()
        _check(self.lib.orc_get_info(self.h, C.byref(inf)))
        return inf

    def add_particle(self, params) -> int:
        pid = C.c_int32()
        _check(self.lib.orc_add_particle(self.h, C.byref(params), C.byref(pid)))
        return pid.value

    def step(self, n: int) -> None:
        _check(self.lib.orc_step(self.h, int(n)))

    def fields(self):
        rho = np.zeros(self.cells, dtype=np.float64)
        u = np.zeros(self.cells * self.dims, dtype=np.float64)
        _check(self.lib.orc_get_fields(self.h, rho.ctypes.data_as(capi._dp), u.ctypes.data_as(capi._dp)))
        return rho, u.reshape(self.dims, self.cells)

    def stress(self):
        """viscousStressTensor: (d, d, N) with entry [a, b] the field sigma_ab."""
        s = np.zeros(self.cells * self.dims * self.dims, dtype=np.float64)
        _check(self.lib.orc_get_stress(self.h, s.ctypes.data_as(capi._dp)))
        return s.reshape(self.dims, self.dims, self.cells).transpose(1, 0, 2)

    def distributions(self):
        f = np.zeros(self.cells * self.q, dtype=np.float64)
        _check(self.lib.orc_get_distributions(self.h, f.ctypes.data_as(capi._dp)))
        return f.reshape(self.q, self.cells)

    def set_distributions(self, f):
        f = np.ascontiguousarray(f, dtype=np.float64).ravel()
        _check(self.lib.orc_set_distributions(self.h, f.ctypes.data_as(capi._dp)))

    def particles(self):
        cnt = C.c_int32()
        _check(self.lib.orc_get_particles(self.h, None, 0, C.byref(cnt)))
        arr = (capi.LbmParticleState * max(1, cnt.value))()
        _check(self.lib.orc_get_particles(self.h, arr, cnt.value, C.byref(cnt)))
        return list(arr)[:cnt.value]

    def set_particle(self, pid: int, state) -> None:
        """Move particle `pid` to another state (position, velocity, angular velocity,
        swimming direction of an LbmParticleState) and re-voxelise it there."""
        _check(self.lib.orc_set_particle(self.h, pid, C.byref(state)))

    def set_interactions(self, items) -> None:
        """particleInteractions as a list of LbmInteraction items (pairs flattened in order)."""
        arr = (capi.LbmInteraction * max(1, len(items)))(*items)
        _check(self.lib.orc_set_interactions(self.h, arr, len(items)))

    def record_force(self, pid: int, on: bool = True) -> None:
        """Accumulate particle pid's momentum-exchange force even when it is not
        coupled (reported as last_force, never applied): the drag of a held particle."""
        _check(self.lib.orc_record_force(self.h, pid, int(bool(on))))

    def mask(self, pid: int):
        m = np.zeros(self.cells, dtype=np.uint8)
        _check(self.lib.orc_get_mask(self.h, pid, m.ctypes.data_as(capi._u8p)))
        return m

    def links(self, pid: int):
        n = C.c_int64()
        _check(self.lib.orc_get_links(self.h, pid, None, None, 0, C.byref(n)))
        cells = np.zeros(max(1, n.value), dtype=np.int64)
        dirs = np.zeros(max(1, n.value), dtype=np.int8)
        _check(self.lib.orc_get_links(self.h, pid, cells.ctypes.data_as(C.POINTER(C.c_int64)),
                                      dirs.ctypes.data_as(C.POINTER(C.c_int8)), n.value, C.byref(n)))
        return cells[:n.value], dirs[:n.value]

    def close(self):
        if self.h:
            self.lib.orc_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# derivative directions of the dual-number oracle
DIRECTIONS = ("B1", "B2", "tau", "Fx", "Fy", "Fz")


def tau_minus_slope(resolved) -> float:
    """d tau- / d tau+ at fixed magic parameter: tau- = L dt^2 / (tau+ - dt/2) + dt/2 (TRT), 0 for BGK."""
    if resolved.collision != "trt":
        return 0.0
    lam = resolved.kineticParameter
    if isinstance(lam, str):
        raise ValueError("the dual oracle needs a numeric kineticParameter")
    dt = resolved.dt
    return -float(lam) * dt * dt / (resolved.tau - dt / 2) ** 2


class DualOracle:
    """The oracle with forward-mode dual numbers: every quantity carries its
    derivatives along DIRECTIONS (B1 and B2 of the particles added, the
    relaxation time tau+ with tau- following at fixed magic parameter, and the
    three components of the uniform body force).  Values equal the FP64
    oracle's; solid masks are taken as computed (comparisons see values)."""

    def __init__(self, resolved):
        self.lib = load()
        K = int(self.lib.ord_directions())
        assert K == len(DIRECTIONS)
        self.K = K
        e = np.eye(K)
        tp = np.ascontiguousarray(e[2])
        tm = np.ascontiguousarray(e[2] * tau_minus_slope(resolved))
        fs = np.ascontiguousarray(e[3:6])
        self._seeds = (tp, tm, fs)
        self.h = C.c_void_p()
        dp = capi._dp
        _check(self.lib.ord_create(C.byref(resolved.cfg), tp.ctypes.data_as(dp), tm.ctypes.data_as(dp),
                                   fs.ctypes.data_as(dp), C.byref(self.h)))

    def add_particle(self, params) -> int:
        e = np.eye(self.K)
        b1, b2 = np.ascontiguousarray(e[0]), np.ascontiguousarray(e[1])
        pid = C.c_int32()
        _check(self.lib.ord_add_particle(self.h, C.byref(params), b1.ctypes.data_as(capi._dp),
                                         b2.ctypes.data_as(capi._dp), C.byref(pid)))
        return pid.value

    def step(self, n: int) -> None:
        _check(self.lib.ord_step(self.h, int(n)))

    def particle(self, pid: int = 1):
        """(values, derivatives): dicts of position, velocity, angular_velocity,
        swimming_direction -> (3,) values and (3, K) derivatives."""
        v = np.zeros(12)
        d = np.zeros((12, self.K))
        _check(self.lib.ord_particle(self.h, pid, v.ctypes.data_as(capi._dp), d.ctypes.data_as(capi._dp)))
        names = ("position", "velocity", "angular_velocity", "swimming_direction")
        return ({n: v[3 * i:3 * i + 3] for i, n in enumerate(names)},
                {n: d[3 * i:3 * i + 3] for i, n in enumerate(names)})

    def record_force(self, pid: int = 1, on: bool = True) -> None:
        _check(self.lib.ord_record_force(self.h, pid, int(bool(on))))

    def particle_force(self, pid: int = 1):
        """(values (3,), derivatives (3, K)) of the last tick's momentum-exchange force."""
        v = np.zeros(3)
        d = np.zeros((3, self.K))
        _check(self.lib.ord_particle_force(self.h, pid, v.ctypes.data_as(capi._dp), d.ctypes.data_as(capi._dp)))
        return v, d

    def close(self):
        if self.h:
            self.lib.ord_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
