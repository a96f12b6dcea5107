"""ctypes binding of the C ABI declared in include/lbm_b200.h.

The shared library ``liblbm_b200.so`` is built in-tree next to this package
(``lbmengine.jl_b200/liblbm_b200.so``) by ``lbmengine.jl_b200/build.py``.
Loading fails loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

LBM_OK = 0
LBM_ERR_INVALID = -1
LBM_ERR_CUDA = -2
LBM_ERR_OOM = -3
LBM_ERR_UNSUPPORTED = -4
LBM_ERR_NUMERIC = -5
LBM_ERR_TIMEOUT = -6
LBM_ERR_STATE = -7
LBM_ERR_NO_DEVICE = -8

LBM_D2Q9, LBM_D3Q15, LBM_D3Q19, LBM_D3Q27 = 9, 15, 19, 27
LBM_BGK, LBM_TRT = 0, 1
LBM_STORE_F32, LBM_STORE_F16, LBM_STORE_BF16, LBM_STORE_F64 = 0, 1, 2, 3
LBM_BEAD, LBM_SQUIRMER = 0, 1
LBM_FORCE_NONE, LBM_FORCE_UNIFORM, LBM_FORCE_FIELD = 0, 1, 2

STORAGE_NAMES = {"f32": LBM_STORE_F32, "f16": LBM_STORE_F16, "bf16": LBM_STORE_BF16, "f64": LBM_STORE_F64}
LBM_SCHEDULE_AUTO, LBM_SCHEDULE_STREAM, LBM_SCHEDULE_PERSISTENT = 0, 1, 3
SCHEDULE_NAMES = {"auto": LBM_SCHEDULE_AUTO, "stream": LBM_SCHEDULE_STREAM, "persistent": LBM_SCHEDULE_PERSISTENT}
LBM_RULES_GPU_MODULE, LBM_RULES_CPU_MODULE = 0, 1
LBM_BULK_AUTO, LBM_BULK_VECTOR, LBM_BULK_TMA, LBM_BULK_SCALAR = 0, 1, 2, 3
LBM_OBSERVABLE_VELOCITY, LBM_OBSERVABLE_FORCE = 0, 1
LBM_ROUND_STOCHASTIC, LBM_ROUND_NEAREST = 0, 1
(LBM_INTERACTION_LINEAR, LBM_INTERACTION_BISTABLE, LBM_INTERACTION_POLAR, LBM_INTERACTION_LENNARD_JONES,
 LBM_INTERACTION_DIPOLE) = range(5)
ROUNDING_NAMES = {"stochastic": LBM_ROUND_STOCHASTIC, "nearest": LBM_ROUND_NEAREST}
RULES_NAMES = {"gpu": LBM_RULES_GPU_MODULE, "cpu": LBM_RULES_CPU_MODULE}

_dp = C.POINTER(C.c_double)
_u8p = C.POINTER(C.c_uint8)


class LbmConfig(C.Structure):
    _fields_ = [
        ("dims", C.c_int32),
        ("lattice", C.c_int32),
        ("n", C.c_int64 * 3),
        ("coords", _dp * 3),
        ("x0", C.c_double * 3),
        ("dx", C.c_double),
        ("tau", C.c_double),
        ("tau_minus", C.c_double),
        ("collision", C.c_int32),
        ("compressible", C.c_int32),
        ("force_mode", C.c_int32),
        ("storage", C.c_int32),
        ("force", C.c_double * 3),
        ("force_field", _dp),
        ("wall_mask", _u8p),
        ("wall_velocity", _dp),
        ("rho_init", _dp),
        ("u_init", _dp),
        ("rho_uniform", C.c_double),
        ("u_uniform", C.c_double * 3),
        ("rho_ref", C.c_double),
        ("store_scale", C.c_double),
        ("device", C.c_int32),
        ("schedule", C.c_int32),
        ("particle_rules", C.c_int32),
        ("rounding", C.c_int32),
    ]


class LbmParticleParams(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("couple_forces", C.c_int32),
        ("couple_torques", C.c_int32),
        ("reserved", C.c_int32),
        ("radius", C.c_double),
        ("mass_density", C.c_double),
        ("position", C.c_double * 3),
        ("velocity", C.c_double * 3),
        ("angular_velocity", C.c_double * 3),
        ("swimming_direction", C.c_double * 3),
        ("B1", C.c_double),
        ("B2", C.c_double),
    ]


class LbmParticleState(C.Structure):
    _fields_ = [
        ("id", C.c_int32),
        ("kind", C.c_int32),
        ("couple_forces", C.c_int32),
        ("couple_torques", C.c_int32),
        ("radius", C.c_double),
        ("inverse_mass", C.c_double),
        ("inverse_inertia", C.c_double),
        ("B1", C.c_double),
        ("B2", C.c_double),
        ("position", C.c_double * 3),
        ("velocity", C.c_double * 3),
        ("angular_velocity", C.c_double * 3),
        ("swimming_direction", C.c_double * 3),
        ("last_force", C.c_double * 3),
        ("last_torque", C.c_double * 3),
    ]


class LbmInfo(C.Structure):
    _fields_ = [
        ("dims", C.c_int32),
        ("lattice", C.c_int32),
        ("q", C.c_int32),
        ("storage", C.c_int32),
        ("n", C.c_int64 * 3),
        ("cells", C.c_int64),
        ("tick", C.c_int64),
        ("time", C.c_double),
        ("num_particles", C.c_int32),
        ("bytes_per_population", C.c_int32),
        ("device_bytes", C.c_int64),
        ("bulk_kernel", C.c_int32),
        ("bulk_threads", C.c_int32),
        ("bulk_stages", C.c_int32),
        ("reserved", C.c_int32),
    ]


class LbmInteraction(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("id1", C.c_int32),
        ("id2", C.c_int32),
        ("id3", C.c_int32),
        ("p", C.c_double * 4),
    ]


class LbmProfile(C.Structure):
    _fields_ = [
        ("total_ms", C.c_double),
        ("bulk_ms", C.c_double),
        ("fixup_ms", C.c_double),
        ("particles_ms", C.c_double),
        ("steps", C.c_int64),
        ("launches", C.c_int64),
        ("profiled_steps", C.c_int64),
        ("bulk_cells", C.c_int64),
        ("fixup_entries", C.c_int64),
    ]


class LbmBatchTuning(C.Structure):
    _fields_ = [
        ("schedule", C.c_int32),
        ("ctas_per_sm", C.c_int32),
        ("tile_order", C.c_int32),
        ("tile_cta", C.c_int32),
        ("ms_per_tick", C.c_double),
    ]


class LbmAdjointSpec(C.Structure):
    _fields_ = [
        ("ticks", C.c_int64),
        ("window_begin", C.c_int64),
        ("window_end", C.c_int64),
        ("direction", C.c_double * 3),
        ("tau_minus_slope", C.c_double),
        ("snapshots", C.c_int32),
        ("observable", C.c_int32),
    ]


class LbmAdjointResult(C.Structure):
    _fields_ = [
        ("value", C.c_double),
        ("dB1", C.c_double),
        ("dB2", C.c_double),
        ("dtau", C.c_double),
        ("dtau_plus", C.c_double),
        ("dtau_minus", C.c_double),
        ("dF", C.c_double * 3),
        ("forward_ticks", C.c_int64),
        ("snapshots_used", C.c_int32),
        ("reserved", C.c_int32),
        ("ms", C.c_double),
    ]


# (name, restype, argtypes) for every symbol of include/lbm_b200.h
PROTOTYPES = [
    ("lbm_abi_version", C.c_int32, []),
    ("lbm_build_info", C.c_char_p, []),
    ("lbm_create", C.c_int, [C.POINTER(LbmConfig), C.POINTER(C.c_void_p)]),
    ("lbm_add_particle", C.c_int, [C.c_void_p, C.POINTER(LbmParticleParams), C.POINTER(C.c_int32)]),
    ("lbm_step", C.c_int, [C.c_void_p, C.c_int64]),
    ("lbm_get_fields", C.c_int, [C.c_void_p, _dp, _dp]),
    ("lbm_get_distributions", C.c_int, [C.c_void_p, _dp]),
    ("lbm_get_stress", C.c_int, [C.c_void_p, _dp]),
    ("lbm_get_totals", C.c_int, [C.c_void_p, _dp, _dp]),
    ("lbm_record_trajectories", C.c_int, [C.c_void_p, C.c_int64]),
    ("lbm_read_trajectories", C.c_int, [C.c_void_p, _dp, C.c_int64, C.POINTER(C.c_int64)]),
    ("lbm_write_fluid_csv", C.c_int, [C.c_void_p, C.c_char_p]),
    ("lbm_output_flush", C.c_int, [C.c_void_p]),
    ("lbm_set_distributions", C.c_int, [C.c_void_p, _dp]),
    ("lbm_get_particles", C.c_int, [C.c_void_p, C.POINTER(LbmParticleState), C.c_int32, C.POINTER(C.c_int32)]),
    ("lbm_set_particle", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(LbmParticleState)]),
    ("lbm_get_mask", C.c_int, [C.c_void_p, C.c_int32, _u8p]),
    ("lbm_record_force", C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
    ("lbm_set_interactions", C.c_int, [C.c_void_p, C.POINTER(LbmInteraction), C.c_int32]),
    ("lbm_get_links", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int8), C.c_int64,
                                C.POINTER(C.c_int64)]),
    ("lbm_get_info", C.c_int, [C.c_void_p, C.POINTER(LbmInfo)]),
    ("lbm_set_profiling", C.c_int, [C.c_void_p, C.c_int32]),
    ("lbm_get_profile", C.c_int, [C.c_void_p, C.POINTER(LbmProfile)]),
    ("lbm_time_kernel", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_double)]),
    ("lbm_save_state", C.c_int, [C.c_void_p, C.c_char_p]),
    ("lbm_load_state", C.c_int, [C.c_void_p, C.c_char_p]),
    ("lbm_step_noalloc", C.c_int, [C.c_void_p, C.c_int64]),
    ("lbm_set_wait_limit", C.c_int, [C.c_void_p, C.c_int64, C.c_int32]),
    ("lbm_set_memory_limit", C.c_int, [C.c_int64]),
    ("lbm_set_bulk_kernel", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32]),
    ("lbm_last_error", C.c_char_p, [C.c_void_p]),
    ("lbm_last_global_error", C.c_char_p, []),
    ("lbm_destroy", None, [C.c_void_p]),
    ("lbm_adjoint", C.c_int, [C.c_void_p, C.POINTER(LbmAdjointSpec), C.POINTER(LbmAdjointResult)]),
    ("lbm_batch_create", C.c_int, [C.c_int32, C.POINTER(LbmConfig), C.POINTER(C.c_int32),
                                   C.POINTER(LbmParticleParams), C.POINTER(C.c_void_p)]),
    ("lbm_batch_size", C.c_int32, [C.c_void_p]),
    ("lbm_batch_replica", C.c_void_p, [C.c_void_p, C.c_int32]),
    ("lbm_batch_step", C.c_int, [C.c_void_p, C.c_int64]),
    ("lbm_batch_autotune", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(LbmBatchTuning), C.c_int32,
                                     C.POINTER(C.c_int32), C.POINTER(LbmBatchTuning)]),
    ("lbm_batch_set_tuning", C.c_int, [C.c_void_p, C.POINTER(LbmBatchTuning)]),
    ("lbm_batch_get_tuning", C.c_int, [C.c_void_p, C.POINTER(LbmBatchTuning)]),
    ("lbm_batch_set_profiling", C.c_int, [C.c_void_p, C.c_int32]),
    ("lbm_batch_get_profile", C.c_int, [C.c_void_p, C.POINTER(LbmProfile)]),
    ("lbm_batch_status", C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    ("lbm_batch_last_error", C.c_char_p, [C.c_void_p]),
    ("lbm_batch_destroy", None, [C.c_void_p]),
]

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "liblbm_b200.so")

_lib = None


class LbmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def load(path: str | None = None) -> C.CDLL:
    """Load liblbm_b200.so and declare its prototypes (raises if absent)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise FileNotFoundError(
            f"{p} not found: build it with `python lbmengine.jl_b200/build.py` (nvcc, sm_100a)")
    lib = C.CDLL(p)
    for name, res, args in PROTOTYPES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(lib, handle, code: int) -> None:
    if code != LBM_OK:
        if handle:
            msg = lib.lbm_last_error(handle)
        else:
            msg = lib.lbm_last_global_error()
        raise LbmError(code, (msg or b"").decode(errors="replace"))
