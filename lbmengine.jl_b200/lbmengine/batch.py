"""Batches of independent replicas over the C ABI (lbm_batch_* in include/lbm_b200.h).

A replica is a model (modelInit keywords) with its particles (addSquirmer /
addBead keywords).  All replicas share the velocity set, collision model and
storage format; grid sizes, relaxation times, forces and particles may
differ.  Every tick advances all of them: their bulk tiles, boundary fix-up
blocks and particle updates are the items of one GPU work queue.  The
reference has no batch API; a sweep there is a loop over modelInit and
LBMpropagate! (src/gpu/initMethods.jl:440, src/gpu/fluids.jl:228).
"""
from __future__ import annotations

import ctypes as C
from types import SimpleNamespace

from . import _capi as capi
from . import config as cfgmod
from . import model as mdl


class LBMbatch:
    """``replicas``: a list of ``(model_kwargs, [(kind, particle_kwargs), ...])``
    with ``kind`` "squirmer" or "bead"."""

    def __init__(self, replicas, lib=None):
        self._lib = lib or capi.load()
        self._b = C.c_void_p()
        resolved, params, counts = [], [], []
        for mkw, parts in replicas:
            res = cfgmod.resolve_model(**mkw)
            resolved.append(res)
            counts.append(len(parts))
            for kind, pkw in parts:
                if kind == "squirmer":
                    params.append(cfgmod.resolve_squirmer(res.dims, **pkw))
                elif kind == "bead":
                    params.append(cfgmod.resolve_bead(res.dims, **pkw))
                else:
                    raise ValueError(f"unknown particle kind {kind!r}")
        n = len(resolved)
        if n == 0:
            raise ValueError("a batch needs at least one replica")
        cfgs = (capi.LbmConfig * n)(*[r.cfg for r in resolved])
        cnt = (C.c_int32 * n)(*counts)
        prm = (capi.LbmParticleParams * max(1, len(params)))(*params)
        self._res = resolved  # keeps the host arrays the configurations point to alive
        capi.check(self._lib, None, self._lib.lbm_batch_create(n, cfgs, cnt, prm, C.byref(self._b)))
        self.replicas = []
        for i, res in enumerate(resolved):
            m = mdl.LBMmodel(res, lib=self._lib, handle=self._lib.lbm_batch_replica(self._b, i))
            if counts[i]:
                m.schemes += [s for s in ("ladd", "bounceBack") if s not in m.schemes]
            self.replicas.append(m)
        self.cells = sum(m._cells for m in self.replicas)

    def _check(self, code):
        if code != capi.LBM_OK:
            raise capi.LbmError(code, (self._lib.lbm_batch_last_error(self._b) or b"").decode(errors="replace"))

    def __len__(self):
        return len(self.replicas)

    def step(self, n: int) -> None:
        """Advance every replica by n ticks."""
        self._check(self._lib.lbm_batch_step(self._b, int(n)))

    def status(self):
        """Per replica: LBM_OK, or LBM_ERR_NUMERIC once its density went non-finite or negative."""
        st = (C.c_int32 * len(self))()
        self._lib.lbm_batch_status(self._b, st)
        return list(st)

    def autotune(self, ticks: int = 16):
        """Time every tuning candidate and keep the fastest: (chosen, [candidates])."""
        cap = 64
        res = (capi.LbmBatchTuning * cap)()
        count = C.c_int32()
        chosen = capi.LbmBatchTuning()
        self._check(self._lib.lbm_batch_autotune(self._b, int(ticks), res, cap, C.byref(count), C.byref(chosen)))
        return _tuning(chosen), [_tuning(res[i]) for i in range(min(cap, count.value))]

    @property
    def tuning(self):
        t = capi.LbmBatchTuning()
        self._check(self._lib.lbm_batch_get_tuning(self._b, C.byref(t)))
        return _tuning(t)

    def set_tuning(self, schedule="persistent", ctas_per_sm=8, tile_order=0, tile_cta=0) -> None:
        t = capi.LbmBatchTuning(schedule=capi.SCHEDULE_NAMES[schedule], ctas_per_sm=int(ctas_per_sm),
                                tile_order=int(tile_order), tile_cta=int(tile_cta))
        self._check(self._lib.lbm_batch_set_tuning(self._b, C.byref(t)))

    def set_profiling(self, level: int) -> None:
        self._check(self._lib.lbm_batch_set_profiling(self._b, int(level)))

    def profile(self):
        p = capi.LbmProfile()
        self._check(self._lib.lbm_batch_get_profile(self._b, C.byref(p)))
        return p

    def close(self):
        for m in getattr(self, "replicas", []):
            m.close()
        if self._b:
            self._lib.lbm_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_SCHEDULES = {v: k for k, v in capi.SCHEDULE_NAMES.items()}


def _tuning(t):
    return SimpleNamespace(schedule=_SCHEDULES.get(t.schedule, t.schedule), ctas_per_sm=t.ctas_per_sm,
                           tile_order=t.tile_order, tile_cta=t.tile_cta, ms_per_tick=t.ms_per_tick)
