"""Allocation-free stepping: lbm_step_noalloc against lbm_step, through the C ABI.

Some callers cannot allocate device memory once their run has started: they
reserve all of it up front (another library's memory pool, a fixed budget per
process) or run under a policy that forbids allocation after initialisation.
lbm_step_noalloc serves them; it must produce the same ticks as lbm_step,
whose first call (and first call after adding a particle) instantiates CUDA
graphs.  The momentum-exchange partials live in a fixed device array compiled
into the library and shared by all calls in the process.

This file is named so that pytest collects it last: if it fails, a run that
stops at the first failure has already run every other test.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from parity_cases import CASES, build_pair

pytestmark = pytest.mark.gpu


def _twins(name, storage="f32"):
    case = CASES[name]
    res, ref, _ = build_pair(case, storage=storage)
    _, nal, _ = build_pair(case, storage=storage)
    return res, ref, nal


# The two entry points launch the same kernels on the same inputs in the same
# order (lbm_step from CUDA graphs, lbm_step_noalloc directly), so populations
# and particle state must agree bit for bit.  The cases cover one and several
# particles, a wall, FP16 storage, a link list longer than the fix-up's 32 CTAs
# per particle, and the chunk-walking fix-up of many particles (the largest
# users of the shared array).
@pytest.mark.parametrize("name,storage", [("d3q19_trt_guo_squirmer", "f32"), ("d3q19_multi", "f32"),
                                          ("d2q9_bgk_lid_bead", "f32"), ("d3q19_trt_guo_squirmer", "f16"),
                                          ("d3q19_large_squirmer", "f32"), ("d3q19_twelve_squirmers", "f32")])
def test_noalloc_matches_lbm_step_on_two_calls(lib, name, storage):
    res, ref, nal = _twins(name, storage)
    for n in (7, 13):  # two calls in a row; the second reuses the shared array
        ref.step(n)
        rc = lib.lbm_step_noalloc(nal.handle, n)
        assert rc == 0, lib.lbm_last_error(nal.handle).decode()
        assert nal.tick == ref.tick
        np.testing.assert_array_equal(nal.distributions, ref.distributions)
        for a, b in zip(nal.particle_states(), ref.particle_states()):
            for field in ("position", "velocity", "angular_velocity", "swimming_direction", "last_force",
                          "last_torque"):
                assert list(getattr(a, field)) == list(getattr(b, field)), field


def test_noalloc_rejects_models_beyond_the_fixed_array(lib):
    """A particle whose near box needs more partial slots than the array holds."""
    from lbmengine import _capi, config, model
    res = config.resolve_model(dims=2, latticeParameter=1.0, relaxationTimeRatio=0.8, collisionModel="bgk",
                               xlims=(-520.0, 519.0), storage="f32")
    m = model.LBMmodel(res)
    model._add(m, config.resolve_bead(2, radius=515.0, position=[0.0, 0.0]))
    rc = lib.lbm_step_noalloc(m.handle, 1)
    assert rc == _capi.LBM_ERR_UNSUPPORTED
    assert b"fixed array holds 16384" in lib.lbm_last_error(m.handle)
    assert m.tick == 0
