"""Failure detection through the C ABI.

Every failure is made on the host: a non-finite value in the initial density
field, a wait target that no count of the persistent tick kernel reaches
(set by lbm_set_wait_limit's test knob, with a short poll limit so the wait
gives up quickly), and a device-memory cap.  No test faults, traps or hangs
the GPU: the kernels' waits are bounded and report through the error word.
"""
from __future__ import annotations

import os
import tempfile

import numpy as np
import pytest

from lbmengine import _capi, config, model as M


def _small(storage="f32", schedule="auto", **kw):
    res = config.resolve_model(dims=3, velocities="D3Q19", collisionModel="trt", latticeParameter=1.0,
                               relaxationTimeRatio=0.7, xlims=(-12.0, 11.0), storage=storage, schedule=schedule, **kw)
    m = M.LBMmodel(res)
    M._add(m, config.resolve_squirmer(3, radius=4.0, position=[0.3, 0.1, -0.2], swimmingSpeed=1e-3, beta=2.0,
                                      coupleForces=True, coupleTorques=True))
    return m


def test_limits_reject_bad_arguments_without_gpu(lib):
    assert lib.lbm_set_memory_limit(-1) == _capi.LBM_ERR_INVALID
    assert lib.lbm_set_wait_limit(None, 100, 0) == _capi.LBM_ERR_INVALID
    assert lib.lbm_set_memory_limit(0) == _capi.LBM_OK


@pytest.mark.gpu
def test_nonfinite_initial_density_raises_numeric(lib):
    rho = np.ones((24, 24, 24))
    rho[5, 7, 9] = np.nan
    m = _small(massDensity=rho, fluidVelocity=np.zeros((24, 24, 24, 3)))
    with pytest.raises(_capi.LbmError) as e:
        m.step(1)
    assert e.value.code == _capi.LBM_ERR_NUMERIC
    assert "density" in str(e.value)
    # the context and other models stay usable
    ok = _small()
    ok.step(3)
    assert np.isfinite(ok.fluidVelocity).all()


@pytest.mark.gpu
@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_diverging_run_raises_numeric(lib, storage):
    """A negative initial density (far below the sentinel's -1e-3) is caught in the first tick."""
    rho = np.ones((24, 24, 24))
    rho[:, :, 3] = -0.5
    m = _small(storage=storage, massDensity=rho, fluidVelocity=np.zeros((24, 24, 24, 3)))
    with pytest.raises(_capi.LbmError) as e:
        m.step(2)
    assert e.value.code == _capi.LBM_ERR_NUMERIC


@pytest.mark.gpu
def test_walls_hold_zero_density_without_raising(lib):
    """Wall nodes carry zero density (as in the reference); the sentinel leaves them alone."""
    res = config.resolve_model(dims=2, latticeParameter=1.0, relaxationTimeRatio=0.9, collisionModel="trt",
                               xlims=(0.0, 15.0), ylims=(0.0, 20.0), walledDimensions=[2], forceDensity=[1e-5, 0.0])
    m = M.LBMmodel(res)
    m.step(50)
    assert float(m.massDensity[:, 0].max()) == 0.0


@pytest.mark.gpu
def test_tick_kernel_wait_gives_up_with_timeout(lib):
    m = _small(schedule="persistent")
    m.step(2)
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "s.lbm")
        m.save_state(path)
        u_ref = None
        assert lib.lbm_set_wait_limit(m.handle, 2000, 1) == 0
        with pytest.raises(_capi.LbmError) as e:
            m.step(1)
        assert e.value.code == _capi.LBM_ERR_TIMEOUT
        # back to normal limits: the handle recovers from its checkpoint
        assert lib.lbm_set_wait_limit(m.handle, 1 << 22, 0) == 0
        m.load_state(path)
        m.step(3)
        ref = _small(schedule="persistent")
        ref.step(5)
        u_ref = ref.fluidVelocity
        np.testing.assert_array_equal(m.fluidVelocity, u_ref)


@pytest.mark.gpu
def test_memory_limit_raises_oom(lib):
    try:
        assert lib.lbm_set_memory_limit(1 << 20) == 0
        with pytest.raises(_capi.LbmError) as e:
            _small()
        assert e.value.code == _capi.LBM_ERR_OOM
        assert "memory limit" in str(e.value)
    finally:
        lib.lbm_set_memory_limit(0)
    _small().step(1)
