"""The bulk stream-collide kernels give bit-identical ticks.

The vector kernel (in every CTA shape) and the TMA kernel (bulk copies
through a shared-memory ring) run the same collision on the same values and
store with the same rounding, so whole runs must agree bit for bit, in every
storage format and launch shape.  The FP16/BF16 stores round stochastically with a dither that
is a function of (cell, direction, value) only, so results do not depend on
how the ticks are split into calls either.
"""
from __future__ import annotations

import numpy as np
import pytest

from lbmengine import _capi, config, model as M
from parity_cases import CASES, build_pair

pytestmark = pytest.mark.gpu


def _box(side, storage, particles=True):
    h = side // 2
    res = config.resolve_model(dims=3, velocities="D3Q19", collisionModel="trt", kineticParameter=3 / 16,
                               latticeParameter=1.0, relaxationTimeRatio=0.7, xlims=(-float(h), float(side - h - 1)),
                               forceDensity=[1e-5, 0.0, 0.0], storage=storage)
    m = M.LBMmodel(res)
    if particles:
        M._add(m, config.resolve_squirmer(3, radius=5.0, position=[0.3, -0.2, 0.1], swimmingSpeed=1e-3, beta=-3.0,
                                          swimmingDirection=[0.6, 0.0, 0.8], coupleForces=True,
                                          coupleTorques=True))
    return m


def _kernel(m, kind, threads=0, stages=0):
    rc = m._lib.lbm_set_bulk_kernel(m.handle, kind, threads, stages)
    assert rc == 0, m._lib.lbm_last_error(m.handle).decode()
    return m.info()


@pytest.mark.parametrize("storage", ["f32", "f16", "bf16"])
@pytest.mark.parametrize("side,threads,stages", [(64, 0, 0), (64, 128, 4), (32, 256, 2), (64, 256, 2)])
def test_tma_kernel_matches_vector_kernel(lib, storage, side, threads, stages):
    ref, tma = _box(side, storage), _box(side, storage)
    assert _kernel(ref, _capi.LBM_BULK_VECTOR).bulk_kernel == _capi.LBM_BULK_VECTOR
    inf = _kernel(tma, _capi.LBM_BULK_TMA, threads, stages)
    assert inf.bulk_kernel == _capi.LBM_BULK_TMA
    for n in (1, 6, 17):
        ref.step(n)
        tma.step(n)
        np.testing.assert_array_equal(tma.distributions, ref.distributions)
    for a, b in zip(tma.particle_states(), ref.particle_states()):
        assert list(a.position) == list(b.position) and list(a.last_force) == list(b.last_force)


@pytest.mark.parametrize("name", ["d3q19_trt_guo_squirmer", "d2q9_trt_channel", "d2q9_incompressible",
                                  "d2q9_bgk_squirmer", "d3q19_multi"])
def test_tma_kernel_on_parity_cases(lib, name):
    """Other velocity sets, walls and several particles: the TMA kernel where it applies."""
    case = CASES[name]
    _, ref, _ = build_pair(case, storage="f32")
    _, tma, _ = build_pair(case, storage="f32")
    rc_ref = lib.lbm_set_bulk_kernel(ref.handle, _capi.LBM_BULK_VECTOR, 0, 0)
    rc = lib.lbm_set_bulk_kernel(tma.handle, _capi.LBM_BULK_TMA, 0, 0)
    if rc == _capi.LBM_ERR_UNSUPPORTED:
        assert b"TMA" in lib.lbm_last_error(tma.handle)
        pytest.skip("x-rows of this case do not fit the TMA kernel")
    assert rc == 0 and rc_ref == 0
    ref.step(case["steps"])
    tma.step(case["steps"])
    np.testing.assert_array_equal(tma.distributions, ref.distributions)


def test_tma_kernel_rejects_rows_it_cannot_take(lib):
    res = config.resolve_model(dims=3, velocities="D3Q19", collisionModel="trt", latticeParameter=1.0,
                               relaxationTimeRatio=0.7, xlims=(-12.0, 11.0))  # 24 nodes: 6 threads per row
    m = M.LBMmodel(res)
    assert lib.lbm_set_bulk_kernel(m.handle, _capi.LBM_BULK_TMA, 0, 0) == _capi.LBM_ERR_UNSUPPORTED
    assert m.info().bulk_kernel == _capi.LBM_BULK_VECTOR
    assert lib.lbm_set_bulk_kernel(m.handle, 7, 0, 0) == _capi.LBM_ERR_INVALID


@pytest.mark.parametrize("storage", ["f16", "bf16"])
def test_dithered_rounding_does_not_depend_on_call_chunking(lib, storage):
    a, b = _box(32, storage), _box(32, storage)
    a.step(23)
    for n in (1, 4, 2, 16):
        b.step(n)
    np.testing.assert_array_equal(a.distributions, b.distributions)
    c = _box(32, storage)
    for _ in range(23):
        assert lib.lbm_step_noalloc(c.handle, 1) == 0
    np.testing.assert_array_equal(a.distributions, c.distributions)



@pytest.mark.parametrize("storage", ["f32", "f16", "bf16"])
@pytest.mark.parametrize("vel,nx,threads", [("D3Q19", 128, 128), ("D3Q19", 64, 128), ("D3Q19", 32, 256),
                                            ("D3Q27", 32, 128), ("D2Q9", 64, 256), ("D2Q9", 16, 32)])
@pytest.mark.parametrize("rounding", ["stochastic", "nearest"])
def test_vector_kernel_cta_shapes_agree(lib, storage, vel, nx, threads, rounding):
    """The default shape (64 threads) against another CTA size."""
    if storage == "f32" and rounding == "nearest":
        pytest.skip("FP32 stores do not round")
    d = 2 if vel == "D2Q9" else 3
    ms = []
    for t in (0, threads):
        h = nx // 2
        res = config.resolve_model(dims=d, velocities=vel, collisionModel="trt", kineticParameter=3 / 16,
                                   latticeParameter=1.0, relaxationTimeRatio=0.7,
                                   xlims=(-float(h), float(nx - h - 1)), ylims=(-8.0, 7.0), zlims=(-6.0, 5.0),
                                   forceDensity=[1e-5] + [0.0] * (d - 1), storage=storage, rounding=rounding)
        m = M.LBMmodel(res)
        M._add(m, config.resolve_squirmer(d, radius=4.0, position=[0.3, -0.2, 0.1][:d], swimmingSpeed=1e-3,
                                          beta=-3.0, swimmingDirection=[0.6, 0.0, 0.8] if d == 3 else [0.6, 0.8],
                                          coupleForces=True, coupleTorques=True))
        inf = _kernel(m, _capi.LBM_BULK_VECTOR, t)
        assert inf.bulk_threads == (threads if t else 64)
        ms.append(m)
    ref, other = ms
    for n in (1, 6, 17):
        ref.step(n)
        other.step(n)
        np.testing.assert_array_equal(other.distributions, ref.distributions)
    for a, b in zip(other.particle_states(), ref.particle_states()):
        assert list(a.position) == list(b.position) and list(a.last_force) == list(b.last_force)


@pytest.mark.parametrize("storage", ["f32", "f16"])
@pytest.mark.parametrize("vel,nx", [("D3Q19", 96), ("D3Q19", 192), ("D2Q9", 192), ("D2Q9", 48)])
def test_96_thread_ctas_against_the_oracle(lib, oracle_mod, storage, vel, nx):
    """Rows of 96 or 192 nodes (24 or 48 threads) fill 96-thread CTAs without
    idle threads; checked against the FP64 oracle with the parity tolerances
    (FP16 density to 3e-5)."""
    from test_parity_gpu import TOL, compare_state
    d = 2 if vel == "D2Q9" else 3
    h = nx // 2
    model = dict(dims=d, velocities=vel, collisionModel="trt", kineticParameter=3 / 16, latticeParameter=1.0,
                 relaxationTimeRatio=0.7, xlims=(-float(h), float(nx - h - 1)), ylims=(-16.0, 15.0),
                 forceDensity=[1e-5] + [0.0] * (d - 1))
    if d == 3:
        model["zlims"] = (-16.0, 15.0)
    sq = dict(radius=4.5, position=[0.3, -0.2, 0.1][:d], swimmingSpeed=5e-4 / 1.5 * 4, beta=-5.0,
              swimmingDirection=[0.6, 0.0, 0.8] if d == 3 else [0.6, 0.8], coupleForces=True, coupleTorques=True)
    res = config.resolve_model(**model, storage=storage)
    m = M.LBMmodel(res)
    orc = oracle_mod.OracleModel(res)
    for tgt in (m, orc):
        prm = config.resolve_squirmer(d, **sq)
        M._add(tgt, prm) if tgt is m else tgt.add_particle(prm)
    inf = m.info()
    assert inf.bulk_kernel == _capi.LBM_BULK_VECTOR and inf.bulk_threads == 96
    m.step(40)
    orc.step(40)
    tol = dict(TOL[storage], field=3e-5) if storage == "f16" else TOL[storage]
    compare_state(res, m, orc, tol, f"{vel} nx={nx} {storage}")
