"""Particle-particle interactions (molecularDynamicsTick!, src/gpu/particles.jl:100-197)
on the GPU against the FP64 oracle, and a known answer for the oracle itself."""
from __future__ import annotations

import math

import numpy as np
import pytest

from lbmengine import _capi, config
from parity_cases import build_pair

TOL = {"f64": dict(field=1e-10, pos=1e-10, force=1e-8), "f32": dict(field=1e-5, pos=1e-7, force=5e-4)}


def _item(kind, id1, id2, p, id3=0):
    e = _capi.LbmInteraction()
    e.kind, e.id1, e.id2, e.id3 = kind, id1, id2, id3
    for k, v in enumerate(p):
        e.p[k] = v
    return e


def test_oracle_linear_bond_force_known_answer(oracle_mod):
    """One tick: the bond adds k (d - d0) r^ to particle 1 and its opposite to particle 2."""
    kw = dict(dims=2, latticeParameter=1.0, relaxationTimeRatio=0.8, collisionModel="bgk", xlims=(-16.0, 15.0))
    forces = []
    for bonded in (False, True):
        res = config.resolve_model(**kw)
        m = oracle_mod.OracleModel(res)
        m.add_particle(config.resolve_bead(2, radius=3.0, position=[-5.0, 0.5], coupleForces=True))
        m.add_particle(config.resolve_bead(2, radius=3.0, position=[5.5, -0.5], coupleForces=True))
        if bonded:
            m.set_interactions([_item(_capi.LBM_INTERACTION_LINEAR, 1, 2, [8.0, 1e-4])])
        m.step(1)
        forces.append([np.array(p.last_force[:2]) for p in m.particles()])
    d = np.array([10.5, -1.0])
    expect = 1e-4 * (np.hypot(*d) - 8.0) * d / np.hypot(*d)
    np.testing.assert_allclose(forces[1][0] - forces[0][0], expect, rtol=1e-12, atol=1e-20)
    np.testing.assert_allclose(forces[1][1] - forces[0][1], -expect, rtol=1e-12, atol=1e-20)


def _case3d():
    sq = lambda pos, e, beta: dict(kind="squirmer", radius=3.5, position=pos, swimmingSpeed=2e-3, beta=beta,
                                   coupleForces=True, coupleTorques=True, swimmingDirection=e, massDensity=2.0)
    return dict(model=dict(dims=3, velocities="D3Q19", collisionModel="trt", latticeParameter=1.0,
                           relaxationTimeRatio=0.7, xlims=(-16.0, 15.0), forceDensity=[1e-5, 0.0, 0.0]),
                particles=[sq([-7.0, 0.3, 0.1], [1.0, 0.2, 0.0], 2.0), sq([0.4, -0.2, 0.3], [0.0, 1.0, 0.3], -1.0),
                           sq([6.8, 1.1, -0.4], [0.5, 0.5, 0.5], 0.5)], steps=40)


def _case2d():
    bead = lambda pos: dict(kind="bead", radius=3.0, position=pos, coupleForces=True, coupleTorques=True,
                            massDensity=2.0)
    return dict(model=dict(dims=2, latticeParameter=1.0, relaxationTimeRatio=0.8, collisionModel="bgk",
                           xlims=(-24.0, 23.0), ylims=(-16.0, 15.0)),
                particles=[bead([-8.3, 0.2]), bead([0.1, -0.4]), bead([8.2, 1.3]), bead([0.2, 8.6])], steps=60)


def _interactions(dims):
    L, B, P, LJ, DP = (_capi.LBM_INTERACTION_LINEAR, _capi.LBM_INTERACTION_BISTABLE, _capi.LBM_INTERACTION_POLAR,
                       _capi.LBM_INTERACTION_LENNARD_JONES, _capi.LBM_INTERACTION_DIPOLE)
    items = [_item(L, 1, 2, [6.5, 2e-4]), _item(P, 1, 2, [2.5, 1e-4], id3=3), _item(B, 2, 3, [7.0, 1e-5, 2e-4])]
    field = [0.0, 0.3, 0.2] if dims == 3 else [0.4, -0.2, 0.0]
    n = 3 if dims == 3 else 4
    for a in range(1, n + 1):  # the pairs of one dipole interaction, then of one WCA interaction
        for b in range(a + 1, n + 1):
            items.append(_item(DP, a, b, [5e-2] + field))
    for a in range(1, n + 1):
        for b in range(a + 1, n + 1):
            items.append(_item(LJ, a, b, [1e-4, 8.0, 2 ** (1 / 6) * 8.0]))
    return items


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["3d", "2d"])
@pytest.mark.parametrize("storage", ["f64", "f32"])
def test_interactions_against_oracle(lib, oracle_mod, which, storage):
    case = _case3d() if which == "3d" else _case2d()
    res, gpu, orc = build_pair(case, storage=storage, oracle_mod=oracle_mod)
    items = _interactions(res.dims)
    arr = (_capi.LbmInteraction * len(items))(*items)
    assert lib.lbm_set_interactions(gpu.handle, arr, len(items)) == 0, lib.lbm_last_error(gpu.handle)
    orc.set_interactions(items)
    tol = TOL[storage]
    d = res.dims
    for chunk in (1, case["steps"] - 1):
        gpu.step(chunk)
        orc.step(chunk)
        for a, b in zip(gpu.particle_states(), orc.particles()):
            assert np.max(np.abs(np.array(a.position[:d]) - np.array(b.position[:d]))) <= tol["pos"]
            fo = np.array(b.last_force[:d])
            assert np.max(np.abs(np.array(a.last_force[:d]) - fo)) <= tol["force"] * np.max(np.abs(fo)) + 1e-15
    rho_o, u_o = orc.fields()
    assert np.max(np.abs(gpu.massDensity.ravel(order="F") - rho_o)) <= tol["field"]
    # the interactions moved the particles: without them the trajectories differ
    _, ref, _ = build_pair(case, storage=storage)
    ref.step(case["steps"])
    moved = max(abs(a.position[k] - b.position[k]) for a, b in zip(gpu.particle_states(), ref.particle_states())
                for k in range(d))
    assert moved > 1e-6


@pytest.mark.gpu
def test_interaction_api_defaults_and_limits(lib):
    from lbmengine import addBistableBond, addDipoles, addLinearBond, addPolarBond, addSquirmer, addWCA, modelInit
    m = modelInit(dims=2, latticeParameter=1.0, relaxationTimeRatio=0.8, collisionModel="bgk", xlims=(-20.0, 19.0))
    for x in (-8.0, 0.0, 8.0):
        addSquirmer(m, radius=3.0, position=[x, 0.5], coupleForces=True)
    addLinearBond(m, 1, 2)
    assert m.particleInteractions[0].params[0] == 8.0  # equilibrium = the current distance
    addPolarBond(m, 1, 2, 3)
    assert abs(m.particleInteractions[1].params[0] - math.pi) < 1e-12
    addBistableBond(m, 2, 3)
    addDipoles(m, magneticField=[0.0, 1.0])
    addWCA(m)
    wca = m.particleInteractions[-1]
    assert wca.sigma == 7.0 and abs(wca.cutoff - 2 ** (1 / 6) * 7.0) < 1e-15 and abs(wca.epsilon - 1.0) < 1e-6
    m.step(5)
    # the CPU module has no interactions; batches and the adjoint reject them
    res = config.resolve_model(dims=2, latticeParameter=1.0, relaxationTimeRatio=0.8, collisionModel="bgk",
                               xlims=(-20.0, 19.0), particleRules="cpu")
    from lbmengine import model as M
    c = M.LBMmodel(res)
    for x in (-8.0, 8.0):
        M._add(c, config.resolve_bead(2, radius=3.0, position=[x, 0.5]))
    arr = (_capi.LbmInteraction * 1)(_item(_capi.LBM_INTERACTION_LINEAR, 1, 2, [16.0, 1.0]))
    assert lib.lbm_set_interactions(c.handle, arr, 1) == _capi.LBM_ERR_UNSUPPORTED
    bad = (_capi.LbmInteraction * 1)(_item(_capi.LBM_INTERACTION_LINEAR, 1, 9, [16.0, 1.0]))
    assert lib.lbm_set_interactions(m.handle, bad, 1) == _capi.LBM_ERR_INVALID
