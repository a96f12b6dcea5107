"""Particle-particle interactions (src/gpu/initMethods.jl:224-414, applied by
molecularDynamicsTick!, src/gpu/particles.jl:100-197).

The ``add*`` functions resolve the reference's keywords and defaults and keep
``model.particleInteractions`` in the reference's order; the flattened items
(one per bond, one per pair of a pair potential) go to the library with
lbm_set_interactions, which evaluates them on the GPU every tick.
"""
from __future__ import annotations

import ctypes as C
import math
from types import SimpleNamespace

import numpy as np

from . import _capi as capi


def _assert(cond, msg):
    if not cond:
        raise AssertionError(msg)


def _norm(v):
    v = np.asarray(v, dtype=np.float64)
    return float(np.sqrt((v * v).sum())) if np.any(v != 0) else 0.0


def _positions(model):
    d = model._dims
    return [np.array(s.position[:d]) for s in model.particle_states()]


def _items(model, t=None):
    """The flattened items of model.particleInteractions (dipole fields evaluated at time t)."""
    items = []
    t = model.time if t is None else t
    for it in model.particleInteractions:
        if it.kind in ("linear", "bistable", "polar"):
            e = capi.LbmInteraction()
            e.kind = {"linear": capi.LBM_INTERACTION_LINEAR, "bistable": capi.LBM_INTERACTION_BISTABLE,
                      "polar": capi.LBM_INTERACTION_POLAR}[it.kind]
            e.id1, e.id2 = it.id1, it.id2
            e.id3 = it.id3 if it.kind == "polar" else 0
            for k, v in enumerate(it.params):
                e.p[k] = v
            items.append(e)
            continue
        if it.kind == "dipole":
            B = it.magneticField(t) if callable(it.magneticField) else it.magneticField
            B = list(np.asarray(B, dtype=np.float64).ravel()) + [0.0] * 3
            params = [it.dipoleConstant] + B[:3]
        else:
            params = [it.epsilon, it.sigma, it.cutoff]
        for a, b in it.pairs:
            e = capi.LbmInteraction()
            e.kind = capi.LBM_INTERACTION_DIPOLE if it.kind == "dipole" else capi.LBM_INTERACTION_LENNARD_JONES
            e.id1, e.id2 = a, b
            for k, v in enumerate(params):
                e.p[k] = v
            items.append(e)
    return items


def push(model, t=None):
    """Send the flattened interaction list to the library."""
    items = _items(model, t)
    arr = (capi.LbmInteraction * max(1, len(items)))(*items)
    model._check(model._lib.lbm_set_interactions(model.handle, arr, len(items)))


def time_dependent(model) -> bool:
    return any(it.kind == "dipole" and callable(it.magneticField) for it in model.particleInteractions)


def addLinearBond(model, id1: int, id2: int, equilibriumDisplacement=None, stiffness=1):
    """addLinearBond! (src/gpu/initMethods.jl:229-246)."""
    R = _positions(model)
    if equilibriumDisplacement is None:
        equilibriumDisplacement = _norm(R[id2 - 1] - R[id1 - 1])
    _assert(isinstance(equilibriumDisplacement, (int, float)), "equilibriumDisplacement must be a number!")
    _assert(isinstance(stiffness, (int, float)), "stiffness must be a number!")
    model.particleInteractions.append(SimpleNamespace(kind="linear", id1=id1, id2=id2,
                                                      params=[float(equilibriumDisplacement), float(stiffness)]))
    push(model)


def addPolarBond(model, id1: int, id2: int, id3: int, equilibriumAngle=None, stiffness=1):
    """addPolarBond! (src/gpu/initMethods.jl:248-274)."""
    R = _positions(model)
    vecA, vecB = R[id1 - 1] - R[id2 - 1], R[id3 - 1] - R[id2 - 1]
    cos_alpha = float((vecA * vecB).sum()) / (_norm(vecA) * _norm(vecB))
    if equilibriumAngle is None:
        equilibriumAngle = math.acos(cos_alpha)
    _assert(isinstance(equilibriumAngle, (int, float)), "equilibriumAngle must be a number!")
    _assert(isinstance(stiffness, (int, float)), "stiffness must be a number!")
    model.particleInteractions.append(SimpleNamespace(kind="polar", id1=id1, id2=id2, id3=id3,
                                                      params=[float(equilibriumAngle), float(stiffness)]))
    push(model)


def addBistableBond(model, id1: int, id2: int, lowDisp=None, highDisp=None, hillHeight=1):
    """addBistableBond! (src/gpu/initMethods.jl:283-309)."""
    R = _positions(model)
    if lowDisp is None:
        lowDisp = _norm(R[id2 - 1] - R[id1 - 1])
    if highDisp is None:
        highDisp = lowDisp + model.spaceTime.latticeParameter
    _assert(isinstance(lowDisp, (int, float)), "lowDisp must be a number!")
    _assert(isinstance(highDisp, (int, float)), "highDisp must be a number!")
    trap_radius = (highDisp + lowDisp) / 2
    trap_width = highDisp - lowDisp
    _assert(isinstance(hillHeight, (int, float)), "hillHeight must be a number!")
    a = 4 * 16 * hillHeight / trap_width ** 4
    b = 2 * 8 * hillHeight / trap_width ** 2
    model.particleInteractions.append(SimpleNamespace(kind="bistable", id1=id1, id2=id2,
                                                      params=[float(trap_radius), float(a), float(b)]))
    push(model)


def _pairs(ids):
    return [(ids[i], ids[j]) for i in range(len(ids)) for j in range(len(ids)) if i < j]


def addDipoles(model, *ids, magneticField=(1, 0), susceptibility=0.5, permeability=400 * math.pi, rewrite=False):
    """addDipoles! (src/gpu/initMethods.jl:317-360); no ids: every particle.
    magneticField: a vector or a function of time returning one."""
    ids = list(ids) if ids else list(range(1, len(model.particle_states()) + 1))
    old = [k for k, it in enumerate(model.particleInteractions) if it.kind == "dipole"]
    write_new = not old or rewrite
    if not write_new:
        prev = model.particleInteractions[old[0]]
        ids = sorted(set(ids + [i for p in prev.pairs for i in p]))
    _assert(len(ids) > 1, "There must be at least two dipoles!")
    pairs = _pairs(ids)
    if write_new:
        if rewrite and old:
            del model.particleInteractions[old[0]]
        r = model.particle_states()[ids[0] - 1].radius
        model.particleInteractions.append(SimpleNamespace(
            kind="dipole", pairs=pairs, dipoleConstant=4 * math.pi * r ** 6 * susceptibility ** 2 / (3 * permeability),
            magneticField=magneticField))
    else:
        prev.pairs = pairs
    push(model)


def _default_epsilon(model):
    rho = model.massDensity
    nz = rho[rho != 0.0]
    return float(nz.sum() / nz.size) * model.spaceTime.latticeParameter ** 5 / model.spaceTime.timeStep ** 2


def addLennardJones(model, epsilon=None, sigma=None, cutoff=None):
    """addLennardJones! (src/gpu/initMethods.jl:362-397): all pairs of the model's particles."""
    ids = list(range(1, len(model.particle_states()) + 1))
    old = [k for k, it in enumerate(model.particleInteractions) if it.kind == "lennard_jones"]
    if old:
        del model.particleInteractions[old[0]]
    if epsilon is None:
        epsilon = _default_epsilon(model)
    if sigma is None:
        r = model.particle_states()[0].radius
        sigma = 2 * r + model.spaceTime.latticeParameter
    if cutoff is None:
        cutoff = math.inf
    _assert(isinstance(epsilon, (int, float)), "epsilon must be a number!")
    _assert(isinstance(sigma, (int, float)), "sigma must be a number!")
    model.particleInteractions.append(SimpleNamespace(kind="lennard_jones", pairs=_pairs(ids), epsilon=float(epsilon),
                                                      sigma=float(sigma), cutoff=float(cutoff)))
    push(model)


def addWCA(model, epsilon=None, sigma=None):
    """addWCA! (src/gpu/initMethods.jl:399-413): Lennard-Jones cut at its minimum 2^(1/6) sigma."""
    if epsilon is None:
        epsilon = _default_epsilon(model)
    if sigma is None:
        r = model.particle_states()[0].radius
        sigma = 2 * r + model.spaceTime.latticeParameter
    addLennardJones(model, epsilon=epsilon, sigma=sigma, cutoff=2 ** (1 / 6) * sigma)
