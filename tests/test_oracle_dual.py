"""The dual-number oracle: values identical to the FP64 oracle, derivatives equal to central differences.

The dual oracle is the reference for the adjoint's gradients; it is pinned here
against finite differences of the FP64 oracle on small cases (no GPU needed).
"""
from __future__ import annotations

import numpy as np
import pytest

from lbmengine import config as cfgmod


def swimmer_case(dims):
    if dims == 3:
        model = dict(dims=3, velocities="D3Q19", collisionModel="trt", kineticParameter=3 / 16,
                     latticeParameter=1.0, relaxationTimeRatio=0.7, xlims=(-7.0, 6.0),
                     forceDensity=[2e-5, 1e-5, 0.0])
        sq = dict(radius=3.2, position=[0.21, -0.13, 0.07], swimmingSpeed=2e-3, beta=-2.0,
                  swimmingDirection=[0.6, 0.64, 0.48], coupleForces=True, coupleTorques=True, massDensity=2.0)
    else:
        model = dict(dims=2, collisionModel="trt", kineticParameter=0.25, latticeParameter=1.0,
                     relaxationTimeRatio=0.8, xlims=(-10.0, 9.0), forceDensity=[3e-5, -1e-5])
        sq = dict(radius=3.7, position=[0.3, -0.2], swimmingSpeed=3e-3, beta=3.0, swimmingDirection=[0.8, 0.6],
                  coupleForces=True, coupleTorques=True, massDensity=0.5)
    return model, sq


def run_double(oracle_mod, model, sq, ticks, **over):
    mkw = dict(model)
    skw = dict(sq)
    for k, v in over.items():
        if k in ("B1", "B2"):
            continue
        mkw[k] = v
    res = cfgmod.resolve_model(**mkw)
    orc = oracle_mod.OracleModel(res)
    p = cfgmod.resolve_squirmer(res.dims, **skw)
    if "B1" in over:
        p.B1 = over["B1"]
    if "B2" in over:
        p.B2 = over["B2"]
    orc.add_particle(p)
    orc.step(ticks)
    st = orc.particles()[0]
    mask = orc.mask(1)
    orc.close()
    return np.array(st.velocity[:res.dims]), np.array(st.position[:res.dims]), mask


@pytest.mark.parametrize("dims", [2, 3])
def test_dual_values_equal_fp64_oracle(oracle_mod, dims):
    model, sq = swimmer_case(dims)
    res = cfgmod.resolve_model(**model)
    dual = oracle_mod.DualOracle(res)
    dual.add_particle(cfgmod.resolve_squirmer(dims, **sq))
    dual.step(25)
    val, _ = dual.particle(1)
    v, r, _ = run_double(oracle_mod, model, sq, 25)
    assert np.array_equal(val["velocity"][:dims], v)
    assert np.array_equal(val["position"][:dims], r)


@pytest.mark.parametrize("dims", [2, 3])
def test_dual_derivatives_match_central_differences(oracle_mod, dims):
    model, sq = swimmer_case(dims)
    ticks = 30
    res = cfgmod.resolve_model(**model)
    p0 = cfgmod.resolve_squirmer(dims, **sq)
    dual = oracle_mod.DualOracle(res)
    dual.add_particle(p0)
    dual.step(ticks)
    _, der = dual.particle(1)
    dv = der["velocity"][:dims]  # (dims, K)
    tau = res.relaxationTimeRatio
    F = list(model["forceDensity"])
    checks = {"B1": (p0.B1, lambda h: dict(B1=p0.B1 + h)),
              "B2": (p0.B2, lambda h: dict(B2=p0.B2 + h)),
              "tau": (tau, lambda h: dict(relaxationTimeRatio=tau + h)),
              "Fx": (F[0], lambda h: dict(forceDensity=[F[0] + h] + F[1:]))}
    for j, name in enumerate(oracle_mod.DIRECTIONS):
        if name not in checks:
            continue
        x0, over = checks[name]
        h = 1e-6 * abs(x0)
        vp, _, mp = run_double(oracle_mod, model, sq, ticks, **over(h))
        vm, _, mm = run_double(oracle_mod, model, sq, ticks, **over(-h))
        assert np.array_equal(mp, mm), f"{name}: a mask flipped inside the difference step"
        fd = (vp - vm) / (2 * h)
        scale = max(np.max(np.abs(fd)), 1e-30)
        assert np.max(np.abs(dv[:, j] - fd)) <= 1e-5 * scale, f"{name}: dual {dv[:, j]} vs FD {fd}"
