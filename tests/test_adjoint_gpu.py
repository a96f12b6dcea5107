"""Adjoint gradients (lbm_adjoint) against forward-mode dual numbers through the oracle, and checkpoint invariance.

The observable is the squirmer's velocity along its initial orientation,
averaged over a window of ticks; the parameters are B1, B2, the relaxation
time tau (tau- following at fixed magic parameter) and the body force.  Both
the adjoint and the dual oracle hold the solid masks as the forward run
computes them, so with FP64 storage they agree to rounding; with FP32
storage the linearisation point itself differs at the FP32 level.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = {
    "d3q19_trt": dict(
        model=dict(dims=3, velocities="D3Q19", collisionModel="trt", kineticParameter=3 / 16, latticeParameter=1.0,
                   relaxationTimeRatio=0.7, xlims=(-10.0, 9.0), forceDensity=[2e-5, 1e-5, 0.0]),
        squirmer=dict(radius=3.5, position=[0.3, -0.2, 0.1], swimmingSpeed=2e-3, beta=-2.0,
                      swimmingDirection=[0.6, 0.64, 0.48], coupleForces=True, coupleTorques=True, massDensity=2.0),
        ticks=60, window=(20, 60)),
    "d2q9_bgk": dict(
        model=dict(dims=2, collisionModel="bgk", latticeParameter=1.0, relaxationTimeRatio=0.8,
                   xlims=(-24.0, 23.0), forceDensity=[1e-5, 0.0]),
        squirmer=dict(radius=5.0, position=[0.4, -0.3], swimmingSpeed=2e-3, beta=3.0, swimmingDirection=[0.8, 0.6],
                      coupleForces=True, coupleTorques=True, massDensity=1.5),
        ticks=80, window=(40, 80)),
    # walls on y (halfway bounce-back) and a moving lid: the wall links' bounce-back
    # copy and moving-wall term in the adjoint
    "d2q9_trt_walls_lid": dict(
        model=dict(dims=2, collisionModel="trt", kineticParameter=3 / 16, latticeParameter=1.0,
                   relaxationTimeRatio=0.75, xlims=(-20.0, 19.0), ylims=(-12.0, 11.0), walledDimensions=[2],
                   movingWalls=lambda x, y: [2e-3, 0.0] if y >= 11.0 else [0.0, 0.0], forceDensity=[1e-5, 0.0]),
        squirmer=dict(radius=4.0, position=[0.3, -1.2], swimmingSpeed=2e-3, beta=2.0, swimmingDirection=[0.8, 0.6],
                      coupleForces=True, coupleTorques=True, massDensity=1.5),
        ticks=80, window=(30, 80)),
    "d3q19_walls": dict(
        model=dict(dims=3, velocities="D3Q19", collisionModel="bgk", latticeParameter=1.0, relaxationTimeRatio=0.8,
                   xlims=(-10.0, 9.0), ylims=(-10.0, 9.0), zlims=(-8.0, 7.0), walledDimensions=[3],
                   forceDensity=[2e-5, 0.0, 0.0]),
        squirmer=dict(radius=3.5, position=[0.3, -0.2, -0.4], swimmingSpeed=2e-3, beta=-1.0,
                      swimmingDirection=[0.6, 0.0, 0.8], coupleForces=True, coupleTorques=True, massDensity=2.0),
        ticks=50, window=(20, 50)),
}


def dual_gradient(oracle_mod, case):
    from lbmengine import config as cfgmod
    res = cfgmod.resolve_model(**case["model"])
    dual = oracle_mod.DualOracle(res)
    p = cfgmod.resolve_squirmer(res.dims, **case["squirmer"])
    dual.add_particle(p)
    d = res.dims
    e0 = np.array(p.swimming_direction[:d], dtype=float)
    J, dJ = 0.0, np.zeros(len(oracle_mod.DIRECTIONS))
    lo, hi = case["window"]
    K = hi - lo + 1
    for t in range(1, case["ticks"] + 1):
        dual.step(1)
        if lo <= t <= hi:
            val, der = dual.particle(1)
            J += float(val["velocity"][:d] @ e0) / K
            dJ += (e0 @ der["velocity"][:d]) / K
    dual.close()
    return J, dict(zip(oracle_mod.DIRECTIONS, dJ))


def gpu_gradient(case, storage, snapshots):
    from lbmengine.adjoint import build_swimmer, swimming_speed_gradient
    m = build_swimmer(dict(case["model"], storage=storage), case["squirmer"])
    out = swimming_speed_gradient(m, case["ticks"], case["window"], snapshots=snapshots)
    assert m.tick == 0  # the model is left as it was
    m.close()
    return out


@pytest.mark.parametrize("name", list(CASES))
def test_adjoint_matches_dual_numbers_fp64(lib, oracle_mod, name):
    case = CASES[name]
    J, dJ = dual_gradient(oracle_mod, case)
    out = gpu_gradient(case, "f64", snapshots=4)
    assert abs(out.value - J) <= 1e-10 * abs(J)
    scale = max(abs(v) for v in dJ.values())
    for k, v in dJ.items():
        assert abs(out.grad[k] - v) <= 1e-6 * abs(v) + 1e-9 * scale, f"{k}: adjoint {out.grad[k]:.9e} dual {v:.9e}"


def test_adjoint_fp32_storage_close_to_dual(lib, oracle_mod):
    case = CASES["d3q19_trt"]
    _, dJ = dual_gradient(oracle_mod, case)
    out = gpu_gradient(case, "f32", snapshots=8)
    scale = max(abs(v) for v in dJ.values())
    for k, v in dJ.items():
        assert abs(out.grad[k] - v) <= 2e-3 * abs(v) + 1e-4 * scale, f"{k}: adjoint {out.grad[k]:.6e} dual {v:.6e}"


def test_gradient_does_not_depend_on_the_checkpoint_budget(lib):
    case = CASES["d2q9_bgk"]
    a = gpu_gradient(case, "f64", snapshots=2)
    b = gpu_gradient(case, "f64", snapshots=64)
    assert a.value == b.value
    for k in a.grad:
        assert a.grad[k] == b.grad[k]
    assert a.forward_ticks > b.forward_ticks  # fewer snapshots, more recomputation
    assert a.snapshots_used <= 2 and b.snapshots_used <= 64


def test_autograd_function(lib):
    import torch
    from lbmengine.adjoint import PARAMETERS, make_autograd_function
    case = CASES["d2q9_bgk"]
    fn = make_autograd_function()
    theta = torch.tensor([3e-3, 9e-3, 0.8, 1e-5, 0.0, 0.0], dtype=torch.float64, requires_grad=True)
    mkw = dict(case["model"], storage="f64")
    J = fn.apply(theta, mkw, case["squirmer"], case["ticks"], case["window"], 8)
    J.backward()
    out = gpu_gradient(case, "f64", snapshots=8)
    assert abs(J.item() - out.value) <= 1e-12 * abs(out.value)
    for k, name in enumerate(PARAMETERS[:5]):
        assert abs(theta.grad[k].item() - out.grad[name]) <= 1e-9 * (abs(out.grad[name]) + 1e-30)


def forward_observable(case, theta):
    """The observable from a plain FP64 forward run of the model built from theta."""
    from lbmengine.adjoint import build_swimmer
    m = build_swimmer(dict(case["model"], storage="f64"), case["squirmer"], theta)
    lo, hi = case["window"]
    d = m._dims
    e0 = np.array(case["squirmer"]["swimmingDirection"][:d], dtype=float)
    e0 /= np.linalg.norm(e0)
    J = 0.0
    for t in range(1, case["ticks"] + 1):
        m.step(1)
        if lo <= t <= hi:
            J += float(np.dot(np.array(m.particle_states()[0].velocity[:d]), e0)) / (hi - lo + 1)
    m.close()
    return J


@pytest.mark.parametrize("name", list(CASES))
def test_adjoint_matches_central_differences(lib, name):
    """Central differences of FP64 forward runs, with a step small enough (1e-6
    relative) that no solid node changes sides between the two runs.  A force
    component whose gradient is far below the others' is compared with an
    absolute term of 1e-7 of the largest force gradient (the quotient's
    rounding at steps of 1e-11)."""
    case = CASES[name]
    out = gpu_gradient(case, "f64", snapshots=4)
    sq, mo = case["squirmer"], case["model"]
    B1 = 1.5 * sq["swimmingSpeed"]
    F = list(mo["forceDensity"]) + [0.0] * (3 - len(mo["forceDensity"]))
    theta = np.array([B1, sq["beta"] * B1, mo["relaxationTimeRatio"], F[0], F[1], F[2]])
    for k, nm in enumerate(("B1", "B2", "tau", "Fx", "Fy")):
        h = 1e-6 * max(abs(theta[k]), 1e-5)
        tp, tm = theta.copy(), theta.copy()
        tp[k] += h
        tm[k] -= h
        fd = (forward_observable(case, tp) - forward_observable(case, tm)) / (2 * h)
        fscale = max(abs(out.grad["Fx"]), abs(out.grad["Fy"])) if nm.startswith("F") else 0.0
        assert abs(out.grad[nm] - fd) <= 1e-5 * abs(fd) + 1e-7 * fscale, f"{nm}: adjoint {out.grad[nm]:.9e} FD {fd:.9e}"


# ---- the force observable: drag of a held squirmer -------------------------
DRAG_CASES = {
    "d3q19_held": dict(
        model=dict(dims=3, velocities="D3Q19", collisionModel="trt", kineticParameter=3 / 16, latticeParameter=1.0,
                   relaxationTimeRatio=0.7, xlims=(-10.0, 9.0), forceDensity=[2e-5, 1e-5, 0.0]),
        squirmer=dict(radius=3.5, position=[0.3, -0.2, 0.1], swimmingSpeed=2e-3, beta=-2.0,
                      swimmingDirection=[0.6, 0.64, 0.48], coupleForces=False, coupleTorques=False),
        ticks=60, window=(20, 60)),
    "d2q9_held": dict(
        model=dict(dims=2, collisionModel="bgk", latticeParameter=1.0, relaxationTimeRatio=0.8,
                   xlims=(-24.0, 23.0), forceDensity=[1e-5, 0.0]),
        squirmer=dict(radius=5.0, position=[0.4, -0.3], swimmingSpeed=2e-3, beta=3.0, swimmingDirection=[0.8, 0.6],
                      coupleForces=False, coupleTorques=False),
        ticks=80, window=(40, 80)),
    # a held squirmer in a channel driven by the body force, walls on y
    "d2q9_held_channel": dict(
        model=dict(dims=2, collisionModel="trt", kineticParameter=3 / 16, latticeParameter=1.0,
                   relaxationTimeRatio=0.8, xlims=(-20.0, 19.0), ylims=(-10.0, 9.0), walledDimensions=[2],
                   forceDensity=[2e-5, 0.0]),
        squirmer=dict(radius=4.0, position=[0.2, 0.4], swimmingSpeed=2e-3, beta=1.0, swimmingDirection=[1.0, 0.0],
                      coupleForces=False, coupleTorques=False),
        ticks=80, window=(40, 80)),
}


def dual_drag(oracle_mod, case):
    from lbmengine import config as cfgmod
    res = cfgmod.resolve_model(**case["model"])
    dual = oracle_mod.DualOracle(res)
    p = cfgmod.resolve_squirmer(res.dims, **case["squirmer"])
    dual.add_particle(p)
    dual.record_force(1)
    d = res.dims
    e0 = np.array(p.swimming_direction[:d], dtype=float)
    J, dJ = 0.0, np.zeros(len(oracle_mod.DIRECTIONS))
    lo, hi = case["window"]
    K = hi - lo + 1
    for t in range(1, case["ticks"] + 1):
        dual.step(1)
        if lo <= t <= hi:
            val, der = dual.particle_force(1)
            J += float(val[:d] @ e0) / K
            dJ += (e0 @ der[:d]) / K
    dual.close()
    return J, dict(zip(oracle_mod.DIRECTIONS, dJ))


def gpu_drag(case, storage, snapshots, theta=None):
    from lbmengine.adjoint import build_swimmer, drag_gradient
    m = build_swimmer(dict(case["model"], storage=storage), case["squirmer"], theta)
    out = drag_gradient(m, case["ticks"], case["window"], snapshots=snapshots)
    assert m.tick == 0
    assert all(x == 0.0 for x in m.particle_states()[0].last_force)  # ordinary stepping records no force
    m.close()
    return out


@pytest.mark.parametrize("name", list(DRAG_CASES))
def test_drag_adjoint_matches_dual_numbers_fp64(lib, oracle_mod, name):
    case = DRAG_CASES[name]
    J, dJ = dual_drag(oracle_mod, case)
    out = gpu_drag(case, "f64", snapshots=4)
    assert J != 0.0 and abs(out.value - J) <= 1e-10 * abs(J)
    scale = max(abs(v) for v in dJ.values())
    for k, v in dJ.items():
        assert abs(out.grad[k] - v) <= 1e-6 * abs(v) + 1e-9 * scale, f"{k}: adjoint {out.grad[k]:.9e} dual {v:.9e}"


def forward_drag(case, theta):
    """The drag from a plain FP64 forward run, the particle's force recorded (lbm_record_force)."""
    from lbmengine.adjoint import build_swimmer
    m = build_swimmer(dict(case["model"], storage="f64"), case["squirmer"], theta)
    m.record_force(1)
    lo, hi = case["window"]
    d = m._dims
    e0 = np.array(case["squirmer"]["swimmingDirection"][:d], dtype=float)
    e0 /= np.linalg.norm(e0)
    J = 0.0
    for t in range(1, case["ticks"] + 1):
        m.step(1)
        if lo <= t <= hi:
            J += float(np.dot(np.array(m.particle_states()[0].last_force[:d]), e0)) / (hi - lo + 1)
    m.close()
    return J


@pytest.mark.parametrize("name", list(DRAG_CASES))
def test_drag_adjoint_matches_central_differences_at_relative_step_1e4(lib, name):
    """A held particle never moves, so no node changes sides between the +-h
    runs and central differences at h = 1e-4 relative are exact to O(h^2)."""
    case = DRAG_CASES[name]
    out = gpu_drag(case, "f64", snapshots=4)
    sq, mo = case["squirmer"], case["model"]
    B1 = 1.5 * sq["swimmingSpeed"]
    F = list(mo["forceDensity"]) + [0.0] * (3 - len(mo["forceDensity"]))
    theta = np.array([B1, sq["beta"] * B1, mo["relaxationTimeRatio"], F[0], F[1], F[2]])
    for k, nm in enumerate(("B1", "B2", "tau", "Fx")):
        h = 1e-4 * abs(theta[k])
        tp, tm = theta.copy(), theta.copy()
        tp[k] += h
        tm[k] -= h
        fd = (forward_drag(case, tp) - forward_drag(case, tm)) / (2 * h)
        assert abs(out.grad[nm] - fd) <= 1e-5 * abs(fd), f"{nm}: adjoint {out.grad[nm]:.9e} FD {fd:.9e}"


def test_force_observable_of_a_coupled_squirmer_matches_dual_numbers(lib, oracle_mod):
    """The force observable of a free squirmer: its momentum exchange feeds its motion as well."""
    from lbmengine.adjoint import build_swimmer, drag_gradient
    case = CASES["d3q19_trt"]
    J, dJ = dual_drag(oracle_mod, case)
    m = build_swimmer(dict(case["model"], storage="f64"), case["squirmer"])
    out = drag_gradient(m, case["ticks"], case["window"], snapshots=4)
    m.close()
    assert abs(out.value - J) <= 1e-10 * abs(J)
    scale = max(abs(v) for v in dJ.values())
    for k, v in dJ.items():
        assert abs(out.grad[k] - v) <= 1e-6 * abs(v) + 1e-9 * scale, f"{k}: adjoint {out.grad[k]:.9e} dual {v:.9e}"
