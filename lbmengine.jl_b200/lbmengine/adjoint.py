"""Gradients of a squirmer observable through the C ABI (lbm_adjoint in include/lbm_b200.h).

``swimming_speed_gradient`` runs the hand-written discrete adjoint with
binomial checkpointing.  ``make_autograd_function`` wraps it as a
torch.autograd.Function (the PyTorch counterpart of a ChainRulesCore.rrule):
its input is the parameter vector (B1, B2, tau, Fx, Fy, Fz), its output the
observable, and its backward pass returns the adjoint gradients.  The
reference has no differentiation; what is differentiated is the reference's
tick as this library runs it (src/gpu/fluids.jl:132-226,
src/gpu/particles.jl:7-92).
"""
from __future__ import annotations

import ctypes as C
from types import SimpleNamespace

from . import _capi as capi
from . import config as cfgmod
from . import model as mdl

PARAMETERS = ("B1", "B2", "tau", "Fx", "Fy", "Fz")


def tau_minus_slope(resolved) -> float:
    """d tau- / d tau+ at fixed magic parameter (TRT: tau- = L dt^2 / (tau+ - dt/2) + dt/2)."""
    if resolved.collision != "trt":
        return 0.0
    lam = resolved.kineticParameter
    if isinstance(lam, str):
        raise ValueError("gradients need a numeric kineticParameter")
    dt = resolved.dt
    return -float(lam) * dt * dt / (resolved.tau - dt / 2) ** 2


def swimming_speed_gradient(model: mdl.LBMmodel, ticks: int, window, direction=None, snapshots: int = 32,
                            observable: int = capi.LBM_OBSERVABLE_VELOCITY):
    """Average over ticks window[0]..window[1] of the particle velocity along
    ``direction`` (default: its initial swimming direction), over ``ticks``
    ticks from the model's initial state, and its gradient.  The model is left
    as it was."""
    spec = capi.LbmAdjointSpec(ticks=int(ticks), window_begin=int(window[0]), window_end=int(window[1]),
                               tau_minus_slope=tau_minus_slope(model._res), snapshots=int(snapshots),
                               observable=int(observable))
    if direction is not None:
        for k, v in enumerate(direction):
            spec.direction[k] = float(v)
    res = capi.LbmAdjointResult()
    model._check(model._lib.lbm_adjoint(model.handle, C.byref(spec), C.byref(res)))
    grad = dict(B1=res.dB1, B2=res.dB2, tau=res.dtau, Fx=res.dF[0], Fy=res.dF[1], Fz=res.dF[2])
    return SimpleNamespace(value=res.value, grad=grad, dtau_plus=res.dtau_plus, dtau_minus=res.dtau_minus,
                           forward_ticks=res.forward_ticks, snapshots_used=res.snapshots_used, ms=res.ms)


def drag_gradient(model: mdl.LBMmodel, ticks: int, window, direction=None, snapshots: int = 32):
    """Average over ticks window[0]..window[1] of the momentum-exchange force on
    the particle along ``direction`` (default: its initial swimming direction)
    and its gradient; for a held particle (coupleForces false) this is its
    drag.  The model is left as it was."""
    return swimming_speed_gradient(model, ticks, window, direction, snapshots, capi.LBM_OBSERVABLE_FORCE)


def build_swimmer(model_kw: dict, squirmer_kw: dict, theta=None) -> mdl.LBMmodel:
    """A model with one squirmer; theta = (B1, B2, tau, Fx, Fy, Fz) overrides
    B1, B2, the relaxation time (relaxationTimeRatio * latticeParameter) and
    the body force when given."""
    mkw = dict(model_kw)
    if theta is not None:
        dims = mkw.get("dims", 2)
        mkw["relaxationTimeRatio"] = float(theta[2]) / float(mkw.get("latticeParameter", 1.0))
        mkw["forceDensity"] = [float(theta[3 + k]) for k in range(dims)]
    m = mdl.LBMmodel(cfgmod.resolve_model(**mkw))
    p = cfgmod.resolve_squirmer(m._dims, **squirmer_kw)
    if theta is not None:
        p.B1 = float(theta[0])
        p.B2 = float(theta[1])
    mdl._add(m, p)
    return m


def make_autograd_function():
    """A torch.autograd.Function: the swimming-speed observable of a squirmer
    model built from the parameter tensor, with the adjoint as its backward
    pass (what a ChainRulesCore.rrule is to the Julia front end)."""
    import torch

    class SwimmingSpeed(torch.autograd.Function):
        @staticmethod
        def forward(ctx, theta, model_kw, squirmer_kw, ticks, window, snapshots=32):
            m = build_swimmer(model_kw, squirmer_kw, theta.detach().cpu().double().tolist())
            out = swimming_speed_gradient(m, ticks, window, snapshots=snapshots)
            m.close()
            g = torch.tensor([out.grad[k] for k in PARAMETERS], dtype=theta.dtype, device=theta.device)
            ctx.save_for_backward(g)
            return torch.tensor(out.value, dtype=theta.dtype, device=theta.device)

        @staticmethod
        def backward(ctx, grad_out):
            (g,) = ctx.saved_tensors
            return grad_out * g, None, None, None, None, None

    return SwimmingSpeed
