"""Keyword resolution of the reference's model-construction API.

Pure host logic, no device work: turns the keyword sets of ``modelInit``,
``addSquirmer!`` and ``addBead!`` into the resolved C structs of
include/lbm_b200.h.  Each step cites the reference lines it restates.
"""
from __future__ import annotations

import math
from fractions import Fraction
from types import SimpleNamespace

import numpy as np

from . import _capi as capi

DEFAULT = None  # stands for the reference's `:default`

_VELOCITY_SETS = {"D2Q9": (2, capi.LBM_D2Q9), "D3Q15": (3, capi.LBM_D3Q15),
                  "D3Q19": (3, capi.LBM_D3Q19), "D3Q27": (3, capi.LBM_D3Q27)}


def _assert(cond, msg):
    if not cond:
        raise AssertionError(msg)


def _exact_fraction(x: float):
    """Rational with a short decimal form equal to x, or None (Julia's `rat` use in ranges)."""
    fr = Fraction(repr(float(x)))
    return fr if float(fr) == float(x) else None


def julia_float_range(start, stop, step):
    """Values of Julia's `range(start, stop=stop, step=step)` for Float64 inputs.

    Follows base/twiceprecision.jl `(:)(start, step, stop)`: when start, step and
    stop have exact rational forms the length is computed in rational arithmetic
    and every element is the correctly rounded value of start + (i-1)*step;
    otherwise the floating-point fallback is used.
    """
    start, stop, step = float(start), float(stop), float(step)
    if step == 0:
        raise ValueError("range step cannot be zero")
    fs, ft, fp = _exact_fraction(start), _exact_fraction(stop), _exact_fraction(step)
    if fs is not None and ft is not None and fp is not None:
        length = max(0, math.floor((ft - fs) / fp) + 1)
        # start + i*step = (a d + i c b) / (b d) for start = a/b, step = c/d;
        # int / int is correctly rounded, as float(Fraction) is
        a, b, c, d = fs.numerator, fs.denominator, fp.numerator, fp.denominator
        num0, dnum, den = a * d, c * b, b * d
        return np.array([(num0 + i * dnum) / den for i in range(length)], dtype=np.float64)
    lf = (stop - start) / step
    if lf < 0:
        length = 0
    elif lf == 0:
        length = 1
    else:
        length = round(lf) + 1
        stop2 = start + (length - 1) * step
        length -= int(start < stop < stop2) + int(start > stop > stop2)
    return np.array([start + i * step for i in range(length)], dtype=np.float64)


def resolve_time_parameters(timeStep=DEFAULT, relaxationTimeRatio=DEFAULT, viscosity=DEFAULT,
                            latticeParameter=DEFAULT):
    """src/gpu/initMethods.jl:471-492: returns (dt, tau_ratio, viscosity)."""
    _assert(any(v is DEFAULT for v in (timeStep, relaxationTimeRatio, viscosity)),
            "timeStep, relaxationTimeRatio, and viscosity cannot be all simultaneously defined!")
    _assert(any(v is DEFAULT for v in (timeStep, latticeParameter)),
            "timeStep, and latticeParameter cannot be both simultaneously defined!")
    if latticeParameter is not DEFAULT:
        _assert(isinstance(latticeParameter, (int, float)), "latticeParameter must be a number!")
        timeStep = latticeParameter
    if timeStep is DEFAULT:
        if relaxationTimeRatio is DEFAULT:
            relaxationTimeRatio = 15
        if viscosity is DEFAULT:
            viscosity = 1
        timeStep = 3 * viscosity / (relaxationTimeRatio - 0.5)
    else:
        if relaxationTimeRatio is DEFAULT:
            if viscosity is DEFAULT:
                viscosity = 1
            relaxationTimeRatio = 3 * viscosity / timeStep + 0.5
        else:
            viscosity = timeStep / 3 * (relaxationTimeRatio - 0.5)
    return float(timeStep), float(relaxationTimeRatio), float(viscosity)


def wall_nodes(shape, walled_dimensions):
    """wallNodes, src/gpu/misc.jl:7-31: first and last slab of each walled axis (1-based axes)."""
    w = np.zeros(shape, dtype=np.uint8, order="F")
    for a in walled_dimensions:
        idx = [slice(None)] * len(shape)
        idx[a - 1] = 0
        w[tuple(idx)] = 1
        idx[a - 1] = shape[a - 1] - 1
        w[tuple(idx)] = 1
    return w


def resolve_model(massDensity=DEFAULT, fluidVelocity=DEFAULT, velocities=DEFAULT, collisionModel=DEFAULT,
                  relaxationTimeRatio=DEFAULT, viscosity=DEFAULT, timeStep=DEFAULT, latticeParameter=DEFAULT,
                  kineticParameter=0.25, xlims=DEFAULT, ylims=DEFAULT, zlims=DEFAULT, dims=2,
                  walledDimensions=DEFAULT, dampenEcho=False, walls=DEFAULT, movingWalls=DEFAULT,
                  isFluidCompressible=True, forceDensity=DEFAULT, forcingScheme=DEFAULT, saveData=False,
                  storage="f32", rho_ref=DEFAULT, store_scale=DEFAULT, device=DEFAULT, schedule="auto",
                  particleRules="gpu", rounding="stochastic"):
    """Resolve modelInit's keywords (src/gpu/initMethods.jl:440-702) into an LbmConfig.

    Returns a namespace with ``cfg`` (capi.LbmConfig), ``keep`` (arrays the
    config points into; keep them alive while the config is used) and the
    resolved scalars (dt, tau, viscosity, coordinates, schemes ...).
    """
    dt, ratio, nu = resolve_time_parameters(timeStep, relaxationTimeRatio, viscosity, latticeParameter)
    if xlims is DEFAULT:
        xlims = (-1, 1)
    if ylims is DEFAULT:
        ylims = xlims
    if zlims is DEFAULT:
        zlims = xlims
    _assert(all(t[1] != t[0] for t in (xlims, ylims, zlims)),
            f"Coordinate lower and upper limits cannot be equal! Current limits are {[xlims, ylims, zlims][:dims]}")
    axes = [julia_float_range(l[0], l[1], dt) for l in (xlims, ylims, zlims)][:dims]
    shape = tuple(len(a) for a in axes)
    # velocity set (initMethods.jl:528-541)
    if velocities is DEFAULT:
        _assert(dims > 1, "1 dimensional LBM is not implemented in CUDA!")
        _assert(dims <= 3, "for dimensions higher than 3 a velocity set must be defined using a NamedTuple!")
        velocities = ["D1Q3", "D2Q9", "D3Q15"][dims - 1]
    vname = str(velocities).lstrip(":")
    _assert(vname in _VELOCITY_SETS or vname == "D1Q3",
            "If a default velocity set is chosen, it must be one of the following: [:D1Q3, :D2Q9, :D3Q15, :D3Q19, :D3Q27]")
    vdims, lattice = _VELOCITY_SETS.get(vname, (1, 3))
    _assert(vdims == dims, f"The chosen velocity must be {dims}-dimensional!")
    # collision (initMethods.jl:550-566)
    if collisionModel is DEFAULT:
        collisionModel = "trt"
    cm = str(collisionModel).lstrip(":")
    _assert(cm in ("bgk", "trt"), f"Collision model {collisionModel} is not implemented!")
    c2_s, c4_s = 1.0 / 3, 1.0 / 9
    tau = ratio * dt
    tau_minus = 0.0
    if cm == "trt":
        lam = kineticParameter
        if isinstance(lam, str) and lam.lstrip(":") == "debug":
            lam = nu ** 2 / (c4_s * dt ** 2)
        tau_minus = lam * c2_s * dt ** 2 / nu + dt / 2
    schemes = [cm]
    keep = []
    # walls (initMethods.jl:568-628)
    wall = None
    if walledDimensions is not DEFAULT and len(walledDimensions) != 0:
        if dampenEcho:
            raise NotImplementedError(":cbc is not currently implemented in the gpu modules! "
                                      "Please use the cpu modules instead.")
        wall = wall_nodes(shape, walledDimensions)
        schemes.append("bounceBack")
    # coordinate grids, only for the wall functions that are evaluated on them
    grids = np.meshgrid(*axes, indexing="ij") if (walls is not DEFAULT or movingWalls is not DEFAULT) else None
    if walls is not DEFAULT:
        _assert(callable(walls), "walls must be a function!")
        new = np.vectorize(walls, otypes=[object])(*grids)
        _assert(all(isinstance(b, (bool, np.bool_)) for b in new.ravel()), "walls must return boolean values!")
        new = new.astype(np.uint8)
        wall = new if wall is None else (wall | new)
        schemes.append("bounceBack")
    uw = None
    if movingWalls is not DEFAULT:
        _assert(callable(movingWalls), "movingWalls must be a function!")
        vals = [np.asarray(movingWalls(*[g[idx] for g in grids]), dtype=np.float64)
                for idx in np.ndindex(*shape)]
        _assert(len(vals[0]) == dims, f"movingWalls must return a vector of dimension {dims}!")
        uw = np.zeros(shape + (dims,), dtype=np.float64, order="F")
        for idx, v in zip(np.ndindex(*shape), vals):
            uw[idx] = v
        if wall is None:
            wall = np.zeros(shape, dtype=np.uint8, order="F")
        schemes += ["movingWalls", "bounceBack"]
    # forcing (initMethods.jl:631-654)
    if forcingScheme is DEFAULT:
        forcingScheme = "guo"
    fsch = str(forcingScheme).lstrip(":")
    force_mode, force_vec, force_field = capi.LBM_FORCE_NONE, (0.0, 0.0, 0.0), None
    if forceDensity is not DEFAULT:
        if fsch != "guo":
            raise NotImplementedError(f"forcing scheme :{fsch} has no collision term in the gpu modules")
        fd = np.asarray(forceDensity, dtype=np.float64)
        if fd.ndim == 1 and len(fd) == dims:
            force_mode = capi.LBM_FORCE_UNIFORM
            force_vec = tuple(list(fd) + [0.0] * (3 - dims))
        elif fd.shape == shape + (dims,):
            force_mode = capi.LBM_FORCE_FIELD
            force_field = np.asfortranarray(fd)
        else:
            raise ValueError("force density does not have consistent dimensions!")
        schemes.append(fsch)
    if saveData:  # initMethods.jl:671-675: the output directory is made by the front end
        schemes.append("saveData")
    cfg = capi.LbmConfig()
    cfg.dims = dims
    cfg.lattice = lattice
    for a in range(3):
        cfg.n[a] = shape[a] if a < dims else 1
    coord_arrays = [np.ascontiguousarray(a, dtype=np.float64) for a in axes]
    keep += coord_arrays
    for a in range(dims):
        cfg.coords[a] = coord_arrays[a].ctypes.data_as(capi._dp)
        cfg.x0[a] = float(coord_arrays[a][0])
    cfg.dx = dt
    cfg.tau = tau
    cfg.tau_minus = tau_minus
    cfg.collision = capi.LBM_BGK if cm == "bgk" else capi.LBM_TRT
    cfg.compressible = 1 if isFluidCompressible else 0
    cfg.force_mode = force_mode
    cfg.storage = capi.STORAGE_NAMES[storage] if isinstance(storage, str) else int(storage)
    for a in range(3):
        cfg.force[a] = force_vec[a]
    if force_field is not None:
        keep.append(force_field)
        cfg.force_field = force_field.ctypes.data_as(capi._dp)
    if wall is not None:
        wall = np.asfortranarray(wall.astype(np.uint8))
        keep.append(wall)
        cfg.wall_mask = wall.ctypes.data_as(capi._u8p)
    if uw is not None:
        keep.append(uw)
        cfg.wall_velocity = uw.ctypes.data_as(capi._dp)
    # initial hydrodynamic fields (initMethods.jl:507-526)
    if massDensity is DEFAULT:
        cfg.rho_uniform = 1.0
    elif np.isscalar(massDensity):
        cfg.rho_uniform = float(massDensity)
    else:
        rho = np.asfortranarray(np.asarray(massDensity, dtype=np.float64))
        _assert(rho.shape == shape, f"The mass density given has the wrong size! {shape} expected.")
        keep.append(rho)
        cfg.rho_init = rho.ctypes.data_as(capi._dp)
    if fluidVelocity is not DEFAULT:
        fv = np.asarray(fluidVelocity, dtype=np.float64)
        if fv.ndim == 1:
            for a in range(dims):
                cfg.u_uniform[a] = fv[a]
        else:
            fv = np.asfortranarray(fv)
            _assert(fv.shape[:dims] == shape, f"The fluid velocity given has the wrong size! {shape} expected.")
            keep.append(fv)
            cfg.u_init = fv.ctypes.data_as(capi._dp)
    cfg.rho_ref = 0.0 if rho_ref is DEFAULT else float(rho_ref)
    cfg.store_scale = 0.0 if store_scale is DEFAULT else float(store_scale)
    cfg.device = -1 if device is DEFAULT else int(device)
    if schedule not in capi.SCHEDULE_NAMES:
        raise ValueError(f"schedule must be one of {sorted(capi.SCHEDULE_NAMES)}")
    cfg.schedule = capi.SCHEDULE_NAMES[schedule]
    # particleRules: "gpu" follows moveParticles! of src/gpu/particles.jl:7-92 (the module the
    # reference loads when CUDA is functional), "cpu" that of src/cpu/particles.jl:48-100
    if particleRules not in capi.RULES_NAMES:
        raise ValueError(f"particleRules must be one of {sorted(capi.RULES_NAMES)}")
    cfg.particle_rules = capi.RULES_NAMES[particleRules]
    # rounding of the F16/BF16 stores: "stochastic" (unbiased, the default) or "nearest"
    if rounding not in capi.ROUNDING_NAMES:
        raise ValueError(f"rounding must be one of {sorted(capi.ROUNDING_NAMES)}")
    cfg.rounding = capi.ROUNDING_NAMES[rounding]
    return SimpleNamespace(cfg=cfg, keep=keep, dt=dt, tau=tau, tau_minus=tau_minus, viscosity=nu,
                           relaxationTimeRatio=ratio, coordinates=axes, shape=shape, dims=dims,
                           velocities=vname, collision=cm, schemes=list(dict.fromkeys(schemes)),
                           kineticParameter=kineticParameter)


def _norm(v):
    return math.sqrt(sum(float(x) * float(x) for x in v))


def resolve_squirmer(dims, massDensity=1.0, radius=0.1, position=DEFAULT, velocity=DEFAULT,
                     angularVelocity=DEFAULT, slipSpeed=DEFAULT, swimmingSpeed=DEFAULT,
                     swimmingDirection=DEFAULT, B1=DEFAULT, B2=DEFAULT, beta=DEFAULT,
                     coupleTorques=False, coupleForces=False, scheme=DEFAULT, kind=capi.LBM_SQUIRMER):
    """addSquirmer! keyword resolution (src/gpu/initMethods.jl:91-173) -> LbmParticleParams."""
    p = capi.LbmParticleParams()
    p.kind = kind
    p.couple_forces = int(bool(coupleForces))
    p.couple_torques = int(bool(coupleTorques))
    p.radius = float(radius)
    p.mass_density = float(massDensity)
    pos = [0.0] * dims if position is DEFAULT else [float(x) for x in position]
    vel = [0.0] * dims if velocity is DEFAULT else [float(x) for x in velocity]
    if len(pos) != len(vel) or len(pos) != dims:
        raise ValueError("The position and velocity dimensions must match the dimensionality of the model! "
                         f"dims = {dims}")
    for a in range(dims):
        p.position[a] = pos[a]
        p.velocity[a] = vel[a]
    if dims == 2:
        om = 0.0 if angularVelocity is DEFAULT else angularVelocity
        _assert(np.isscalar(om), "In two dimensions, angularVelocity must be a number!")
        p.angular_velocity[0] = float(om)
    else:
        om = [0.0, 0.0, 0.0] if angularVelocity is DEFAULT else angularVelocity
        _assert(not np.isscalar(om), "In three dimensions, angularVelocity must be an array!")
        for a in range(3):
            p.angular_velocity[a] = float(om[a])
    if scheme is not DEFAULT:
        s = str(scheme).lstrip(":")
        _assert(s in ("psm", "ladd"), f"{scheme} cannot be used as a particle-fluid collision scheme!")
        _assert(s == "ladd", f"{scheme} is not implemented in the gpu modules!")
    if kind == capi.LBM_BEAD:
        return p
    # B1 / B2 (initMethods.jl:132-148)
    _assert(any(v is DEFAULT for v in (B1, B2, beta)), "B1, B2, and beta cannot be all simultaneously defined!")
    if beta is DEFAULT:
        B1 = 1 if B1 is DEFAULT else B1
        B2 = 0 if B2 is DEFAULT else B2
        beta = B2 / B1
    else:
        if B2 is DEFAULT:
            B1 = 1 if B1 is DEFAULT else B1
            B2 = B1 * beta
        else:
            _assert(beta != 0, "if beta = 0, then B2 can only be zero! In this case, do not declare both.")
            B1 = B2 / beta
    # swimming direction (:150-157)
    if swimmingDirection is DEFAULT:
        swimmingDirection = [1.0] + [0.0] * (dims - 1)
    _assert(len(swimmingDirection) == dims, f"the swimming direction must be {dims}-dimensional!")
    nrm = _norm(swimmingDirection)
    e = [float(x) / nrm for x in swimmingDirection]
    # B1/B2 rescaling (:159-173)
    _assert(slipSpeed is DEFAULT or swimmingSpeed is DEFAULT,
            "slipSpeed and swimmingSpeed cannot be all simultaneously defined!")
    if slipSpeed is DEFAULT:
        if swimmingSpeed is DEFAULT:
            swimmingSpeed = 1e-3
        sgn = float(np.sign(swimmingSpeed))
        e = [x * sgn for x in e]
        B1 = abs(3 / 2 * swimmingSpeed)
        B2 = B1 * beta
    else:
        thetas = np.linspace(-math.pi, math.pi, 100)
        normFactor = max(abs((B1 + B2 * math.cos(t)) * math.sin(t)) for t in thetas)
        B1 = B1 * (slipSpeed / normFactor)
        B2 = B2 * (slipSpeed / normFactor)
    p.B1 = float(B1)
    p.B2 = float(B2)
    for a in range(dims):
        p.swimming_direction[a] = e[a]
    return p


def resolve_bead(dims, massDensity=1.0, radius=0.1, position=DEFAULT, velocity=DEFAULT,
                 angularVelocity=DEFAULT, coupleTorques=False, coupleForces=False, scheme=DEFAULT):
    """addBead! keyword resolution (src/gpu/initMethods.jl:7-53) -> LbmParticleParams."""
    return resolve_squirmer(dims, massDensity=massDensity, radius=radius, position=position, velocity=velocity,
                            angularVelocity=angularVelocity, coupleTorques=coupleTorques,
                            coupleForces=coupleForces, scheme=scheme, kind=capi.LBM_BEAD)


def propagate_ticks(dt, simulationTime=DEFAULT, ticks=DEFAULT):
    """Number of ticks LBMpropagate! runs (src/gpu/fluids.jl:231-241)."""
    _assert(simulationTime is DEFAULT or ticks is DEFAULT,
            "simulationTime and ticks cannot be simultaneously chosen, as the time step is defined already in the model!")
    if simulationTime is DEFAULT and ticks is DEFAULT:
        return 100
    if ticks is DEFAULT:
        return len(julia_float_range(dt, simulationTime, dt))
    return int(ticks)
