"""Python mirror of LBMengine.jl's model API over the C ABI.

Names, keywords, defaults and error behaviour follow the reference's exported
API (src/LBMengine.jl:27-41); Julia's `f!` functions are spelled without the
bang.  Arrays are numpy views in the reference's column-major layout:
``model.massDensity[i, j, k]`` is the reference's ``massDensity[i+1, j+1, k+1]``.
All computation happens in liblbm_b200.so on the GPU; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
from types import SimpleNamespace

import numpy as np

from . import _capi as capi
from . import config as cfgmod
from . import interactions
from . import output
from .config import DEFAULT


class LBMparticle(SimpleNamespace):
    """Snapshot of LBMparticle (src/gpu/structs.jl:85-95) after a tick."""


class LBMmodel:
    """A model living on the GPU (LBMmodel, src/gpu/structs.jl:52-76)."""

    def __init__(self, resolved, lib=None, handle=None):
        """Create the model on the GPU, or (``handle``) wrap a replica handle a
        batch owns; such a view never destroys it."""
        self._lib = lib or capi.load()
        self._res = resolved
        self._owned = handle is None
        if handle is None:
            self._h = C.c_void_p()
            capi.check(self._lib, None, self._lib.lbm_create(C.byref(resolved.cfg), C.byref(self._h)))
        else:
            self._h = C.c_void_p(handle)
        self.schemes = list(resolved.schemes)
        self.spaceTime = SimpleNamespace(coordinates=resolved.coordinates, latticeParameter=resolved.dt,
                                         timeStep=resolved.dt, latticeSpeed=1.0, dims=resolved.dims)
        self.fluidParams = SimpleNamespace(relaxationTime=resolved.tau, viscosity=resolved.viscosity,
                                           relaxationTimePlus=resolved.tau, relaxationTimeMinus=resolved.tau_minus,
                                           c_s=3 ** -0.5, c2_s=1 / 3, c4_s=1 / 9, invC_s=3 ** 0.5, invC2_s=3.0,
                                           invC4_s=9.0)
        self.particleInteractions = []
        self._shape = resolved.shape
        self._dims = resolved.dims
        info = self.info()
        self._q = info.q
        self._cells = info.cells
        if self._owned and "saveData" in self.schemes:  # modelInit: fresh output.lbm, the initial fluid
            output.prepare_directory()
            output.write_fluid(self)
            self._check(self._lib.lbm_output_flush(self._h))

    # ---- handle plumbing -------------------------------------------------
    def _check(self, code):
        capi.check(self._lib, self._h, code)

    def info(self):
        inf = capi.LbmInfo()
        self._check(self._lib.lbm_get_info(self._h, C.byref(inf)))
        return inf

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h and self._owned:
            self._lib.lbm_destroy(self._h)
        self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- reference fields --------------------------------------------------
    @property
    def tick(self) -> int:
        return int(self.info().tick)

    @property
    def time(self) -> float:
        return float(self.info().time)

    def read_fields(self, rho=None, u=None) -> None:
        """Write rho (shape N...) and u (N..., d) into caller-owned float64
        arrays in column-major order (a Julia array's layout, e.g. numpy
        arrays made with order="F", or pinned host memory); either may be None."""
        for a, shape in ((rho, self._shape), (u, self._shape + (self._dims,))):
            if a is not None and (a.dtype != np.float64 or a.shape != shape or not a.flags.f_contiguous
                                  or not a.flags.writeable):
                raise ValueError(f"expected a writeable column-major float64 array of shape {shape}")
        self._check(self._lib.lbm_get_fields(self._h, None if rho is None else rho.ctypes.data_as(capi._dp),
                                             None if u is None else u.ctypes.data_as(capi._dp)))

    @property
    def massDensity(self) -> np.ndarray:
        rho = np.empty(self._shape, dtype=np.float64, order="F")
        self.read_fields(rho=rho)
        return rho

    @property
    def fluidVelocity(self) -> np.ndarray:
        u = np.empty(self._shape + (self._dims,), dtype=np.float64, order="F")
        self.read_fields(u=u)
        return u

    @property
    def distributions(self) -> np.ndarray:
        f = np.empty(self._cells * self._q, dtype=np.float64)
        self._check(self._lib.lbm_get_distributions(self._h, f.ctypes.data_as(capi._dp)))
        return f.reshape(self._shape + (self._q,), order="F")

    @distributions.setter
    def distributions(self, f):
        f = np.asfortranarray(np.asarray(f, dtype=np.float64))
        if f.shape != self._shape + (self._q,):
            raise ValueError(f"distributions must have shape {self._shape + (self._q,)}")
        flat = np.ascontiguousarray(f.ravel(order="F"))
        self._check(self._lib.lbm_set_distributions(self._h, flat.ctypes.data_as(capi._dp)))

    def totals(self):
        """(sum of rho, sum of rho u): global FP64 sums on the device (lbm_get_totals)."""
        m = C.c_double()
        p = (C.c_double * 3)()
        self._check(self._lib.lbm_get_totals(self._h, C.byref(m), p))
        return m.value, np.array(p[:self._dims])

    def viscous_stress_tensor(self) -> np.ndarray:
        """viscousStressTensor(model) (src/cpu/fluids.jl:507-520): array (N..., d, d)."""
        d = self._dims
        s = np.empty(self._cells * d * d, dtype=np.float64)
        self._check(self._lib.lbm_get_stress(self._h, s.ctypes.data_as(capi._dp)))
        return s.reshape(self._shape + (d, d), order="F")

    def particle_states(self):
        cnt = C.c_int32()
        self._check(self._lib.lbm_get_particles(self._h, None, 0, C.byref(cnt)))
        if cnt.value == 0:
            return []
        arr = (capi.LbmParticleState * cnt.value)()
        self._check(self._lib.lbm_get_particles(self._h, arr, cnt.value, C.byref(cnt)))
        return list(arr)

    @property
    def particles(self):
        d = self._dims
        out = []
        for s in self.particle_states():
            props = ["spherical", "bead" if s.kind == capi.LBM_BEAD else "squirmer"]
            pp = SimpleNamespace(radius=s.radius, inverseMass=s.inverse_mass,
                                 inverseMomentOfInertia=s.inverse_inertia, properties=props,
                                 coupleForces=bool(s.couple_forces), coupleTorques=bool(s.couple_torques))
            if s.kind == capi.LBM_SQUIRMER:
                pp.B1, pp.B2 = s.B1, s.B2
                pp.swimmingDirection = np.array(s.swimming_direction[:d])
            out.append(LBMparticle(
                id=s.id, particleParams=pp,
                position=np.array(s.position[:d]), velocity=np.array(s.velocity[:d]),
                angularVelocity=(s.angular_velocity[0] if d == 2 else np.array(s.angular_velocity[:3])),
                forceInput=np.zeros(d), torqueInput=(0.0 if d == 2 else np.zeros(3)),
                lastForce=np.array(s.last_force[:d]),
                lastTorque=(s.last_torque[0] if d == 2 else np.array(s.last_torque[:3]))))
        return out

    def solid_region(self, pid: int) -> np.ndarray:
        m = np.empty(self._cells, dtype=np.uint8)
        self._check(self._lib.lbm_get_mask(self._h, pid, m.ctypes.data_as(capi._u8p)))
        return m.reshape(self._shape, order="F").astype(bool)

    def boundary_links(self, pid: int):
        n = C.c_int64()
        self._check(self._lib.lbm_get_links(self._h, pid, None, None, 0, C.byref(n)))
        cells = np.empty(max(1, n.value), dtype=np.int64)
        dirs = np.empty(max(1, n.value), dtype=np.int8)
        self._check(self._lib.lbm_get_links(self._h, pid, cells.ctypes.data_as(C.POINTER(C.c_int64)),
                                            dirs.ctypes.data_as(C.POINTER(C.c_int8)), n.value, C.byref(n)))
        return cells[:n.value], dirs[:n.value]

    def step(self, n: int) -> None:
        self._check(self._lib.lbm_step(self._h, int(n)))

    def record_force(self, pid: int, on: bool = True) -> None:
        """Report the momentum-exchange force of particle pid even when it is held
        (coupleForces false), without applying it: its drag (lbm_record_force)."""
        self._check(self._lib.lbm_record_force(self._h, int(pid), int(bool(on))))

    def save_state(self, path: str) -> None:
        self._check(self._lib.lbm_save_state(self._h, path.encode()))

    def load_state(self, path: str) -> None:
        self._check(self._lib.lbm_load_state(self._h, path.encode()))


def modelInit(**kw) -> LBMmodel:
    """modelInit(; ...) — src/gpu/initMethods.jl:440-702.

    Extra keywords of this build: ``storage`` ("f32" default, "f16", "bf16",
    "f64"), ``rho_ref`` and ``store_scale`` (shifted-storage parameters),
    ``device`` and ``schedule`` ("auto", "stream", "persistent": how
    the kernels of a tick are launched; results do not depend on it).
    """
    return LBMmodel(cfgmod.resolve_model(**kw))


def _add(model: LBMmodel, params) -> int:
    pid = C.c_int32()
    model._check(model._lib.lbm_add_particle(model._h, C.byref(params), C.byref(pid)))
    for s in ("ladd", "bounceBack"):
        if s not in model.schemes:
            model.schemes.append(s)
    if "saveData" in model.schemes:  # writeParticleTrajectory of the new particle (initMethods.jl:86, 219)
        output.write_particle(model, model.particle_states()[pid.value - 1])
    return pid.value


def addSquirmer(model: LBMmodel, **kw) -> None:
    """addSquirmer!(model; ...) — src/gpu/initMethods.jl:91-222 (src/cpu/initMethods.jl:89-222
    under the CPU module's particle rules, whose addSquirmer! has no angularVelocity keyword)."""
    if model._res.cfg.particle_rules == capi.LBM_RULES_CPU_MODULE and "angularVelocity" in kw:
        raise TypeError('addSquirmer! got unsupported keyword argument "angularVelocity"')
    _add(model, cfgmod.resolve_squirmer(model._dims, **kw))


def addBead(model: LBMmodel, **kw) -> None:
    """addBead!(model; ...) — src/gpu/initMethods.jl:7-89."""
    _add(model, cfgmod.resolve_bead(model._dims, **kw))


def LBMpropagate(model: LBMmodel, simulationTime=DEFAULT, ticks=DEFAULT, verbose=False, ticksSaved=DEFAULT) -> None:
    """LBMpropagate!(model; simulationTime, ticks, verbose, ticksSaved) — src/gpu/fluids.jl:228-264."""
    n = cfgmod.propagate_ticks(model.spaceTime.timeStep, simulationTime, ticks)
    if interactions.time_dependent(model):  # a field B(t) of dipoles: evaluated at each tick's time
        if "saveData" in model.schemes:
            raise NotImplementedError("saveData with a time-dependent magnetic field")
        for _ in range(n):
            interactions.push(model, model.time + model.spaceTime.timeStep)
            model.step(1)
    elif "saveData" in model.schemes:
        output.propagate(model, n, None if ticksSaved is DEFAULT else ticksSaved)
    else:
        model.step(n)
    if verbose:
        print(f"\r t = {round(model.time, 2)}")


def viscousStressTensor(model: LBMmodel):
    """viscousStressTensor(model) — src/cpu/fluids.jl:507-520: a d x d matrix
    whose entry (alpha, beta) is the field sigma_alpha_beta (N...)."""
    s = model.viscous_stress_tensor()
    d = model._dims
    return [[s[..., a, b] for b in range(d)] for a in range(d)]


def hydroVariablesUpdate(model: LBMmodel, useEquilibriumScheme=False) -> None:
    """hydroVariablesUpdate! — src/gpu/fluids.jl:32-37.

    The library keeps rho and u consistent with the populations at all times
    (they are evaluated from model.distributions on read), so this is a no-op
    kept for API compatibility.
    """
    return None
