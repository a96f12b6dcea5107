"""lbmengine — B200 lattice-Boltzmann time step behind LBMengine.jl's model API.

    import lbmengine as lbm
    model = lbm.modelInit(dims=3, velocities="D3Q19", collisionModel="trt", ...)
    lbm.addSquirmer(model, radius=8, position=[0.0, 0.0, 0.0], coupleForces=True)
    lbm.LBMpropagate(model, ticks=1000)
    rho, u = model.massDensity, model.fluidVelocity

The compute path is liblbm_b200.so (CUDA, sm_100a), loaded through ctypes.
"""
from .config import DEFAULT, julia_float_range, resolve_bead, resolve_model, resolve_squirmer  # noqa: F401
from .model import (LBMmodel, LBMparticle, LBMpropagate, addBead, addSquirmer,  # noqa: F401
                    hydroVariablesUpdate, modelInit, viscousStressTensor)
from .interactions import (addBistableBond, addDipoles, addLennardJones, addLinearBond,  # noqa: F401
                           addPolarBond, addWCA)
from .batch import LBMbatch  # noqa: F401
from . import _capi  # noqa: F401

__all__ = ["modelInit", "addSquirmer", "addBead", "LBMpropagate", "hydroVariablesUpdate", "LBMmodel",
           "LBMparticle", "LBMbatch", "DEFAULT", "viscousStressTensor", "addLinearBond", "addPolarBond",
           "addBistableBond", "addDipoles", "addLennardJones", "addWCA"]
