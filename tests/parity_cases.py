"""Shared builders for the GPU-vs-oracle parity tests.

A case is a resolved modelInit keyword set plus a list of particle keyword
sets; `build_pair` instantiates it once on the CUDA library and once on the
FP64 CPU oracle from the very same C config struct.
"""
from __future__ import annotations

import numpy as np

from lbmengine import config as cfgmod
from lbmengine import model as lbmmodel


def unit(v):
    v = np.asarray(v, dtype=np.float64)
    return v / np.sqrt((v * v).sum())


def seeded_direction(seed, dims):
    rng = np.random.default_rng(seed)
    return list(unit(rng.standard_normal(dims)))


CASES = {
    # D2Q9 BGK squirmer (the 256x128 plain-method configuration, shrunk)
    "d2q9_bgk_squirmer": dict(
        model=dict(dims=2, latticeParameter=1.0, relaxationTimeRatio=0.8, collisionModel="bgk",
                   xlims=(-32.0, 31.0), ylims=(-16.0, 15.0)),
        particles=[dict(kind="squirmer", radius=5, position=[-12.0, 0.5], swimmingSpeed=1e-3 / 1.5, beta=3.0,
                        coupleForces=True, coupleTorques=True, swimmingDirection=[1.0, 0.3])],
        steps=150),
    # D3Q19 TRT + Guo squirmer (the 128^3 plain GPU configuration, shrunk)
    "d3q19_trt_guo_squirmer": dict(
        model=dict(dims=3, velocities="D3Q19", collisionModel="trt", kineticParameter=3 / 16,
                   latticeParameter=1.0, relaxationTimeRatio=0.7, xlims=(-16.0, 15.0),
                   forceDensity=[1e-5, 0.0, 0.0]),
        particles=[dict(kind="squirmer", radius=4.5, position=[0.3, -0.2, 0.1], swimmingSpeed=5e-4 / 1.5 * 4,
                        beta=-5.0, coupleForces=True, coupleTorques=True, swimmingDirection=seeded_direction(7, 3))],
        steps=80),
    # walls: Poiseuille channel, walls on y, body force along x
    "d2q9_trt_channel": dict(
        model=dict(dims=2, latticeParameter=1.0, relaxationTimeRatio=0.9, collisionModel="trt",
                   kineticParameter=3 / 16, xlims=(0.0, 15.0), ylims=(0.0, 20.0), walledDimensions=[2],
                   forceDensity=[1e-5, 0.0]),
        particles=[], steps=200),
    # moving walls (a lid along the top row) with a bead near it.  Coordinates are
    # centred on the origin: the reference computes a particle's mass from the
    # sphere around the ORIGIN (initMethods.jl:108), so in an all-positive domain
    # a particle would be 4x (2D) / 8x (3D) too light and Ladd coupling unstable.
    "d2q9_bgk_lid_bead": dict(
        model=dict(dims=2, latticeParameter=1.0, relaxationTimeRatio=0.7, collisionModel="bgk",
                   xlims=(-12.0, 11.0), ylims=(-12.0, 11.0), walledDimensions=[2],
                   movingWalls=lambda x, y: [1e-3, 0.0] if y >= 11.0 else [0.0, 0.0]),
        particles=[dict(kind="bead", radius=3.5, position=[-0.7, 0.0], coupleForces=True, coupleTorques=True,
                        massDensity=2.0)],
        steps=120),
    # several particles, 3D, beads and squirmers; the first touches the x edge so
    # its links cross the periodic boundary while its mask is clipped
    "d3q19_multi": dict(
        model=dict(dims=3, velocities="D3Q19", collisionModel="trt", latticeParameter=1.0,
                   relaxationTimeRatio=0.65, xlims=(-20.0, 19.0), ylims=(-12.0, 11.0), zlims=(-12.0, 11.0)),
        particles=[
            dict(kind="squirmer", radius=3.6, position=[-16.5, -0.8, -0.3], swimmingSpeed=2e-3, beta=2.0,
                 coupleForces=True, coupleTorques=True, swimmingDirection=seeded_direction(1, 3), massDensity=3.0),
            dict(kind="bead", radius=3.0, position=[0.2, -6.9, 5.3], velocity=[1e-3, 0.0, 0.0],
                 angularVelocity=[0.0, 0.0, 1e-3], coupleForces=False, coupleTorques=False),
            dict(kind="squirmer", radius=4.2, position=[10.5, 4.0, -5.6], swimmingSpeed=-1.5e-3, beta=-3.0,
                 coupleForces=True, coupleTorques=True, swimmingDirection=seeded_direction(3, 3), massDensity=2.0),
        ],
        steps=60),
    "d3q15_bgk_bead": dict(
        model=dict(dims=3, velocities="D3Q15", collisionModel="bgk", latticeParameter=1.0,
                   relaxationTimeRatio=0.9, xlims=(-10.0, 9.0), forceDensity=[0.0, 2e-5, 0.0]),
        particles=[dict(kind="bead", radius=3.2, position=[0.0, 0.0, 0.0], coupleForces=True,
                        coupleTorques=True)],
        steps=60),
    "d3q27_trt_squirmer": dict(
        model=dict(dims=3, velocities="D3Q27", collisionModel="trt", latticeParameter=1.0,
                   relaxationTimeRatio=0.75, xlims=(-10.0, 9.0)),
        particles=[dict(kind="squirmer", radius=3.7, position=[0.2, 0.1, -0.3], swimmingSpeed=2e-3, beta=1.0,
                        coupleForces=True, coupleTorques=True, swimmingDirection=seeded_direction(5, 3))],
        steps=60),
    # a squirmer whose link list (~2,300 entries) is longer than the 32 fix-up
    # CTAs of a particle cover in one pass, so each walks several chunks
    "d3q19_large_squirmer": dict(
        model=dict(dims=3, velocities="D3Q19", collisionModel="trt", latticeParameter=1.0,
                   relaxationTimeRatio=0.8, xlims=(-20.0, 19.0)),
        particles=[dict(kind="squirmer", radius=13.5, position=[0.4, -0.3, 0.2], swimmingSpeed=1e-3, beta=2.0,
                        coupleForces=True, coupleTorques=True, swimmingDirection=seeded_direction(9, 3),
                        massDensity=3.0)],
        steps=30),
    # twelve squirmers: more fix-up CTAs than the one-chunk-per-CTA launch
    # takes (nparts x capacity chunks >= 1024), so the chunk-walking fix-up runs
    "d3q19_twelve_squirmers": dict(
        model=dict(dims=3, velocities="D3Q19", collisionModel="trt", latticeParameter=1.0,
                   relaxationTimeRatio=0.8, xlims=(-24.0, 23.0), ylims=(-16.0, 15.0), zlims=(-16.0, 15.0)),
        particles=[dict(kind="squirmer", radius=5.0, position=[-16.0 + 16.0 * i + 0.3, -8.0 + 16.0 * j - 0.2,
                                                                -8.0 + 16.0 * k + 0.1],
                        swimmingSpeed=1e-3, beta=float(2 * i - j - k), coupleForces=True, coupleTorques=True,
                        swimmingDirection=seeded_direction(20 + 4 * i + 2 * j + k, 3), massDensity=3.0)
                   for i in range(3) for j in range(2) for k in range(2)],
        steps=30),
    "d2q9_incompressible": dict(
        model=dict(dims=2, latticeParameter=1.0, relaxationTimeRatio=0.8, collisionModel="trt",
                   xlims=(-16.0, 15.0), isFluidCompressible=False, massDensity=1.0,
                   fluidVelocity=[2e-3, -1e-3]),
        particles=[dict(kind="squirmer", radius=4, position=[0.0, 0.0], coupleForces=True, coupleTorques=True)],
        steps=80),
}


def particle_params(dims, p):
    p = dict(p)
    kind = p.pop("kind")
    if kind == "bead":
        return cfgmod.resolve_bead(dims, **p)
    return cfgmod.resolve_squirmer(dims, **p)


def build_pair(case, storage="f64", oracle_mod=None, with_gpu=True, rules="gpu"):
    res = cfgmod.resolve_model(**case["model"], storage=storage, particleRules=rules)
    gpu = lbmmodel.LBMmodel(res) if with_gpu else None
    orc = oracle_mod.OracleModel(res) if oracle_mod is not None else None
    for p in case["particles"]:
        prm = particle_params(res.dims, p)
        if gpu is not None:
            lbmmodel._add(gpu, prm)
        if orc is not None:
            orc.add_particle(prm)
    return res, gpu, orc


def rel_l2(a, b, floor=0.0):
    """||a - b|| / max(||b||, floor * sqrt(n)); `floor` is a characteristic magnitude
    of the field, so that a reference field that is zero up to rounding is not
    divided by its rounding residue."""
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    den = max(np.sqrt((b * b).sum()), floor * np.sqrt(b.size))
    return float(np.sqrt(((a - b) ** 2).sum()) / (den if den > 0 else 1.0))
