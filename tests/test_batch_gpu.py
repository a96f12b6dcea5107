"""Batches of replicas (lbm_batch_*) against the same models stepped one by one, and against the oracle.

A batch runs every replica's bulk tiles, fix-up blocks and particle updates as
items of one work queue; the per-node arithmetic is the one of the
single-model kernels, so a replica must follow the same model stepped alone
(to FP32 rounding), under either schedule, and the FP64 oracle within the FP32
parity tolerances of tests/test_parity_gpu.py.
"""
from __future__ import annotations

import numpy as np
import pytest

from parity_cases import rel_l2

pytestmark = pytest.mark.gpu


def replica_specs():
    """Six D2Q9 TRT squirmer replicas of uneven size, radius, beta and tau (a small sweep)."""
    rng = np.random.default_rng(11)
    specs = []
    for side, ny in ((64, 64), (96, 48), (128, 64), (64, 96), (256, 40), (32, 32)):
        r = float(rng.integers(4, 8)) if side > 32 else 3.0
        tau = float(rng.uniform(0.6, 1.0))
        beta = float(rng.uniform(-5, 5))
        ang = float(rng.uniform(0, 2 * np.pi))
        hx, hy = side // 2, ny // 2
        model = dict(dims=2, latticeParameter=1.0, relaxationTimeRatio=tau, collisionModel="trt",
                     xlims=(-float(hx), float(side - hx - 1)), ylims=(-float(hy), float(ny - hy - 1)))
        sq = dict(radius=r, position=[float(rng.uniform(-2, 2)), float(rng.uniform(-2, 2))],
                  swimmingSpeed=1e-3 / 1.5, beta=beta, swimmingDirection=[np.cos(ang), np.sin(ang)],
                  coupleForces=True, coupleTorques=True)
        specs.append((model, [("squirmer", sq)]))
    return specs


def alone(spec):
    from lbmengine import config as cfgmod, model as mdl
    mkw, parts = spec
    m = mdl.LBMmodel(cfgmod.resolve_model(**mkw))
    for kind, pkw in parts:
        mdl._add(m, (cfgmod.resolve_squirmer if kind == "squirmer" else cfgmod.resolve_bead)(2, **pkw))
    return m


def assert_close(a, b, tol_field=1e-6, tol_pos=1e-9):
    assert rel_l2(a.massDensity, b.massDensity) <= tol_field
    assert rel_l2(a.fluidVelocity, b.fluidVelocity, floor=1e-4) <= tol_field * 10
    for pa, pb in zip(a.particle_states(), b.particle_states()):
        assert np.max(np.abs(np.array(pa.position[:2]) - np.array(pb.position[:2]))) <= tol_pos
        assert np.max(np.abs(np.array(pa.velocity[:2]) - np.array(pb.velocity[:2]))) <= tol_pos


@pytest.mark.parametrize("schedule,order,cta", [("persistent", 0, 0), ("persistent", 1, 0), ("stream", 0, 0), ("stream", 1, 1)])
def test_batch_matches_models_stepped_alone(lib, schedule, order, cta):
    from lbmengine import LBMbatch
    specs = replica_specs()
    batch = LBMbatch(specs)
    batch.set_tuning(schedule=schedule, ctas_per_sm=4, tile_order=order, tile_cta=cta)
    singles = [alone(s) for s in specs]
    for n in (17, 23):  # a graph of 16 ticks plus tail ticks, then an odd count
        batch.step(n)
        for m in singles:
            m.step(n)
    for rep, m in zip(batch.replicas, singles):
        assert rep.tick == m.tick == 40
        assert_close(rep, m)
    batch.close()


def test_batch_replica_against_oracle(lib, oracle_mod):
    from lbmengine import LBMbatch, config as cfgmod
    specs = replica_specs()[:3]
    batch = LBMbatch(specs)
    batch.step(60)
    for spec, rep in zip(specs, batch.replicas):
        mkw, parts = spec
        orc = oracle_mod.OracleModel(cfgmod.resolve_model(**mkw))
        for _, pkw in parts:
            orc.add_particle(cfgmod.resolve_squirmer(2, **pkw))
        orc.step(60)
        rho_o, u_o = orc.fields()
        assert rel_l2(rep.massDensity.ravel(order="F"), rho_o) <= 1e-5
        assert rel_l2(rep.fluidVelocity.reshape(-1, 2, order="F").T, u_o, floor=1e-4) <= 1e-4
        po = orc.particles()[0]
        pg = rep.particle_states()[0]
        assert np.max(np.abs(np.array(pg.position[:2]) - np.array(po.position[:2]))) <= 1e-7
    batch.close()


def test_replica_stepped_alone_then_batch(lib):
    """Stepping one replica by itself flips its buffer parity; the batch rebuilds its queue."""
    from lbmengine import LBMbatch
    specs = replica_specs()[:3]
    batch = LBMbatch(specs)
    singles = [alone(s) for s in specs]
    batch.replicas[1].step(3)
    singles[1].step(3)
    batch.step(20)
    for m in singles:
        m.step(20)
    assert [r.tick for r in batch.replicas] == [20, 23, 20]
    for rep, m in zip(batch.replicas, singles):
        assert_close(rep, m)
    batch.close()


def test_autotune_restores_the_state(lib):
    from lbmengine import LBMbatch
    batch = LBMbatch(replica_specs()[:4])
    batch.step(5)
    before = [r.distributions.copy() for r in batch.replicas]
    pos = [r.particle_states()[0].position[:2] for r in batch.replicas]
    chosen, cands = batch.autotune(ticks=4)
    assert len(cands) >= 4 and all(c.ms_per_tick > 0 for c in cands)
    assert chosen.ms_per_tick == min(c.ms_per_tick for c in cands)
    assert batch.tuning.schedule == chosen.schedule
    for r, d, p in zip(batch.replicas, before, pos):
        assert r.tick == 5
        assert np.array_equal(r.distributions, d)
        assert list(r.particle_states()[0].position[:2]) == list(p)
    batch.close()
