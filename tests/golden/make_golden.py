"""Generate the golden fixtures under tests/golden/.

    python tests/golden/make_golden.py --reference <checkout of LBMengine.jl>

1. velocity_sets.json — the D2Q9/D3Q15/D3Q19/D3Q27 tables (direction order,
   lattice vectors, weights) read as TEXT from the reference's
   src/gpu/misc.jl:195-272 and expanded with Julia's comprehension order
   (first iterator fastest, `|> vec` column-major).  The reference ships no
   tests or fixtures, so these tables are the part of its behaviour that can
   be pinned without running Julia.
2. oracle_small.json — outputs of the FP64 CPU oracle on three tiny cases
   (regression pins of the oracle itself; regenerated only on purpose).
"""
from __future__ import annotations

import argparse
import itertools
import json
import os
import re
import sys
from fractions import Fraction

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def _expand_entry(line: str):
    """Expand one `cs` entry of misc.jl into a list of vectors."""
    line = line.strip().rstrip(",")
    if not line or line.startswith("#"):
        return []
    line = line.replace("|>vec", "")
    m = re.fullmatch(r"\[\s*\[([^\]]*)\]\s*for\s+(.*)\]", line)
    if not m:
        lit = re.fullmatch(r"\[\s*\[([^\]]*)\]\s*\]", line)
        if not lit:
            raise ValueError(f"unrecognised entry: {line!r}")
        return [[int(v) for v in lit.group(1).split(",")]]
    template = [t.strip() for t in m.group(1).split(",")]
    iters = re.findall(r"(\w+)\s+in\s+\[([^\]]*)\]", m.group(2))
    names = [n for n, _ in iters]
    ranges = [[int(v) for v in r.split(",")] for _, r in iters]
    out = []
    # Julia's multi-iterator comprehension builds an array whose first index is
    # the first iterator; `vec` reads it column-major, so the first varies fastest
    for combo in itertools.product(*reversed(ranges)):
        env = dict(zip(reversed(names), combo))
        out.append([env[t] if t in env else int(t) for t in template])
    return out


def _expand_weights(line: str):
    line = line.strip().rstrip(",")
    if not line or line.startswith("#"):
        return []
    m = re.fullmatch(r"fill\(\s*([\d/\.]+)\s*,\s*(\d+)\s*\)", line)
    if m:
        return [str(Fraction(m.group(1)))] * int(m.group(2))
    return [str(Fraction(line))]


def parse_velocity_sets(misc_text: str):
    sets = {}
    pattern = re.compile(r"cs\s*=\s*\[(.*?)\n\]\s*ws\s*=\s*\[(.*?)\n\]\s*(D\dQ\d+)\s*=\s*\(;\s*cs,\s*ws\)", re.S)
    for cs_block, ws_block, name in pattern.findall(misc_text):
        cs = []
        for ln in cs_block.splitlines():
            ln = re.sub(r"#=+#", "", ln)
            cs += _expand_entry(ln)
        ws = []
        for ln in ws_block.splitlines():
            ln = re.sub(r"#=+#", "", ln)
            ws += _expand_weights(ln)
        sets[name] = {"c": cs, "w": ws}
    return sets


def make_velocity_sets(ref_root: str):
    path = os.path.join(ref_root, "src", "gpu", "misc.jl")
    text = open(path).read()
    sets = parse_velocity_sets(text)
    out = {"source": "src/gpu/misc.jl:195-272 (read as text)", "sets": sets}
    with open(os.path.join(HERE, "velocity_sets.json"), "w") as f:
        json.dump(out, f, indent=1)
    return sets


def make_oracle_small():
    sys.path.insert(0, os.path.join(REPO, "lbmengine.jl_b200"))
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    sys.path.insert(0, os.path.join(REPO, "tests"))
    import numpy as np
    import oracle
    from parity_cases import build_pair
    cases = {
        "d2q9_bgk_squirmer_tiny": dict(
            model=dict(dims=2, latticeParameter=1.0, relaxationTimeRatio=0.8, collisionModel="bgk",
                       xlims=(-8.0, 7.0), ylims=(-6.0, 5.0)),
            particles=[dict(kind="squirmer", radius=3, position=[-1.5, 0.25], swimmingSpeed=2e-3, beta=3.0,
                            coupleForces=True, coupleTorques=True, swimmingDirection=[1.0, 0.2])],
            steps=30),
        "d3q19_trt_guo_bead_tiny": dict(
            model=dict(dims=3, velocities="D3Q19", collisionModel="trt", kineticParameter=3 / 16,
                       latticeParameter=1.0, relaxationTimeRatio=0.7, xlims=(-5.0, 4.0),
                       forceDensity=[1e-4, 0.0, 0.0]),
            particles=[dict(kind="bead", radius=2.2, position=[0.1, -0.2, 0.3], coupleForces=True,
                            coupleTorques=True)],
            steps=20),
        "d2q9_trt_channel_tiny": dict(
            model=dict(dims=2, latticeParameter=1.0, relaxationTimeRatio=0.9, collisionModel="trt",
                       kineticParameter=3 / 16, xlims=(0.0, 5.0), ylims=(0.0, 9.0), walledDimensions=[2],
                       forceDensity=[1e-4, 0.0]),
            particles=[], steps=40),
    }
    out = {}
    for name, case in cases.items():
        _, _, orc = build_pair(case, oracle_mod=oracle, with_gpu=False)
        orc.step(case["steps"])
        rho, u = orc.fields()
        parts = [{"position": list(p.position), "velocity": list(p.velocity),
                  "angular_velocity": list(p.angular_velocity), "swimming_direction": list(p.swimming_direction),
                  "last_force": list(p.last_force), "last_torque": list(p.last_torque)} for p in orc.particles()]
        out[name] = {"case": {k: v for k, v in case.items()}, "rho": rho.tolist(), "u": u.tolist(),
                     "particles": parts}
    with open(os.path.join(HERE, "oracle_small.json"), "w") as f:
        json.dump(out, f)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="path of a checkout of david16correa/LBMengine.jl")
    ap.add_argument("--skip-oracle", action="store_true")
    a = ap.parse_args()
    sets = make_velocity_sets(a.reference)
    print({k: len(v["c"]) for k, v in sets.items()})
    if not a.skip_oracle:
        make_oracle_small()
        print("oracle_small.json written")


if __name__ == "__main__":
    main()
