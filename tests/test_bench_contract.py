"""bench.py's contract on the CPU: the reference arm's JSON line, and the
multi-rank plumbing (gloo, world size 2) that `bench.py --gpus N` uses under
torchrun: every rank joins, the timings are reduced to their maximum, only
rank 0 prints."""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env():
    env = dict(os.environ)
    env["OMP_NUM_THREADS"] = "2"
    return env


def test_reference_arm_prints_one_json_line():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--side", "16", "--steps", "2",
                          "--warmup", "1"], cwd=REPO, env=_env(), capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["unit"] == "MLUPS" and line["value"] > 0
    assert line["higher_is_better"] is True and line["n_gpus"] == 1
    assert line["config"]["cells"] == 16 ** 3 and line["config"]["parallelism"] == "single"
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


_WORKER = r"""
import os, sys, json
sys.path.insert(0, {repo!r})
import bench
world, rank, local, dist = bench.dist_setup()
m = bench.reduce_max(dist, float(rank + 1))
bench.barrier(dist)
print(json.dumps({{"rank": rank, "world": world, "max": m}}), flush=True)
dist.destroy_process_group()
"""


def test_ranks_reduce_their_timings_to_the_maximum():
    port = _free_port()
    procs = []
    for rank in range(2):
        env = _env()
        env.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2", RANK=str(rank),
                   LOCAL_RANK=str(rank))
        procs.append(subprocess.Popen([sys.executable, "-c", _WORKER.format(repo=REPO)], cwd=REPO, env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=300) for p in procs]
    for p, (o, e) in zip(procs, outs):
        assert p.returncode == 0, e[-2000:]
    got = sorted((json.loads(o.strip().splitlines()[-1]) for o, _ in outs), key=lambda d: d["rank"])
    assert [g["rank"] for g in got] == [0, 1]
    assert all(g["world"] == 2 and g["max"] == 2.0 for g in got)


def test_reference_arm_under_torchrun_prints_once():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference", "--gpus", "2", "--side", "16",
           "--steps", "1", "--warmup", "1"]
    out = subprocess.run(cmd, cwd=REPO, env=_env(), capture_output=True, text=True, timeout=900)
    if out.returncode != 0 and "torch.distributed" in out.stderr and "No module" in out.stderr:
        pytest.skip("torchrun is not available")
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.strip().startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
