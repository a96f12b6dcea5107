"""Build liblbm_b200.so in-tree (nvcc, sm_100a).

    python lbmengine.jl_b200/build.py [--jobs N] [--force]

Each translation unit under csrc/ is compiled to an object under _build/ and
linked into lbmengine.jl_b200/liblbm_b200.so, the library the Python mirror
(lbmengine/_capi.py) and the Julia shim (julia/LBMengineB200.jl) load.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "liblbm_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "--expt-relaxed-constexpr",
              "-Xcompiler", "-fPIC,-ffp-contract=off", f"-I{os.path.join(REPO, 'include')}", f"-I{CSRC}"]
UNITS = ["lbm_capi.cu", "inst_d2q9.cu", "inst_d3q15.cu", "inst_d3q19.cu", "inst_d3q27.cu"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _deps_mtime() -> float:
    paths = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    paths.append(os.path.join(REPO, "include", "lbm_b200.h"))
    return max(os.path.getmtime(p) for p in paths)


def _compile(unit: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-c", os.path.join(CSRC, unit), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {unit}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr.strip():
        print(r.stderr)
    return obj


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> str:
    """Compile and link the library unless it is newer than every source."""
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= _deps_mtime():
        return OUT
    # the sources as of now are what gets compiled; the library is stamped with
    # this time, so a source edited while the build runs makes it stale
    stamp = _deps_mtime()
    os.makedirs(BUILD, exist_ok=True)
    jobs = jobs or min(len(UNITS), os.cpu_count() or 1)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda u: _compile(u, verbose), UNITS))
    tmp = OUT + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.utime(tmp, (stamp, stamp))
    os.replace(tmp, OUT)
    return OUT


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--verbose", action="store_true")
    args = ap.parse_args(argv)
    out = build(force=args.force, jobs=args.jobs, verbose=args.verbose)
    print(out)
    return 0


if __name__ == "__main__":
    sys.exit(main())
